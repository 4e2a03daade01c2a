"""The server's continuous wavefront on a B200 (rt_server_options.continuous), through the C-ABI.

* A request's image is a session's render of the same view and seed taken first to one pass, then to its target: the
  same samples with the same random numbers, each pixel's passes added in pass order into a chunk accumulator that
  goes into the sums after the first pass, at every chunk's end and at the target. For the books' tree-searched
  scenes the kernels compute the same values as the session's, so the images are equal bit for bit; under NEE/MIS the
  batch shade kernel (its integrator chosen per job at run time) is compiled apart from the session's, so the images
  agree to rounding; the flat-searched scenes are walked through their tree in the continuous run, so their closest
  hits agree up to the order of exact ties.
  The batched server's steps may end inside a chunk (its step time decides), so its images equal these to rounding.
* Every request gets its first frame before it is refined, and reaches its target.
* The rings wrap: more sample values than the values ring holds and more segments than the segment table holds pass
  through them, and the images stay right.
* A request cancelled while its samples are in flight frees its memory; the others are not disturbed.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same_render(img, ref):
    """Equal to the rounding of separately compiled kernels: nearly every value to 1e-5 relative, the means to 1e-5."""
    close = np.isclose(img, ref, rtol=1e-5, atol=1e-7)
    assert close.mean() >= 0.995, close.mean()
    assert abs(img.mean() - ref.mean()) <= 1e-5 * max(abs(ref.mean()), 1e-3), (img.mean(), ref.mean())


def _session_split(rt, scene, camera, seed, target):
    sess = rt.Session(scene, seed=seed)
    sess.set_camera(camera)
    sess.render_to(1)
    sess.render_to(target)
    return sess.pixels()


def _serve(rt, views, continuous, step_seconds=0.002, budget=1 << 30):
    server = rt.Server(hbm_budget_bytes=budget, step_seconds=step_seconds, continuous=continuous)
    ids = [server.submit(scene, cam, seed, target) for scene, cam, seed, target in views]
    steps = 0
    while any(server.poll(i)["state"] != "done" for i in ids):
        server.step()
        steps += 1
        assert steps < 20000
    images = [server.fetch(i) for i in ids]
    stats = server.stats()
    server.close()
    return images, stats, steps


def _bit_equal(img, ref):
    same = img == ref
    assert same.all(), (f"{same.mean():.6f} of values equal; largest difference "
                        f"{np.abs(img - ref).max():.3e}, image means {img.mean():.9f} {ref.mean():.9f}")


def test_continuous_tree_scenes_equal_sessions_bit_for_bit(rt):
    weekend = rt.builtin_scene("weekend", width=96, spp=16)
    mesh = rt.builtin_scene("mesh-ggx", width=64, spp=16, mesh_level=5, env_width=64)
    w, m = rt.Scene(weekend), rt.Scene(mesh)
    orbit = rt.builtin_camera("weekend", width=72, spp=16, orbit=(120.0, 20.0))
    views = [(w, weekend.camera, 3, 40), (m, mesh.camera, 4, 17), (w, orbit, 5, 33), (m, mesh.camera, 6, 1)]
    cont, cstats, _ = _serve(rt, views, continuous=True)
    batched, bstats, _ = _serve(rt, views, continuous=False)
    for (scene, cam, seed, target), img, other in zip(views, cont, batched):
        ref = _session_split(rt, scene, cam, seed, target)
        assert img.shape == ref.shape
        if scene is w:
            _bit_equal(img, ref)  # the books' integrator
        else:
            _same_render(img, ref)  # NEE/MIS
        _same_render(other, img)
    assert cstats["rays"] == bstats["rays"] and cstats["shadow_rays"] == bstats["shadow_rays"]
    assert cstats["completed"] == 4 and cstats["used_bytes"] == 0


def test_continuous_mixed_scenes_equal_sessions(rt):
    glass = rt.builtin_scene("glass", width=64, spp=16)
    mis = rt.builtin_scene("cornell-mis", width=48, spp=16)
    cover = rt.builtin_scene("weekend", width=56, spp=16)
    g, c, k = rt.Scene(glass), rt.Scene(mis), rt.Scene(cover)
    orbit = rt.builtin_camera("glass", width=80, spp=16, orbit=(40.0, 15.0))
    views = [(g, glass.camera, 5, 40), (c, mis.camera, 6, 33), (g, orbit, 7, 17), (k, cover.camera, 8, 48)]
    images, stats, _ = _serve(rt, views, continuous=True)
    for (scene, cam, seed, target), img in zip(views, images):
        _same_render(img, _session_split(rt, scene, cam, seed, target))
    assert stats["completed"] == 4 and stats["rays"] > 0 and stats["shadow_rays"] > 0


def test_continuous_first_frames_then_targets(rt):
    glass = rt.builtin_scene("glass", width=64, spp=16)
    g = rt.Scene(glass)
    server = rt.Server(hbm_budget_bytes=1 << 30, step_seconds=0.001, continuous=True)
    ids = [server.submit(g, glass.camera, s, 400) for s in range(3)]
    first = server.step()
    assert first["admitted"] == 3
    # every first frame is published at admission: each has its first pass after at most a few steps
    steps = 1
    while any(server.poll(i)["passes"] == 0 for i in ids):
        server.step()
        steps += 1
        assert steps < 50
    seen = {i: server.poll(i)["passes"] for i in ids}
    assert all(p >= 1 for p in seen.values())
    while any(server.poll(i)["state"] != "done" for i in ids):
        server.step()
        for i in ids:
            p = server.poll(i)["passes"]
            assert p >= seen[i]
            # the passes shown: 1, then multiples of the 16-pass chunk, then the target
            assert p in (1, 400) or p % 16 == 0, p
            seen[i] = p
        steps += 1
        assert steps < 20000
    for i in ids:
        st = server.poll(i)
        assert st["passes"] == 400 and st["done_seconds"] >= st["first_frame_seconds"] >= 0
    server.close()


def test_continuous_rings_wrap(rt):
    """About 1.6 x 2^26 sample values (the values ring holds 2^26) and 5,000 segments (the table holds 4,096)."""
    cover = rt.builtin_scene("weekend", width=256, spp=16)
    k = rt.Scene(cover)
    big = [(k, cover.camera, 100 + i, 200) for i in range(8)]  # 8 x 65,536 x 200 samples
    tiny_cam = rt.builtin_camera("weekend", width=16, spp=16, orbit=(30.0, 10.0))
    tiny = [(k, tiny_cam, 1000 + i, 2) for i in range(2500)]  # two segments each
    views = big + tiny
    images, stats, _ = _serve(rt, views, continuous=True, step_seconds=0.005, budget=8 << 30)
    assert stats["completed"] == len(views)
    for idx in (0, 7, 8, 1000, len(views) - 1):
        scene, cam, seed, target = views[idx]
        _bit_equal(images[idx], _session_split(rt, scene, cam, seed, target))


def test_continuous_cancel_in_flight(rt):
    cover = rt.builtin_scene("weekend", width=64, spp=16)
    k = rt.Scene(cover)
    big_cam = rt.builtin_camera("weekend", width=1024, spp=16)
    server = rt.Server(hbm_budget_bytes=1 << 30, step_seconds=0.001, continuous=True)
    big = server.submit(k, big_cam, 1, 4096)
    small = server.submit(k, cover.camera, 2, 48)
    server.step()
    server.step()
    assert server.poll(big)["state"] == "active" and server.poll(big)["passes"] < 4096
    used = server.stats()["used_bytes"]
    server.cancel(big)
    assert server.poll(big)["state"] == "cancelled"
    assert server.stats()["used_bytes"] == used - (1024 * 576 * 48 + 16)
    while server.poll(small)["state"] != "done":
        server.step()
    img = server.fetch(small)
    _bit_equal(img, _session_split(rt, k, cover.camera, 2, 48))
    assert server.stats()["used_bytes"] == 0
    server.close()


def test_continuous_budget_counts_the_accumulator(rt):
    """A continuous request holds its sums and its chunk accumulator: 48 bytes a pixel."""
    glass = rt.builtin_scene("glass", width=64, spp=16)
    g = rt.Scene(glass)
    one = glass.width * glass.height * 48 + 16
    server = rt.Server(hbm_budget_bytes=one + one // 2, step_seconds=0.001, continuous=True)
    ids = [server.submit(g, glass.camera, s, 16) for s in range(2)]
    r = server.step()
    assert r["admitted"] == 1 and r["queued"] == 1
    while server.poll(ids[0])["state"] != "done":
        server.step()
    server.fetch(ids[0])
    r = server.step()
    assert r["admitted"] == 1
    while server.poll(ids[1])["state"] != "done":
        server.step()
    _same_render(server.fetch(ids[1]), _session_split(rt, g, glass.camera, 1, 16))
    server.close()
