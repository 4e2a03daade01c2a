"""Batched rendering and serving on a B200, through the C-ABI.

* A job rendered in a batch beside other jobs (other scenes, sizes, integrators) gives the image a plain render of
  the same scene and seed gives: the same samples with the same random numbers, its steps ending on chunk boundaries
  and each pixel's chunks added in chunk order whatever the step they came in; equal to the rounding of the two
  separately compiled kernels.
* The captured graph of a step gives the same images as the step launched directly, bit for bit, and so does a
  small partials arena that takes more steps.
* A batch job's image passes ImageCompare against the oracle (the parity of the shared kernel path).
* The server: admission under the HBM budget in arrival order, a first frame before refinement, a request done at
  its target with an image equal (to rounding of a split first chunk) to a session's render of the same view.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mixed_scenes(rt):
    return [
        (rt.builtin_scene("glass", width=48, spp=64), 11, 64),
        (rt.builtin_scene("cornell-mis", width=40, spp=16), 12, 20),
        (rt.builtin_scene("cover-40", width=56, spp=16, sampling="mixture", scene_seed=3), 13, 33),
        (rt.builtin_scene("materials", width=24, spp=4), 14, 16),
        (rt.builtin_scene("furnace", width=16, spp=4), 15, 5),
    ]


def _same_render(img, ref):
    """The batch kernel traces the same samples with the same random numbers as the plain kernel; the two are compiled
    separately, so the compiler's fused multiply-adds may round a few values differently. Nearly every value is equal
    to 1e-5 relative, and the image means agree to 1e-5 (a rounding that flips one path's branch moves one value)."""
    close = np.isclose(img, ref, rtol=1e-5, atol=1e-7)
    assert close.mean() >= 0.995, close.mean()
    assert abs(img.mean() - ref.mean()) <= 1e-5 * max(abs(ref.mean()), 1e-3), (img.mean(), ref.mean())


def test_batch_equals_plain_renders(rt):
    jobs = _mixed_scenes(rt)
    b = rt.batch_render(jobs)
    assert b.graph
    # per step: the four persistent groups' launches and the reduction, and for the jobs in the wavefront form (the
    # lit Cornell boxes, the cover scene) each group's shade and trace launches of each wavefront step and its partials
    assert b.steps >= 1 and b.launches > 5 * b.steps
    for (scene, seed, passes), img in zip(jobs, b.images):
        ref = rt.render(scene, seed=seed, passes=passes)
        assert img.shape == ref.pixels.shape
        _same_render(img, ref.pixels)
    assert np.all(b.images[4] == 1.0)


def test_batch_graph_equals_direct_launches(rt):
    jobs = _mixed_scenes(rt)
    a = rt.batch_render(jobs, use_graph=True)
    b = rt.batch_render(jobs, use_graph=False)
    assert a.graph and not b.graph
    for x, y in zip(a.images, b.images):
        assert np.array_equal(x, y)
    assert a.rays == b.rays and a.shadow_rays == b.shadow_rays


def test_batch_jobs_take_their_forms(rt):
    # a bare flat scene in the persistent groups; a tree in the wavefront's groups; a lit flat scene in the persistent
    # kernel in a short step (one wavefront run a step at most) and in the wavefront's flat-searched group in a long one
    bare = rt.batch_render([(rt.builtin_scene("quads", width=32, spp=4), 1, 4)])
    assert bare.launches == 5 * bare.steps  # the four persistent groups' launches and the reduction
    short = rt.batch_render([(rt.builtin_scene("glass", width=32, spp=4), 1, 4)])
    assert short.launches == 5 * short.steps
    tree = rt.batch_render([(rt.builtin_scene("cover-40", width=32, spp=4), 1, 4)])
    assert tree.launches >= 8 * tree.steps  # and a wavefront run's steps (two launches each) and its partials


def test_long_step_flat_jobs_take_the_wavefront(rt):
    """A step of more than 12M samples renders a lit flat scene (the glass Cornell box, 13M samples) in the wavefront's
    flat-searched group; its image is a session's (the session's wavefront and flat search, to the rounding of
    separately compiled kernels)."""
    scene = rt.builtin_scene("glass", width=320, spp=128)
    b = rt.batch_render([(scene, 31, 128)])
    assert b.launches >= 8 * b.steps
    ref = rt.render(scene, seed=31, passes=128).pixels
    img = b.images[0]
    close = np.isclose(img, ref, rtol=1e-4, atol=1e-5 * max(abs(ref.mean()), 1e-3))
    assert close.mean() >= 0.99, close.mean()
    assert abs(img.mean() - ref.mean()) <= 2e-4 * max(abs(ref.mean()), 1e-3), (img.mean(), ref.mean())


def _same_wavefront_render(img, ref):
    """The wavefront's tolerance (tests/test_gpu_wavefront.py): through glass and smoke a last-bit difference between
    separately compiled kernels can send a few paths elsewhere."""
    close = np.isclose(img, ref, rtol=1e-4, atol=1e-5 * max(abs(ref.mean()), 1e-3))
    assert close.mean() >= 0.99, close.mean()
    assert abs(img.mean() - ref.mean()) <= 2e-4 * max(abs(ref.mean()), 1e-3), (img.mean(), ref.mean())


def test_long_step_flat_scene_with_smoke(rt):
    # the Cornell box with smoke, 256 x 256 x 256 passes (16.8M samples, a long step): the wavefront's flat-searched
    # group with the second book's features (free flights, transmittance on the lamps' shadow rays)
    scene = rt.builtin_scene("smoke", width=256, spp=256, combination="mis")
    b = rt.batch_render([(scene, 41, 256)])
    assert b.launches >= 8 * b.steps
    _same_wavefront_render(b.images[0], rt.render(scene, seed=41, passes=256).pixels)


def test_short_step_tree_jobs_share_one_group(rt):
    # a short step's tree jobs in one wavefront group: the sphere cover scene renders with the textured, moving
    # spheres and smoke of the second book's final scene, in its feature kernels, and gives its own session's image
    jobs = [(rt.builtin_scene("final", width=64, spp=16), 51, 16),
            (rt.builtin_scene("weekend", width=64, spp=16), 52, 16)]
    b = rt.batch_render(jobs)
    # one step: the persistent groups' four launches and the reduction, and ONE wavefront run (two launches a step
    # and its partials: an even count; a second run would make it odd)
    assert b.steps == 1 and b.launches >= 8 and b.launches % 2 == 0
    for (scene, seed, passes), img in zip(jobs, b.images):
        _same_wavefront_render(img, rt.render(scene, seed=seed, passes=passes).pixels)


def test_batch_small_arena_takes_more_steps_same_images(rt):
    jobs = _mixed_scenes(rt)[:3]
    a = rt.batch_render(jobs)
    # room for about one chunk of the largest job: the jobs are cut back to fewer chunks per step
    b = rt.batch_render(jobs, partial_budget_bytes=48 * 48 * 24 * 2)
    assert b.steps > a.steps
    for x, y in zip(a.images, b.images):
        assert np.array_equal(x, y)


def test_batch_job_matches_oracle(rt, oracle):
    s = rt.builtin_scene("cover-40", width=64, spp=64, sampling="mixture", scene_seed=5)
    others = [(rt.builtin_scene("glass", width=40, spp=16), 1, 16)]
    for gpu_seed, cpu_seed in ((101, 202), (303, 404)):
        b = rt.batch_render([(s, gpu_seed, 64)] + others)
        c, _ = oracle.render(s.desc, s.width, s.height, seed=cpu_seed, passes=64)
        r = oracle.image_compare(c, b.images[0])
        if r["verdict"] == 0:
            return
    raise AssertionError(f"a batch job failed ImageCompare twice: {r}")


def _session_image(rt, scene_handle, camera, seed, passes):
    sess = rt.Session(scene_handle, seed=seed)
    sess.set_camera(camera)
    sess.render_to(passes)
    return sess.pixels()


def test_server_serves_first_frames_then_targets(rt):
    glass = rt.builtin_scene("glass", width=64, spp=16)
    mis = rt.builtin_scene("cornell-mis", width=48, spp=16)
    g = rt.Scene(glass)
    m = rt.Scene(mis)
    orbit = rt.builtin_camera("glass", width=80, spp=16, orbit=(40.0, 15.0))
    server = rt.Server(hbm_budget_bytes=1 << 30, step_seconds=0.002)
    ids = [server.submit(g, glass.camera, 5, 40), server.submit(m, mis.camera, 6, 33), server.submit(g, orbit, 7, 17)]
    first = server.step()
    assert first["admitted"] == 3 and first["first_frames"] == 3 and first["refined"] == 0
    for i in ids:
        st = server.poll(i)
        assert st["state"] == "active" and st["passes"] == 1 and st["first_frame_seconds"] >= 0
    steps = 1
    while any(server.poll(i)["state"] != "done" for i in ids):
        server.step()
        steps += 1
        assert steps < 500
    views = [(g, glass.camera, 5, 40), (m, mis.camera, 6, 33), (g, orbit, 7, 17)]
    for i, (scene, cam, seed, target) in zip(ids, views):
        st = server.poll(i)
        assert st["passes"] == target and st["done_seconds"] >= st["first_frame_seconds"] >= 0
        img = server.fetch(i)
        ref = _session_image(rt, scene, cam, seed, target)
        _same_render(img, ref)
    stats = server.stats()
    assert stats["completed"] == 3 and stats["used_bytes"] == 0 and stats["rays"] > 0 and stats["shadow_rays"] > 0
    server.close()


def test_server_admits_under_the_budget_in_order(rt):
    glass = rt.builtin_scene("glass", width=64, spp=16)
    g = rt.Scene(glass)
    one = glass.width * glass.height * 24 + 16
    server = rt.Server(hbm_budget_bytes=one + one // 2, step_seconds=0.002)
    ids = [server.submit(g, glass.camera, s, 16) for s in range(3)]
    r = server.step()
    assert r["admitted"] == 1 and r["queued"] == 2
    assert server.poll(ids[1])["state"] == "queued"
    with pytest.raises(rt.LogicError):
        server.fetch(ids[1])
    server.cancel(ids[2])
    assert server.poll(ids[2])["state"] == "cancelled"
    while server.poll(ids[0])["state"] != "done":
        server.step()
    server.fetch(ids[0])  # frees its memory: the next step admits the second
    r = server.step()
    assert r["admitted"] == 1 and r["queued"] == 0
    while server.poll(ids[1])["state"] != "done":
        server.step()
    img = server.fetch(ids[1])
    _same_render(img, _session_image(rt, g, glass.camera, 1, 16))
    with pytest.raises(rt.CapacityError):
        server.submit(g, rt.builtin_camera("glass", width=4000), 1, 1)
    server.close()


def test_large_tree_jobs_take_the_wavefront(rt):
    """A job of a large tree (the mesh at 82k triangles) renders in the batch's wavefront groups beside jobs of other
    groups; its image is a session's render of the same view and seed (the session's wavefront: the same samples, to
    the rounding of separately compiled kernels)."""
    jobs = [(rt.builtin_scene("mesh-ggx", width=64, spp=16, mesh_level=6, env_width=64), 21, 16),
            (rt.builtin_scene("cover-40", width=40, spp=16, scene_seed=5), 22, 16),
            (rt.builtin_scene("glass", width=32, spp=16), 23, 16)]
    b = rt.batch_render(jobs)
    assert b.launches > 8 * b.steps  # the wavefront groups' steps beside the persistent groups' launches and the reduction
    for (scene, seed, passes), img in zip(jobs, b.images):
        ref = rt.render(scene, seed=seed, passes=passes).pixels
        close = np.isclose(img, ref, rtol=1e-4, atol=1e-5 * max(abs(ref.mean()), 1e-3))
        assert close.mean() >= 0.99, close.mean()
        assert abs(img.mean() - ref.mean()) <= 2e-4 * max(abs(ref.mean()), 1e-3), (img.mean(), ref.mean())
