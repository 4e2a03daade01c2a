"""Parity of the CUDA path with the oracle, through the C-ABI, on a B200.

* The white furnace renders exactly 1.0 in every pixel (src/gpu_scenes.ixx:33-55; docs/image-compare.md:145).
* Primary-ray first hits: the same float camera rays go to the GPU's closest-hit queries and to the oracle's
  double-precision brute force; ids are compared in source index space and must agree on >= 99.99% of the rays,
  and every difference must be a hit-distance tie within 1e-6 relative (the reference's tracer-parity classes,
  tests/optix_tests.cu:461-475, tests/tracer_check_layout.h).
* Images: ImageCompare (the restated src/image_compare.cpp) between a GPU render and an oracle render of the same
  scene, strategy and passes, with different seeds; a failure is re-run once with fresh seeds, the reference's
  re-run rule (scripts/verify/compare.ps1), so a chance alarm (<= 1/100 per comparison) does not fail the suite.
* A seed fixes the image bit for bit; passes grouped into launches on chunk boundaries give the same image bit for
  bit (renderer.h:582-584).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _compare_with_rerun(rt, oracle, name, passes, seeds, **kw):
    s = rt.builtin_scene(name, **kw)
    reports = []
    for gpu_seed, cpu_seed in seeds:
        g = rt.render(s, seed=gpu_seed, passes=passes)
        c, cstats = oracle.render(s.desc, s.width, s.height, seed=cpu_seed, passes=passes)
        r = oracle.image_compare(c, g.pixels)
        reports.append((r, g, cstats))
        if r["verdict"] == 0:
            return r, g, cstats
    raise AssertionError(f"{name} {kw}: ImageCompare failed twice: {[x[0] for x in reports]}")


def test_device_is_a_b200(rt):
    info = rt.query_device()
    assert info["compute_capability"] == (10, 0), info
    assert info["multiprocessors"] >= 100


def test_furnace_is_exactly_one(rt):
    s = rt.builtin_scene("furnace", width=480, spp=64)
    r = rt.render(s, seed=7)
    assert r.pixels.shape == (270, 480, 3)
    assert np.all(r.pixels == 1.0), (r.pixels.min(), r.pixels.max())
    assert r.passes == 64
    n = 480 * 270 * 64
    assert n <= r.rays <= 2 * n
    assert r.kernel["name"] == "persistent books"


@pytest.mark.parametrize("name,width", [("weekend", 400), ("glass", 300), ("cornell", 300), ("materials", 320),
                                        ("quads", 256)])
def test_first_hit_ids_match_oracle(rt, oracle, name, width):
    s = rt.builtin_scene(name, width=width, spp=16)
    scene = rt.Scene(s)
    for p in (0, 5):
        o, d = scene.camera_rays(seed=3, pass_index=p)
        ids, ts = scene.closest_hits(o, d)
        ref_ids, ref_ts = oracle.closest_hits(s.desc, o.astype(np.float64), d.astype(np.float64), brute_force=True)
        both = (ids == ref_ids) & (ids >= 0)
        assert np.allclose(ts[both], ref_ts[both], rtol=2e-4, atol=1e-5)
        # >= 99.99% equal, and every difference a tie: both hit at distances within 1e-6 relative
        r = oracle.first_hit_mismatches(s.desc, o, d, ids, ref_ids, ts, ref_ts, tie_rel=1e-6)
        assert r["mismatches"] <= 1e-4 * r["rays"] and r["non_tie_mismatches"] == 0, r


@pytest.mark.parametrize("name,kw,passes", [
    ("weekend", dict(width=200, spp=16), 32),
    ("glass", dict(width=128, spp=64), 64),
    ("cornell", dict(width=128, spp=64), 64),
    ("cornell", dict(width=96, spp=64, sampling="material"), 64),
    ("cornell", dict(width=96, spp=64, sampling="uniform"), 64),
    ("cornell", dict(width=96, spp=64, sampling="lights"), 64),
    ("cornell", dict(width=128, spp=64, combination="mis"), 64),
    ("cornell", dict(width=96, spp=64, combination="nee"), 64),
    ("cornell-mis", dict(width=128, spp=64), 64),
    ("materials", dict(width=160, spp=16), 32),
    ("quads", dict(width=128, spp=16), 16),
])
def test_image_matches_oracle(rt, oracle, name, kw, passes):
    r, g, cstats = _compare_with_rerun(rt, oracle, name, passes, [(101, 202), (303, 404)], **kw)
    # The same estimator traces the same number of segments per sample, up to noise
    gpu_rays = g.rays / g.pixels[..., 0].size / passes
    cpu_rays = cstats["rays"] / g.pixels[..., 0].size / passes
    assert gpu_rays == pytest.approx(cpu_rays, rel=0.03), (gpu_rays, cpu_rays)
    if kw.get("combination") in ("mis", "nee") or name == "cornell-mis":
        assert g.shadow_rays > 0
        assert g.shadow_rays / cstats["shadow_rays"] == pytest.approx(1.0, rel=0.05)


def test_seed_fixes_the_image(rt):
    s = rt.builtin_scene("glass", width=96, spp=16)
    a = rt.render(s, seed=9, passes=32).pixels
    b = rt.render(s, seed=9, passes=32, launch_seconds=0.001).pixels
    c = rt.render(s, seed=10, passes=32).pixels
    assert np.array_equal(a, b)
    assert not np.array_equal(a, c)


def test_grouping_of_passes_does_not_change_the_image(rt):
    s = rt.builtin_scene("weekend", width=128, spp=16)
    scene = rt.Scene(s)
    one = rt.Session(scene, seed=4)
    one.render_to(64)
    steps = rt.Session(scene, seed=4)
    for target in (16, 32, 48, 64):
        steps.render_to(target)
    assert np.array_equal(one.pixels(), steps.pixels())
    # passes split inside a chunk: the same samples, summed in another grouping
    odd = rt.Session(scene, seed=4)
    for target in (5, 21, 40, 64):
        odd.render_to(target)
    assert np.allclose(one.pixels(), odd.pixels(), rtol=1e-12, atol=1e-15)
    assert one.counters()["rays"] == steps.counters()["rays"] == odd.counters()["rays"]


def test_session_semantics(rt):
    s = rt.builtin_scene("cornell", width=64, spp=16)
    scene = rt.Scene(s)
    session = rt.Session(scene, seed=1)
    with pytest.raises(rt.LogicError):
        session.pixels()
    report = session.render_to(16)
    assert report["passes"] == 16 and report["launches"] >= 1
    with pytest.raises(ValueError):
        session.render_to(8)
    report = session.render_for(0.05, 10_000)
    assert session.state() >= 17
    cam = s.camera
    cam.sampling = rt.SAMPLING["material"]
    with pytest.raises(ValueError):
        session.set_camera(cam)
    cam.sampling = rt.SAMPLING["mixture"]
    session.set_camera(cam)
    assert session.state() == 0
    assert session.counters()["rays"] == 0


def test_counting_build_counts_fetches(rt):
    s = rt.builtin_scene("weekend", width=128, spp=16)
    session = rt.Session(rt.Scene(s), seed=2)
    session.set_counting(True)
    session.render_to(16)
    counts = session.fetch_counts()
    rays = session.counters()["rays"]
    assert counts["nodes"] > rays  # every segment fetches at least the root
    assert counts["spheres"] > rays
    assert counts["quads"] == 0 and counts["triangles"] == 0


def test_env_furnace_is_exactly_one(rt):
    s = rt.builtin_scene("env-furnace", width=480, spp=64)
    r = rt.render(s, seed=5)
    assert np.all(r.pixels == 1.0), (r.pixels.min(), r.pixels.max())
    assert r.kernel["name"].endswith("nee-mis")


def test_ggx_furnace_keeps_the_light(rt):
    s = rt.builtin_scene("ggx-furnace", width=320, spp=256)
    r = rt.render(s, seed=6)
    h, w = s.height, s.width
    centre = r.pixels[h // 2 - 3:h // 2 + 3, w // 2 - 3:w // 2 + 3].mean(axis=2).ravel()
    se = centre.std(ddof=1) / np.sqrt(centre.size)
    assert abs(centre.mean() - 1.0) < 0.005 + 4 * se, (centre.mean(), se)


def test_mesh_first_hits_match_oracle(rt, oracle):
    s = rt.builtin_scene("mesh-ggx", width=320, spp=16, mesh_level=5, env_width=256)
    scene = rt.Scene(s)
    assert scene.stats()["triangles"] == 20 * 4 ** 5
    o, d = scene.camera_rays(seed=4, pass_index=3)
    ids, ts = scene.closest_hits(o, d)
    ref_ids, ref_ts = oracle.closest_hits(s.desc, o.astype(np.float64), d.astype(np.float64), brute_force=False)
    same = ids == ref_ids
    assert np.allclose(ts[same & (ids >= 0)], ref_ts[same & (ids >= 0)], rtol=2e-4, atol=1e-5)
    r = oracle.first_hit_mismatches(s.desc, o, d, ids, ref_ids, ts, ref_ts, tie_rel=1e-6)
    assert r["mismatches"] <= 1e-4 * r["rays"] and r["non_tie_mismatches"] == 0, r


def test_mesh_ggx_image_matches_oracle(rt, oracle):
    """The mesh workload reduced: the displaced icosphere (level 4), GGX metal, glossy-coat plane, the sun-lit sky
    sampled by its alias table, NEE with power-heuristic MIS."""
    r, g, cstats = _compare_with_rerun(rt, oracle, "mesh-ggx", 64, [(11, 12), (13, 14)], width=128, spp=64,
                                       mesh_level=4, env_width=256)
    assert g.shadow_rays > 0
    per_sample = g.pixels[..., 0].size * 64
    assert g.rays / per_sample == pytest.approx(cstats["rays"] / per_sample, rel=0.03)
