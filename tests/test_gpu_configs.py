"""Parity at the sizes of the workloads themselves, on a B200, through the C-ABI.

* The first book's cover scene at 400 x 225, 32 passes (two rounds of 4 x 4 strata), depth 50: ImageCompare against
  the oracle (src/camera.ixx's CPU renderer in double) and against the reference's own CUDA renderer.
* The Cornell box with a glass ball at 600 x 600, 1024 spp, depth 50: under the mixture of light and cosine sampling
  against the CPU oracle and the reference's all-books kernel, and under NEE with power-heuristic MIS against the
  reference's quality kernel (src/gpu/quality.cu), the image the benchmark times.
* The displaced icosphere of 1,310,720 triangles (level 8) with GGX metal, the glossy-coat plane and the sun-lit
  environment: first hits of all 1920 x 1080 primary rays against the oracle's double BVH search, and ImageCompare of
  a reduced image (480 x 270, 64 spp) against the oracle.
* First hits three ways on the same float camera rays: this library's kernel, the reference's own device closest_hit
  (src/gpu/bvh.cuh:576-706) over the reference's BVH, and the oracle's double brute force. At least 99.99% of the ids
  agree, and every disagreement is a hit-distance tie within 1e-6 relative (another primitive hit at the same t: the
  reference's tracer-check class `ties`, tests/tracer_check_layout.h).

ImageCompare runs with independent seeds; a failure is re-run once with fresh seeds (the reference's re-run rule), so
a chance alarm does not fail the suite.
"""
import numpy as np
import pytest

from oracle import ref_gpu

pytestmark = pytest.mark.gpu

needs_reference = pytest.mark.skipif(not ref_gpu.available(), reason="the reference's renderer was not built here")

TIE_REL = 1e-6


def _consistent(oracle, a_fn, b_fn, seeds):
    reports = []
    for sa, sb in seeds:
        r = oracle.image_compare(a_fn(sa), b_fn(sb))
        reports.append({k: r[k] for k in ("verdict", "whole_image_z", "all_tiles_z", "largest_tile_z",
                                           "tiles_over_3", "tested_tiles")})
        if r["verdict"] == 0:
            return r
    raise AssertionError(f"ImageCompare failed twice: {reports}")


def _assert_first_hits(oracle, desc, o, d, ids, ref_ids, ts=None, ref_ts=None):
    r = oracle.first_hit_mismatches(desc, o, d, ids, ref_ids, ts, ref_ts, tie_rel=TIE_REL)
    assert r["mismatches"] <= 1e-4 * r["rays"], r
    assert r["non_tie_mismatches"] == 0, r
    return r


def test_cover_scene_at_config_size_matches_oracle(rt, oracle):
    s = rt.builtin_scene("weekend", width=400, spp=16, depth=50)
    assert (s.width, s.height) == (400, 225) and s.camera.sqrt_spp == 4
    ours = lambda seed: rt.render(s, seed=seed, passes=32).pixels  # noqa: E731
    cpu = lambda seed: oracle.render(s.desc, s.width, s.height, seed=seed, passes=32)[0]  # noqa: E731
    _consistent(oracle, cpu, ours, [(1, 2), (3, 4)])


@needs_reference
def test_cover_scene_at_config_size_matches_reference(rt, oracle):
    s = rt.builtin_scene("weekend", width=400, spp=16, depth=50)
    ours = lambda seed: rt.render(s, seed=seed, passes=32).pixels  # noqa: E731
    ref = lambda seed: ref_gpu.render(s.desc, s.width, s.height, seed=seed, passes=32)[0]  # noqa: E731
    _consistent(oracle, ref, ours, [(5, 6), (7, 8)])


def test_glass_at_config_size_matches_oracle(rt, oracle):
    """The benchmark's workload, mixture sampling, against the CPU oracle at its full size (about 10^9 segments on
    the host's cores)."""
    s = rt.builtin_scene("glass", width=600, spp=1024, depth=50)
    assert (s.width, s.height, s.round_passes) == (600, 600, 1024)
    ours = lambda seed: rt.render(s, seed=seed, launch_seconds=0.5).pixels  # noqa: E731
    cpu = lambda seed: oracle.render(s.desc, s.width, s.height, seed=seed)[0]  # noqa: E731
    _consistent(oracle, cpu, ours, [(9, 10), (11, 12)])


@needs_reference
@pytest.mark.parametrize("name", ["glass", "cornell-mis"])
def test_glass_at_config_size_matches_reference(rt, oracle, name):
    """Mixture sampling against the reference's all-books kernel, NEE+MIS against its quality kernel: same scene
    tables, same spp, independent seeds."""
    s = rt.builtin_scene(name, width=600, spp=1024, depth=50)
    ours = lambda seed: rt.render(s, seed=seed, launch_seconds=0.5).pixels  # noqa: E731
    ref = lambda seed: ref_gpu.render(s.desc, s.width, s.height, seed=seed)[0]  # noqa: E731
    _consistent(oracle, ref, ours, [(13, 14), (15, 16)])


def test_mesh_first_hits_at_config_size_match_oracle(rt, oracle):
    """All primary rays of the 1920 x 1080 mesh view (level 8: 1,310,720 triangles) against the oracle's double BVH."""
    s = rt.builtin_scene("mesh-ggx")
    scene = rt.Scene(s)
    assert scene.stats()["triangles"] == 1_310_720
    assert (s.width, s.height) == (1920, 1080)
    o, d = scene.camera_rays(seed=4, pass_index=3)
    ids, ts = scene.closest_hits(o, d)
    ref_ids, ref_ts = oracle.closest_hits(s.desc, o.astype(np.float64), d.astype(np.float64), brute_force=False)
    assert np.count_nonzero(ids >= 0) > 0.3 * ids.size
    same = (ids == ref_ids) & (ids >= 0)
    assert np.allclose(ts[same], ref_ts[same], rtol=2e-4, atol=1e-5)
    _assert_first_hits(oracle, s.desc, o, d, ids, ref_ids, ts, ref_ts)


def test_mesh_image_at_level_8_matches_oracle(rt, oracle):
    """The mesh workload's scene itself (level 8, the 1024 x 512 environment) at a reduced image: 480 x 270, 64 spp,
    depth 16, NEE with MIS."""
    s = rt.builtin_scene("mesh-ggx", width=480, spp=64)
    assert (s.width, s.height) == (480, 270) and s.camera.max_depth == 16
    ours = lambda seed: rt.render(s, seed=seed).pixels  # noqa: E731
    cpu = lambda seed: oracle.render(s.desc, s.width, s.height, seed=seed)[0]  # noqa: E731
    _consistent(oracle, cpu, ours, [(17, 18), (19, 20)])


@needs_reference
@pytest.mark.parametrize("name,width", [("weekend", 400), ("glass", 300), ("cornell", 300), ("materials", 320),
                                        ("quads", 256), ("final", 200), ("bouncing", 200)])
def test_first_hits_three_ways(rt, oracle, name, width):
    """This library's kernel, the reference's device closest_hit and the oracle's double brute force, on the same
    float camera rays (two passes' rays: jittered and on the lens)."""
    s = rt.builtin_scene(name, width=width, spp=16)
    scene = rt.Scene(s)
    for p in (0, 5):
        o, d = scene.camera_rays(seed=3, pass_index=p)
        ids, ts = scene.closest_hits(o, d)
        ref_ids, ref_ts = ref_gpu.closest_hits(s.desc, o, d)
        cpu_ids, cpu_ts = oracle.closest_hits(s.desc, o.astype(np.float64), d.astype(np.float64), brute_force=True)
        _assert_first_hits(oracle, s.desc, o, d, ids, ref_ids, ts, ref_ts)
        _assert_first_hits(oracle, s.desc, o, d, ids, cpu_ids, ts, cpu_ts)
        _assert_first_hits(oracle, s.desc, o, d, ref_ids, cpu_ids, ref_ts, cpu_ts)


@needs_reference
def test_error_against_the_fp64_oracle_matches_the_references(rt):
    """The glass box at its full size, 1024 spp: this library's image and the reference renderer's (same spp and
    strategy) have the same error against the FP64 65,536-spp oracle render (tests/golden/fp64_glass.npz, made by the
    reference's own renderer in double): PfmStats' trimmed RMS (tests/pfm_stats.cpp:344-367) within 5%."""
    from pathlib import Path

    z = np.load(Path(__file__).resolve().parent / "golden" / "fp64_glass.npz")
    truth = z["image"].astype(np.float64)
    s = rt.builtin_scene("glass", width=600, spp=1024, depth=50)

    def trimmed(img):
        d = img.mean(axis=2) - truth.mean(axis=2)
        d2 = np.sort((d * d).ravel())
        return float(np.sqrt(d2[: d2.size - int(d2.size * 0.01)].mean()))

    ours = trimmed(rt.render(s, seed=31, launch_seconds=0.5).pixels)
    ref = trimmed(ref_gpu.render(s.desc, s.width, s.height, seed=32)[0])
    assert abs(ours / ref - 1.0) <= 0.05, (ours, ref)
