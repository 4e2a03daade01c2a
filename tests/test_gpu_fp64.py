"""The books' integrator in double (precision::float64, renderer.h:402-409) on a B200, through the C-ABI.

The reference renders its books' scenes in double as a mode to compare with (all_books_kernel<double>, renderer.cu:
445-451), and the cover scene's workload asks for FP32 and FP64 renders against the CPU renderer. Here:

* the white furnace is exactly 1.0 in every pixel in double too (furnace: docs/image-compare.md:145);
* ImageCompare finds the double render consistent with the CPU oracle (the CPU renderer in double) on the cover scene
  at its workload's size (400 x 225, 32 passes, depth 50), on the glass Cornell box under the mixture, and on the
  second book's scenes (moving spheres, checker, image and marble textures, smoke, the final scene);
* and consistent with the reference's own float64 render (its renderer built from its sources, fp64 mode);
* the double image of N passes is the same bit for bit however its passes are grouped into launches;
* what the reference computes in float only is refused in float64 with its error class: the quality kernel's scenes,
  triangle meshes, and a tone map other than the books' bytes (renderer.cu:1203-1220, 2047-2078).

Independent seeds; a failure is re-run once with fresh seeds (the reference's re-run rule).
"""
import numpy as np
import pytest

from oracle import ref_gpu

pytestmark = pytest.mark.gpu

needs_reference = pytest.mark.skipif(not ref_gpu.available(), reason="the reference's renderer was not built here")


def _consistent(oracle, a_fn, b_fn, seeds):
    reports = []
    for sa, sb in seeds:
        r = oracle.image_compare(a_fn(sa), b_fn(sb))
        reports.append({k: r[k] for k in ("verdict", "whole_image_z", "all_tiles_z", "largest_tile_z",
                                           "tiles_over_3", "tested_tiles")})
        if r["verdict"] == 0:
            return r
    raise AssertionError(f"ImageCompare failed twice: {reports}")


def test_furnace_is_exactly_one_in_double(rt):
    s = rt.builtin_scene("furnace", width=96, spp=16)
    r = rt.render(s, seed=3, arithmetic="float64")
    assert np.all(r.pixels == 1.0), (r.pixels.min(), r.pixels.max())
    assert r.kernel["name"] == "persistent books fp64"
    assert r.rays > 0


def test_cover_scene_in_double_matches_oracle(rt, oracle):
    """The cover scene's workload (400 x 225, 32 passes of 4 x 4 strata, depth 50), FP64 against the CPU renderer."""
    s = rt.builtin_scene("weekend", width=400, spp=16, depth=50)
    assert (s.width, s.height) == (400, 225)
    ours = lambda seed: rt.render(s, seed=seed, passes=32, arithmetic="float64").pixels  # noqa: E731
    cpu = lambda seed: oracle.render(s.desc, s.width, s.height, seed=seed, passes=32)[0]  # noqa: E731
    _consistent(oracle, cpu, ours, [(21, 22), (23, 24)])


@needs_reference
def test_cover_scene_in_double_matches_reference_double(rt, oracle):
    s = rt.builtin_scene("weekend", width=400, spp=16, depth=50)
    ours = lambda seed: rt.render(s, seed=seed, passes=32, arithmetic="float64").pixels  # noqa: E731
    ref = lambda seed: ref_gpu.render(s.desc, s.width, s.height, seed=seed, passes=32, fp64=True)[0]  # noqa: E731
    _consistent(oracle, ref, ours, [(25, 26), (27, 28)])


@needs_reference
def test_glass_in_double_matches_reference_double(rt, oracle):
    s = rt.builtin_scene("glass", width=128, spp=64)
    ours = lambda seed: rt.render(s, seed=seed, arithmetic="float64").pixels  # noqa: E731
    ref = lambda seed: ref_gpu.render(s.desc, s.width, s.height, seed=seed, fp64=True)[0]  # noqa: E731
    _consistent(oracle, ref, ours, [(29, 30), (31, 32)])


CASES = [
    ("glass", dict(width=128, spp=64), 64),
    ("materials", dict(width=96, spp=16), 16),
    ("quads", dict(width=96, spp=16), 16),
    ("bouncing", dict(width=96, spp=16), 16),
    ("checker", dict(width=96, spp=16), 16),
    ("earth", dict(width=96, spp=16, env_width=128), 16),
    ("perlin", dict(width=96, spp=16), 16),
    ("smoke", dict(width=64, spp=64), 64),
    ("final", dict(width=64, spp=16, env_width=128), 16),
]


@pytest.mark.parametrize("name,kw,passes", CASES)
def test_books_scenes_in_double_match_oracle(rt, oracle, name, kw, passes):
    s = rt.builtin_scene(name, **kw)
    ours = lambda seed: rt.render(s, seed=seed, passes=passes, arithmetic="float64").pixels  # noqa: E731
    cpu = lambda seed: oracle.render(s.desc, s.width, s.height, seed=seed, passes=passes)[0]  # noqa: E731
    _consistent(oracle, cpu, ours, [(41, 42), (43, 44)])


def test_double_and_float_agree(rt, oracle):
    """The same estimator in both precisions: the double image is consistent with the float image."""
    s = rt.builtin_scene("weekend", width=200, spp=16)
    f64 = lambda seed: rt.render(s, seed=seed, passes=32, arithmetic="float64").pixels  # noqa: E731
    f32 = lambda seed: rt.render(s, seed=seed, passes=32).pixels  # noqa: E731
    _consistent(oracle, f64, f32, [(51, 52), (53, 54)])


def test_double_grouping_of_passes_does_not_change_the_image(rt):
    s = rt.builtin_scene("bouncing", width=64, spp=8)
    scene = rt.Scene(s)
    one = rt.Session(scene, seed=5, arithmetic="float64")
    one.render_to(64)
    many = rt.Session(scene, seed=5, arithmetic="float64")
    for target in (16, 32, 48, 64):
        many.render_to(target)
    assert np.array_equal(one.pixels(), many.pixels())
    assert one.kernel()["name"] == "persistent books fp64"
    assert one.counters()["rays"] == many.counters()["rays"]
    again = rt.render(s, seed=5, passes=64, arithmetic="float64")
    assert np.array_equal(again.pixels, one.pixels())


def test_double_display_takes_the_books_bytes_only(rt):
    s = rt.builtin_scene("glass", width=48, spp=4)
    scene = rt.Scene(s)
    session = rt.Session(scene, seed=1, arithmetic="float64")
    session.render_to(16)
    rgba = session.display("books")
    assert rgba.shape == (48, 48, 4) and np.all(rgba[..., 3] == 255)
    with pytest.raises(ValueError, match="float only"):
        session.display("agx", exposure=0.0)
    with pytest.raises(rt.LogicError):
        session.set_counting(True)


def test_what_computes_in_float_only_is_refused_in_double(rt):
    quality = rt.Scene(rt.builtin_scene("cornell-mis", width=32, spp=4))
    with pytest.raises(ValueError, match="quality kernel computes in float only"):
        rt.Session(quality, arithmetic="float64")
    mesh = rt.Scene(rt.builtin_scene("mesh-ggx", width=32, spp=4, mesh_level=2))
    with pytest.raises(ValueError):
        rt.Session(mesh, arithmetic="float64")
    books = rt.Scene(rt.builtin_scene("weekend", width=32, spp=4))
    with pytest.raises(ValueError, match="wavefront"):
        rt.Session(books, arithmetic="float64", form="wavefront")
