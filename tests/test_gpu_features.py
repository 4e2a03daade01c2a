"""The second book's features on a B200, through the C-ABI: textures (checker, image, marble), moving spheres (motion
blur) and volumes of smoke (constant media with isotropic scattering), in both integrators.

* feature-furnace: a moving checker sphere, an image-textured quad and two volumes of white smoke in the white
  furnace; every pixel is exactly 1 (every bounce and scattering keeps all of the light), in the books' kernel and in
  the NEE/MIS kernel.
* ImageCompare against the CPU oracle (the reference's CPU estimator restated, double) for the reference's scenes
  that use them: bouncing, checker, earth, perlin, light, smoke, final, aluminum; the smoke and light scenes also under
  NEE with MIS (shadow rays through smoke weighted by its transmittance, shadow.cuh:129-165). Independent seeds, one
  re-run on a chance alarm.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("combination", [None, "mis"])
def test_feature_furnace_is_exactly_one(rt, combination):
    kw = {"combination": combination} if combination else {}
    s = rt.builtin_scene("feature-furnace", width=160, spp=64, **kw)
    r = rt.render(s, seed=9)
    assert np.all(r.pixels == 1.0), (r.pixels.min(), r.pixels.max())
    assert r.rays > 1.05 * s.width * s.height * 64


CASES = [
    ("bouncing", dict(width=96, spp=16), 16),
    ("checker", dict(width=96, spp=16), 16),
    ("earth", dict(width=96, spp=16, env_width=128), 16),
    ("perlin", dict(width=96, spp=16), 16),
    ("light", dict(width=96, spp=64), 64),
    ("smoke", dict(width=64, spp=64), 64),
    ("final", dict(width=64, spp=16, env_width=128), 16),
    ("aluminum", dict(width=64, spp=64), 64),
    ("smoke", dict(width=64, spp=64, combination="mis"), 64),
    ("light", dict(width=96, spp=64, combination="mis"), 64),
]


@pytest.mark.parametrize("name,kw,passes", CASES)
def test_features_match_oracle(rt, oracle, name, kw, passes):
    s = rt.builtin_scene(name, **kw)
    reports = []
    for gpu_seed, cpu_seed in ((41, 42), (43, 44)):
        g = rt.render(s, seed=gpu_seed, passes=passes)
        c, _ = oracle.render(s.desc, s.width, s.height, seed=cpu_seed, passes=passes)
        r = oracle.image_compare(c, g.pixels)
        reports.append(r)
        if r["verdict"] == 0:
            return
    raise AssertionError(f"{name} {kw}: ImageCompare failed twice: {reports}")


def test_motion_blurs(rt):
    """The bouncing spheres move while the shutter is open: the image differs from the same scene held still."""
    moving = rt.builtin_scene("bouncing", width=96, spp=16)
    still = rt.builtin_scene("bouncing", width=96, spp=16)
    d = still.desc.contents
    for i in range(d.sphere_count):
        d.spheres[i].displacement.x = d.spheres[i].displacement.y = d.spheres[i].displacement.z = 0.0
    a = rt.render(moving, seed=3, passes=16).pixels
    b = rt.render(still, seed=3, passes=16).pixels
    assert np.abs(a - b).mean() > 1e-3
