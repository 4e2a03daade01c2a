"""The wavefront form against the persistent kernel on a B200, through the C-ABI.

A session in the wavefront form renders the samples the persistent kernel renders: the same work items, the same
random numbers, each sample's segments shaded by the same code in the same order, its shadow rays' light added before
its next vertex, its passes added into the item's partial in pass order. The trace kernel's search is the persistent
kernel's (the tree's leaf tests and self-intersection rules, four wide; or every primitive in turn for a flat scene),
so the hits are the same. The two forms are compiled as different kernels, so the compiler's fused multiply-adds may
round a few values differently.

Covered: spheres in a tree (books and NEE/MIS), the triangle mesh with GGX and the environment map's shadow rays,
the flat-searched Cornell boxes (books with the lights list, NEE/MIS with lamp shadow rays), and the second book's
textures, smoke (free flights, transmittance on shadow rays) and motion blur; more samples than slots (a slot renders
several samples in turn); many short launches; paths of one and two segments.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same_render(img, ref):
    """99% of the values equal to 1e-4 relative (1e-5 of the image's mean near black: a last-bit difference in a
    texture's noise or a hit point moves a dark pixel by more than its own 1e-4); the means within 2e-4 relative: the
    reach of the few samples whose path a different rounding sent elsewhere (through glass and smoke a last-bit
    difference can grow into another branch; one sample of a 16-pass pixel moves the mean of a 48 x 27 image by
    1e-5). A slip of the logic (a lost shadow ray, a sample counted twice or in another order) moves far more than 1%
    of the values."""
    close = np.isclose(img, ref, rtol=1e-4, atol=1e-5 * max(abs(ref.mean()), 1e-3))
    assert close.mean() >= 0.99, close.mean()
    assert abs(img.mean() - ref.mean()) <= 2e-4 * max(abs(ref.mean()), 1e-3), (img.mean(), ref.mean())


CASES = [
    ("weekend", dict(width=64, spp=16), 16),
    ("weekend", dict(width=48, spp=16, combination="mis"), 16),
    ("mesh-ggx", dict(width=64, spp=16, mesh_level=4, env_width=64), 16),
    ("cornell-mis", dict(width=48, spp=16), 16),
    ("glass", dict(width=48, spp=16), 16),
    ("final", dict(width=64, spp=16), 16),
    ("smoke", dict(width=48, spp=16, combination="mis"), 16),
    ("bouncing", dict(width=48, spp=16), 16),
    ("perlin", dict(width=48, spp=16), 8),
]


def _pair(rt, name, kw, passes, seed=5, launch_seconds=0.05):
    scene = rt.Scene(rt.builtin_scene(name, **kw))
    a = rt.Session(scene, seed=seed, form="persistent", launch_seconds=launch_seconds)
    a.render_to(passes)
    b = rt.Session(scene, seed=seed, form="wavefront", launch_seconds=launch_seconds)
    b.render_to(passes)
    return a, b


@pytest.mark.parametrize("name,kw,passes", CASES, ids=[f"{c[0]}-{c[1].get('combination', 'plain')}" for c in CASES])
def test_wavefront_equals_persistent(rt, name, kw, passes):
    a, b = _pair(rt, name, kw, passes)
    assert a.kernel()["name"].startswith("persistent")
    assert b.kernel()["name"].startswith("wavefront")
    _same_render(b.pixels(), a.pixels())
    # the same paths: their segment and shadow-ray counts agree but for the few paths a rounding sent elsewhere
    ca, cb = a.counters(), b.counters()
    assert abs(ca["rays"] - cb["rays"]) <= 1e-3 * ca["rays"], (ca, cb)
    assert abs(ca["shadow_rays"] - cb["shadow_rays"]) <= 1e-3 * max(ca["shadow_rays"], 100), (ca, cb)


def test_auto_form_follows_the_scene(rt):
    # the wavefront for a tree (weekend) and for a flat scene with lights (the glass Cornell box); the persistent
    # kernel for a bare flat scene (five quads under the sky)
    tree = rt.Session(rt.Scene(rt.builtin_scene("weekend", width=32, spp=1)), seed=1)
    lit = rt.Session(rt.Scene(rt.builtin_scene("glass", width=32, spp=1)), seed=1)
    bare = rt.Session(rt.Scene(rt.builtin_scene("quads", width=32, spp=1)), seed=1)
    assert tree.kernel()["name"].startswith("wavefront")
    assert lit.kernel()["name"].startswith("wavefront")
    assert bare.kernel()["name"].startswith("persistent")
    rep = lit.render_to(1)
    assert rep["kernel_launches"] >= 3 and rep["kernel_launches"] % 2 == 1  # shade and trace per step, the reduction


def test_more_items_than_slots(rt):
    # 1024 x 576 pixels, 16 passes: 9.4M samples for 2^20 slots, so slots take samples in turn
    a, b = _pair(rt, "weekend", dict(width=1024, spp=16), 16)
    _same_render(b.pixels(), a.pixels())


def test_many_short_launches(rt):
    # launches of a chunk each, the first a probe: every launch clears the slots and ends when its queue empties
    a, b = _pair(rt, "weekend", dict(width=40, spp=64), 64, launch_seconds=1e-4)
    _same_render(b.pixels(), a.pixels())
    assert b.counters()["rays"] > 0


@pytest.mark.parametrize("depth", [1, 2])
def test_short_paths(rt, depth):
    # paths cut at one or two segments: the last vertex's shadow ray still lands before the sample ends
    a, b = _pair(rt, "mesh-ggx", dict(width=48, spp=16, depth=depth, mesh_level=3, env_width=64), 16)
    _same_render(b.pixels(), a.pixels())
