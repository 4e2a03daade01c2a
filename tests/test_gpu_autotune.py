"""The wavefront autotuner on a B200: it picks a launch shape among its candidates by measuring renders of the
session's view, and a later session of the same scene class takes the remembered shape.

* The slot pool, the trace grid and the shade kernel's block size move no sample's arithmetic: the image is the same
  bit for bit (samples go to whichever slot claims them; each is computed and summed the same way).
* The trace kernel's register cap selects a separately compiled instantiation of the walk, which the compiler may
  schedule and contract differently: the image is the same to that rounding (as the wavefront and persistent forms
  are, tests/test_gpu_wavefront.py), and the same bit for bit again under the same shape.
* Per-kernel CUDA-event times account for the launches' GPU time.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KNOBS = ("slots", "trace_blocks_per_sm", "shade_block", "trace_min_blocks")


def _same_to_rounding(img, ref):
    close = np.isclose(img, ref, rtol=1e-4, atol=1e-5 * max(abs(ref.mean()), 1e-3))
    assert close.mean() >= 0.99, close.mean()
    assert abs(img.mean() - ref.mean()) <= 2e-4 * max(abs(ref.mean()), 1e-3), (img.mean(), ref.mean())


@pytest.mark.parametrize("name,kw", [("glass", dict(width=200, spp=16)), ("weekend", dict(width=200, spp=16))])
def test_autotune_picks_a_shape_and_is_remembered(rt, name, kw):
    s = rt.builtin_scene(name, **kw)
    scene = rt.Scene(s)
    plain = rt.Session(scene, seed=21, form="wavefront")
    default = plain.tuning()
    assert default["trials"] == 0
    plain.render_to(32)
    reference = plain.pixels()

    tuned = rt.Session(scene, seed=21, form="wavefront")
    t = tuned.autotune(trial_passes=16)
    assert t["trials"] >= 8
    assert t["slots"] in (1 << 19, 1 << 20, 3 << 19, 1 << 21, 3 << 20)
    assert t["shade_block"] in (64, 128) and t["trace_min_blocks"] in (6, 8)
    assert 1 <= t["trace_blocks_per_sm"] <= 16 and t["trace_registers"] > 0
    assert t["samples_per_second"] >= t["default_samples_per_second"] > 0
    assert tuned.state() == 0  # the view starts over after the trials
    tuned.render_to(32)
    if t["trace_min_blocks"] == default["trace_min_blocks"]:
        assert np.array_equal(tuned.pixels(), reference)
    else:
        _same_to_rounding(tuned.pixels(), reference)

    later = rt.Session(scene, seed=21, form="wavefront")
    c = later.tuning()
    assert c["from_cache"] == 1
    assert {k: c[k] for k in KNOBS} == {k: t[k] for k in KNOBS}
    later.render_to(16)
    with pytest.raises(rt.LogicError):
        later.autotune(16)  # a view with passes cannot be tuned


@pytest.mark.parametrize("name,kw", [("glass", dict(width=200, spp=16)), ("weekend", dict(width=200, spp=16)),
                                     ("mesh-ggx", dict(width=160, spp=16, mesh_level=5, env_width=256))])
def test_shapes_set_by_hand(rt, name, kw):
    s = rt.builtin_scene(name, **kw)
    scene = rt.Scene(s)
    base = rt.Session(scene, seed=5, form="wavefront")
    default = base.tuning()
    base.render_to(32)
    reference = base.pixels()
    # the pool, the grid and the block size: bit for bit
    for change in (dict(slots=1 << 19), dict(shade_block=64), dict(trace_blocks_per_sm=4)):
        sess = rt.Session(scene, seed=5, form="wavefront")
        shape = {k: default[k] for k in KNOBS}
        shape.update(change)
        sess.set_tuning(shape)
        assert {k: sess.tuning()[k] for k in KNOBS} == shape
        sess.render_to(32)
        assert np.array_equal(sess.pixels(), reference), change
    # the roomier register cap: the same to rounding, and reproducible under the same shape
    roomy = {k: default[k] for k in KNOBS}
    roomy.update(trace_min_blocks=6, trace_blocks_per_sm=4)
    images = []
    for _ in range(2):
        sess = rt.Session(scene, seed=5, form="wavefront")
        sess.set_tuning(roomy)
        sess.render_to(32)
        images.append(sess.pixels())
    assert np.array_equal(images[0], images[1])
    _same_to_rounding(images[0], reference)
    sess = rt.Session(scene, seed=5, form="wavefront")
    with pytest.raises(ValueError):
        sess.set_tuning(dict(slots=1000, trace_blocks_per_sm=4, shade_block=64, trace_min_blocks=6))
    with pytest.raises(ValueError):
        sess.set_tuning(dict(slots=1 << 20, trace_blocks_per_sm=64, shade_block=128, trace_min_blocks=8))


def test_kernel_times_add_up(rt):
    """Per-kernel CUDA-event timing: the kernels' times account for the launches' GPU time."""
    for form in ("wavefront", "persistent"):
        s = rt.builtin_scene("glass", width=160, spp=16)
        sess = rt.Session(rt.Scene(s), seed=2, form=form)
        sess.set_timing(True)
        rep = sess.render_to(64)
        kt = sess.kernel_times()
        total = sum(v[0] for v in kt.values())
        assert 0.7 * rep["gpu_seconds"] <= total <= 1.01 * rep["gpu_seconds"], (kt, rep)
        if form == "wavefront":
            assert kt["shade"][1] == kt["trace"][1] > 0 and kt["render"][1] == 0
        else:
            assert kt["render"][1] == rep["launches"] and kt["shade"][1] == 0
        assert kt["reduce"][1] == rep["launches"]
