"""The wavefront autotuner on a B200: it picks a launch shape among its candidates by measuring short renders of the
session's view, the image does not depend on the shape (bit for bit), and a later session of the same scene class
takes the remembered shape."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,kw", [("glass", dict(width=200, spp=16)), ("weekend", dict(width=200, spp=16))])
def test_autotune_keeps_the_image_and_is_remembered(rt, name, kw):
    s = rt.builtin_scene(name, **kw)
    scene = rt.Scene(s)
    plain = rt.Session(scene, seed=21, form="wavefront")
    before = plain.tuning()
    plain.render_to(32)
    reference = plain.pixels()

    tuned = rt.Session(scene, seed=21, form="wavefront")
    t = tuned.autotune(trial_passes=16)
    assert t["trials"] >= 8
    assert t["slots"] in (1 << 19, 1 << 20, 3 << 19, 1 << 21, 3 << 20)
    assert t["shade_block"] in (64, 128) and t["trace_min_blocks"] in (6, 8) and t["shade_sort"] in (0, 1)
    assert 1 <= t["trace_blocks_per_sm"] <= 16 and t["trace_registers"] > 0
    assert t["samples_per_second"] >= t["default_samples_per_second"] > 0
    assert tuned.state() == 0  # the view starts over after the trials
    tuned.render_to(32)
    assert np.array_equal(tuned.pixels(), reference)
    assert before["trials"] == 0

    # a shape set by hand gives the same image too
    manual = rt.Session(scene, seed=21, form="wavefront")
    manual.set_tuning(dict(slots=1 << 19, trace_blocks_per_sm=4, shade_block=64, trace_min_blocks=6, shade_sort=1))
    assert manual.tuning()["slots"] == 1 << 19 and manual.tuning()["shade_sort"] == 1
    manual.render_to(32)
    assert np.array_equal(manual.pixels(), reference)
    with pytest.raises(ValueError):
        manual.set_tuning(dict(slots=1000, trace_blocks_per_sm=4, shade_block=64, trace_min_blocks=6, shade_sort=1))

    later = rt.Session(scene, seed=21, form="wavefront")
    c = later.tuning()
    assert c["from_cache"] == 1
    assert {k: c[k] for k in ("slots", "trace_blocks_per_sm", "shade_block", "trace_min_blocks", "shade_sort")} == \
        {k: t[k] for k in ("slots", "trace_blocks_per_sm", "shade_block", "trace_min_blocks", "shade_sort")}
    with pytest.raises(rt.LogicError):
        later.render_to(16)
        later.autotune(16)  # a view with passes cannot be tuned


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
