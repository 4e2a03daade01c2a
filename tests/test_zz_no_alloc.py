"""rt_render_passes_no_alloc: the render kernel with its scratch in a fixed array of the library's device image, for
callers that cannot call cudaMalloc (a program that owns all of its device memory through its own pool, or a thread
that must not block on the allocator). Its output, two calls in a row accumulating into one caller-owned device
buffer, must equal what a session renders with the same seed and passes.

Collected last (test_zz_...), so a run that stops at the first failure has run everything else before it; it also
passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_buffer(n):
    import torch

    return torch.zeros(n, dtype=torch.float64, device="cuda")


def test_no_alloc_matches_session_on_two_calls_in_a_row(rt):
    import torch

    from raytracing_b200 import _abi

    lib = _abi.load()
    rt.set_device(0)
    desc = rt.builtin_scene("glass", width=160, spp=16)
    scene = rt.Scene(desc)
    w, h = scene.width, scene.height
    camera = desc.camera
    seed = 77

    # The existing entry point: a session rendered to 48, then 96 passes, in the persistent form (the no-allocation
    # render runs the same persistent kernel; a session would take the wavefront for this scene by default)
    session = rt.Session(scene, seed=seed, form="persistent")
    session.render_to(48)
    expected_48 = session.pixels().copy()
    session.render_to(96)
    expected_96 = session.pixels().copy()

    sums = _device_buffer(h * w * 3)
    rays = C.c_uint64()
    shadow = C.c_uint64()
    for begin, end, expected in ((0, 48, expected_48), (48, 96, expected_96)):
        status = lib.rt_render_passes_no_alloc(scene._handle, C.byref(camera), seed, begin, end,
                                               C.c_void_p(sums.data_ptr()), C.byref(rays), C.byref(shadow))
        assert status == 0, lib.rt_last_error_message()
        torch.cuda.synchronize()
        got = sums.cpu().numpy().reshape(h, w, 3) / end
        assert rays.value > 0
        # The same kernels over the same chunks: equal within the tolerance the parity tests use for regrouped
        # sums (they are in fact bit for bit equal)
        np.testing.assert_allclose(got, expected, rtol=1e-12, atol=1e-15)


def test_no_alloc_splits_a_call_into_launches_that_fit_its_scratch(rt):
    """An image whose padded pixels nearly fill the scratch (1920 x 1400: 2,688,000 of 2,796,192 entries) takes one
    16-pass chunk a launch, so passes 0-48 are three render+reduce launches in one call; the sums and the ray counts
    equal a persistent-form session's of the same seed and passes."""
    import torch

    from raytracing_b200 import _abi

    lib = _abi.load()
    rt.set_device(0)
    desc = rt.builtin_scene("cornell", width=1920, height=1400, spp=1)
    scene = rt.Scene(desc)
    w, h = scene.width, scene.height
    assert (w, h) == (1920, 1400)
    session = rt.Session(scene, seed=5, form="persistent")
    session.render_to(48)
    expected = session.pixels()
    expected_rays = session.counters()["rays"]
    sums = _device_buffer(h * w * 3)
    rays = C.c_uint64()
    status = lib.rt_render_passes_no_alloc(scene._handle, C.byref(desc.camera), 5, 0, 48, C.c_void_p(sums.data_ptr()),
                                           C.byref(rays), None)
    assert status == 0, lib.rt_last_error_message()
    torch.cuda.synchronize()
    got = sums.cpu().numpy().reshape(h, w, 3) / 48
    np.testing.assert_allclose(got, expected, rtol=1e-12, atol=1e-15)
    assert rays.value == expected_rays


def test_no_alloc_refuses_images_beyond_its_scratch(rt):
    from raytracing_b200 import _abi

    lib = _abi.load()
    desc = rt.builtin_scene("cornell", width=64, spp=4)
    scene = rt.Scene(desc)
    camera = desc.camera
    camera.image_width = 4096
    camera.image_height = 4096
    sums = _device_buffer(16)
    status = lib.rt_render_passes_no_alloc(scene._handle, C.byref(camera), 1, 0, 4, C.c_void_p(sums.data_ptr()),
                                           None, None)
    assert status == _abi.RT_ERR_CAPACITY
    assert b"no-allocation scratch" in lib.rt_last_error_message()
