"""The drop-in, end to end on a B200: the reference's own gpu:: API (src/gpu/renderer.h, unchanged), served by this
library through the shim INTEGRATION.md documents (built from that document into oracle/_ref/librenderer_b200.so by
oracle/build_ref.py), renders what the C-ABI renders, bit for bit: gpu::render's pixels and rays, a tone map's bytes,
and a gpu::session's pixels() and display()."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

SHIM = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "librenderer_b200.so"

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not SHIM.exists(), reason="the shim was not built here")]


def _lib():
    lib = C.CDLL(str(SHIM))
    lib.shim_render.restype = C.c_int
    lib.shim_render.argtypes = [C.c_void_p, C.c_uint64, C.c_int64, C.c_int32, C.c_double, C.POINTER(C.c_double),
                                C.POINTER(C.c_uint8), C.POINTER(C.c_uint64), C.c_char_p, C.c_int32]
    lib.shim_session.restype = C.c_int
    lib.shim_session.argtypes = [C.c_void_p, C.c_uint64, C.c_int64, C.c_int32, C.c_double, C.POINTER(C.c_double),
                                 C.POINTER(C.c_uint8), C.c_char_p, C.c_int32]
    return lib


@pytest.mark.parametrize("name,kw", [("glass", dict(width=96, spp=16)), ("cornell-mis", dict(width=64, spp=16)),
                                     ("final", dict(width=64, spp=4, env_width=64))])
def test_reference_render_through_the_shim_equals_the_c_abi(rt, name, kw):
    s = rt.builtin_scene(name, **kw)
    lib = _lib()
    pixels = np.zeros((s.height, s.width, 3))
    rays = C.c_uint64()
    err = C.create_string_buffer(512)
    status = lib.shim_render(C.cast(s.desc, C.c_void_p), 7, 32, 0, 0.0, pixels.ctypes.data_as(C.POINTER(C.c_double)),
                             None, C.byref(rays), err, 512)
    assert status == 0, err.value
    ours = rt.render(s, seed=7, passes=32)
    assert np.array_equal(pixels, ours.pixels)
    assert rays.value == ours.rays


def test_reference_session_and_tone_map_through_the_shim(rt):
    s = rt.builtin_scene("glass", width=80, spp=16)
    lib = _lib()
    err = C.create_string_buffer(512)
    pixels = np.zeros((s.height, s.width, 3))
    rgba = np.zeros((s.height, s.width, 4), dtype=np.uint8)
    rays = C.c_uint64()
    assert lib.shim_render(C.cast(s.desc, C.c_void_p), 3, 16, 2, -1.0, pixels.ctypes.data_as(C.POINTER(C.c_double)),
                           rgba.ctypes.data_as(C.POINTER(C.c_uint8)), C.byref(rays), err, 512) == 0, err.value
    session = rt.Session(rt.Scene(s), seed=3)
    session.render_to(16)
    assert np.array_equal(pixels, session.pixels())
    assert np.array_equal(rgba, session.display("agx", -1.0))

    p2 = np.zeros_like(pixels)
    b2 = np.zeros_like(rgba)
    assert lib.shim_session(C.cast(s.desc, C.c_void_p), 3, 16, 0, 0.0, p2.ctypes.data_as(C.POINTER(C.c_double)),
                            b2.ctypes.data_as(C.POINTER(C.c_uint8)), err, 512) == 0, err.value
    assert np.array_equal(p2, pixels)
    assert np.array_equal(b2, session.display())


def test_reference_float64_render_through_the_shim_equals_the_c_abi(rt):
    """precision::float64 through the reference's gpu::render reaches this library's FP64 integrator; a quality scene
    in float64 is refused there with the reference's error class (std::invalid_argument)."""
    s = rt.builtin_scene("bouncing", width=64, spp=4)
    lib = _lib()
    lib.shim_render_precision.restype = C.c_int
    lib.shim_render_precision.argtypes = [C.c_void_p, C.c_uint64, C.c_int64, C.c_int32, C.POINTER(C.c_double),
                                          C.POINTER(C.c_uint64), C.c_char_p, C.c_int32]
    pixels = np.zeros((s.height, s.width, 3))
    rays = C.c_uint64()
    err = C.create_string_buffer(512)
    assert lib.shim_render_precision(C.cast(s.desc, C.c_void_p), 11, 32, 1, pixels.ctypes.data_as(
        C.POINTER(C.c_double)), C.byref(rays), err, 512) == 0, err.value
    ours = rt.render(s, seed=11, passes=32, arithmetic="float64")
    assert ours.kernel["name"] == "persistent books fp64"
    assert np.array_equal(pixels, ours.pixels)
    assert rays.value == ours.rays

    q = rt.builtin_scene("cornell-mis", width=32, spp=4)
    p2 = np.zeros((q.height, q.width, 3))
    assert lib.shim_render_precision(C.cast(q.desc, C.c_void_p), 1, 4, 1, p2.ctypes.data_as(C.POINTER(C.c_double)),
                                     C.byref(rays), err, 512) == 1
    assert b"float only" in err.value
