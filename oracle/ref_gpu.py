"""TEST INFRASTRUCTURE — ctypes binding of the reference's own CUDA renderer (oracle/_ref/libref_gpu.so, built from
the reference's src/gpu sources by oracle/build_ref.py).

A second, independent oracle: the reference itself, rendering the same scene tables on the same GPU. Tests use it for
image parity (ImageCompare between its render and this library's), for first-hit parity (its device closest_hit on
the same rays) and for the display transform's bytes (its display.cu / tonemap.cu kernels on the same sums); bench.py
reports its speed beside this library's on the same workload and checks the timed image against its render. The
product (raytracing_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIBRARY = Path(__file__).resolve().parent / "_ref" / "libref_gpu.so"


class RefResult(C.Structure):
    _fields_ = [("seconds", C.c_double), ("kernel_seconds", C.c_double), ("rays", C.c_uint64),
                ("shadow_rays", C.c_uint64), ("registers", C.c_int32), ("blocks_per_multiprocessor", C.c_int32),
                ("kernel", C.c_char * 32)]


_lib = None


def available() -> bool:
    return LIBRARY.exists()


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            raise RuntimeError(f"{LIBRARY} is missing: build it with `python oracle/build_ref.py` where the "
                               "reference's sources are")
        lib = C.CDLL(str(LIBRARY))
        lib.ref_gpu_render.restype = C.c_int
        lib.ref_gpu_render.argtypes = [C.c_void_p, C.c_uint64, C.c_int64, C.c_int32, C.c_int32,
                                       C.POINTER(C.c_double), C.c_int64, C.POINTER(RefResult), C.c_char_p, C.c_int32]
        lib.ref_gpu_closest_hits.restype = C.c_int
        lib.ref_gpu_closest_hits.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int64,
                                             C.POINTER(C.c_int32), C.POINTER(C.c_float), C.c_char_p, C.c_int32]
        lib.ref_gpu_display_bytes.restype = C.c_int
        lib.ref_gpu_display_bytes.argtypes = [C.POINTER(C.c_double), C.c_int32, C.c_int32, C.c_double, C.c_int32,
                                              C.c_double, C.POINTER(C.c_uint8), C.c_char_p, C.c_int32]
        _lib = lib
    return _lib


def render(desc, width: int, height: int, seed: int = 0, passes: int = 0, fp64: bool = False,
           all_books: bool = False) -> tuple[np.ndarray, dict]:
    """gpu::render (renderer.h:526) of the reference on a scene desc pointer: (pixels HxWx3, its render_result)."""
    lib = load()
    pixels = np.zeros((height, width, 3), dtype=np.float64)
    result = RefResult()
    error = C.create_string_buffer(512)
    status = lib.ref_gpu_render(C.cast(desc, C.c_void_p), seed, passes, 1 if fp64 else 0, 1 if all_books else 0,
                                pixels.ctypes.data_as(C.POINTER(C.c_double)), pixels.size, C.byref(result), error,
                                len(error))
    if status != 0:
        raise RuntimeError(error.value.decode("utf-8", "replace"))
    return pixels, {"seconds": result.seconds, "kernel_seconds": result.kernel_seconds, "rays": result.rays,
                    "shadow_rays": result.shadow_rays, "registers": result.registers,
                    "blocks_per_multiprocessor": result.blocks_per_multiprocessor,
                    "kernel": result.kernel.decode()}


def closest_hits(desc, origins: np.ndarray, directions: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """The reference's device closest_hit (src/gpu/bvh.cuh:576-706) over its own BVH, for float rays: (ids in source
    index space, -1 for a miss; t as float)."""
    lib = load()
    o = np.ascontiguousarray(origins, dtype=np.float32).reshape(-1, 3)
    d = np.ascontiguousarray(directions, dtype=np.float32).reshape(-1, 3)
    n = o.shape[0]
    ids = np.empty(n, dtype=np.int32)
    ts = np.empty(n, dtype=np.float32)
    error = C.create_string_buffer(512)
    status = lib.ref_gpu_closest_hits(C.cast(desc, C.c_void_p), o.ctypes.data_as(C.POINTER(C.c_float)),
                                      d.ctypes.data_as(C.POINTER(C.c_float)), n,
                                      ids.ctypes.data_as(C.POINTER(C.c_int32)),
                                      ts.ctypes.data_as(C.POINTER(C.c_float)), error, len(error))
    if status != 0:
        raise RuntimeError(error.value.decode("utf-8", "replace"))
    return ids, ts


TONE_MAPS = {"books": 0, "none": 1, "agx": 2, "neutral": 3}


def display_bytes(sums: np.ndarray, scale: float, tone: str = "books", exposure: float = 0.0) -> np.ndarray:
    """The reference's display transform (display.cu rgba8_kernel, tonemap.cu tone_map_kernel) of per-pixel sums
    (height x width x 3 doubles) times `scale`: height x width x 4 bytes."""
    lib = load()
    s = np.ascontiguousarray(sums, dtype=np.float64)
    h, w, _ = s.shape
    out = np.empty((h, w, 4), dtype=np.uint8)
    error = C.create_string_buffer(512)
    status = lib.ref_gpu_display_bytes(s.ctypes.data_as(C.POINTER(C.c_double)), w, h, scale, TONE_MAPS[tone],
                                       exposure, out.ctypes.data_as(C.POINTER(C.c_uint8)), error, len(error))
    if status != 0:
        raise RuntimeError(error.value.decode("utf-8", "replace"))
    return out
