"""TEST INFRASTRUCTURE — ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module, as the checker and the CPU
baseline; the product (raytracing_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
LIBRARY = ORACLE_DIR / "_build" / "liboracle.so"


class OracleStats(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("seconds", C.c_double),
                ("threads", C.c_int32), ("rows_rendered", C.c_int32)]


class CompareResult(C.Structure):
    _fields_ = [("verdict", C.c_int), ("mean_a", C.c_double), ("mean_b", C.c_double),
                ("channel_mean", C.c_double * 4), ("channel_se", C.c_double * 4), ("channel_z", C.c_double * 4),
                ("channel_level", C.c_double * 4), ("channel_rms", C.c_double * 4),
                ("whole_image_z", C.c_double), ("all_tiles_z", C.c_double), ("largest_tile_z", C.c_double),
                ("tiles_over_3", C.c_int), ("tested_tiles", C.c_int), ("identical_tiles", C.c_int),
                ("threshold_whole_image", C.c_double), ("threshold_all_tiles", C.c_double),
                ("threshold_largest_tile", C.c_double), ("threshold_tiles_over_3", C.c_int),
                ("failed_whole_image", C.c_int), ("failed_all_tiles", C.c_int), ("failed_largest_tile", C.c_int),
                ("failed_tile_count", C.c_int), ("sign_b_brighter", C.c_int64), ("sign_a_brighter", C.c_int64),
                ("sign_z", C.c_double), ("noise_shapes_differ", C.c_int), ("non_finite", C.c_int),
                ("largest_tile_x0", C.c_int), ("largest_tile_y0", C.c_int)]


_lib = None


def build() -> Path:
    """Compiles the oracle (make -C oracle) if its sources changed."""
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)
    return LIBRARY


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            build()
        lib = C.CDLL(str(LIBRARY))
        lib.oracle_last_error.restype = C.c_char_p
        lib.oracle_render.restype = C.c_int
        lib.oracle_render.argtypes = [C.c_void_p, C.c_uint64, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                                      C.POINTER(C.c_double), C.POINTER(OracleStats)]
        lib.oracle_closest_hits.restype = C.c_int
        lib.oracle_closest_hits.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int64,
                                            C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
        lib.oracle_hit_distances.restype = C.c_int
        lib.oracle_hit_distances.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int64,
                                             C.POINTER(C.c_int32), C.c_double, C.POINTER(C.c_double)]
        lib.oracle_image_compare.restype = C.c_int
        lib.oracle_image_compare.argtypes = [C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int32, C.c_int32,
                                             C.c_int32, C.POINTER(CompareResult)]
        lib.oracle_thresholds.restype = C.c_int
        lib.oracle_thresholds.argtypes = [C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                          C.POINTER(C.c_double), C.POINTER(C.c_int32)]
        lib.oracle_sizeof_compare_result.restype = C.c_int32
        if lib.oracle_sizeof_compare_result() != C.sizeof(CompareResult):
            raise RuntimeError("oracle compare_result layout mismatch")
        _lib = lib
    return _lib


def _desc_pointer(desc) -> C.c_void_p:
    return C.cast(desc, C.c_void_p)


def render(desc, width: int, height: int, seed: int = 0, passes: int = 0, threads: int = 0, row_begin: int = 0,
           row_end: int = 0) -> tuple[np.ndarray, dict]:
    """The CPU renderer (camera.ixx render) on a scene desc pointer; returns (pixels HxWx3, stats)."""
    lib = load()
    pixels = np.zeros((height, width, 3), dtype=np.float64)
    stats = OracleStats()
    status = lib.oracle_render(_desc_pointer(desc), seed, passes, threads, row_begin, row_end,
                               pixels.ctypes.data_as(C.POINTER(C.c_double)), C.byref(stats))
    if status != 0:
        raise RuntimeError(lib.oracle_last_error().decode())
    return pixels, {"rays": stats.rays, "shadow_rays": stats.shadow_rays, "seconds": stats.seconds,
                    "threads": stats.threads, "rows": stats.rows_rendered}


def closest_hits(desc, origins: np.ndarray, directions: np.ndarray, brute_force: bool = True):
    lib = load()
    o = np.ascontiguousarray(origins, dtype=np.float64).reshape(-1, 3)
    d = np.ascontiguousarray(directions, dtype=np.float64).reshape(-1, 3)
    n = o.shape[0]
    ids = np.empty(n, dtype=np.int32)
    ts = np.empty(n, dtype=np.float64)
    status = lib.oracle_closest_hits(_desc_pointer(desc), o.ctypes.data_as(C.POINTER(C.c_double)),
                                     d.ctypes.data_as(C.POINTER(C.c_double)), n, 1 if brute_force else 0,
                                     ids.ctypes.data_as(C.POINTER(C.c_int32)),
                                     ts.ctypes.data_as(C.POINTER(C.c_double)))
    if status != 0:
        raise RuntimeError(lib.oracle_last_error().decode())
    return ids, ts


def hit_distances(desc, origins: np.ndarray, directions: np.ndarray, ids: np.ndarray, slack: float = 0.0) -> np.ndarray:
    """Where, in double, each ray meets primitive ids[i] (source index space) over (0.001, inf); inf where it does
    not or ids[i] < 0. slack: a quad's or triangle's barycentrics accepted that far outside their bounds."""
    lib = load()
    o = np.ascontiguousarray(origins, dtype=np.float64).reshape(-1, 3)
    d = np.ascontiguousarray(directions, dtype=np.float64).reshape(-1, 3)
    k = np.ascontiguousarray(ids, dtype=np.int32).reshape(-1)
    ts = np.empty(k.size, dtype=np.float64)
    status = lib.oracle_hit_distances(_desc_pointer(desc), o.ctypes.data_as(C.POINTER(C.c_double)),
                                      d.ctypes.data_as(C.POINTER(C.c_double)), k.size,
                                      k.ctypes.data_as(C.POINTER(C.c_int32)), slack,
                                      ts.ctypes.data_as(C.POINTER(C.c_double)))
    if status != 0:
        raise RuntimeError(lib.oracle_last_error().decode())
    return ts


EDGE_SLACK = 1e-4  # barycentric slack of a float search's hit on an edge two primitives share


def first_hit_mismatches(desc, origins, directions, ids, ref_ids, ts=None, ref_ts=None, tie_rel: float = 1e-6) -> dict:
    """First-hit parity of `ids` against `ref_ids` on the same rays (both source index space, -1 a miss). Of the rays
    whose ids differ, a tie is one where both searches hit a surface at the same distance within `tie_rel` relative
    (the reference's tracer-check class `ties`, tests/tracer_check_layout.h: another primitive at the same t): either
    the double search meets both primitives within `tie_rel` of each other (each quad or triangle taken with its
    edges widened by EDGE_SLACK of its size, the float rounding of a hit on the edge it shares with its neighbour), or
    the two searches' own distances (`ts`, `ref_ts`, where given) agree within `tie_rel`. Every other difference is a
    mismatch; `examples` lists a few (ray, ids, distances)."""
    ids = np.asarray(ids).reshape(-1)
    ref_ids = np.asarray(ref_ids).reshape(-1)
    bad = np.flatnonzero(ids != ref_ids)
    ties = 0
    if bad.size:
        o = np.asarray(origins, dtype=np.float64).reshape(-1, 3)[bad]
        d = np.asarray(directions, dtype=np.float64).reshape(-1, 3)[bad]
        ta = hit_distances(desc, o, d, ids[bad], EDGE_SLACK)
        tb = hit_distances(desc, o, d, ref_ids[bad], EDGE_SLACK)

        def close(a, b):
            both = np.isfinite(a) & np.isfinite(b) & (ids[bad] >= 0) & (ref_ids[bad] >= 0)
            a0 = np.where(both, a, 1.0)
            b0 = np.where(both, b, 1.0)
            return both & (np.abs(a0 - b0) <= tie_rel * np.minimum(np.abs(a0), np.abs(b0)))

        tie = close(ta, tb)
        if ts is not None and ref_ts is not None:
            tie |= close(np.asarray(ts, dtype=np.float64).reshape(-1)[bad],
                         np.asarray(ref_ts, dtype=np.float64).reshape(-1)[bad])
        ties = int(np.count_nonzero(tie))
        others = np.flatnonzero(~tie)[:5]
        examples = [{"ray": int(bad[k]), "ids": [int(ids[bad[k]]), int(ref_ids[bad[k]])],
                     "double_t": [float(ta[k]), float(tb[k])],
                     "own_t": [float(np.asarray(ts).reshape(-1)[bad[k]]) if ts is not None else None,
                               float(np.asarray(ref_ts).reshape(-1)[bad[k]]) if ref_ts is not None else None]}
                    for k in others]
    else:
        examples = []
    return {"rays": int(ids.size), "mismatches": int(bad.size), "ties": ties,
            "non_tie_mismatches": int(bad.size) - ties, "tie_rel": tie_rel, "examples": examples}


def image_compare(a: np.ndarray, b: np.ndarray, tile: int = 32) -> dict:
    """ImageCompare A B (image_compare.cpp): the verdict (0 consistent, 1 different, 2 error) and its numbers.
    a and b are height x width x 3; they are rounded to float32 as a PFM file stores them."""
    lib = load()
    fa = np.ascontiguousarray(a, dtype=np.float32)
    fb = np.ascontiguousarray(b, dtype=np.float32)
    if fa.shape != fb.shape or fa.ndim != 3 or fa.shape[2] != 3:
        raise ValueError("images must have the same shape (height, width, 3)")
    r = CompareResult()
    lib.oracle_image_compare(fa.ctypes.data_as(C.POINTER(C.c_float)), fb.ctypes.data_as(C.POINTER(C.c_float)),
                             fa.shape[1], fa.shape[0], tile, C.byref(r))
    out = {}
    for name, _ in CompareResult._fields_:
        v = getattr(r, name)
        out[name] = list(v) if hasattr(v, "__len__") else v
    return out


def thresholds(tested_tiles: int) -> dict:
    lib = load()
    w, a, l = C.c_double(), C.c_double(), C.c_double()
    k = C.c_int32()
    lib.oracle_thresholds(tested_tiles, C.byref(w), C.byref(a), C.byref(l), C.byref(k))
    return {"whole_image": w.value, "all_tiles": a.value, "largest_tile": l.value, "tiles_over_3": k.value}


def save_pfm(path: str, pixels: np.ndarray) -> None:
    """image.ixx:157-203 save_pfm: 'PF', the size, -1.0 (little-endian), rows from the bottom as float32."""
    h, w, _ = pixels.shape
    with open(path, "wb") as f:
        f.write(f"PF\n{w} {h}\n-1.0\n".encode())
        f.write(np.ascontiguousarray(pixels[::-1], dtype="<f4").tobytes())


def load_pfm(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        if f.readline().strip() != b"PF":
            raise ValueError("not a color PFM")
        w, h = (int(x) for x in f.readline().split())
        scale = float(f.readline())
        data = np.frombuffer(f.read(), dtype="<f4" if scale < 0 else ">f4").reshape(h, w, 3)
    return data[::-1].astype(np.float64)
