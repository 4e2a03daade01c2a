"""Benchmark of the path-tracing integrator: path segments per second on the Cornell box with a glass ball.

The workload is the configuration the metric is quoted on that fits one GPU: the reference's `glass` scene
(src/scenes.ixx:484-501), 600 x 600 pixels, 1024 samples per pixel (32 x 32 strata), depth 50, the mixture of half
light / half cosine sampling. A step renders that whole image from zero passes. Inputs are synthetic (the scene is
procedural and fully specified); the scene tables are resident in HBM before the timed region starts.

Arms:
  default          this library: `value` from a resident scene (device-timed steps), `e2e` through the C-ABI's
                   render() with host tables in and host pixels out, copies included;
  --impl reference the reference's CPU renderer on this box's host cores (its algorithm restated as the oracle,
                   as the reference's MSVC-module build cannot compile here), on a bounded band of rows of the
                   same workload each step.

One process per GPU under torchrun: every rank renders its own independent image (its own seed) of the same
workload, so per-GPU work is fixed as N grows (weak scaling); the step times are max-reduced over ranks.

After the timed region (rank 0, untimed): the last timed image is checked at its full size against the reference's
own renderer (ImageCompare, `parity`) and both images' error against the FP64 65,536-spp oracle render is reported;
the same workload under NEE with power-heuristic MIS is measured and checked the same way (`nee_mis`); one more render
with CUDA events around every kernel gives the dominant kernel's roofline; then the triangle mesh, the 64 batched jobs
(each job ImageCompared with a plain render) and the served stream.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

from raytracing_b200 import shard  # noqa: E402  (pure Python: the split of the work over ranks)

METRIC = "path segments/s at matched ImageCompare error; served p50/p99 vs plain launch"
UNIT = "segments/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--scene", default="glass")
    p.add_argument("--width", type=int, default=600)
    p.add_argument("--spp", type=int, default=1024)
    p.add_argument("--depth", type=int, default=50)
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="target length of the CPU-baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-mis", action="store_true", help="skip the NEE/MIS integrator on the same workload")
    p.add_argument("--no-batched", action="store_true", help="skip the 64-job batched measurement")
    p.add_argument("--no-reference-gpu", action="store_true",
                   help="skip timing the reference's own CUDA renderer on the same workload")
    p.add_argument("--no-mesh", action="store_true", help="skip the triangle-mesh (GGX, environment) measurement")
    p.add_argument("--no-served", action="store_true", help="skip the served request stream's measurement")
    p.add_argument("--served-rate", type=float, default=200.0)
    p.add_argument("--served-window", type=float, default=0.25, help="seconds of arrivals (a bounded sample)")
    p.add_argument("--served-step", type=float, default=0.01, help="GPU seconds a batched server step aims at")
    p.add_argument("--served-continuous-step", type=float, default=0.002,
                   help="GPU seconds a step of the continuous server runs before it returns to take arrivals")
    p.add_argument("--served-limit", type=float, default=300.0, help="wall seconds after which serving stops")
    p.add_argument("--served-long-window", type=float, default=5.0,
                   help="seconds of arrivals of the long stream (first frames of about 1,000 requests)")
    return p.parse_args()


def workload_config(args, scene) -> dict:
    return {"workload": f"cornell box with glass ball ({args.scene}), {scene.width}x{scene.height}, {args.spp} spp, "
                        f"depth {args.depth}, mixture sampling",
            "scene": args.scene, "width": scene.width, "height": scene.height, "spp": args.spp,
            "max_depth": args.depth, "strategy": "mixture (0.5 lights list / 0.5 cosine)",
            "arithmetic": "fp32 (fp64 for large-sphere quadratics and per-pixel sums)",
            "l2": "L2 flushed between timed steps (512 MiB write); the scene itself is a few KB and cache-resident "
                  "by nature"}


def rank_info():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"rt_b200_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.out.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def read_peaks() -> dict:
    path = REPO / "MEASURED_PEAKS.json"
    if path.exists():
        peaks = json.loads(path.read_text())
        return {"hbm_gbs": peaks["hbm_gbs"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


# The wavefront's state per unit of work, by the layout of its slots and queues (raytracing_b200/csrc/kernels.cu): what
# the shade kernel must move through HBM for each segment (the slot's 16-byte rows in and out: five, or for a scene
# without the second book's features, whose paths carry no time or job, three for the books' integrator and four for
# NEE/MIS; the walk's answer; the next query of 48 bytes), for each shadow ray (its answer, its three rows out and back in, its query) and for each sample
# (its value). These are the bytes that bind the shade kernel: the scene itself (a few KB) is read from L1.
def shade_bytes_per_segment(slot_rows: int) -> int:
    return 2 * slot_rows * 16 + 16 + 48


SHADE_BYTES_PER_SHADOW_RAY = 4 + 2 * 3 * 16 + 48
SHADE_BYTES_PER_SAMPLE = 16


def slot_rows_of(desc, kernel_name: str) -> int:
    """The rows of a session's wavefront slot for a scene without moving spheres, textures or smoke (kernels.cu
    compact_slots): three for the books' integrator, four for NEE/MIS; five otherwise."""
    d = desc.contents
    moving = any(d.spheres[i].displacement.x or d.spheres[i].displacement.y or d.spheres[i].displacement.z
                 for i in range(d.sphere_count))
    textured = any(d.materials[i].kind in (0, 3, 4) and d.textures[d.materials[i].texture].kind != 0
                   for i in range(d.material_count))
    features = moving or textured or d.medium_count > 0
    if features:
        return 5
    return {"wavefront books": 3, "wavefront nee-mis": 4}.get(kernel_name, 5)
# FP32 operations per primitive test and per node visit (slab test: 6 FMA + 6 min/max), the trace kernels' arithmetic
FLOPS_PER_NODE, FLOPS_PER_SPHERE, FLOPS_PER_QUAD, FLOPS_PER_TRIANGLE = 12, 20, 25, 30


def roofline_of(times: dict, counts: dict, samples: int, fetched: dict, counted: int, scene_bytes_per_query: float,
                peaks: dict, fp32_peak: float, render_seconds: float, slot_rows: int = 5) -> dict:
    """The roofline of the render's dominant kernel, from per-kernel CUDA-event times of one render of the workload.
    The wavefront's shade kernel is bound by HBM on the slot state it streams; the trace kernel (and the persistent
    kernel) by FP32 arithmetic on the scene's primitives, which sit in L1."""
    active = {k: v for k, v in times.items() if v[1] > 0 and v[0] > 0}
    total = sum(v[0] for v in active.values())
    dominant = max(active, key=lambda k: active[k][0])
    rays, shadow = counts["rays"], counts["shadow_rays"]
    queries = rays + shadow
    flops_per_query = (FLOPS_PER_NODE * fetched["nodes"] + FLOPS_PER_SPHERE * fetched["spheres"] +
                       FLOPS_PER_QUAD * fetched["quads"] + FLOPS_PER_TRIANGLE * fetched["triangles"]) / max(counted, 1)
    kernels = {k: {"seconds": v[0], "launches": v[1], "avg_launch_us": 1e6 * v[0] / v[1], "share": v[0] / total}
               for k, v in active.items()}

    def fp32_roof(kind: str) -> dict:
        sec = active[kind][0]
        achieved = flops_per_query * queries / sec / 1e12
        return {"bound": "fp32", "kernel": kind, "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": achieved / fp32_peak, "flops_per_query": flops_per_query,
                "peak_source": "measured here: FP32 GEMM through cuBLAS, TF32 off"}

    if dominant == "shade":
        state = (rays * shade_bytes_per_segment(slot_rows) + shadow * SHADE_BYTES_PER_SHADOW_RAY +
                 samples * SHADE_BYTES_PER_SAMPLE)
        sec = active["shade"][0]
        achieved = state / sec / 1e9
        out = {"bound": "hbm", "kernel": "wave_shade_kernel", "achieved": achieved, "peak": peaks["hbm_gbs"],
               "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": None,
               "peak_source": peaks["source"], "algorithmic_bytes_per_segment": state / rays,
               "algorithmic_bytes_per_launch": state / active["shade"][1],
               "note": "the slot state the shade kernel streams per segment (rows in and out, answer, next query), "
                       "per shadow ray and per sample, over its CUDA-event time; the scene's own bytes "
                       f"({scene_bytes_per_query:.0f} per query) are served from L1. DRAM traffic per launch is in "
                       "the committed ncu summary under profiles/"}
        if "trace" in active:
            out["trace_kernel"] = fp32_roof("trace")
    else:
        out = fp32_roof(dominant)
        out["traffic"] = None
    out["kernels"] = kernels
    out["events_total_over_render"] = total / render_seconds
    return out


GOLDEN = REPO / "tests" / "golden"


def trimmed_rms(a: np.ndarray, b: np.ndarray, trim: float = 0.01) -> tuple[float, float]:
    """PfmStats' RMS of the channel average's difference (tests/pfm_stats.cpp:344-367): (trimmed, full), the trimmed
    one leaving out the largest share `trim` of the squared differences (fireflies, lamp edges)."""
    d = a.mean(axis=2) - b.mean(axis=2)
    d2 = np.sort((d * d).ravel())
    drop = int(np.floor(d2.size * trim))
    return float(np.sqrt(d2[: d2.size - drop].mean())), float(np.sqrt(d2.mean()))


def error_vs_fp64(name: str, images: dict) -> dict:
    """Each image's error against the FP64 high-spp oracle render of the same scene and view (tests/golden/fp64_*.npz,
    made by tests/golden/make_fp64_oracle.py): PfmStats' trimmed RMS, and the ratio of this library's error to the
    reference renderer's at the same spp and strategy ("matched" within 5%)."""
    path = GOLDEN / f"fp64_{name}.npz"
    if not path.exists():
        return {"unavailable": f"{path.name} is missing (tests/golden/make_fp64_oracle.py makes it)"}
    z = np.load(path)
    oracle_img = z["image"].astype(np.float64)
    out = {"oracle": f"{z['renderer']}, {int(z['width'])}x{int(z['height'])}, {int(z['passes'])} passes",
           "metric": "RMS of the channel average's difference, trimmed by 1% (PfmStats)"}
    for key, img in images.items():
        if img is None or img.shape != oracle_img.shape:
            continue
        t, full = trimmed_rms(img, oracle_img)
        out[key] = {"trimmed_rms": t, "rms": full}
    if "this_library" in out and "reference_gpu" in out:
        ratio = out["this_library"]["trimmed_rms"] / out["reference_gpu"]["trimmed_rms"]
        out["ratio"] = ratio
        out["matched"] = bool(abs(ratio - 1.0) <= 0.05)
    return out


def image_parity(reference_fn, ours: np.ndarray, seeds=(6, 7)) -> dict:
    """ImageCompare (src/image_compare.cpp, restated in the oracle) between this library's image and an independent
    render of the same scene, spp and strategy by the reference's renderer; a failure is re-run once with a fresh seed
    (the reference's re-run rule)."""
    from oracle import binding as oracle

    attempts = []
    for seed in seeds:
        r = oracle.image_compare(reference_fn(seed), ours)
        attempts.append({"verdict": "consistent" if r["verdict"] == 0 else "different",
                         "whole_image_z": r["whole_image_z"], "all_tiles_z": r["all_tiles_z"],
                         "largest_tile_z": r["largest_tile_z"], "tiles_over_3": r["tiles_over_3"],
                         "tested_tiles": r["tested_tiles"],
                         "thresholds": [r["threshold_whole_image"], r["threshold_all_tiles"],
                                        r["threshold_largest_tile"], r["threshold_tiles_over_3"]]})
        if r["verdict"] == 0:
            break
    return {"verdict": attempts[-1]["verdict"], "attempts": attempts}


def fp32_peak_tflops(torch) -> float:
    """The FP32 (non-tensor) arithmetic peak measured on this GPU: a plain FP32 GEMM through cuBLAS with TF32 off,
    8192^3, the best of five after warm-up."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    a = torch.randn(8192, 8192, device="cuda", dtype=torch.float32)
    b = torch.randn(8192, 8192, device="cuda", dtype=torch.float32)
    for _ in range(2):
        torch.mm(a, b)
    best = 0.0
    for _ in range(5):
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        torch.mm(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2 * 8192 ** 3 / (s.elapsed_time(e) / 1000.0) / 1e12)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    return best


def config_errors(rt, seed: int) -> dict:
    """The other workloads' error against their FP64 oracle renders (tests/golden/fp64_*.npz), beside an independent
    render of the same spp and strategy: the first book's cover scene at 400x225, 32 passes (against the reference's
    float renderer), and the mesh scene (level 8, GGX, environment) reduced to 240x135 at 256 spp (against the CPU
    oracle, as the reference traces triangles only through OptiX)."""
    from oracle import binding as oracle
    from oracle import ref_gpu

    out = {}
    w = rt.builtin_scene("weekend", width=400, spp=16, depth=50)
    ours = rt.render(w, seed=seed, passes=32).pixels
    ref = ref_gpu.render(w.desc, w.width, w.height, seed=seed + 1, passes=32)[0] if ref_gpu.available() else None
    out["cover_400x225_32spp"] = error_vs_fp64("weekend", {"this_library": ours, "reference_gpu": ref})
    # The same workload in FP64 (precision::float64: the books' integrator in double), this library's and the
    # reference's, against the same oracle; and both double renderers' speed on 256 passes of the view
    ours64 = rt.render(w, seed=seed + 3, passes=32, arithmetic="float64").pixels
    ref64 = (ref_gpu.render(w.desc, w.width, w.height, seed=seed + 4, passes=32, fp64=True)[0]
             if ref_gpu.available() else None)
    e64 = error_vs_fp64("weekend", {"this_library": ours64, "reference_gpu": ref64})
    timed = rt.render(w, seed=seed + 5, passes=256, arithmetic="float64")
    e64["this_library_segments_per_s"] = timed.rays / timed.kernel_seconds
    e64["kernel"] = timed.kernel["name"]
    if ref_gpu.available():
        _, info = ref_gpu.render(w.desc, w.width, w.height, seed=seed + 6, passes=256, fp64=True)
        e64["reference_gpu_segments_per_s"] = info["rays"] / info["kernel_seconds"]
        e64["this_library_over_reference"] = e64["this_library_segments_per_s"] / e64["reference_gpu_segments_per_s"]
    out["cover_400x225_32spp_fp64"] = e64
    m = rt.builtin_scene("mesh-ggx", width=240, spp=16)
    ours = rt.render(m, seed=seed, passes=256).pixels
    cpu, _ = oracle.render(m.desc, m.width, m.height, seed=seed + 2, passes=256)
    e = error_vs_fp64("mesh-ggx", {"this_library": ours, "cpu_oracle": cpu})
    if "this_library" in e and "cpu_oracle" in e:
        e["ratio"] = e["this_library"]["trimmed_rms"] / e["cpu_oracle"]["trimmed_rms"]
        e["matched"] = bool(abs(e["ratio"] - 1.0) <= 0.05)
    out["mesh_240x135_256spp"] = e
    return out


def leg(line, key: str, run) -> None:
    """line[key] = run(), or, when the leg raises, the error in its place: one workload's failure is recorded in the
    line instead of ending the run before the line is printed."""
    try:
        line[key] = run()
    except Exception as e:  # noqa: BLE001 - any failure of an auxiliary leg
        line[key] = {"error": f"{type(e).__name__}: {e}"}


def row_band(height: int, threads: int, per_thread: int) -> tuple[int, int]:
    """(first row, rows) of the CPU legs' band of rows about the image's middle: `per_thread` rows a thread where the
    image has them, and always a whole number of rows a thread when the image has at least one a thread (rows are the
    unit of threading, so no thread idles in the last round)."""
    per_thread = max(1, per_thread)
    rows = threads * min(per_thread, height // threads) if height >= threads else height
    return max(0, height // 2 - rows // 2), rows


def cpu_baseline(scene, args, threads: int) -> dict:
    """The reference's CPU renderer (restated as the oracle) on a bounded band of rows of the same workload."""
    from oracle import binding as oracle

    h = scene.height
    mid = h // 2
    # Probe one row (one thread: rows are the unit of threading), then size the band to about --cpu-seconds on all
    # threads
    _, probe = oracle.render(scene.desc, scene.width, h, seed=11, passes=args.spp, threads=threads,
                             row_begin=mid, row_end=mid + 1)
    begin, rows = row_band(h, threads, int(args.cpu_seconds / max(probe["seconds"], 1e-3)))
    _, stats = oracle.render(scene.desc, scene.width, h, seed=12, passes=args.spp, threads=threads,
                             row_begin=begin, row_end=begin + rows)
    value = stats["rays"] / stats["seconds"]
    return {"value": value, "unit": UNIT, "cores": stats["threads"], "kind": "port",
            "sample": f"rows {begin}-{begin + rows - 1} of {scene.width}x{h} at {args.spp} spp "
                      f"({stats['rays']} segments in {stats['seconds']:.2f} s)"}


def reference_gpu_measurement(scene_desc, passes: int, value: float) -> dict:
    """The reference's own CUDA renderer (src/gpu, built unmodified into oracle/_ref) on the same workload and GPU:
    gpu::render's rays over its kernel_seconds (the passes alone, timed on the GPU) — the reference's own figure."""
    from oracle import ref_gpu

    if not ref_gpu.available():
        return {"unavailable": "oracle/_ref/libref_gpu.so was not built (needs the reference's sources)"}
    w, h = scene_desc.width, scene_desc.height
    ref_gpu.render(scene_desc.desc, w, h, seed=5, passes=16)  # warm-up: module load, allocations
    image, info = ref_gpu.render(scene_desc.desc, w, h, seed=6, passes=passes)
    segments_per_s = info["rays"] / info["kernel_seconds"]
    return {"image": image, "segments_per_s": segments_per_s, "e2e_segments_per_s": info["rays"] / info["seconds"],
            "kernel": info["kernel"], "registers": info["registers"],
            "blocks_per_multiprocessor": info["blocks_per_multiprocessor"],
            "segments_per_sample": info["rays"] / (w * h * passes),
            "this_library_over_reference": value / segments_per_s,
            "note": "the reference's gpu::render built from its src/gpu sources for sm_100a, same scene tables"}


def mesh_measurement(rt, torch, peaks: dict) -> dict:
    """The triangle-mesh workload (an icosphere of 1.31M triangles displaced by Perlin noise, GGX metal on a glossy
    plane, a 1024x512 environment map with a sun, importance-sampled; 1920x1080, 256 spp, depth 16, NEE with MIS)
    in both forms of a session: the wavefront (its default on a tree-searched scene) and the persistent kernel.
    Timed on the GPU by the session's own events; the scene is far larger than L2."""
    desc = rt.builtin_scene("mesh-ggx")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    scene = rt.Scene(desc)  # validation, the BVH build on the host's threads, the upload
    torch.cuda.synchronize()
    create_s = time.perf_counter() - t0
    passes = desc.round_passes  # sqrt_spp^2: 256
    out = {"workload": f"mesh-ggx {desc.width}x{desc.height}, {passes} spp, depth {desc.camera.max_depth}, "
                       f"{scene.stats()['triangles']} triangles, NEE/MIS with the environment map",
           "scene_stats": scene.stats(),
           "scene_create_s": create_s, "host_threads": os.cpu_count()}
    # The tree's algorithmic bytes per query: node visits (64 B) and triangle tests (48 B) counted on the workload's
    # own rays by the counting build (the binary walk; the four-wide walk reads 128-B nodes about half as often)
    counting = rt.Session(scene, seed=4, launch_seconds=0.5)
    counting.set_counting(True)
    counting.render_to(2)
    fetched = counting.fetch_counts()
    cc = counting.counters()
    counting.close()
    queries = max(cc["rays"] + cc["shadow_rays"], 1)
    bytes_per_query = (64 * fetched["nodes"] + 16 * fetched["spheres"] + 48 * fetched["quads"] +
                       48 * fetched["triangles"]) / queries
    for form in ("wavefront", "persistent"):
        sess = rt.Session(scene, seed=3, form=form, launch_seconds=0.5)
        if form == "wavefront":
            out["autotune"] = sess.autotune()
        sess.render_to(16)  # warm-up: module load, buffers
        sess.set_camera(desc.camera)
        torch.cuda.synchronize()
        rep = sess.render_to(passes)
        cnt = sess.counters()
        out[form] = {"segments_per_s": cnt["rays"] / rep["gpu_seconds"],
                     "queries_per_s": (cnt["rays"] + cnt["shadow_rays"]) / rep["gpu_seconds"],
                     "gpu_s": rep["gpu_seconds"], "launches": rep["launches"], "segments": cnt["rays"],
                     "shadow_rays": cnt["shadow_rays"], "kernel": sess.kernel()}
        if form == "wavefront":
            # the walks' bytes over the trace kernel's own CUDA-event time, against the HBM roofline
            sess.set_timing(True)
            sess.set_camera(desc.camera)
            sess.render_to(min(passes, 64))
            kt = sess.kernel_times()
            tc = sess.counters()
            sess.set_timing(False)
            walks = tc["rays"] + tc["shadow_rays"]
            achieved = bytes_per_query * walks / kt["trace"][0] / 1e9
            out["bvh_fetch_roofline"] = {
                "bound": "hbm", "kernel": "wave_trace_kernel (four-wide walk)", "achieved": achieved,
                "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                "peak_source": peaks["source"], "algorithmic_bytes_per_query": bytes_per_query,
                "node_visits_per_query": fetched["nodes"] / queries,
                "triangle_tests_per_query": fetched["triangles"] / queries,
                "trace_share": kt["trace"][0] / (kt["trace"][0] + kt["shade"][0] + kt["reduce"][0]),
                "note": "BVH node and triangle bytes a walk reads (counting build, binary walk) over the trace "
                        "kernel's event time; the tree (49 MB of nodes, 63 MB of triangles) is about L2's size, so "
                        "part of these bytes come from L2"}
        sess.close()
    out["wavefront_over_persistent"] = out["wavefront"]["segments_per_s"] / out["persistent"]["segments_per_s"]
    return out


def mis_measurement(rt, torch, args, steps: int, seed: int) -> tuple[dict, np.ndarray]:
    """The same workload under NEE with power-heuristic MIS (the quality integrator; the reference's quality kernel,
    src/gpu/quality.cu): the glass Cornell box at the same size, spp and depth, its lamp the light NEE samples.
    Device-timed renders from zero with the scene resident; returns the measurement and the last image."""
    desc = rt.builtin_scene("cornell-mis", width=args.width, spp=args.spp, depth=args.depth)
    passes = desc.round_passes if args.spp <= 0 else args.spp
    sess = rt.Session(rt.Scene(desc), seed=seed, launch_seconds=0.5)
    sess.render_to(min(passes, 64))  # warm-up: buffers, module load
    seconds = 0.0
    rays = shadow = launches = 0
    for _ in range(steps):
        sess.set_camera(desc.camera)
        torch.cuda.synchronize()
        rep = sess.render_to(passes)
        c = sess.counters()
        seconds += rep["gpu_seconds"]
        rays += c["rays"]
        shadow += c["shadow_rays"]
        launches += rep["kernel_launches"]
    image = sess.pixels()
    samples = steps * passes * desc.width * desc.height
    out = {"workload": f"cornell-mis (the glass box, NEE + power-heuristic MIS), {desc.width}x{desc.height}, "
                       f"{passes} spp, depth {desc.camera.max_depth}",
           "segments_per_s": rays / seconds, "shadow_rays_per_s": shadow / seconds,
           "queries_per_s": (rays + shadow) / seconds, "ms_per_render": 1000 * seconds / steps, "renders": steps,
           "segments_per_sample": rays / samples, "shadow_rays_per_sample": shadow / samples,
           "kernel": sess.kernel(), "gpu_launches_per_render": launches // steps}
    sess.close()
    return out, image, desc, passes


def log_uniform(rng, lo: float, hi: float) -> float:
    return float(np.exp(rng.uniform(np.log(lo), np.log(hi))))


def batched_jobs(rt, count: int = 64, seed: int = 2024):
    """The batched workload: `count` cover-scene variants, job j with seed j; W and H each log-uniform in
    [64, 1024], spp log-uniform in [16, 1024] (whole passes), N log-uniform in [50, 2000] spheres."""
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(count):
        w = int(round(log_uniform(rng, 64, 1024)))
        h = int(round(log_uniform(rng, 64, 1024)))
        spp = int(round(log_uniform(rng, 16, 1024)))
        n = int(round(log_uniform(rng, 50, 2000)))
        jobs.append((rt.builtin_scene(f"cover-{n}", width=w, height=h, spp=spp, scene_seed=j), j, spp))
    return jobs


def batched_measurement(rt, torch, rank: int = 0, world: int = 1) -> dict:
    """64 jobs in one batched render (the jobs' wavefront runs sharing one slot pool, per step) against the plain
    form (one render per job), on the same jobs and seeds; every job's image compared bit for bit. With N ranks the
    jobs are split by cost (pixels x passes, longest first to the least loaded rank) and each rank renders its share
    on its own GPU: the times are the slowest rank's, the segments everyone's (no collective on the data)."""
    all_jobs = batched_jobs(rt)
    costs = [s.width * s.height * p for s, _, p in all_jobs]
    jobs = [all_jobs[i] for i in shard.my_units(costs, world, rank)]
    rt.batch_render(jobs[:4])  # warm-up (graph capture, module load)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b = rt.batch_render(jobs)
    batch_wall = time.perf_counter() - t0
    plain_kernel = 0.0
    plain_wall = 0.0
    plain_rays = 0
    identical = 0
    max_diff = 0.0
    consistent = 0
    reruns = 0
    worst_z = 0.0
    from oracle import binding as oracle

    for (scene, seed, passes), img in zip(jobs, b.images):
        t0 = time.perf_counter()
        r = rt.render(scene, seed=seed, passes=passes)
        plain_wall += time.perf_counter() - t0
        plain_kernel += r.kernel_seconds
        plain_rays += r.rays
        identical += int(np.array_equal(r.pixels, img))
        max_diff = max(max_diff, abs(float(img.mean()) - float(r.pixels.mean())) / max(float(r.pixels.mean()), 1e-9))
        # Per-job ImageCompare against a plain render with an independent seed (untimed); one re-run on an alarm
        for attempt in range(2):
            other = rt.render(scene, seed=seed + 100_000 * (attempt + 1), passes=passes).pixels
            cmp = oracle.image_compare(other, img)
            if cmp["verdict"] == 0:
                consistent += 1
                worst_z = max(worst_z, abs(cmp["whole_image_z"]))
                break
            reruns += 1
    pixels = sum(s.width * s.height for s, _, _ in all_jobs)
    samples = sum(costs)
    batch_gpu, batch_rays = shard.combine(b.gpu_seconds, b.rays)
    batch_wall, _ = shard.combine(batch_wall, 0)
    plain_kernel, plain_rays = shard.combine(plain_kernel, plain_rays)
    plain_wall, _ = shard.combine(plain_wall, 0)
    _, identical = shard.combine(0, identical)
    _, consistent = shard.combine(0, consistent)
    reference = {}
    from oracle import ref_gpu

    if ref_gpu.available() and world == 1:
        ref_rays = 0
        ref_kernel = 0.0
        ref_wall = 0.0
        for scene, seed, passes in jobs:
            _, info = ref_gpu.render(scene.desc, scene.width, scene.height, seed=seed, passes=passes)
            ref_rays += info["rays"]
            ref_kernel += info["kernel_seconds"]
            ref_wall += info["seconds"]
        reference = {"reference_plain_segments_per_s": ref_rays / ref_kernel, "reference_plain_gpu_s": ref_kernel,
                     "reference_plain_e2e_s": ref_wall,
                     "speedup_gpu_over_reference": (batch_rays / batch_gpu) / (ref_rays / ref_kernel),
                     "speedup_e2e_over_reference": ref_wall / batch_wall}
    return {**reference, "workload": "64 cover-scene variants (50-2000 spheres, W,H log-uniform 64-1024, spp log-uniform "
                        "16-1024, seeds 0-63), mixture of sizes sharing one wavefront run per step",
            "ranks": world, "pixels": pixels, "samples": samples, "segments": batch_rays,
            "batched_segments_per_s": batch_rays / batch_gpu, "batched_gpu_s": batch_gpu,
            "batched_e2e_segments_per_s": batch_rays / batch_wall, "batched_e2e_s": batch_wall,
            "batched_setup_s": b.setup_seconds, "batched_steps": b.steps, "batched_launches": b.launches,
            "graph": b.graph,
            "plain_segments_per_s": plain_rays / plain_kernel, "plain_gpu_s": plain_kernel,
            "plain_e2e_segments_per_s": plain_rays / plain_wall, "plain_e2e_s": plain_wall,
            "speedup_gpu": (batch_rays / batch_gpu) / (plain_rays / plain_kernel),
            "speedup_e2e": plain_wall / batch_wall,
            "jobs_bit_identical_to_plain": f"{int(identical)}/{len(all_jobs)}",
            "jobs_image_compare_consistent_with_plain": f"{int(consistent)}/{len(all_jobs)}",
            "image_compare_reruns": reruns, "largest_whole_image_z": worst_z,
            "image_compare_note": "each job against a plain render of the same scene and passes with an independent "
                                  "seed, one re-run on an alarm (the reference's rule)",
            "max_relative_mean_difference_to_plain": max_diff}


SERVED_RESOLUTIONS = [((256, 256), 4), ((512, 512), 3), ((1920, 1080), 2), ((3840, 2160), 1)]
SERVED_SCENES = ["weekend", "glass", "mesh-ggx"]


def served_requests(rt, rate: float, window: float, seed: int = 7):
    """The served stream: Poisson arrivals at `rate` per second over `window` seconds; each request a scene from
    {cover (weekend), cornell glass, mesh+GGX} uniform, an orbit camera (azimuth U(0, 360), elevation U(5, 40)
    degrees), a resolution from {256^2, 512^2, 1920x1080, 3840x2160} weighted 4:3:2:1, target spp log-uniform in
    [1, 4096]."""
    rng = np.random.default_rng(seed)
    weights = np.array([w for _, w in SERVED_RESOLUTIONS], dtype=float)
    out = []
    t = 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > window:
            break
        name = SERVED_SCENES[int(rng.integers(0, 3))]
        (w, h) = SERVED_RESOLUTIONS[int(rng.choice(4, p=weights / weights.sum()))][0]
        spp = max(1, int(round(log_uniform(rng, 1, 4096))))
        orbit = (float(rng.uniform(0, 360)), float(rng.uniform(5, 40)))
        cam = rt.builtin_camera(name, width=w, height=h, spp=spp, orbit=orbit)
        out.append({"arrival": t, "scene": name, "camera": cam, "target": spp, "seed": len(out) + 1})
    return out


def serve_stream(rt, scenes, requests, continuous: bool, step_seconds: float, limit: float) -> dict:
    """The requests submitted at their arrival times to a server (the continuous wavefront, or batched steps) and
    served until every one is done or `limit` wall seconds have passed: time-to-first-frame and time-to-target
    percentiles, and the server's segments per GPU second and per wall second."""
    server = rt.Server(hbm_budget_bytes=120 << 30, step_seconds=step_seconds, continuous=continuous)
    pending = list(range(len(requests)))
    ids = {}
    start = time.perf_counter()
    submitted = {}
    step_log = []  # (wall s, GPU s, first frames, refined, admitted) of each step
    while True:
        now = time.perf_counter() - start
        while pending and requests[pending[0]]["arrival"] <= now:
            i = pending.pop(0)
            q = requests[i]
            ids[i] = server.submit(scenes[q["scene"]], q["camera"], q["seed"], q["target"])
            submitted[i] = time.perf_counter() - start
        if len(ids) == len(requests) and all(server.poll(r)["state"] == "done" for r in ids.values()):
            break
        if now > limit:
            break
        rep = server.step()
        step_log.append((round(time.perf_counter() - start, 4), round(rep["gpu_seconds"], 5), rep["first_frames"],
                         rep["refined"], rep["admitted"]))
        if rep["active"] == 0 and rep["queued"] == 0 and pending:
            time.sleep(max(0.0, requests[pending[0]]["arrival"] - (time.perf_counter() - start)))
    wall = time.perf_counter() - start
    ttff, ttt = [], []
    by_size = {}
    for i, rid in ids.items():
        st = server.poll(rid)
        lag = submitted[i] - requests[i]["arrival"]
        if st["first_frame_seconds"] >= 0:
            ttff.append(lag + st["first_frame_seconds"])
            cam = requests[i]["camera"]
            by_size.setdefault(f"{cam.image_width}x{cam.image_height}", []).append(lag + st["first_frame_seconds"])
        if st["done_seconds"] >= 0:
            ttt.append(lag + st["done_seconds"])
    stats = server.stats()
    server.close()
    return {"server": "continuous wavefront" if continuous else "batched steps",
            "requests": len(requests), "completed": len(ttt), "first_frames": len(ttff), "wall_s": wall,
            "ttff_p50_s": pct(ttff, 50), "ttff_p99_s": pct(ttff, 99),
            "ttff_by_resolution": {k: {"requests": len(v), "p50_s": pct(v, 50), "p99_s": pct(v, 99)}
                                   for k, v in sorted(by_size.items())},
            "step_seconds": step_seconds,
            "step_gpu_seconds_max": max((s[1] for s in step_log), default=None),
            "steps_over_twice_the_budget": sum(1 for s in step_log if s[1] > 2 * step_seconds),
            "first_steps": step_log[:12],
            "time_to_target_p50_s": pct(ttt, 50), "time_to_target_p99_s": pct(ttt, 99),
            "served_segments_per_s": stats["rays"] / stats["gpu_seconds"] if stats["gpu_seconds"] else None,
            "served_segments_per_wall_s": stats["rays"] / wall if wall > 0 else None,
            "served_gpu_s": stats["gpu_seconds"], "served_steps": stats["steps"],
            "served_launches": stats["launches"], "groups_of_steps": stats["groups"],
            "busy_slots": stats["busy_slots"]}


def pct(v, p):
    return float(np.percentile(v, p)) if v else None


def served_measurement(rt, torch, args) -> dict:
    """The served stream through the request server against the plain form (one render per request, FIFO, one at a
    time), on the same requests: the continuous wavefront (the headline), the batched steps beside it, and the plain
    form's latencies from its measured per-request GPU times and the arrival times (a single FIFO server)."""
    requests = served_requests(rt, args.served_rate, args.served_window)
    scenes = {name: rt.Scene(rt.builtin_scene(name)) for name in SERVED_SCENES}
    out = serve_stream(rt, scenes, requests, True, args.served_continuous_step, args.served_limit)
    batched = serve_stream(rt, scenes, requests, False, args.served_step, args.served_limit)
    out["batched_server"] = {k: batched[k] for k in ("step_seconds", "ttff_p50_s", "ttff_p99_s", "wall_s",
                                                     "time_to_target_p50_s", "time_to_target_p99_s",
                                                     "served_segments_per_s", "served_segments_per_wall_s",
                                                     "served_steps", "served_launches", "completed")}

    # The plain form: one session render per request on the resident scene, timed on the GPU, then FIFO queueing
    service = []
    plain_rays = 0
    for q in requests:
        sess = rt.Session(scenes[q["scene"]], seed=q["seed"], launch_seconds=0.05)
        sess.set_camera(q["camera"])
        rep = sess.render_to(q["target"])
        sess.pixels()
        plain_rays += sess.counters()["rays"]
        service.append(rep["gpu_seconds"])
        sess.close()
    finish = 0.0
    plain_latency = []
    for q, s in zip(requests, service):
        finish = max(finish, q["arrival"]) + s
        plain_latency.append(finish - q["arrival"])
    out.update({
        "workload": f"Poisson arrivals at {args.served_rate}/s over {args.served_window} s "
                    f"({len(requests)} requests), scenes cover/glass/mesh-ggx, orbit cameras, 256^2..3840x2160 "
                    f"4:3:2:1, target spp log-uniform 1-4096, HBM budget 120 GB",
        "plain_ttff_p50_s": pct(plain_latency, 50), "plain_ttff_p99_s": pct(plain_latency, 99),
        "plain_time_to_target_p50_s": pct(plain_latency, 50),
        "plain_time_to_target_p99_s": pct(plain_latency, 99),
        "plain_segments_per_s": plain_rays / sum(service) if service else None,
        "plain_note": "one render per request (a session on the resident scene), FIFO, first frame = final image"})
    return out


def served_first_frames(rt, args, continuous: bool = True) -> dict:
    """The served stream over a long window (default 5 s of Poisson arrivals at 200/s, about 1,000 requests of the
    same distributions), served until every request has its first frame: time-to-first-frame percentiles over all of
    them (by resolution too), with the server refining the earlier requests meanwhile. Time to target is reported for
    the requests that reached it in that time (the rest are cancelled: the full stream holds about 100x what one GPU
    renders in real time)."""
    requests = served_requests(rt, args.served_rate, args.served_long_window, seed=11)
    scenes = {name: rt.Scene(rt.builtin_scene(name)) for name in SERVED_SCENES}
    server = rt.Server(hbm_budget_bytes=120 << 30,
                       step_seconds=args.served_continuous_step if continuous else args.served_step,
                       continuous=continuous)
    pending = list(range(len(requests)))
    ids, submitted = {}, {}
    start = time.perf_counter()
    steps = 0
    log = []  # (wall s at the step's start, wall s it took, GPU s, first frames, refined, admitted, queued)
    while True:
        now = time.perf_counter() - start
        while pending and requests[pending[0]]["arrival"] <= now:
            i = pending.pop(0)
            q = requests[i]
            ids[i] = server.submit(scenes[q["scene"]], q["camera"], q["seed"], q["target"])
            submitted[i] = time.perf_counter() - start
        if not pending and all(server.poll(r)["first_frame_seconds"] >= 0 for r in ids.values()):
            break
        if now > args.served_long_window + 60:
            break
        t0 = time.perf_counter()
        rep = server.step()
        log.append((round(t0 - start, 4), round(time.perf_counter() - t0, 4), round(rep["gpu_seconds"], 5),
                    rep["first_frames"], rep["refined"], rep["admitted"], rep["queued"]))
        steps += 1
        if rep["active"] == 0 and rep["queued"] == 0 and pending:
            time.sleep(max(0.0, requests[pending[0]]["arrival"] - (time.perf_counter() - start)))
    wall = time.perf_counter() - start
    ttff, ttt, by_size = [], [], {}
    for i, rid in ids.items():
        st = server.poll(rid)
        lag = submitted[i] - requests[i]["arrival"]
        if st["first_frame_seconds"] >= 0:
            ttff.append(lag + st["first_frame_seconds"])
            cam = requests[i]["camera"]
            by_size.setdefault(f"{cam.image_width}x{cam.image_height}", []).append(lag + st["first_frame_seconds"])
        if st["done_seconds"] >= 0:
            ttt.append(lag + st["done_seconds"])
    stats = server.stats()
    server.close()

    def pct(v, p):
        return float(np.percentile(v, p)) if v else None

    return {"server": "continuous wavefront" if continuous else "batched steps",
            "workload": f"Poisson arrivals at {args.served_rate}/s over {args.served_long_window} s "
                        f"({len(requests)} requests), the served stream's distributions, served until every request "
                        f"has its first frame",
            "requests": len(requests), "first_frames": len(ttff), "wall_s": wall, "steps": steps,
            "ttff_p50_s": pct(ttff, 50), "ttff_p99_s": pct(ttff, 99), "ttff_max_s": max(ttff) if ttff else None,
            "ttff_by_resolution": {k: {"requests": len(v), "p50_s": pct(v, 50), "p99_s": pct(v, 99)}
                                   for k, v in sorted(by_size.items())},
            "reached_target": len(ttt), "time_to_target_p50_s": pct(ttt, 50), "gpu_s": stats["gpu_seconds"],
            "busy_slots": stats["busy_slots"],
            "longest_steps": sorted(log, key=lambda e: -e[1])[:8],
            "step_log_fields": "wall start s, wall s, GPU s, first frames, refined, admitted, queued"}


def run_reference(args):
    world, rank, _ = rank_info()
    if rank != 0:
        return 0
    import raytracing_b200 as rt

    scene = rt.builtin_scene(args.scene, width=args.width, spp=args.spp, depth=args.depth)
    threads = os.cpu_count() or 1
    from oracle import binding as oracle

    h = scene.height
    mid = h // 2
    _, probe = oracle.render(scene.desc, scene.width, h, seed=1, passes=args.spp, threads=threads, row_begin=mid,
                             row_end=mid + 1)
    # Each step is a band of rows of about 2 s on all threads (one row per thread at a time), so that warm-up +
    # steps end within a few minutes
    begin, rows = row_band(h, threads, int(2.0 / max(probe["seconds"], 1e-3)))
    for w in range(args.warmup):
        oracle.render(scene.desc, scene.width, h, seed=100 + w, passes=args.spp, threads=threads, row_begin=begin,
                      row_end=begin + rows)
    rays = 0
    seconds = 0.0
    for k in range(args.steps):
        _, st = oracle.render(scene.desc, scene.width, h, seed=200 + k, passes=args.spp, threads=threads,
                              row_begin=begin, row_end=begin + rows)
        rays += st["rays"]
        seconds += st["seconds"]
    value = rays / seconds
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * seconds / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args, scene), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"rows {begin}-{begin + rows - 1} of {scene.width}x{h} at {args.spp} spp, "
                                       f"each step"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_b200(args):
    world, rank, local = rank_info()
    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import raytracing_b200 as rt

    rt.set_device(local)
    scene_desc = rt.builtin_scene(args.scene, width=args.width, spp=args.spp, depth=args.depth)
    passes = scene_desc.round_passes if args.spp <= 0 else args.spp
    scene = rt.Scene(scene_desc)
    stats = scene.stats()
    seed = 1000 + 17 * rank

    # The roofline's algorithmic bytes per segment: a counting render on the workload's own rays (untimed)
    counting = rt.Session(scene, seed=seed + 999, launch_seconds=0.5)
    counting.set_counting(True)
    counting.render_to(min(passes, 64))
    fetched = counting.fetch_counts()
    c = counting.counters()
    segments_counted = c["rays"] + c["shadow_rays"]
    bytes_per_segment = (64 * fetched["nodes"] + 16 * fetched["spheres"] + 48 * fetched["quads"] +
                         48 * fetched["triangles"]) / max(segments_counted, 1)
    counting.close()

    session = rt.Session(scene, seed=seed, launch_seconds=0.5)
    camera = scene_desc.camera
    # The wavefront's launch shape chosen by the library's autotuner on this view (untimed, before the warm-up)
    tuning = session.autotune()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step():
        session.set_camera(camera)
        return session.render_to(passes)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    times = []
    rays0 = session.counters()
    launches = 0
    kernel_launches = 0
    kernel_seconds = 0.0
    total_rays = 0
    total_shadow = 0
    for _ in range(args.steps):
        flush.fill_(1.0)  # evict L2 between steps
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record()
        report = step()
        torch.cuda.synchronize()
        end.record()
        end.synchronize()
        times.append(start.elapsed_time(end) / 1000.0)
        cnt = session.counters()
        total_rays += cnt["rays"]
        total_shadow += cnt["shadow_rays"]
        kernel_seconds += report["gpu_seconds"]
        launches += report["launches"]
        kernel_launches += report["kernel_launches"]
    clock_info = clocks.stop()
    del rays0
    timed_image = session.pixels()  # the last timed render (every step renders the same seed), for the parity check

    # Per-kernel times of the same workload (untimed: CUDA events around every kernel), for the roofline
    session.set_timing(True)
    session.set_camera(camera)
    profiled = session.render_to(passes)
    kernel_times = session.kernel_times()
    prof_counts = session.counters()
    session.set_timing(False)
    # the slowest rank's time, every rank's segments (no collective on the data path: each rank's image is its own)
    step_seconds, all_rays = shard.combine(sum(times), total_rays)
    value = all_rays / step_seconds

    peaks = read_peaks()
    fp32_peak = fp32_peak_tflops(torch)
    roofline = roofline_of(kernel_times, prof_counts, passes * scene.width * scene.height, fetched,
                           segments_counted, bytes_per_segment, peaks, fp32_peak, profiled["gpu_seconds"],
                           slot_rows=slot_rows_of(scene_desc.desc, session.kernel()["name"]))

    line = None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1000 * step_seconds / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": workload_config(args, scene_desc), "roofline": roofline, "clocks": clock_info,
                "gpu_launches": kernel_launches,
                "segments_per_sample": total_rays / (args.steps * passes * scene.width * scene.height),
                "shadow_rays_per_sample": total_shadow / (args.steps * passes * scene.width * scene.height),
                "kernel": session.kernel(), "scene_stats": stats, "autotune": tuning}
    session.close()
    del flush

    # e2e: the same metric through the public render() call, host tables in, host pixels out, copies inside
    if not args.no_e2e:
        e2e_steps = max(1, args.steps)
        out = np.empty((scene.height, scene.width, 3), dtype=np.float64)
        for w in range(max(1, args.warmup)):  # warm-up calls, as the timed steps have theirs
            rt.render(scene_desc, seed=seed + 100 + w, passes=passes, launch_seconds=0.5, out=out)
        e_seconds = 0.0
        e_rays = 0
        e_each = []
        for k in range(e2e_steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            start = torch.cuda.Event(enable_timing=True)
            end = torch.cuda.Event(enable_timing=True)
            start.record()
            res = rt.render(scene_desc, seed=seed + k, passes=passes, launch_seconds=0.5, out=out)
            torch.cuda.synchronize()
            end.record()
            end.synchronize()
            e_each.append(start.elapsed_time(end))
            e_seconds += e_each[-1] / 1000.0
            e_rays += res.rays
            del t0
        e_seconds, e_rays = shard.combine(e_seconds, e_rays)
        if rank == 0:
            line["e2e"] = {"value": e_rays / e_seconds, "unit": UNIT, "h2d_bytes_per_step": int(stats["device_bytes"]),
                           "d2h_bytes_per_step": int(out.nbytes),
                           "ms_per_step": 1000 * e_seconds / e2e_steps,
                           # each call's time: the host's share (scene build, teardown: about 7 ms) is the difference
                           # to the kernels' time; a call far above it met host interference
                           "ms_each": [round(x, 1) for x in e_each], "kernel_ms_last": round(1000 * res.kernel_seconds, 1),
                           "path": "raytracing_b200.render -> rt_render (validate, BVH build, upload, launches, "
                                   "download of width*height*3 doubles)"}

    # The other workloads' legs (NEE/MIS, the FP64 errors, the mesh, the served streams, the CPU baseline) run on rank 0
    # of a one-GPU run only: under torchrun they would hold the other ranks' GPUs idle in the closing barrier for
    # minutes, and the scaled metric is the image's alone
    single = world == 1
    mis = mis_image = mis_desc = None
    mis_passes = 0
    if rank == 0 and single and not args.no_mis:
        def run_mis():
            nonlocal mis, mis_image, mis_desc, mis_passes
            mis, mis_image, mis_desc, mis_passes = mis_measurement(rt, torch, args, max(1, min(args.steps, 3)), seed)
            return mis

        leg(line, "nee_mis", run_mis)

    if rank == 0 and not args.no_reference_gpu:
        def run_reference_gpu():
            ref = reference_gpu_measurement(scene_desc, passes, line["value"])
            ref_image = ref.pop("image", None)
            # Parity of the timed image at its full size: ImageCompare against the reference's own renderer (the
            # same scene tables, spp and strategy, another seed), and both images' error against the FP64 oracle
            if ref_image is not None:
                from oracle import ref_gpu

                w, h = scene.width, scene.height
                leg(line, "parity", lambda: {
                    "workload": line["config"]["workload"],
                    "image_compare_vs_reference": image_parity(
                        lambda sd: ref_image if sd == 6 else ref_gpu.render(scene_desc.desc, w, h, seed=sd,
                                                                             passes=passes)[0], timed_image),
                    "error_vs_fp64": error_vs_fp64(args.scene, {"this_library": timed_image,
                                                                "reference_gpu": ref_image})})
                if mis is not None and mis_image is not None:
                    def run_mis_parity():
                        mis_ref_fn = lambda sd: ref_gpu.render(mis_desc.desc, mis_desc.width,  # noqa: E731
                                                               mis_desc.height, seed=sd, passes=mis_passes)[0]
                        mis_ref = mis_ref_fn(8)
                        return {"image_compare_vs_reference": image_parity(
                                    lambda sd: mis_ref if sd == 8 else mis_ref_fn(sd), mis_image, seeds=(8, 9)),
                                "error_vs_fp64": error_vs_fp64(args.scene, {"this_library": mis_image,
                                                                            "reference_gpu": mis_ref})}

                    leg(mis, "parity", run_mis_parity)
            return ref

        leg(line, "reference_gpu", run_reference_gpu)
    if rank == 0 and single and not args.no_reference_gpu:
        leg(line, "error_vs_fp64_by_config", lambda: config_errors(rt, seed))
    if rank == 0 and single and not args.no_mesh:
        leg(line, "mesh", lambda: mesh_measurement(rt, torch, peaks))
    if not args.no_batched:
        if single:
            leg(line, "batched", lambda: batched_measurement(rt, torch, rank, world))
        else:
            # every rank its share of the 64 jobs, with collectives inside: not guarded, so that no rank leaves them
            batched = batched_measurement(rt, torch, rank, world)
            if rank == 0:
                line["batched"] = batched
    if rank == 0 and single and not args.no_served:
        def run_served():
            served = served_measurement(rt, torch, args)
            if args.served_long_window > 0:
                served["long_stream"] = served_first_frames(rt, args)
                batched_long = served_first_frames(rt, args, continuous=False)
                served["long_stream"]["batched_server"] = {
                    k: batched_long[k] for k in ("ttff_p50_s", "ttff_p99_s", "ttff_max_s", "ttff_by_resolution",
                                                 "reached_target", "time_to_target_p50_s", "gpu_s", "wall_s",
                                                 "steps", "longest_steps")}
            return served

        leg(line, "served", run_served)

    if rank == 0 and single and not args.no_cpu_baseline:
        leg(line, "cpu_baseline", lambda: cpu_baseline(scene_desc, args, os.cpu_count() or 1))
    if rank == 0 and not single:
        line["single_gpu_legs"] = "nee_mis, error_vs_fp64_by_config, mesh, served and cpu_baseline are measured in the " \
                                  "one-GPU run"

    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
