"""bench.py's own logic without a GPU: the roofline's arithmetic, the slot layout it counts bytes by, the CPU legs'
band of rows, the error statistic, the batched and served workloads' generators, the reference arm's JSON line
(the oracle on a small image, on the CPU), and a failing auxiliary leg recorded in the line instead of ending the run."""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import bench

REPO = Path(__file__).resolve().parent.parent


def test_shade_bytes_follow_the_slot_rows():
    # rows in and out, the walk's answer (16 B) and the next query (48 B)
    assert bench.shade_bytes_per_segment(3) == 160
    assert bench.shade_bytes_per_segment(4) == 192
    assert bench.shade_bytes_per_segment(5) == 224
    # a shadow ray: its answer, its three rows out and back in, its query
    assert bench.SHADE_BYTES_PER_SHADOW_RAY == 148


@pytest.mark.parametrize("name, kernel, rows", [
    ("glass", "wavefront books", 3),
    ("glass", "wavefront nee-mis", 4),
    ("cornell-mis", "wavefront nee-mis", 4),
    ("glass", "persistent books", 5),
    ("final", "wavefront books", 5),      # moving spheres, textures and smoke: the full slot
    ("perlin", "wavefront books", 5),     # a marble texture
    ("bouncing", "wavefront books", 5),   # moving spheres
    ("smoke", "wavefront nee-mis", 5),    # constant media
])
def test_slot_rows_of_scenes(rt, name, kernel, rows):
    s = rt.builtin_scene(name, width=32, spp=1)
    assert bench.slot_rows_of(s.desc, kernel) == rows


def _times(shade, trace, reduce_=0.001):
    # (seconds, launches) per kernel kind, as the session's per-kernel timing reports them
    return {"shade": (shade, 100), "trace": (trace, 100), "reduce": (reduce_, 4), "render": (0.0, 0)}


FETCHED = {"nodes": 0, "spheres": 400, "quads": 900, "triangles": 0}


def test_roofline_of_a_shade_bound_render():
    counts = {"rays": 2_000_000_000, "shadow_rays": 0}
    samples = 600 * 600 * 1024
    r = bench.roofline_of(_times(0.12, 0.06), counts, samples, FETCHED, 100, 592.0, {"hbm_gbs": 6500.0,
                          "source": "measured"}, 60.0, 0.2, slot_rows=3)
    state = counts["rays"] * 160 + samples * 16
    assert r["bound"] == "hbm" and r["kernel"] == "wave_shade_kernel" and r["unit"] == "GB/s"
    assert r["achieved"] == pytest.approx(state / 0.12 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / 6500.0)
    assert r["algorithmic_bytes_per_segment"] == pytest.approx(state / counts["rays"])
    assert r["algorithmic_bytes_per_launch"] == pytest.approx(state / 100)
    assert r["traffic"] is None and r["peak_source"] == "measured"
    # the trace kernel beside it, against the FP32 peak: flops per query from the counting build's visits
    flops = (20 * 400 + 25 * 900) / 100
    assert r["trace_kernel"]["flops_per_query"] == pytest.approx(flops)
    assert r["trace_kernel"]["achieved"] == pytest.approx(flops * counts["rays"] / 0.06 / 1e12)
    # kernels with no launches are left out; the shares add to one
    assert set(r["kernels"]) == {"shade", "trace", "reduce"}
    assert sum(k["share"] for k in r["kernels"].values()) == pytest.approx(1.0)
    assert r["events_total_over_render"] == pytest.approx(0.181 / 0.2)


def test_roofline_of_a_trace_bound_render_is_fp32():
    counts = {"rays": 10**9, "shadow_rays": 5 * 10**8}
    r = bench.roofline_of(_times(0.02, 0.09), counts, 10**6, FETCHED, 100, 592.0, {"hbm_gbs": 6500.0,
                          "source": "fallback"}, 60.0, 0.12)
    assert r["bound"] == "fp32" and r["kernel"] == "trace" and r["unit"] == "TFLOP/s"
    queries = counts["rays"] + counts["shadow_rays"]
    assert r["achieved"] == pytest.approx((20 * 400 + 25 * 900) / 100 * queries / 0.09 / 1e12)
    assert r["frac"] == pytest.approx(r["achieved"] / 60.0)
    assert r["traffic"] is None


@pytest.mark.parametrize("height, threads, per_thread", [
    (600, 16, 2), (600, 16, 40), (600, 16, 1000), (600, 7, 90), (225, 16, 1), (225, 64, 5), (10, 16, 3), (1, 4, 1),
    (600, 16, 0),
])
def test_row_band_is_whole_rows_a_thread(height, threads, per_thread):
    begin, rows = bench.row_band(height, threads, per_thread)
    assert 0 <= begin and begin + rows <= height and rows >= 1
    if height >= threads:
        assert rows % threads == 0
        assert rows == threads * min(max(per_thread, 1), height // threads)
    else:
        assert rows == height
    # centred on the middle row
    assert abs((begin + rows / 2) - height / 2) <= 1


def test_trimmed_rms():
    rng = np.random.default_rng(3)
    a = rng.random((40, 50, 3))
    assert bench.trimmed_rms(a, a) == (0.0, 0.0)
    b = a + 0.01
    t, full = bench.trimmed_rms(a, b)
    assert t == pytest.approx(0.01) and full == pytest.approx(0.01)
    # one firefly: the full RMS sees it, the 1% trim leaves it out
    c = b.copy()
    c[7, 9] += 100.0
    t2, full2 = bench.trimmed_rms(a, c)
    assert t2 == pytest.approx(0.01) and full2 > 1.0


def test_batched_jobs_are_the_stated_distribution(rt):
    jobs = bench.batched_jobs(rt, count=12)
    again = bench.batched_jobs(rt, count=12)
    assert [j[1] for j in jobs] == list(range(12))
    for (s, j, spp), (s2, j2, spp2) in zip(jobs, again):
        assert (s.width, s.height, spp) == (s2.width, s2.height, spp2)
        assert 64 <= s.width <= 1024 and 64 <= s.height <= 1024 and 16 <= spp <= 1024


def test_served_requests_are_poisson_arrivals_in_the_window(rt):
    reqs = bench.served_requests(rt, 200.0, 0.25)
    assert reqs == [] or reqs[-1]["arrival"] <= 0.25
    arrivals = [r["arrival"] for r in reqs]
    assert arrivals == sorted(arrivals) and len(reqs) > 20
    sizes = {(w, h) for (w, h), _ in bench.SERVED_RESOLUTIONS}
    for k, r in enumerate(reqs):
        assert r["scene"] in bench.SERVED_SCENES and 1 <= r["target"] <= 4096 and r["seed"] == k + 1
        assert (r["camera"].image_width, r["camera"].image_height) in sizes
    again = bench.served_requests(rt, 200.0, 0.25)
    assert [(r["arrival"], r["scene"], r["target"]) for r in again] == [(r["arrival"], r["scene"], r["target"])
                                                                        for r in reqs]


def _run_reference(extra_env=None):
    env = dict(os.environ)
    env.update(extra_env or {})
    return subprocess.run([sys.executable, str(REPO / "bench.py"), "--impl", "reference", "--steps", "2", "--warmup",
                           "1", "--width", "24", "--spp", "4", "--depth", "8"], capture_output=True, text=True,
                          env=env, cwd=REPO, timeout=300)


def test_reference_arm_prints_one_line_of_the_contract():
    out = _run_reference()
    assert out.returncode == 0, out.stderr
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["higher_is_better"] is True and line["steps"] == 2 and line["warmup"] == 1
    assert line["value"] > 0 and line["ms_per_step"] > 0
    assert line["config"]["width"] == 24 and line["config"]["spp"] == 4
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_without_work():
    out = _run_reference({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert out.returncode == 0, out.stderr
    assert not [ln for ln in out.stdout.splitlines() if ln.startswith("{")]


def test_a_failing_leg_is_recorded_and_the_rest_still_run():
    line = {"value": 1.0}

    def broken():
        raise RuntimeError("the reference renderer is not built")

    bench.leg(line, "reference_gpu", broken)
    bench.leg(line, "mesh", lambda: {"segments_per_s": 2.0})
    assert line["reference_gpu"] == {"error": "RuntimeError: the reference renderer is not built"}
    assert line["mesh"] == {"segments_per_s": 2.0}
    assert json.loads(json.dumps(line)) == line  # the line still prints as JSON
