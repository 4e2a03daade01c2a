"""The wavefront autotuner's search, on the CPU: the library's own coordinate descent (csrc/tuner.cpp) driven by a
synthetic speed model instead of GPU renders.

* With a separable model it finds the best value of every knob: the trace kernel's register cap and grid, the slot
  pool, the shade kernel's block size.
* It keeps the defaults when no candidate is more than 1% faster (a trial's noise), and never proposes more trace
  blocks a multiprocessor than the kernel's occupancy allows.
"""
import raytracing_b200 as rt

DEFAULT = {"slots": 1 << 20, "trace_blocks_per_sm": 8, "shade_block": 128, "trace_min_blocks": 8}


def _shape(s):
    return {k: s[k] for k in DEFAULT}


def test_finds_the_best_of_every_knob():
    trace_gain = {(8, 10): 1.00, (8, 8): 1.05, (8, 6): 0.97, (8, 4): 0.9, (6, 6): 1.12, (6, 4): 1.0}
    slot_gain = {1 << 19: 0.8, 1 << 20: 1.0, 3 << 19: 1.04, 1 << 21: 1.09, 3 << 20: 1.07}
    block_gain = {128: 1.0, 64: 1.03}
    seen = []

    def measure(s):
        seen.append(dict(s))
        assert s["trace_blocks_per_sm"] <= (10 if s["trace_min_blocks"] == 8 else 6)
        return 1e9 * trace_gain[(s["trace_min_blocks"], s["trace_blocks_per_sm"])] * slot_gain[s["slots"]] * \
            block_gain[s["shade_block"]]

    t = rt.autotune_simulate(measure, max_trace_blocks=10, max_trace_blocks_roomy=6)
    assert (t["trace_min_blocks"], t["trace_blocks_per_sm"]) == (6, 6)
    assert t["slots"] == 1 << 21 and t["shade_block"] == 64
    assert t["samples_per_second"] == measure(t)
    assert t["default_samples_per_second"] == 1e9 * 1.05
    assert _shape(seen[0]) == DEFAULT  # the built-in defaults are measured first
    # 1 default + 5 other trace shapes + 4 other slot pools + 1 other block size
    assert t["trials"] == 11 == len(seen) - 1


def test_keeps_the_defaults_within_noise():
    def measure(s):
        return 1e9 * (1.0 if _shape(s) == DEFAULT else 1.009)

    t = rt.autotune_simulate(measure)
    assert _shape(t) == DEFAULT
    assert t["samples_per_second"] == t["default_samples_per_second"] == 1e9


def test_respects_the_occupancy_of_each_register_cap():
    shapes = []
    rt.autotune_simulate(lambda s: shapes.append(dict(s)) or 1e9, max_trace_blocks=5, max_trace_blocks_roomy=3)
    assert all(s["trace_blocks_per_sm"] <= (5 if s["trace_min_blocks"] == 8 else 3) for s in shapes)
    assert {(s["trace_min_blocks"], s["trace_blocks_per_sm"]) for s in shapes} == {(8, 5), (8, 4), (6, 3)}
