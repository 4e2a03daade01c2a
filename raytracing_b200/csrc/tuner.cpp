// The wavefront's autotuner: how a session's steps are launched (the slot pool, which is the query queue's capacity;
// the trace kernel's register cap and grid; the shade kernel's block size), chosen by measuring short renders of the
// session's own view, one knob after another (coordinate descent from the built-in defaults), and remembered per
// device and scene class for the sessions that come after.
//
// No counterpart in the reference, whose launch planner (src/gpu/renderer.cu:201-308) sizes launches from measured
// row times but never the kernels' shapes.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>

#include "host.h"

namespace rtb
{
namespace
{
std::mutex cache_mutex;
std::map<std::tuple<int, int, int, int, int, int, int>, tune_candidate> cache;

// A candidate replaces the best so far only when it is measurably faster: a trial's noise is about 1%
constexpr double improvement = 1.01;
} // namespace

tune_space default_tune_space(int max_trace_blocks, int max_trace_blocks_roomy)
{
    tune_space s;
    // the default cap at its own occupancy and below it, then the roomier cap (more registers a thread, fewer blocks)
    for (const int b : {max_trace_blocks, 8, 6, 4})
    {
        const std::pair<int, int> t{RTB_TRACE_MIN_BLOCKS_DEFAULT, b};
        if (b >= 1 && b <= max_trace_blocks && std::find(s.trace.begin(), s.trace.end(), t) == s.trace.end())
        {
            s.trace.push_back(t);
        }
    }
    for (const int b : {max_trace_blocks_roomy, 4})
    {
        const std::pair<int, int> t{wave_trace_roomy_blocks, b};
        if (b >= 1 && b <= max_trace_blocks_roomy && std::find(s.trace.begin(), s.trace.end(), t) == s.trace.end())
        {
            s.trace.push_back(t);
        }
    }
    s.slots = {1 << 19, 1 << 20, 3 << 19, 1 << 21, 3 << 20};
    s.shade_blocks = {render_block, render_block / 2};
    return s;
}

tune_candidate default_candidate(int slots, int max_trace_blocks)
{
    return {slots, std::min(RTB_TRACE_MIN_BLOCKS_DEFAULT, std::max(1, max_trace_blocks)), render_block,
            RTB_TRACE_MIN_BLOCKS_DEFAULT};
}

rt_tuning to_tuning(const tune_candidate& c)
{
    rt_tuning t{};
    t.slots = c.slots;
    t.trace_blocks_per_sm = c.trace_blocks_per_sm;
    t.shade_block = c.shade_block;
    t.trace_min_blocks = c.trace_min_blocks;
    return t;
}

tune_outcome coordinate_descent(const tune_candidate& start, const tune_space& space,
                                const std::function<double(const tune_candidate&)>& measure)
{
    tune_outcome out{};
    out.best = start;
    out.default_speed = measure(start);
    out.best_speed = out.default_speed;
    out.trials = 1;
    const auto consider = [&](const tune_candidate& c) {
        if (c.slots == out.best.slots && c.trace_blocks_per_sm == out.best.trace_blocks_per_sm &&
            c.shade_block == out.best.shade_block && c.trace_min_blocks == out.best.trace_min_blocks)
        {
            return;
        }
        const double speed = measure(c);
        ++out.trials;
        if (speed > improvement * out.best_speed)
        {
            out.best = c;
            out.best_speed = speed;
        }
    };
    // 1. the trace kernel: its register cap and how many of its blocks share a multiprocessor
    for (const auto& [min_blocks, blocks] : space.trace)
    {
        tune_candidate c = out.best;
        c.trace_min_blocks = min_blocks;
        c.trace_blocks_per_sm = blocks;
        consider(c);
    }
    // 2. the slot pool (the paths in flight; the query queue holds two queries a slot)
    const tune_candidate after_trace = out.best;
    for (const int slots : space.slots)
    {
        tune_candidate c = after_trace;
        c.slots = slots;
        consider(c);
    }
    // 3. the shade kernel's block size
    const tune_candidate after_slots = out.best;
    for (const int block : space.shade_blocks)
    {
        tune_candidate c = after_slots;
        c.shade_block = block;
        consider(c);
    }
    return out;
}

std::tuple<int, int, int, int, int, int, int> tune_key(int device, const scene_view& v, bool quality)
{
    const bool triangles = v.prim_count > v.triangle_base;
    const int size = v.prim_count > 0 ? static_cast<int>(std::log2(static_cast<double>(v.prim_count))) : 0;
    return {device, v.flat != 0, quality, has_features(v), v.wide_nodes != nullptr, triangles, size};
}

bool cached_tuning(const std::tuple<int, int, int, int, int, int, int>& key, tune_candidate& out)
{
    std::lock_guard<std::mutex> lock(cache_mutex);
    const auto it = cache.find(key);
    if (it == cache.end())
    {
        return false;
    }
    out = it->second;
    return true;
}

void remember_tuning(const std::tuple<int, int, int, int, int, int, int>& key, const tune_candidate& c)
{
    std::lock_guard<std::mutex> lock(cache_mutex);
    cache[key] = c;
}

void forget_tunings()
{
    std::lock_guard<std::mutex> lock(cache_mutex);
    cache.clear();
}
} // namespace rtb

extern "C" {

rt_status rt_autotune_simulate(int32_t max_trace_blocks, int32_t max_trace_blocks_roomy, rt_tune_measure_fn measure,
                               void* user, rt_tuning* result)
{
    try
    {
        if (!measure || !result)
        {
            rtb::fail(RT_ERR_INVALID, "measure and result must not be null");
        }
        const rtb::tune_space space = rtb::default_tune_space(max_trace_blocks, max_trace_blocks_roomy);
        const rtb::tune_outcome o = rtb::coordinate_descent(rtb::default_candidate(1 << 20, max_trace_blocks), space,
                                                            [&](const rtb::tune_candidate& c) {
                                                                const rt_tuning t = rtb::to_tuning(c);
                                                                return measure(&t, user);
                                                            });
        *result = rtb::to_tuning(o.best);
        result->trials = o.trials;
        result->samples_per_second = o.best_speed;
        result->default_samples_per_second = o.default_speed;
        return RT_OK;
    }
    catch (const rtb::rt_error& e)
    {
        rtb::remember_error(e.what());
        return e.status;
    }
    catch (const std::exception& e)
    {
        rtb::remember_error(e.what());
        return RT_ERR_RUNTIME;
    }
}
}
