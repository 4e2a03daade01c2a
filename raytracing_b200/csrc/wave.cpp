// The wavefront's host side, shared by sessions and the batch engine: its buffers (grown to the launch, never shrunk)
// and the loop of steps that ends when a step queues no ray.
#include <algorithm>
#include <functional>
#include <map>
#include <mutex>
#include <vector>

#include "host.h"

namespace rtb
{
void retain_pool_memory()
{
    int device = 0;
    check(cudaGetDevice(&device), "querying the device");
    cudaMemPool_t pool = nullptr;
    check(cudaDeviceGetDefaultMemPool(&pool, device), "querying the memory pool");
    uint64_t keep = UINT64_MAX;
    check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "setting the memory pool");
}

namespace
{
std::mutex pinned_mutex;
std::map<size_t, std::vector<void*>>& pinned_free()
{
    static auto* blocks = new std::map<size_t, std::vector<void*>>(); // lives to the process's end, as the blocks do
    return *blocks;
}
} // namespace

void* acquire_pinned(size_t bytes)
{
    {
        const std::lock_guard<std::mutex> lock(pinned_mutex);
        auto& list = pinned_free()[bytes];
        if (!list.empty())
        {
            void* block = list.back();
            list.pop_back();
            return block;
        }
    }
    void* block = nullptr;
    check(cudaHostAlloc(&block, bytes, cudaHostAllocDefault), "allocating pinned memory");
    return block;
}

void release_pinned(void* block, size_t bytes)
{
    if (block)
    {
        const std::lock_guard<std::mutex> lock(pinned_mutex);
        pinned_free()[bytes].push_back(block);
    }
}

cudaStream_t allocation_stream()
{
    static std::mutex mutex;
    static auto* streams = new std::map<int, cudaStream_t>(); // one per device, to the process's end
    int device = 0;
    check(cudaGetDevice(&device), "querying the device");
    const std::lock_guard<std::mutex> lock(mutex);
    const auto it = streams->find(device);
    if (it != streams->end())
    {
        return it->second;
    }
    cudaStream_t s = nullptr;
    check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "creating a CUDA stream");
    retain_pool_memory();
    (*streams)[device] = s;
    return s;
}

wave_runner::wave_runner(int max_slots_, int group_) : max_slots(max_slots_), group(group_) { retain_pool_memory(); }

wave_runner::~wave_runner()
{
    // the blocks go back to the cache once no copy into them is in flight (each group's readback records done_)
    for (auto& e : done_)
    {
        if (e)
        {
            cudaEventSynchronize(e);
            cudaEventDestroy(e);
        }
    }
    release_pinned(queued_, 8 * sizeof(unsigned));
    release_pinned(claimed_, 2 * sizeof(unsigned long long));
}

wave_buffers wave_runner::setup(int64_t samples, cudaStream_t stream)
{
    if (!queued_)
    {
        queued_ = static_cast<unsigned*>(acquire_pinned(8 * sizeof(unsigned)));
        claimed_ = static_cast<unsigned long long*>(acquire_pinned(2 * sizeof(unsigned long long)));
        for (auto& e : done_)
        {
            check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "creating a CUDA event");
        }
        control_.allocate_async(4, stream);
    }
    if (samples >= (int64_t{1} << 32))
    {
        fail(RT_ERR_CAPACITY, "a wavefront run holds fewer than 2^32 samples (a slot keeps its sample's number in 32 bits)");
    }
    const int64_t wanted = (samples + render_block - 1) / render_block * render_block;
    const auto n = static_cast<size_t>(std::min<int64_t>(max_slots, std::max<int64_t>(wanted, render_block)));
    // grown by doubling, never shrunk: a stream of launches of growing size reallocates a few times, not every time
    if (ext_result_.size() < n)
    {
        const size_t c = std::min<size_t>(static_cast<size_t>(max_slots), std::max(n, 2 * ext_result_.size()));
        slots_.allocate_async(c * wave_slot_bytes(), stream);
        query_o_.allocate_async(2 * c, stream);
        query_d_.allocate_async(2 * c, stream);
        query_meta_.allocate_async(2 * c, stream);
        ext_result_.allocate_async(c, stream);
        shadow_result_.allocate_async(c, stream);
    }
    if (samples_.size() < static_cast<size_t>(samples))
    {
        samples_.allocate_async(std::max(static_cast<size_t>(samples), 2 * samples_.size()), stream);
    }
    wave_buffers b{};
    b.slots = slots_.data();
    b.slot_count = static_cast<int32_t>(n);
    b.samples = samples_.data();
    b.sample_count = samples;
    b.query_o = query_o_.data();
    b.query_d = query_d_.data();
    b.query_meta = query_meta_.data();
    b.ext_result = ext_result_.data();
    b.shadow_result = shadow_result_.data();
    b.control = control_.data();
    return b;
}

int64_t wave_runner::run(const wave_buffers& b, int max_depth, cudaStream_t stream,
                         const std::function<cudaError_t(bool draining)>& step, const unsigned long long* work_counter)
{
    check(clear_wave_slots(b, stream), "clearing the path slots");
    // A sample takes at most max_depth + 1 steps (its segments, then the one that adds its last shadow ray) and a slot
    // renders at most its share of the samples one after another: twice that bounds a launch that works
    const int64_t samples_per_slot = (b.sample_count + b.slot_count - 1) / b.slot_count;
    const int64_t step_limit = 2 * (samples_per_slot * (max_depth + 2) + 4 * group);
    // Groups of steps, two in flight: the host reads one group's queue length while the next group runs; a group
    // after the end finds every slot out of work and costs a few microseconds a step
    int64_t steps = 0;
    bool draining = false;
    for (int g = 0;; ++g)
    {
        for (int s = 0; s < group; ++s)
        {
            check(step(draining), "launching a wavefront step");
        }
        steps += group;
        const int k = g & 1;
        check(cudaMemcpyAsync(queued_ + 4 * k, b.control, 3 * sizeof(unsigned), cudaMemcpyDeviceToHost, stream),
              "reading the queue's length");
        if (work_counter)
        {
            check(cudaMemcpyAsync(claimed_ + k, work_counter, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                  stream),
                  "reading the work counter");
        }
        check(cudaEventRecord(done_[k], stream), "recording a CUDA event");
        if (g > 0)
        {
            check(cudaEventSynchronize(done_[k ^ 1]), "rendering on the GPU");
            const unsigned* q = queued_ + 4 * (k ^ 1);
            if (q[0] + q[2] == 0) // no next ray, shadow ray or camera ray queued
            {
                break;
            }
            draining = draining || (work_counter && claimed_[k ^ 1] >= static_cast<unsigned long long>(b.sample_count));
        }
        if (steps > step_limit)
        {
            fail(RT_ERR_RUNTIME, "the wavefront's paths did not finish within their steps");
        }
    }
    return steps;
}
} // namespace rtb
