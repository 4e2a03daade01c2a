// The server's continuous wavefront (no counterpart in the reference, whose one session renders one view,
// src/gpu/renderer.h:585-590): one pool of path slots that lives as long as the server, into which the requests'
// samples are published as they are scheduled, so that no refinement step ends with a drain of its last paths while
// the rest of the GPU idles.
//
// * Samples. Each request's samples are numbered pass-major within the request (its pixels in 8x4 tiles); the host
//   publishes them in segments, each a contiguous range of one request's numbers mapped to a contiguous range of the
//   run's sample space, and raises the published limit. The shade kernel's slots claim samples up to that limit (a
//   claim beyond it waits in its slot until it is published). A first frame is published the moment its request is
//   added; refinement only while the unclaimed backlog is short (`lookahead_seconds_` of the measured claim rate,
//   or three groups' worth if more), so that a first frame waits behind little and the pool does not starve.
// * Segments sit in a ring of job-table entries; each writes its samples' values to its own range of a ring of values
//   and counts its finished samples. After every group of steps the host reads the counts; a request's finished
//   segments are reduced in order (stream_reduce_kernel, on a stream of their own, beside the next group: pixel by
//   pixel, pass after pass, into the request's chunk accumulator, which goes into its sums at every chunk's end,
//   after its first pass and at its target), and their entries and values are reused by later groups only.
// * Steps run in groups of group_steps_, two groups in flight: the host reads one group's counts while the next runs.
//
// A request's image equals a session's of the same view and seed rendered first to one pass, then to its target
// (the same samples; the first chunk's sum split after the first pass). Flat-searched scenes are walked through their
// tree here, as the run's one trace kernel walks every scene: the same closest hits up to the order of exact ties.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "batch.h"

namespace rtb
{
namespace
{
constexpr int segment_ring = 4096;                  // job-table entries (segments in flight), a power of two
constexpr int64_t piece_samples = int64_t{1} << 21; // a refinement segment's samples at most
} // namespace

stream_engine::stream_engine(int slots, int64_t value_capacity, int group_steps, double lookahead_seconds)
    : slot_count_(slots), value_capacity_(value_capacity), group_steps_(group_steps),
      lookahead_seconds_(lookahead_seconds)
{
    if (slots <= 0 || slots % render_block != 0 || value_capacity <= 0 || group_steps < 1)
    {
        fail(RT_ERR_INVALID, "the stream engine needs a positive multiple of 128 slots, a values ring and steps");
    }
    retain_pool_memory();
    check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "creating a CUDA stream");
    check(cudaStreamCreateWithFlags(&reduce_stream_, cudaStreamNonBlocking), "creating a CUDA stream");
    for (int k = 0; k < 2; ++k)
    {
        check(cudaEventCreate(&group_start_[k]), "creating a CUDA event");
        check(cudaEventCreate(&group_done_[k]), "creating a CUDA event");
    }
    check(cudaEventCreateWithFlags(&reduced_, cudaEventDisableTiming), "creating a CUDA event");
    const size_t n = static_cast<size_t>(slot_count_);
    slots_.allocate_async(n * wave_slot_bytes(), stream_);
    query_o_.allocate_async(2 * n, stream_);
    query_d_.allocate_async(2 * n, stream_);
    query_meta_.allocate_async(2 * n, stream_);
    ext_result_.allocate_async(n, stream_);
    shadow_result_.allocate_async(n, stream_);
    control_.allocate_async(4, stream_);
    counters_.allocate_async(3, stream_); // [0] samples claimed, [1] samples published, [2] the segments' window
    table_.allocate_async(segment_ring, stream_);
    done_.allocate_async(segment_ring, stream_);
    starts_.allocate_async(segment_ring, stream_);
    values_.allocate_async(static_cast<size_t>(value_capacity_), stream_);
    check(cudaMemsetAsync(counters_.data(), 0, counters_.bytes(), stream_), "clearing the stream's counters");
    check(cudaMemsetAsync(done_.data(), 0, done_.bytes(), stream_), "clearing the segments' counts");
    check(cudaMemsetAsync(control_.data(), 0, control_.bytes(), stream_), "clearing the queue");
    check(cudaMemsetAsync(table_.data(), 0, table_.bytes(), stream_), "clearing the segment table");
    check(cudaMemsetAsync(starts_.data(), 0, starts_.bytes(), stream_), "clearing the segment starts");
    check(cudaHostAlloc(reinterpret_cast<void**>(&readback_), 2 * readback_bytes(), cudaHostAllocDefault),
          "allocating pinned memory");
    check(cudaHostAlloc(reinterpret_cast<void**>(&staging_), 2 * sizeof(group_control), cudaHostAllocDefault),
          "allocating pinned memory");
    table_host_.resize(segment_ring);
    segments_.resize(segment_ring);
    buffers_ = wave_buffers{};
    buffers_.slots = slots_.data();
    buffers_.slot_count = slot_count_;
    buffers_.samples = nullptr;
    buffers_.sample_count = 0;
    buffers_.query_o = query_o_.data();
    buffers_.query_d = query_d_.data();
    buffers_.query_meta = query_meta_.data();
    buffers_.ext_result = ext_result_.data();
    buffers_.shadow_result = shadow_result_.data();
    buffers_.control = control_.data();
    check(clear_wave_slots(buffers_, stream_), "clearing the path slots");
    check(preload_wave_batch(), "loading the wavefront's kernels");
    kernel_attributes shade{}, trace{};
    scene_view tree{};
    tree.node_count = 1;
    check(wave_attributes(tree, false, shade, trace), "querying the wavefront kernels");
    trace_grid_ = trace.multiprocessors * std::max(1, trace.blocks_per_sm);
    // every group graph captured now, not while requests wait
    for (int v = 0; v < 4; ++v)
    {
        features_ = (v & 2) != 0;
        wide_ = (v & 1) != 0;
        group_graph(0);
        group_graph(1);
    }
    features_ = false;
    wide_ = true;
    check(cudaStreamSynchronize(stream_), "setting up the stream engine");
}

stream_engine::~stream_engine()
{
    cudaStreamSynchronize(stream_);
    cudaStreamSynchronize(reduce_stream_);
    requests_.clear();
    slots_.release();
    query_o_.release();
    query_d_.release();
    query_meta_.release();
    ext_result_.release();
    shadow_result_.release();
    control_.release();
    counters_.release();
    table_.release();
    done_.release();
    starts_.release();
    values_.release();
    reduce_items_.release();
    rgba_.release();
    cudaStreamSynchronize(stream_);
    cudaStreamSynchronize(reduce_stream_);
    for (auto& g : graphs_)
    {
        if (g)
        {
            cudaGraphExecDestroy(g);
        }
    }
    if (readback_)
    {
        cudaFreeHost(readback_);
    }
    if (staging_)
    {
        cudaFreeHost(staging_);
    }
    for (int k = 0; k < 2; ++k)
    {
        cudaEventDestroy(group_start_[k]);
        cudaEventDestroy(group_done_[k]);
    }
    cudaEventDestroy(reduced_);
    cudaStreamDestroy(reduce_stream_);
    cudaStreamDestroy(stream_);
}

void stream_engine::reserve_pool(size_t bytes)
{
    // an allocation and its release: the pool keeps the memory (its release threshold is the maximum)
    void* p = nullptr;
    check(cudaMallocAsync(&p, bytes, stream_), "growing the memory pool");
    check(cudaFreeAsync(p, stream_), "growing the memory pool");
    check(cudaStreamSynchronize(stream_), "growing the memory pool");
}

size_t stream_engine::readback_bytes() { return 16 + 16 + segment_ring * sizeof(unsigned long long); }

size_t stream_engine::job_bytes(const rt_camera_desc& camera)
{
    // the sums and the chunk accumulator, 24 bytes a pixel each, and the counters
    return static_cast<size_t>(camera.image_width) * static_cast<size_t>(camera.image_height) * 6 * sizeof(double) +
           2 * sizeof(unsigned long long);
}

int stream_engine::add(std::shared_ptr<resident_scene> scene, const rt_camera_desc& camera, uint64_t seed,
                       uint32_t job_id, int64_t target, bool first_pass_elsewhere)
{
    if (target < 1)
    {
        fail(RT_ERR_INVALID, "a request needs at least one pass");
    }
    if (camera.sampling != scene->camera().sampling)
    {
        fail(RT_ERR_INVALID, "a request must keep its scene's sampling strategy");
    }
    if (scene->view().node_count == 0)
    {
        fail(RT_ERR_INVALID, "the stream engine renders scenes with a tree (every scene with a primitive)");
    }
    const camera_params cam = to_camera(camera); // checks the camera
    auto r = std::make_unique<request>();
    r->scene = std::move(scene);
    r->camera = camera;
    r->cam = cam;
    r->seed = seed;
    r->id = job_id;
    r->target = target;
    r->tiles_x = (camera.image_width + 7) / 8;
    r->padded = int64_t{(camera.image_height + 3) / 4} * r->tiles_x * 32;
    if (r->padded * target >= (int64_t{1} << 62))
    {
        fail(RT_ERR_INVALID, "the request's samples overflow the run's numbering");
    }
    const size_t px = static_cast<size_t>(camera.image_width) * static_cast<size_t>(camera.image_height);
    r->sums.allocate_async(px * 3, stream_);
    r->acc.allocate_async(px * 3, stream_);
    r->counters.allocate_async(2, stream_);
    check(cudaMemsetAsync(r->sums.data(), 0, r->sums.bytes(), stream_), "clearing the sums");
    check(cudaMemsetAsync(r->acc.data(), 0, r->acc.bytes(), stream_), "clearing the accumulator");
    check(cudaMemsetAsync(r->counters.data(), 0, r->counters.bytes(), stream_), "clearing the counters");
    const int handle = next_handle_++;
    if (camera.max_depth == 0)
    {
        r->published = r->reduced = r->padded * target; // a path of no rays: every sample is 0
        r->passes = target;
    }
    else if (first_pass_elsewhere)
    {
        r->awaiting_first = true;
    }
    else
    {
        fresh_.push_back(handle);
    }
    requests_[handle] = std::move(r);
    return handle;
}

void stream_engine::first_pass_done(int handle)
{
    request& r = *requests_.at(handle);
    if (!r.awaiting_first)
    {
        return; // a request of no rays: its passes were complete at admission
    }
    // the sums hold pass 0, the accumulator is clear: the next flush is at the first chunk's end
    r.awaiting_first = false;
    r.published = r.reduced = r.padded;
    r.passes = 1;
}

void stream_engine::remove(int handle)
{
    const auto it = requests_.find(handle);
    if (it == requests_.end())
    {
        return;
    }
    request& r = *it->second;
    r.cancelled = true; // nothing more of it is published
    fresh_.erase(std::remove(fresh_.begin(), fresh_.end(), handle), fresh_.end());
    // its segments in flight finish first: their samples write into its memory, their reductions read it
    while (!r.segments.empty())
    {
        advance(0.0);
    }
    check(cudaStreamSynchronize(reduce_stream_), "finishing the request's reductions");
    check(cudaStreamSynchronize(stream_), "finishing the request's work");
    requests_.erase(it);
}

// Contiguous room for `count` values in the ring (segments are retired in the order they were published, so the used
// part runs from the oldest live segment's offset to the head, wrapping at most once); -1 if there is none now
int64_t stream_engine::value_room(int64_t count) const
{
    if (oldest_segment_ == next_segment_)
    {
        return count <= value_capacity_ ? 0 : -1;
    }
    const int64_t tail = segments_[static_cast<size_t>(oldest_segment_ & (segment_ring - 1))].value_offset;
    if (value_head_ > tail)
    {
        if (value_capacity_ - value_head_ >= count)
        {
            return value_head_;
        }
        return tail >= count ? 0 : -1;
    }
    return tail - value_head_ >= count ? value_head_ : -1;
}

// Publishes up to `count` of the request's next samples as one segment, if a table entry and room in the values ring
// are free; returns the samples published
int64_t stream_engine::publish(int handle, request& r, int64_t count)
{
    if (count <= 0 || next_segment_ - oldest_segment_ >= segment_ring)
    {
        return 0;
    }
    const int64_t at = value_room(count);
    if (at < 0)
    {
        return 0;
    }
    const int64_t logical = next_segment_++;
    const int slot = static_cast<int>(logical & (segment_ring - 1));
    segment& s = segments_[static_cast<size_t>(slot)];
    s = segment{};
    s.handle = handle;
    s.local_begin = r.published;
    s.local_end = r.published + count;
    s.global_begin = published_;
    s.value_offset = at;
    batch_job& b = table_host_[static_cast<size_t>(slot)];
    b = batch_job{};
    b.scene = r.scene->view();
    b.cam = r.cam;
    b.seed = r.seed;
    b.pass_begin = 0;
    b.pass_end = r.target;
    b.sample_begin = published_;
    b.tiles_x = r.tiles_x;
    b.padded_pixels = static_cast<int32_t>(r.padded);
    b.round_passes = r.camera.sqrt_spp * r.camera.sqrt_spp;
    b.quality = r.scene->quality() ? 1 : 0;
    b.job = r.id;
    b.counters = r.counters.data();
    b.values = values_.data() + at;
    b.done = done_.data() + slot;
    b.local_begin = s.local_begin;
    // the entry and its cleared count, ordered before the group that may first claim its samples (a pageable copy:
    // the host's entry may change as soon as the call returns)
    check(cudaMemsetAsync(done_.data() + slot, 0, sizeof(unsigned long long), stream_), "clearing a count");
    check(cudaMemcpyAsync(table_.data() + slot, &b, sizeof(batch_job), cudaMemcpyHostToDevice, stream_),
          "publishing a segment");
    check(cudaMemcpyAsync(starts_.data() + slot, &b.sample_begin, sizeof(int64_t), cudaMemcpyHostToDevice, stream_),
          "publishing a segment");
    published_ += count;
    value_head_ = at + count;
    ++live_segments_;
    r.published += count;
    r.segments.push_back(logical);
    features_ = features_ || has_features(b.scene);
    wide_ = wide_ && b.scene.wide_nodes != nullptr;
    return count;
}

void stream_engine::schedule()
{
    // An idle run starts its kernels' variant over from the requests that still have work
    if (live_segments_ == 0 && in_flight_ == 0)
    {
        features_ = false;
        wide_ = true;
        for (const auto& [h, r] : requests_)
        {
            if (!r->cancelled && r->published < r->padded * r->target)
            {
                features_ = features_ || has_features(r->scene->view());
                wide_ = wide_ && r->scene->view().wide_nodes != nullptr;
            }
        }
    }
    // First frames, in arrival order: the first pass of every request added since, whatever the backlog
    while (!fresh_.empty())
    {
        const int h = fresh_.front();
        request& r = *requests_.at(h);
        if (r.published < r.padded && publish(h, r, r.padded - r.published) == 0)
        {
            return; // no room now: a later reading frees some
        }
        fresh_.erase(fresh_.begin());
    }
    // Refinement while the unclaimed backlog is short: the requests with the least work left first (shortest
    // remaining processing time, which minimises the mean time to target)
    // enough for the groups a published sample waits through before a slot can claim it (the next but one), with a
    // group's margin: below that the pool starves between readings
    const double ahead = std::max(lookahead_seconds_, 3.0 * group_seconds_);
    const int64_t lookahead = std::max<int64_t>(slot_count_, static_cast<int64_t>(claim_rate_ * ahead));
    int64_t backlog = std::max<int64_t>(0, published_ - taken_);
    if (backlog >= lookahead)
    {
        return;
    }
    std::vector<std::pair<int64_t, int>> order;
    for (const auto& [h, r] : requests_)
    {
        const int64_t total = r->padded * r->target;
        if (!r->cancelled && r->published >= r->padded && r->published < total)
        {
            order.emplace_back(total - r->published, h);
        }
    }
    std::sort(order.begin(), order.end());
    for (const auto& [left, h] : order)
    {
        request& r = *requests_.at(h);
        while (backlog < lookahead && r.published < r.padded * r.target)
        {
            const int64_t got = publish(h, r, std::min(piece_samples, r.padded * r.target - r.published));
            if (got == 0)
            {
                return;
            }
            backlog += got;
        }
        if (backlog >= lookahead)
        {
            return;
        }
    }
}

bool stream_engine::has_work() const { return live_segments_ > 0 || !fresh_.empty(); }

// A group of steps as one graph: the limit and the window copied in from pinned memory (the group's own slot of it),
// group_steps_ wavefront steps, the queue, the counters and the segments' counts copied out to the group's readback.
// One graph per kernel variant and group slot, captured on first use.
cudaGraphExec_t stream_engine::group_graph(int k)
{
    cudaGraphExec_t& exec = graphs_[(features_ ? 4 : 0) + (wide_ ? 2 : 0) + k];
    if (exec)
    {
        return exec;
    }
    wave_batch w{};
    w.jobs = table_.data();
    w.work_counter = counters_.data();
    w.published = counters_.data() + 1;
    w.job_mask = segment_ring - 1;
    w.window = reinterpret_cast<const int32_t*>(counters_.data() + 2);
    w.starts = starts_.data();
    unsigned char* rb = readback_ + static_cast<size_t>(k) * readback_bytes();
    cudaGraph_t graph = nullptr;
    check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capturing a group of steps");
    cudaError_t e = cudaMemcpyAsync(counters_.data() + 1, staging_ + k, sizeof(group_control), cudaMemcpyHostToDevice,
                                    stream_);
    for (int s = 0; s < group_steps_ && e == cudaSuccess; ++s)
    {
        // requests of either integrator share the pool: the kernel that picks it per request
        e = launch_wave_batch_step(w, false, features_, wide_, true, buffers_, trace_grid_, stream_, false);
    }
    if (e == cudaSuccess)
    {
        e = cudaMemcpyAsync(rb, control_.data(), 16, cudaMemcpyDeviceToHost, stream_);
    }
    if (e == cudaSuccess)
    {
        e = cudaMemcpyAsync(rb + 16, counters_.data(), 16, cudaMemcpyDeviceToHost, stream_);
    }
    if (e == cudaSuccess)
    {
        e = cudaMemcpyAsync(rb + 32, done_.data(), segment_ring * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            stream_);
    }
    const cudaError_t end = cudaStreamEndCapture(stream_, &graph);
    check(e, "capturing a group of steps");
    check(end, "capturing a group of steps");
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    check(e, "instantiating a group of steps");
    return exec;
}

void stream_engine::launch_group()
{
    // the window of segments a claim may fall in: from the oldest with a sample that may not have been taken yet
    // (every sample below min(claims, limit) of a finished group has been)
    int64_t first = oldest_segment_;
    while (first < next_segment_)
    {
        const segment& s = segments_[static_cast<size_t>(first & (segment_ring - 1))];
        if (s.global_begin + (s.local_end - s.local_begin) > taken_)
        {
            break;
        }
        ++first;
    }
    first = std::min(first, std::max<int64_t>(next_segment_ - 1, 0));
    // the kernel searches the window unwrapped, masking each index into the ring: counted from a multiple of the
    // ring's size, the window's ends stay small
    const int64_t base = first / segment_ring * segment_ring;
    const int k = group_index_ & 1;
    // this slot's last group has finished (at most two are in flight), so its staging may be written
    staging_[k].published = published_;
    staging_[k].window_first = static_cast<int32_t>(first - base);
    staging_[k].window_end = static_cast<int32_t>(next_segment_ - base);
    group_limit_[k] = published_;
    group_segments_[k] = next_segment_;
    const cudaGraphExec_t graph = group_graph(k);
    // the reductions the last reading enqueued have read every value a segment retired since held
    check(cudaStreamWaitEvent(stream_, reduced_, 0), "ordering the group after the reductions");
    check(cudaEventRecord(group_start_[k], stream_), "recording a CUDA event");
    check(cudaGraphLaunch(graph, stream_), "launching a group of steps");
    check(cudaEventRecord(group_done_[k], stream_), "recording a CUDA event");
    launches_ += 2 * group_steps_;
    ++group_index_;
    ++in_flight_;
}

// The oldest group in flight: its GPU time, then its counts: finished segments reduced in each request's order
double stream_engine::finish_group()
{
    const int k = (group_index_ - in_flight_) & 1;
    check(cudaEventSynchronize(group_done_[k]), "rendering on the GPU");
    --in_flight_;
    float ms = 0;
    check(cudaEventElapsedTime(&ms, group_start_[k], group_done_[k]), "timing the GPU");
    const unsigned char* rb = readback_ + static_cast<size_t>(k) * readback_bytes();
    unsigned queue[4];
    std::memcpy(queue, rb, 16);
    if (queue[3] != 0)
    {
        fail(RT_ERR_RUNTIME, "the continuous wavefront claimed a sample outside its window of segments");
    }
    unsigned long long counts[2];
    std::memcpy(counts, rb + 16, 16);
    ++groups_;
    busy_sum_ += std::min(1.0, static_cast<double>(queue[0] + queue[2]) / static_cast<double>(slot_count_));
    const int64_t taken = std::max(taken_, std::min(static_cast<int64_t>(counts[0]), group_limit_[k]));
    if (ms > 0 && taken > taken_)
    {
        const double rate = static_cast<double>(taken - taken_) / (ms * 1e-3);
        claim_rate_ = claim_rate_ > 0 ? 0.75 * claim_rate_ + 0.25 * rate : rate;
        group_seconds_ = group_seconds_ > 0 ? 0.75 * group_seconds_ + 0.25 * (ms * 1e-3) : ms * 1e-3;
    }
    taken_ = taken;
    // only the segments published before the group was launched: a table entry reused since still shows its
    // previous segment's count in this reading
    const auto* done = reinterpret_cast<const unsigned long long*>(rb + 32);
    for (int64_t l = oldest_segment_; l < group_segments_[k]; ++l)
    {
        segment& s = segments_[static_cast<size_t>(l & (segment_ring - 1))];
        if (s.handle >= 0 && !s.finished &&
            done[l & (segment_ring - 1)] >= static_cast<unsigned long long>(s.local_end - s.local_begin))
        {
            s.finished = true;
        }
    }
    // A run with work whose counts stop moving would spin here for ever: every sample finishes within its path's
    // length of steps, so a long run of groups without a change is an error
    unsigned long long progress = counts[0];
    for (int64_t l = oldest_segment_; l < group_segments_[k]; ++l)
    {
        progress += done[l & (segment_ring - 1)];
    }
    if (progress != last_progress_ || !has_work())
    {
        last_progress_ = progress;
        stalled_groups_ = 0;
    }
    else if (++stalled_groups_ > 4096)
    {
        fail(RT_ERR_RUNTIME, "the continuous wavefront made no progress over 4096 groups of steps");
    }
    if (reduce_finished(k))
    {
        // the passes the host now reports are in the sums
        check(cudaEventSynchronize(reduced_), "reducing finished segments");
    }
    return ms * 1e-3;
}

// Every request's finished segments in order, one segment of each per launch (a pixel's passes must go in order);
// returns whether any launch was made
bool stream_engine::reduce_finished(int group)
{
    bool any = false;
    while (true)
    {
        std::vector<stream_reduce_item> items;
        std::vector<int64_t> retired;
        int64_t pixels = 0;
        for (auto& [h, rp] : requests_)
        {
            request& r = *rp;
            if (r.segments.empty())
            {
                continue;
            }
            segment& s = segments_[static_cast<size_t>(r.segments.front() & (segment_ring - 1))];
            if (!s.finished)
            {
                continue;
            }
            stream_reduce_item it{};
            it.values = values_.data() + s.value_offset;
            it.sums = r.sums.data();
            it.acc = r.acc.data();
            it.local_begin = s.local_begin;
            it.local_end = s.local_end;
            it.pixel_begin = pixels;
            it.target = r.target;
            it.padded_pixels = static_cast<int32_t>(r.padded);
            it.tiles_x = r.tiles_x;
            it.width = r.camera.image_width;
            it.height = r.camera.image_height;
            it.chunk = pass_chunk;
            items.push_back(it);
            pixels += int64_t{r.camera.image_width} * r.camera.image_height;
            retired.push_back(r.segments.front());
            r.segments.pop_front();
            r.reduced = s.local_end;
            // the passes the sums hold: up to the last point the accumulator went into them
            const int64_t whole = r.reduced / r.padded;
            int64_t flushed = whole / pass_chunk * pass_chunk;
            flushed = whole >= 1 ? std::max<int64_t>(flushed, 1) : flushed;
            flushed = whole >= r.target ? r.target : flushed;
            r.passes = std::max(r.passes, flushed);
        }
        if (items.empty())
        {
            return any;
        }
        if (!any)
        {
            // the reductions read values the group just finished wrote
            check(cudaStreamWaitEvent(reduce_stream_, group_done_[group], 0), "ordering the reductions");
            any = true;
        }
        if (reduce_items_.size() < items.size())
        {
            reduce_items_.allocate_async(std::max<size_t>(items.size(), 2 * reduce_items_.size()), reduce_stream_);
        }
        check(cudaMemcpyAsync(reduce_items_.data(), items.data(), items.size() * sizeof(stream_reduce_item),
                              cudaMemcpyHostToDevice, reduce_stream_),
              "copying the reduction's items");
        check(launch_stream_reduce(reduce_items_.data(), static_cast<int32_t>(items.size()), pixels, reduce_stream_),
              "launching the stream's reduction");
        check(cudaEventRecord(reduced_, reduce_stream_), "recording a CUDA event");
        ++launches_;
        // the segments' entries and values go to later groups (which wait for reduced_)
        for (const int64_t l : retired)
        {
            segments_[static_cast<size_t>(l & (segment_ring - 1))].handle = -1;
            --live_segments_;
        }
        while (oldest_segment_ < next_segment_ &&
               segments_[static_cast<size_t>(oldest_segment_ & (segment_ring - 1))].handle < 0)
        {
            ++oldest_segment_;
        }
        if (oldest_segment_ == next_segment_)
        {
            value_head_ = 0;
        }
    }
}

double stream_engine::advance(double seconds)
{
    double gpu = 0;
    schedule();
    while (true)
    {
        if (has_work() && in_flight_ < 2)
        {
            launch_group();
            continue;
        }
        if (in_flight_ == 0)
        {
            break;
        }
        gpu += finish_group();
        schedule();
        if (gpu >= seconds)
        {
            break;
        }
    }
    gpu_seconds_ += gpu;
    return gpu;
}

int64_t stream_engine::passes(int handle) const { return requests_.at(handle)->passes; }

void stream_engine::pixels(int handle, double* out, int64_t count)
{
    request& r = *requests_.at(handle);
    const int64_t n = int64_t{r.camera.image_width} * r.camera.image_height * 3;
    if (count != n)
    {
        fail(RT_ERR_INVALID, "pixels: the buffer must hold width * height * 3 doubles");
    }
    if (r.passes == 0)
    {
        fail(RT_ERR_LOGIC, "pixels: the image has no complete pass");
    }
    // the sums hold r.passes passes once the reductions enqueued so far have run (the accumulator holds the rest)
    check(cudaMemcpyAsync(out, r.sums.data(), static_cast<size_t>(n) * sizeof(double), cudaMemcpyDeviceToHost,
                          reduce_stream_),
          "copying the image");
    check(cudaStreamSynchronize(reduce_stream_), "copying the image");
    const double scale = 1.0 / static_cast<double>(r.passes);
    for (int64_t i = 0; i < n; ++i)
    {
        out[i] *= scale;
    }
}

void stream_engine::display(int handle, const rt_display_options& options, uint8_t* out, int64_t count)
{
    check_display(options);
    request& r = *requests_.at(handle);
    const int64_t n = int64_t{r.camera.image_width} * r.camera.image_height * 4;
    if (count != n)
    {
        fail(RT_ERR_INVALID, "display: the buffer must hold width * height * 4 bytes");
    }
    if (r.passes == 0)
    {
        fail(RT_ERR_LOGIC, "the image has no complete pass to show");
    }
    if (rgba_.size() < static_cast<size_t>(n))
    {
        rgba_.allocate_async(static_cast<size_t>(n), reduce_stream_);
    }
    launch_display(r.sums.data(), r.camera.image_width, r.camera.image_height, 1.0 / static_cast<double>(r.passes),
                   options, rgba_.data(), reduce_stream_);
    check(cudaMemcpyAsync(out, rgba_.data(), static_cast<size_t>(n), cudaMemcpyDeviceToHost, reduce_stream_),
          "copying the display's bytes");
    check(cudaStreamSynchronize(reduce_stream_), "converting the image for the display");
}

uint64_t stream_engine::rays(int handle) const
{
    unsigned long long v[2] = {0, 0};
    check(cudaMemcpy(v, requests_.at(handle)->counters.data(), sizeof(v), cudaMemcpyDeviceToHost), "reading counts");
    return v[0];
}

uint64_t stream_engine::shadow_rays(int handle) const
{
    unsigned long long v[2] = {0, 0};
    check(cudaMemcpy(v, requests_.at(handle)->counters.data(), sizeof(v), cudaMemcpyDeviceToHost), "reading counts");
    return v[1];
}
} // namespace rtb
