// Batched rendering and serving: the batch engine (a job table, a partials arena and a captured CUDA graph of the
// step), rt_batch_render on top of it (many independent jobs in one persistent launch per group and step), and the
// render server (a stream of requests admitted under an HBM budget, first frames before refinement).
#include "batch.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <exception>
#include <new>
#include <string>

#include "scene_store.h"

namespace rtb
{
namespace
{
constexpr size_t default_partial_budget = size_t{1} << 30;
// A step of at most this many samples in the wavefront form (a server's step: about 10 ms) is a short step
constexpr int64_t short_step_samples = int64_t{12} << 20;
} // namespace

// ---- the batch engine ---------------------------------------------------------------------------------------

batch_engine::batch_engine(size_t partial_budget_bytes, bool use_graph, bool high_priority)
    : use_graph_(use_graph),
      max_partial_entries_(static_cast<int64_t>((partial_budget_bytes > 0 ? partial_budget_bytes : default_partial_budget) /
                                                (3 * sizeof(double))))
{
    int least = 0, greatest = 0;
    check(cudaDeviceGetStreamPriorityRange(&least, &greatest), "querying stream priorities");
    check(cudaStreamCreateWithPriority(&stream_, cudaStreamNonBlocking, high_priority ? greatest : least),
          "creating a CUDA stream");
    check(cudaEventCreate(&start_), "creating a CUDA event");
    check(cudaEventCreate(&stop_), "creating a CUDA event");
    kernel_attributes a{};
    for (int g = 0; g < persistent_groups; ++g)
    {
        check(batch_attributes(g, a), "querying the batch kernel");
        grids_[g] = a.multiprocessors * std::max(1, a.blocks_per_sm);
    }
    kernel_attributes shade{}, trace{};
    check(wave_attributes(scene_view{}, false, shade, trace), "querying the wavefront kernels");
    trace_grid_ = trace.multiprocessors * std::max(1, trace.blocks_per_sm);
    wave_ = std::make_unique<wave_runner>(wave_slots_mesh, wave_group); // the wavefront groups' slots, in turn
    work_counter_.allocate(batch_groups);
    header_.allocate(1);
    retain_pool_memory(); // what the jobs free stays in the pool for the next jobs
    header_host_ = static_cast<batch_header*>(acquire_pinned(sizeof(batch_header)));
}

batch_engine::~batch_engine()
{
    jobs_.clear(); // their arrays (and the wavefront's, the arena and the table) are freed on the stream, before it goes
    wave_.reset();
    arena_.release();
    table_.release();
    rgba_.release();
    release_graph();
    cudaStreamSynchronize(stream_); // no copy from the pinned tables is in flight when they go back to the cache
    release_pinned(table_host_, capacity_ * sizeof(batch_job));
    release_pinned(header_host_, sizeof(batch_header));
    if (start_)
    {
        cudaEventDestroy(start_);
    }
    if (stop_)
    {
        cudaEventDestroy(stop_);
    }
    if (stream_)
    {
        cudaStreamDestroy(stream_);
    }
}

int64_t batch_engine::chunks_of(int64_t passes, int64_t pass_end)
{
    return (pass_end + pass_chunk - 1) / pass_chunk - passes / pass_chunk;
}

int64_t batch_engine::padded_of(const rt_camera_desc& camera)
{
    return int64_t{(camera.image_width + 7) / 8} * ((camera.image_height + 3) / 4) * 32;
}

size_t batch_engine::job_bytes(const rt_camera_desc& camera) const
{
    return static_cast<size_t>(camera.image_width) * static_cast<size_t>(camera.image_height) * 3 * sizeof(double) +
           2 * sizeof(unsigned long long);
}

int batch_engine::add(std::shared_ptr<resident_scene> scene, const rt_camera_desc& camera, uint64_t seed,
                      uint32_t job_id)
{
    if (camera.sampling != scene->camera().sampling)
    {
        fail(RT_ERR_INVALID, "a request must keep its scene's sampling strategy");
    }
    rt_scene_desc probe{};
    probe.camera = camera;
    probe.light_count = camera.sampling == RT_SAMPLING_LIGHTS || camera.sampling == RT_SAMPLING_MIXTURE ? 1 : 0;
    rt_light_desc dummy{};
    dummy.kind = RT_LIGHT_QUAD;
    probe.lights = &dummy;
    validate(probe);
    auto j = std::make_unique<job>();
    j->scene = std::move(scene);
    j->camera = camera;
    j->cam = to_camera(camera);
    j->seed = seed;
    j->id = job_id;
    j->tiles_x = (camera.image_width + 7) / 8;
    j->padded = static_cast<int>(padded_of(camera));
    j->sums.allocate_async(static_cast<size_t>(camera.image_width) * camera.image_height * 3, stream_);
    j->counters.allocate_async(2, stream_);
    check(cudaMemsetAsync(j->sums.data(), 0, j->sums.bytes(), stream_), "clearing the sums");
    check(cudaMemsetAsync(j->counters.data(), 0, j->counters.bytes(), stream_), "clearing the counters");
    const int handle = next_handle_++;
    jobs_[handle] = std::move(j);
    return handle;
}

void batch_engine::remove(int handle)
{
    check(cudaStreamSynchronize(stream_), "finishing the batch's work");
    jobs_.erase(handle);
}

void batch_engine::release_graph()
{
    if (graph_exec_)
    {
        cudaGraphExecDestroy(graph_exec_);
        graph_exec_ = nullptr;
    }
    if (graph_)
    {
        cudaGraphDestroy(graph_);
        graph_ = nullptr;
    }
}

void batch_engine::ensure_capacity(size_t jobs, size_t partial_doubles)
{
    bool moved = false;
    if (jobs > capacity_)
    {
        size_t capacity = 64;
        while (capacity < jobs)
        {
            capacity *= 2;
        }
        table_.allocate_async(capacity, stream_);
        check(cudaStreamSynchronize(stream_), "finishing the batch's copies"); // of the old table, before it is reused
        release_pinned(table_host_, capacity_ * sizeof(batch_job));
        table_host_ = static_cast<batch_job*>(acquire_pinned(capacity * sizeof(batch_job)));
        capacity_ = capacity;
        moved = true;
    }
    if (partial_doubles > arena_.size())
    {
        arena_.allocate_async(partial_doubles + partial_doubles / 4, stream_);
        moved = true;
    }
    if (moved)
    {
        release_graph(); // the graph's copies and kernels point at the old buffers
    }
}

// The step as a graph: the job table and header copied from pinned memory, the work counter cleared, the persistent
// kernel and the reduction. Replayed as is; only the pinned tables' contents change between steps.
void batch_engine::capture()
{
    batch_params p{table_.data(), header_.data(), work_counter_.data()};
    check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capturing the batch step");
    cudaMemcpyAsync(table_.data(), table_host_, capacity_ * sizeof(batch_job), cudaMemcpyHostToDevice, stream_);
    cudaMemcpyAsync(header_.data(), header_host_, sizeof(batch_header), cudaMemcpyHostToDevice, stream_);
    cudaMemsetAsync(work_counter_.data(), 0, batch_groups * sizeof(unsigned long long), stream_);
    const cudaError_t launched = launch_batch(p, grids_, 0, persistent_groups, stream_);
    const cudaError_t ended = cudaStreamEndCapture(stream_, &graph_);
    check(launched, "capturing the batch kernels");
    check(ended, "capturing the batch step");
    check(cudaGraphInstantiate(&graph_exec_, graph_, 0), "instantiating the batch step's graph");
}

double batch_engine::step(std::vector<assignment> work)
{
    // A path of no rays: every sample is 0, the job needs no launch (as a session's render_to)
    for (assignment& a : work)
    {
        job& j = *jobs_.at(a.handle);
        if (j.camera.max_depth == 0 && a.pass_end > j.passes)
        {
            j.passes = a.pass_end;
        }
    }
    // Fit the partials arena: each job its chunks, cut back while the total is over budget (at least one chunk each)
    work.erase(std::remove_if(work.begin(), work.end(),
                              [&](const assignment& a) { return a.pass_end <= jobs_.at(a.handle)->passes; }),
               work.end());
    int64_t entries = 0;
    for (const assignment& a : work)
    {
        const job& j = *jobs_.at(a.handle);
        entries += chunks_of(j.passes, a.pass_end) * j.padded;
    }
    while (entries > max_partial_entries_)
    {
        bool cut = false;
        for (assignment& a : work)
        {
            const job& j = *jobs_.at(a.handle);
            const int64_t chunks = chunks_of(j.passes, a.pass_end);
            if (chunks > 1 && entries > max_partial_entries_)
            {
                const int64_t keep = std::max<int64_t>(1, chunks / 2);
                const int64_t end = (j.passes / pass_chunk + keep) * pass_chunk;
                entries -= (chunks - chunks_of(j.passes, end)) * j.padded;
                a.pass_end = end;
                cut = true;
            }
        }
        if (!cut)
        {
            break; // one chunk per job: let it run over, the arena grows
        }
    }
    if (work.empty())
    {
        return 0;
    }
    ensure_capacity(work.size(), static_cast<size_t>(entries) * 3);
    // A short step (a server's) keeps its wavefront runs to one: every run ends with a drain (its last paths finishing
    // while most slots idle, a path's length of steps), so the tree-searched jobs share one group (the kernels with
    // the second book's features render the scenes without them) and the flat-searched ones take the persistent
    // kernel, whose tail overlaps nothing either but is shorter. Measured on the 10 ms steps of the served stream: 2%
    // above the flat scenes in a wavefront group of their own, whose second drain costs more than its walks save.
    int64_t wave_samples = 0;
    bool tree_features = false;
    for (const assignment& a : work)
    {
        const job& j = *jobs_.at(a.handle);
        const scene_view& v = j.scene->view();
        if (wavefront_suits(v))
        {
            wave_samples += (a.pass_end - j.passes) * int64_t{j.padded};
            tree_features = tree_features || (v.flat == 0 && has_features(v));
        }
    }
    const bool short_step = wave_samples <= short_step_samples;
    // The jobs in their groups' order (each group's items form its own launch)
    const auto group_of = [&](const assignment& a) {
        const scene_view& v = jobs_.at(a.handle)->scene->view();
        if (!wavefront_suits(v) || (short_step && v.flat != 0))
        {
            return batch_group(v.flat != 0, has_features(v));
        }
        return short_step ? wave_batch_group(false, tree_features) : wave_batch_group(v.flat != 0, has_features(v));
    };
    std::stable_sort(work.begin(), work.end(),
                     [&](const assignment& a, const assignment& b) { return group_of(a) < group_of(b); });
    batch_header& header = *header_host_;
    header = batch_header{};
    for (size_t i = 0; i < work.size(); ++i)
    {
        header.group_jobs[group_of(work[i]) + 1] = static_cast<int32_t>(i + 1);
    }
    for (int g = 1; g <= batch_groups; ++g)
    {
        header.group_jobs[g] = std::max(header.group_jobs[g], header.group_jobs[g - 1]);
    }
    last_samples_ = 0;
    int64_t items = 0;
    int64_t pixels = 0;
    int64_t partial_offset = 0;
    for (size_t i = 0; i < work.size(); ++i)
    {
        job& j = *jobs_.at(work[i].handle);
        batch_job& b = table_host_[i];
        b = batch_job{};
        b.scene = j.scene->view();
        b.cam = j.cam;
        b.seed = j.seed;
        b.pass_begin = j.passes;
        b.pass_end = work[i].pass_end;
        b.first_chunk = j.passes / pass_chunk;
        b.chunk = pass_chunk;
        b.chunks = static_cast<int32_t>(chunks_of(j.passes, work[i].pass_end));
        b.tiles_x = j.tiles_x;
        b.padded_pixels = j.padded;
        b.round_passes = j.camera.sqrt_spp * j.camera.sqrt_spp;
        b.quality = j.scene->quality() ? 1 : 0;
        b.job = j.id;
        b.item_begin = items;
        b.pixel_begin = pixels;
        b.partials = arena_.data() + 3 * partial_offset;
        b.sums = j.sums.data();
        b.counters = j.counters.data();
        items += int64_t{b.chunks} * b.padded_pixels;
        pixels += int64_t{j.camera.image_width} * j.camera.image_height;
        last_samples_ += int64_t{j.camera.image_width} * j.camera.image_height * (b.pass_end - b.pass_begin);
        partial_offset += int64_t{b.chunks} * b.padded_pixels;
    }
    // Each group's item range: from its first job's start to the next group's
    for (int g = 0; g <= batch_groups; ++g)
    {
        const int32_t first = header.group_jobs[g];
        header.group_items[g] = first < static_cast<int32_t>(work.size()) ? table_host_[first].item_begin : items;
    }
    header.total_pixels = pixels;
    header.job_count = static_cast<int32_t>(work.size());
    // The wavefront groups' samples, numbered job after job within each group, and the wavefront's buffers for the
    // largest (allocated before the timing starts)
    int64_t group_samples[batch_groups] = {};
    int group_depth[batch_groups] = {};
    for (int g = persistent_groups; g < batch_groups; ++g)
    {
        for (int32_t i = header.group_jobs[g]; i < header.group_jobs[g + 1]; ++i)
        {
            batch_job& b = table_host_[i];
            b.sample_begin = group_samples[g];
            group_samples[g] += (b.pass_end - b.pass_begin) * int64_t{b.padded_pixels};
            group_depth[g] = std::max(group_depth[g], b.cam.max_depth);
        }
    }
    wave_->setup(*std::max_element(group_samples, group_samples + batch_groups), stream_);
    check(cudaEventRecord(start_, stream_), "recording a CUDA event");
    if (use_graph_)
    {
        if (!graph_exec_)
        {
            capture();
        }
        check(cudaGraphLaunch(graph_exec_, stream_), "launching the batch step's graph");
    }
    else
    {
        check(cudaMemcpyAsync(table_.data(), table_host_, work.size() * sizeof(batch_job), cudaMemcpyHostToDevice,
                              stream_),
              "copying the job table");
        check(cudaMemcpyAsync(header_.data(), header_host_, sizeof(batch_header), cudaMemcpyHostToDevice, stream_),
              "copying the batch header");
        check(cudaMemsetAsync(work_counter_.data(), 0, batch_groups * sizeof(unsigned long long), stream_),
              "clearing the counters");
        check(launch_batch(batch_params{table_.data(), header_.data(), work_counter_.data()}, grids_, 0,
                           persistent_groups, stream_),
              "launching the batch kernels");
    }
    launches_ += persistent_groups; // each persistent group's launch (an empty group's ends at once)
    for (int g = persistent_groups; g < batch_groups; ++g)
    {
        if (group_samples[g] == 0)
        {
            continue;
        }
        // the group's samples claimed through its own work counter, zeroed with the others at the step's start
        const wave_batch w{table_.data(),          header.group_jobs[g],      header.group_jobs[g + 1],
                           header.group_items[g], header.group_items[g + 1], work_counter_.data() + g};
        const bool flat = g == wave_batch_group(true, false) || g == wave_batch_group(true, true);
        const bool features = g == wave_batch_group(flat, true);
        bool wide = true;
        bool quality = false;
        for (int32_t i = header.group_jobs[g]; i < header.group_jobs[g + 1]; ++i)
        {
            wide = wide && table_host_[i].scene.wide_nodes != nullptr;
            quality = quality || table_host_[i].quality != 0;
        }
        const wave_buffers b = wave_->setup(group_samples[g], stream_);
        const int64_t steps = wave_->run(
            b, group_depth[g], stream_,
            [&](bool draining) {
                return launch_wave_batch_step(w, flat, features, wide, quality, b, trace_grid_, stream_, draining);
            },
            work_counter_.data() + g);
        check(launch_wave_batch_partials(w, b, stream_), "launching the wavefront's partials");
        launches_ += static_cast<int>(2 * steps + 1);
    }
    check(launch_batch_reduce(batch_params{table_.data(), header_.data(), work_counter_.data()}, grids_[0], stream_),
          "launching the batch reduction");
    launches_ += 1;
    check(cudaEventRecord(stop_, stream_), "recording a CUDA event");
    check(cudaEventSynchronize(stop_), "rendering the batch on the GPU");
    float ms = 0;
    check(cudaEventElapsedTime(&ms, start_, stop_), "timing the GPU");
    for (const assignment& a : work)
    {
        jobs_.at(a.handle)->passes = a.pass_end;
    }
    return ms / 1000.0;
}

void batch_engine::reserve_pool(size_t bytes)
{
    // an allocation and its release: the pool keeps the memory (its release threshold is the maximum)
    void* p = nullptr;
    check(cudaMallocAsync(&p, bytes, stream_), "growing the memory pool");
    check(cudaFreeAsync(p, stream_), "growing the memory pool");
    check(cudaStreamSynchronize(stream_), "growing the memory pool");
}

void batch_engine::reserve_wavefront(int64_t samples)
{
    wave_->setup(samples, stream_);
    check(preload_wave_batch(), "loading the wavefront's kernels");
}

int64_t batch_engine::passes(int handle) const { return jobs_.at(handle)->passes; }

void batch_engine::copy_sums(int handle, double* device_out)
{
    const job& j = *jobs_.at(handle);
    check(cudaMemcpyAsync(device_out, j.sums.data(), j.sums.bytes(), cudaMemcpyDeviceToDevice, stream_),
          "copying a job's sums");
    check(cudaStreamSynchronize(stream_), "copying a job's sums");
}

void batch_engine::pixels(int handle, double* out, int64_t count)
{
    job& j = *jobs_.at(handle);
    const int64_t n = int64_t{j.camera.image_width} * j.camera.image_height * 3;
    if (count != n)
    {
        fail(RT_ERR_INVALID, "pixels: the buffer must hold width * height * 3 doubles");
    }
    if (j.passes == 0)
    {
        fail(RT_ERR_LOGIC, "pixels: the image has no complete pass");
    }
    check(cudaMemcpyAsync(out, j.sums.data(), static_cast<size_t>(n) * sizeof(double), cudaMemcpyDeviceToHost, stream_),
          "copying the image");
    check(cudaStreamSynchronize(stream_), "copying the image");
    const double scale = 1.0 / static_cast<double>(j.passes);
    for (int64_t i = 0; i < n; ++i)
    {
        out[i] *= scale;
    }
}

void batch_engine::display(int handle, const rt_display_options& options, uint8_t* out, int64_t count)
{
    check_display(options);
    job& j = *jobs_.at(handle);
    const int64_t n = int64_t{j.camera.image_width} * j.camera.image_height * 4;
    if (count != n)
    {
        fail(RT_ERR_INVALID, "display: the buffer must hold width * height * 4 bytes");
    }
    if (j.passes == 0)
    {
        fail(RT_ERR_LOGIC, "the image has no complete pass to show");
    }
    if (rgba_.size() < static_cast<size_t>(n))
    {
        rgba_.allocate_async(static_cast<size_t>(n), stream_);
    }
    launch_display(j.sums.data(), j.camera.image_width, j.camera.image_height, 1.0 / static_cast<double>(j.passes),
                   options, rgba_.data(), stream_);
    check(cudaMemcpyAsync(out, rgba_.data(), static_cast<size_t>(n), cudaMemcpyDeviceToHost, stream_),
          "copying the display's bytes");
    check(cudaStreamSynchronize(stream_), "converting the image for the display");
}

uint64_t batch_engine::rays(int handle) const
{
    unsigned long long v = 0;
    check(cudaMemcpy(&v, jobs_.at(handle)->counters.data(), sizeof(v), cudaMemcpyDeviceToHost), "reading counts");
    return v;
}

uint64_t batch_engine::shadow_rays(int handle) const
{
    unsigned long long v = 0;
    check(cudaMemcpy(&v, jobs_.at(handle)->counters.data() + 1, sizeof(v), cudaMemcpyDeviceToHost), "reading counts");
    return v;
}

// ---- the render server --------------------------------------------------------------------------------------

render_server::render_server(const rt_server_options& options) : options_(options)
{
    if (!(options_.step_seconds > 0 && options_.step_seconds <= 1))
    {
        fail(RT_ERR_INVALID, "step_seconds must be in (0, 1]");
    }
    if (options_.hbm_budget_bytes <= 0)
    {
        fail(RT_ERR_INVALID, "hbm_budget_bytes must be positive");
    }
    if (options_.continuous < 0 || options_.continuous > 2)
    {
        fail(RT_ERR_INVALID, "continuous must be 0, 1 or 2");
    }
    if (options_.continuous)
    {
        // The pool of the flat-searched scenes (a compromise between the mesh, which gains up to 3 x 2^20 slots, and
        // the sphere trees, which lose past 2^20) and a ring of 2^26 sample values (1 GB: a 4K first frame and the
        // refinement backlog many times over)
        if (options_.slots < 0 || options_.slots % render_block != 0 || options_.group_steps < 0 ||
            options_.group_steps > 16 || !(options_.lookahead_seconds >= 0 && options_.lookahead_seconds <= 1))
        {
            fail(RT_ERR_INVALID, "slots must be a non-negative multiple of 128, group_steps in 0..16 and "
                                 "lookahead_seconds in [0, 1]");
        }
        stream_ = std::make_unique<stream_engine>(options_.slots > 0 ? options_.slots : wave_slots_large,
                                                  int64_t{1} << 26, options_.group_steps > 0 ? options_.group_steps : 2,
                                                  options_.lookahead_seconds > 0 ? options_.lookahead_seconds : 0.002);
        // First frames are rendered in batched steps of their own (a first frame's last paths then advance through
        // steps of a few slots, not of the whole pool), on a stream whose kernels go first, and handed over
        engine_ = std::make_unique<batch_engine>(size_t{256} << 20, options.use_graph != 0, true);
        engine_->reserve_wavefront(int64_t{1} << 24);
        // The requests' memory (48 bytes a pixel) mapped now: a pool grown while requests wait stalls the step that
        // admits them (tens of GB at once when large requests arrive together)
        stream_->reserve_pool(std::min<size_t>(static_cast<size_t>(options_.hbm_budget_bytes), size_t{64} << 30));
        return;
    }
    engine_ = std::make_unique<batch_engine>(std::min<size_t>(default_partial_budget,
                                                              static_cast<size_t>(options.hbm_budget_bytes) / 4),
                                             options.use_graph != 0);
    // What the first requests would otherwise wait for: the wavefront's buffers (its slots and the samples of a step
    // of 64M samples, about 1.3 GB) and its kernels' modules, and the memory pool grown to hold requests' sums (a
    // pool grown while requests wait stalls the step that admits them: tens of GB when large requests arrive together)
    engine_->reserve_wavefront(int64_t{1} << 26);
    engine_->reserve_pool(std::min<size_t>(static_cast<size_t>(options_.hbm_budget_bytes), size_t{64} << 30));
}

int64_t render_server::passes_of(const request& r) const
{
    if (r.handle < 0)
    {
        return r.state == RT_REQUEST_DONE ? r.target : 0;
    }
    return stream_ ? stream_->passes(r.handle) : engine_->passes(r.handle);
}

// A request's device memory back to the budget
void render_server::release(request& r)
{
    if (r.first_handle >= 0)
    {
        engine_->remove(r.first_handle);
        r.first_handle = -1;
    }
    if (r.handle >= 0)
    {
        if (stream_)
        {
            stream_->remove(r.handle);
        }
        else
        {
            engine_->remove(r.handle);
        }
        r.handle = -1;
        used_bytes_ -= r.bytes;
    }
    r.scene.reset();
}

// A step of the continuous wavefront: admission as in a batched step; the first frames of the admitted requests in
// a batched step of their own (arrival order, about max(first_frame_seconds, step_seconds) of them, at least one),
// handed over to the pool; then, if no first frame is left waiting, the pool runs for about step_seconds of GPU time
// and returns with work still running. A request's state follows the passes its sums hold.
rt_server_step_report render_server::step_continuous()
{
    rt_server_step_report report{};
    while (!queue_.empty())
    {
        request& r = requests_.at(queue_.front());
        if (used_bytes_ + r.bytes > static_cast<size_t>(options_.hbm_budget_bytes))
        {
            break;
        }
        // RNG job field 0, as in a batched step: the image equals a session's of the same view and seed
        const bool batched_first = options_.continuous == 1;
        r.handle = stream_->add(r.scene, r.camera, r.seed, 0, r.target, batched_first);
        if (batched_first)
        {
            r.first_handle = engine_->add(r.scene, r.camera, r.seed, 0);
            first_queue_.push_back(r.id);
        }
        r.state = RT_REQUEST_ACTIVE;
        used_bytes_ += r.bytes;
        queue_.pop_front();
        ++report.admitted;
    }
    std::map<int64_t, int64_t> before;
    for (const auto& [id, r] : requests_)
    {
        if (r.state == RT_REQUEST_ACTIVE)
        {
            before[id] = stream_->passes(r.handle);
        }
    }
    // First frames: no group is launched meanwhile, and the groups in flight give way to the batch engine's stream
    std::vector<batch_engine::assignment> work;
    std::vector<std::pair<const resident_scene*, double>> step_samples;
    std::vector<int64_t> firsts;
    double planned = 0;
    // The waiting first frames, cheapest first (shortest job first, equal costs in arrival order): a 1080p frame
    // waits for no 4K frame that arrived before it, only for the cheaper ones and the step in flight
    std::vector<std::pair<double, int64_t>> waiting;
    for (const int64_t id : first_queue_)
    {
        const auto it = requests_.find(id);
        if (it != requests_.end() && it->second.first_handle >= 0)
        {
            const request& r = it->second;
            waiting.emplace_back(double(r.camera.image_width) * r.camera.image_height * cost_of(r.scene.get()), id);
        }
    }
    std::stable_sort(waiting.begin(), waiting.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    for (const auto& [cost, id] : waiting)
    {
        request& r = requests_.at(id);
        if (!work.empty() && planned + cost > std::max(first_frame_seconds, options_.step_seconds))
        {
            break;
        }
        work.push_back({r.first_handle, 1});
        step_samples.emplace_back(r.scene.get(), double(r.camera.image_width) * r.camera.image_height);
        planned += cost;
        firsts.push_back(id);
    }
    // what stays queued: the frames not taken, in arrival order (entries of requests gone or handed over drop out)
    std::deque<int64_t> left;
    for (const int64_t id : first_queue_)
    {
        const auto it = requests_.find(id);
        if (it != requests_.end() && it->second.first_handle >= 0 &&
            std::find(firsts.begin(), firsts.end(), id) == firsts.end())
        {
            left.push_back(id);
        }
    }
    first_queue_.swap(left);
    if (!work.empty())
    {
        const double seconds = engine_->step(std::move(work));
        if (seconds > 0)
        {
            learn_costs(step_samples, seconds);
        }
        report.gpu_seconds += seconds;
        for (const int64_t id : firsts)
        {
            request& r = requests_.at(id);
            engine_->copy_sums(r.first_handle, stream_->sums(r.handle));
            first_rays_ += engine_->rays(r.first_handle);
            first_shadow_rays_ += engine_->shadow_rays(r.first_handle);
            engine_->remove(r.first_handle);
            r.first_handle = -1;
            stream_->first_pass_done(r.handle);
        }
    }
    // Refinement, unless first frames are still waiting: they take the next step too (as in batched steps, a first
    // frame waits for no refinement; the pool's paths wait in their slots meanwhile, without draining)
    if (first_queue_.empty())
    {
        report.gpu_seconds += stream_->advance(options_.step_seconds);
    }
    stats_.gpu_seconds += report.gpu_seconds;
    ++stats_.steps;
    const auto now = clock::now();
    for (auto& [id, r] : requests_)
    {
        if (r.state != RT_REQUEST_ACTIVE)
        {
            continue;
        }
        const int64_t done = stream_->passes(r.handle);
        const int64_t was = before[id];
        report.first_frames += was == 0 && done >= 1 ? 1 : 0;
        report.refined += was >= 1 && done > was ? 1 : 0;
        if (done >= 1 && r.first_frame_seconds < 0)
        {
            r.first_frame_seconds = std::chrono::duration<double>(now - r.submitted).count();
        }
        if (done >= r.target)
        {
            r.state = RT_REQUEST_DONE;
            r.done_seconds = std::chrono::duration<double>(now - r.submitted).count();
            stats_.rays += stream_->rays(r.handle);
            stats_.shadow_rays += stream_->shadow_rays(r.handle);
            ++stats_.completed;
            ++report.completed;
        }
    }
    for (const auto& [id, r] : requests_)
    {
        report.active += r.state == RT_REQUEST_ACTIVE ? 1 : 0;
    }
    report.queued = static_cast<int32_t>(queue_.size());
    stats_.launches = stream_->launches() + engine_->launches();
    stats_.groups = stream_->groups();
    stats_.busy_slots = stream_->busy_slots();
    return report;
}

int64_t render_server::submit(std::shared_ptr<resident_scene> scene, const rt_camera_desc& camera, uint64_t seed,
                              int64_t target)
{
    if (target < 1)
    {
        fail(RT_ERR_INVALID, "a request needs at least one pass");
    }
    request r{};
    r.id = next_id_++;
    r.scene = std::move(scene);
    r.camera = camera;
    r.seed = seed;
    r.target = target;
    r.submitted = clock::now();
    r.bytes = stream_ ? stream_engine::job_bytes(camera) : engine_->job_bytes(camera);
    if (static_cast<int64_t>(r.bytes) > options_.hbm_budget_bytes)
    {
        fail(RT_ERR_CAPACITY, "the request's image alone exceeds the HBM budget");
    }
    queue_.push_back(r.id);
    requests_.emplace(r.id, std::move(r));
    return next_id_ - 1;
}

rt_server_step_report render_server::step()
{
    if (stream_)
    {
        return step_continuous();
    }
    rt_server_step_report report{};
    // Admission, in arrival order, while the budget holds (a request waits rather than overtake an earlier one)
    while (!queue_.empty())
    {
        request& r = requests_.at(queue_.front());
        if (used_bytes_ + r.bytes > static_cast<size_t>(options_.hbm_budget_bytes))
        {
            break;
        }
        // RNG job field 0: a request's image depends on its scene, camera, seed and passes only, so it equals a
        // session's render of the same view and seed
        r.handle = engine_->add(r.scene, r.camera, r.seed, 0);
        r.state = RT_REQUEST_ACTIVE;
        used_bytes_ += r.bytes;
        queue_.pop_front();
        ++report.admitted;
    }
    // First frames, cheapest first (shortest job first, equal costs in arrival order: a 1080p frame waits for no 4K
    // frame that arrived before it), while the step's time allows (at least one): a burst of large first frames
    // spreads over steps rather than holding up the ones behind it for a long step
    std::vector<batch_engine::assignment> work;
    std::vector<std::pair<const resident_scene*, double>> step_samples; // each job's scene and pixel passes
    double planned = 0;
    std::vector<std::pair<double, request*>> waiting;
    for (auto& [id, r] : requests_)
    {
        if (r.state == RT_REQUEST_ACTIVE && engine_->passes(r.handle) == 0)
        {
            waiting.emplace_back(double(r.camera.image_width) * r.camera.image_height * cost_of(r.scene.get()), &r);
        }
    }
    std::stable_sort(waiting.begin(), waiting.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    for (auto& [cost, rp] : waiting)
    {
        request& r = *rp;
        if (report.first_frames > 0 && planned + cost > options_.step_seconds)
        {
            break;
        }
        work.push_back({r.handle, 1});
        step_samples.emplace_back(r.scene.get(), double(r.camera.image_width) * r.camera.image_height);
        planned += cost;
        ++report.first_frames;
    }
    // Refinement: the others, least remaining work first (shortest remaining processing time, which minimises the
    // mean time to target), while the step's time allows. A step with first frames carries nothing else: a first
    // frame waits for no refinement, and the next step refines.
    std::vector<std::pair<double, request*>> refine;
    for (auto& [id, r] : requests_)
    {
        if (report.first_frames > 0)
        {
            break;
        }
        if (r.state != RT_REQUEST_ACTIVE)
        {
            continue;
        }
        const int64_t done = engine_->passes(r.handle);
        if (done > 0 && done < r.target)
        {
            refine.emplace_back(double(r.camera.image_width) * r.camera.image_height * double(r.target - done), &r);
        }
    }
    std::stable_sort(refine.begin(), refine.end(),
                     [](const auto& a, const auto& b) { return a.first < b.first; });
    for (auto& [remaining, rp] : refine)
    {
        request& r = *rp;
        const int64_t done = engine_->passes(r.handle);
        if (planned >= options_.step_seconds)
        {
            break;
        }
        const double per_pass = double(r.camera.image_width) * r.camera.image_height * cost_of(r.scene.get());
        const int64_t want = std::max<int64_t>(1, static_cast<int64_t>((options_.step_seconds - planned) / per_pass));
        int64_t end = std::min(r.target, done + want);
        // finish the chunk the request is in, or stop on a chunk boundary
        const int64_t boundary = (done / pass_chunk + 1) * pass_chunk;
        end = std::min(r.target, std::max(std::min(end, boundary), end / pass_chunk * pass_chunk));
        if (end <= done)
        {
            end = std::min(r.target, boundary);
        }
        work.push_back({r.handle, end});
        step_samples.emplace_back(r.scene.get(), double(r.camera.image_width) * r.camera.image_height *
                                                     double(end - done));
        planned += per_pass * double(end - done);
        ++report.refined;
    }
    if (!work.empty())
    {
        report.gpu_seconds = engine_->step(std::move(work));
        if (report.gpu_seconds > 0)
        {
            learn_costs(step_samples, report.gpu_seconds);
        }
        stats_.gpu_seconds += report.gpu_seconds;
        ++stats_.steps;
    }
    const auto now = clock::now();
    for (auto& [id, r] : requests_)
    {
        if (r.state != RT_REQUEST_ACTIVE)
        {
            continue;
        }
        const int64_t done = engine_->passes(r.handle);
        if (done >= 1 && r.first_frame_seconds < 0)
        {
            r.first_frame_seconds = std::chrono::duration<double>(now - r.submitted).count();
        }
        if (done >= r.target)
        {
            r.state = RT_REQUEST_DONE;
            r.done_seconds = std::chrono::duration<double>(now - r.submitted).count();
            stats_.rays += engine_->rays(r.handle);
            stats_.shadow_rays += engine_->shadow_rays(r.handle);
            ++stats_.completed;
            ++report.completed;
        }
    }
    for (const auto& [id, r] : requests_)
    {
        report.active += r.state == RT_REQUEST_ACTIVE ? 1 : 0;
    }
    report.queued = static_cast<int32_t>(queue_.size());
    stats_.launches = engine_->launches();
    return report;
}

double render_server::cost_of(const resident_scene* scene) const
{
    const auto it = cost_.find(scene);
    return it != cost_.end() ? it->second : (default_cost_ > 0 ? default_cost_ : 1e-9);
}

// The seconds a pixel pass costs, per scene (the mesh costs several times the Cornell box's): a step's measured time
// against its prediction corrects each of its scenes in proportion to that scene's predicted share of the step
void render_server::learn_costs(const std::vector<std::pair<const resident_scene*, double>>& samples, double seconds)
{
    double predicted = 0, total = 0;
    std::map<const resident_scene*, double> share;
    for (const auto& [scene, n] : samples)
    {
        const double c = cost_of(scene) * n;
        share[scene] += c;
        predicted += c;
        total += n;
    }
    if (!(predicted > 0) || !(total > 0))
    {
        return;
    }
    const double measured = seconds / total;
    default_cost_ = default_cost_ > 0 ? 0.5 * default_cost_ + 0.5 * measured : measured;
    const double factor = seconds / predicted;
    for (const auto& [scene, c] : share)
    {
        const bool fresh = cost_.find(scene) == cost_.end();
        const double corrected = cost_of(scene) * std::pow(factor, c / predicted);
        cost_[scene] = fresh ? corrected : 0.5 * cost_of(scene) + 0.5 * corrected;
    }
}

rt_request_status render_server::poll(int64_t id) const
{
    const auto it = requests_.find(id);
    if (it == requests_.end())
    {
        fail(RT_ERR_INVALID, "no request " + std::to_string(id));
    }
    const request& r = it->second;
    rt_request_status s{};
    s.state = r.state;
    s.passes = passes_of(r);
    s.target = r.target;
    s.first_frame_seconds = r.first_frame_seconds;
    s.done_seconds = r.done_seconds;
    return s;
}

void render_server::fetch(int64_t id, double* pixels, int64_t count)
{
    const auto it = requests_.find(id);
    if (it == requests_.end() || it->second.handle < 0 || it->second.state == RT_REQUEST_CANCELLED)
    {
        fail(RT_ERR_LOGIC, "request " + std::to_string(id) + " has no image");
    }
    request& r = it->second;
    if (stream_)
    {
        stream_->pixels(r.handle, pixels, count);
    }
    else
    {
        engine_->pixels(r.handle, pixels, count);
    }
    if (r.state == RT_REQUEST_DONE)
    {
        release(r);
    }
}

void render_server::display(int64_t id, const rt_display_options& options, uint8_t* rgba, int64_t count)
{
    const auto it = requests_.find(id);
    if (it == requests_.end() || it->second.handle < 0 || it->second.state == RT_REQUEST_CANCELLED)
    {
        fail(RT_ERR_LOGIC, "request " + std::to_string(id) + " has no image");
    }
    if (stream_)
    {
        stream_->display(it->second.handle, options, rgba, count);
    }
    else
    {
        engine_->display(it->second.handle, options, rgba, count);
    }
}

void render_server::cancel(int64_t id)
{
    const auto it = requests_.find(id);
    if (it == requests_.end())
    {
        fail(RT_ERR_INVALID, "no request " + std::to_string(id));
    }
    request& r = it->second;
    if (r.state == RT_REQUEST_QUEUED)
    {
        queue_.erase(std::remove(queue_.begin(), queue_.end(), id), queue_.end());
    }
    first_queue_.erase(std::remove(first_queue_.begin(), first_queue_.end(), id), first_queue_.end());
    release(r);
    r.state = RT_REQUEST_CANCELLED;
}

rt_server_stats render_server::stats() const
{
    rt_server_stats s = stats_;
    s.used_bytes = static_cast<int64_t>(used_bytes_);
    // the continuous server's first frames, counted when handed over
    s.rays += first_rays_;
    s.shadow_rays += first_shadow_rays_;
    return s;
}
} // namespace rtb

// ---- the C-ABI of batching and serving ----------------------------------------------------------------------

namespace
{
template <class F>
rt_status guard(F&& f)
{
    try
    {
        rtb::remember_error("");
        f();
        return RT_OK;
    }
    catch (const rtb::rt_error& e)
    {
        rtb::remember_error(e.what());
        return e.status;
    }
    catch (const std::bad_alloc&)
    {
        rtb::remember_error("out of host memory");
        return RT_ERR_RUNTIME;
    }
    catch (const std::exception& e)
    {
        rtb::remember_error(e.what());
        return RT_ERR_RUNTIME;
    }
}

void need(const void* p, const char* name)
{
    if (!p)
    {
        rtb::fail(RT_ERR_INVALID, std::string(name) + " is null");
    }
}
} // namespace

extern "C" {

rt_status rt_batch_render(const rt_batch_job* jobs, int32_t count, const rt_batch_options* options,
                          rt_batch_report* report)
{
    return guard([&] {
        if (count < 0 || (count > 0 && !jobs))
        {
            rtb::fail(RT_ERR_INVALID, "jobs and count");
        }
        const auto start = std::chrono::steady_clock::now();
        const rt_batch_options o = options ? *options : rt_batch_options{0, 1, 0};
        rtb::batch_engine engine(o.partial_budget_bytes > 0 ? static_cast<size_t>(o.partial_budget_bytes) : 0,
                                 o.use_graph != 0);
        std::vector<int> handles;
        std::vector<int64_t> targets;
        for (int32_t i = 0; i < count; ++i)
        {
            need(jobs[i].scene, "jobs[i].scene");
            need(jobs[i].pixels, "jobs[i].pixels");
            auto scene = std::make_shared<rtb::resident_scene>(*jobs[i].scene);
            const rt_camera_desc& c = jobs[i].scene->camera;
            handles.push_back(engine.add(scene, c, jobs[i].seed, 0)); // images as rt_render's for the same seed
            targets.push_back(jobs[i].passes > 0 ? jobs[i].passes : int64_t{c.sqrt_spp} * c.sqrt_spp);
        }
        const auto setup_end = std::chrono::steady_clock::now();
        double gpu = 0;
        int steps = 0;
        while (true)
        {
            std::vector<rtb::batch_engine::assignment> work;
            for (size_t i = 0; i < handles.size(); ++i)
            {
                if (engine.passes(handles[i]) < targets[i])
                {
                    work.push_back({handles[i], targets[i]});
                }
            }
            if (work.empty())
            {
                break;
            }
            gpu += engine.step(std::move(work));
            ++steps;
        }
        uint64_t rays = 0;
        uint64_t shadow = 0;
        for (int32_t i = 0; i < count; ++i)
        {
            const rt_camera_desc& c = jobs[i].scene->camera;
            if (targets[static_cast<size_t>(i)] > 0)
            {
                engine.pixels(handles[static_cast<size_t>(i)], jobs[i].pixels, int64_t{c.image_width} * c.image_height * 3);
            }
            rays += engine.rays(handles[static_cast<size_t>(i)]);
            shadow += engine.shadow_rays(handles[static_cast<size_t>(i)]);
        }
        if (report)
        {
            report->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
            report->setup_seconds = std::chrono::duration<double>(setup_end - start).count();
            report->gpu_seconds = gpu;
            report->rays = rays;
            report->shadow_rays = shadow;
            report->steps = steps;
            report->launches = engine.launches();
            report->graph = engine.graph_used() ? 1 : 0;
        }
    });
}

rt_status rt_server_create(const rt_server_options* options, rt_server** server)
{
    return guard([&] {
        need(options, "options");
        need(server, "server");
        *server = nullptr;
        auto s = std::make_unique<rt_server>();
        s->server = std::make_unique<rtb::render_server>(*options);
        *server = s.release();
    });
}

rt_status rt_server_destroy(rt_server* server)
{
    return guard([&] { delete server; });
}

rt_status rt_server_submit(rt_server* server, rt_scene* scene, const rt_camera_desc* camera, uint64_t seed,
                           int64_t target_passes, int64_t* request_id)
{
    return guard([&] {
        need(server, "server");
        need(scene, "scene");
        need(camera, "camera");
        need(request_id, "request_id");
        *request_id = server->server->submit(scene->scene, *camera, seed, target_passes);
    });
}

rt_status rt_server_step(rt_server* server, rt_server_step_report* report)
{
    return guard([&] {
        need(server, "server");
        const rt_server_step_report r = server->server->step();
        if (report)
        {
            *report = r;
        }
    });
}

rt_status rt_server_poll(const rt_server* server, int64_t request_id, rt_request_status* status)
{
    return guard([&] {
        need(server, "server");
        need(status, "status");
        *status = server->server->poll(request_id);
    });
}

rt_status rt_server_fetch(rt_server* server, int64_t request_id, double* pixels, int64_t pixel_count)
{
    return guard([&] {
        need(server, "server");
        need(pixels, "pixels");
        server->server->fetch(request_id, pixels, pixel_count);
    });
}

rt_status rt_server_display(rt_server* server, int64_t request_id, const rt_display_options* options, uint8_t* rgba,
                            int64_t byte_count)
{
    return guard([&] {
        need(server, "server");
        need(options, "options");
        need(rgba, "rgba");
        server->server->display(request_id, *options, rgba, byte_count);
    });
}

rt_status rt_server_cancel(rt_server* server, int64_t request_id)
{
    return guard([&] {
        need(server, "server");
        server->server->cancel(request_id);
    });
}

rt_status rt_server_stats_get(const rt_server* server, rt_server_stats* stats)
{
    return guard([&] {
        need(server, "server");
        need(stats, "stats");
        *stats = server->server->stats();
    });
}

rt_status rt_builtin_camera(const char* name, const rt_builtin_params* params, rt_camera_desc* camera)
{
    return guard([&] {
        need(name, "name");
        need(camera, "camera");
        rt_builtin_params p{};
        if (params)
        {
            p = *params;
        }
        else
        {
            p.sampling = -1;
            p.combination = -1;
        }
        // The camera depends only on the scene's camera settings and the overrides, not on its geometry: build the
        // scene at its cheapest (a level-0 mesh, a tiny map)
        p.mesh_level = std::string(name) == "mesh-ggx" ? 1 : p.mesh_level;
        p.env_width = 8;
        std::unique_ptr<rtb::scene_store> s;
        std::string error;
        const rt_status status = rtb::build_builtin(name, p, s, error);
        if (status != RT_OK)
        {
            rtb::fail(status, error);
        }
        *camera = s->camera;
    });
}
}
