// A session: one view of a resident scene, its image's sums kept on the device and grown by launches of the
// persistent kernel (renderer.h:591-673; the launch loop of renderer.cu:1315-1334, 1924-1971).
//
// Launch planning. The reference plans ~50 ms launches from measured row times and renders a pass in bands of rows
// when one pass is too long for a launch (renderer.cu:179-308), because Windows stops long kernels. Here a launch is
// a range of whole passes for every pixel, cut into (pixel, chunk) work items that the persistent threads pull, so a
// launch's length is set by its number of passes alone: the first launch is one chunk (a probe of the speed), and
// each later one as many chunks as fit launch_seconds at the last measured speed. A launch may span rounds of
// strata: every sample finds its round, and so its seed, from its own absolute pass.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "host.h"

namespace rtb
{
namespace
{
constexpr double max_launch_seconds = 0.5;              // renderer.h:413
constexpr size_t partial_budget_bytes = size_t{1} << 30; // a launch's chunk partials: at most 1 GiB
constexpr size_t wave_sample_budget_bytes = size_t{2} << 30; // a wavefront launch's samples (16 bytes each): 2 GiB
constexpr double trial_samples = 32e6; // the autotuner's measured launch, by default
} // namespace

session::session(std::shared_ptr<resident_scene> scene, const rt_session_options& options)
    : scene_(std::move(scene)), options_(options)
{
    if (options_.arithmetic != RT_FLOAT32 && options_.arithmetic != RT_FLOAT64)
    {
        fail(RT_ERR_INVALID, "arithmetic must be RT_FLOAT32 or RT_FLOAT64");
    }
    f64_ = options_.arithmetic == RT_FLOAT64;
    if (f64_)
    {
        // What computes in float only, in the reference's order and sense (renderer.cu:2047-2078)
        if (scene_->quality())
        {
            fail(RT_ERR_INVALID, "the quality kernel computes in float only");
        }
        if (scene_->view_f64() == nullptr)
        {
            fail(RT_ERR_INVALID, "a scene with triangle meshes renders in float only");
        }
        if (options_.form == RT_FORM_WAVEFRONT)
        {
            fail(RT_ERR_INVALID, "the wavefront form computes in float only");
        }
    }
    if (!(options_.launch_seconds > 0 && options_.launch_seconds <= max_launch_seconds))
    {
        fail(RT_ERR_INVALID, "launch_seconds must be in (0, 0.5]");
    }
    check(cudaSetDevice(scene_->device()), "selecting the scene's device");
    check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "creating a CUDA stream");
    retain_pool_memory(); // the sums and the launches' scratch come from the pool, stream-ordered
    check(cudaEventCreate(&start_), "creating a CUDA event");
    check(cudaEventCreate(&stop_), "creating a CUDA event");
    if (options_.form < RT_FORM_AUTO || options_.form > RT_FORM_WAVEFRONT)
    {
        fail(RT_ERR_INVALID, "form must be RT_FORM_AUTO, RT_FORM_PERSISTENT or RT_FORM_WAVEFRONT");
    }
    kernel_attributes a{};
    if (f64_)
    {
        check(render_f64_attributes(*scene_->view_f64(), a), "querying the FP64 render kernel");
    }
    else
    {
        check(render_attributes(scene_->view(), scene_->quality(), a), "querying the render kernel");
    }
    grid_ = a.multiprocessors * std::max(1, a.blocks_per_sm);
    const scene_view& view = scene_->view();
    wavefront_ = !f64_ &&
                 (options_.form == RT_FORM_WAVEFRONT || (options_.form == RT_FORM_AUTO && wavefront_suits(view)));
    multiprocessors_ = a.multiprocessors;
    if (wavefront_)
    {
        kernel_attributes shade{}, trace{};
        check(wave_attributes(view, scene_->quality(), shade, trace), "querying the wavefront kernels");
        // The built-in shape, or the one an earlier session's autotuning chose for this scene class
        tune_candidate c = default_candidate(wave_slots_for(view), trace.blocks_per_sm);
        tune_candidate cached{};
        if (cached_tuning(tune_key(scene_->device(), view, scene_->quality()), cached))
        {
            c = cached;
            tuning_.from_cache = 1;
        }
        apply(c);
    }
    counters_.allocate(7);
    set_camera(scene_->camera());
}

void session::apply(const tune_candidate& c)
{
    if (!wave_ || wave_->max_slots != c.slots)
    {
        wave_.reset();
        wave_ = std::make_unique<wave_runner>(c.slots, wave_group);
    }
    tuned_ = c;
    shape_.trace_grid = multiprocessors_ * c.trace_blocks_per_sm;
    shape_.shade_block = c.shade_block;
    shape_.trace_min_blocks = c.trace_min_blocks;
    const int from_cache = tuning_.from_cache;
    const int trials = tuning_.trials;
    const double speed = tuning_.samples_per_second;
    const double base = tuning_.default_samples_per_second;
    tuning_ = to_tuning(c);
    tuning_.from_cache = from_cache;
    tuning_.trials = trials;
    tuning_.samples_per_second = speed;
    tuning_.default_samples_per_second = base;
    kernel_attributes shade{}, trace{};
    check(wave_attributes(scene_->view(), scene_->quality(), shade, trace, c.trace_min_blocks),
          "querying the wavefront kernels");
    tuning_.trace_registers = trace.registers;
}

void session::set_tuning(const rt_tuning& t)
{
    if (!wavefront_)
    {
        fail(RT_ERR_LOGIC, "a persistent-form session has no launch shape to set");
    }
    kernel_attributes shade{}, trace{};
    const scene_view& view = scene_->view();
    if (t.trace_min_blocks != RTB_TRACE_MIN_BLOCKS_DEFAULT && t.trace_min_blocks != wave_trace_roomy_blocks)
    {
        fail(RT_ERR_INVALID, "trace_min_blocks must be 8 or 6");
    }
    check(wave_attributes(view, scene_->quality(), shade, trace, t.trace_min_blocks), "querying the wavefront kernels");
    if (t.trace_blocks_per_sm < 1 || t.trace_blocks_per_sm > trace.blocks_per_sm)
    {
        fail(RT_ERR_INVALID, "trace_blocks_per_sm must be from 1 to the trace kernel's occupancy");
    }
    if (t.slots < render_block || t.slots > (1 << 24) || t.slots % render_block != 0)
    {
        fail(RT_ERR_INVALID, "slots must be a multiple of 128 up to 2^24");
    }
    if (t.shade_block != render_block && t.shade_block != render_block / 2)
    {
        fail(RT_ERR_INVALID, "shade_block must be 64 or 128");
    }
    apply({t.slots, t.trace_blocks_per_sm, t.shade_block, t.trace_min_blocks});
    tuning_.from_cache = 0;
    tuning_.trials = 0;
}

rt_tuning session::autotune(int64_t trial_passes)
{
    if (!wavefront_)
    {
        return rt_tuning{}; // the persistent kernel's launches have no shape to choose
    }
    if (passes_ != 0)
    {
        fail(RT_ERR_LOGIC, "autotune needs a view with no passes yet (it renders trials of its own)");
    }
    if (trial_passes < 0 || trial_passes > 1 << 20)
    {
        fail(RT_ERR_INVALID, "trial_passes must be in [0, 2^20]");
    }
    const scene_view& view = scene_->view();
    kernel_attributes shade{}, trace{}, roomy{};
    check(wave_attributes(view, scene_->quality(), shade, trace), "querying the wavefront kernels");
    check(wave_attributes(view, scene_->quality(), shade, roomy, wave_trace_roomy_blocks),
          "querying the wavefront kernels");
    const tune_space space = default_tune_space(trace.blocks_per_sm, roomy.blocks_per_sm);
    const double pixels = static_cast<double>(camera_.image_width) * camera_.image_height;
    // The measured launch: whole chunks, by default about 32M samples, enough for the pool's largest candidate to
    // reach its steady state (a launch of a few slot generations would favour small pools, which ramp up and drain
    // sooner, over the pools a long render runs best with)
    int64_t measured = trial_passes;
    if (measured == 0)
    {
        measured = static_cast<int64_t>(std::ceil(trial_samples / pixels));
    }
    measured = std::max<int64_t>(pass_chunk, (measured + pass_chunk - 1) / pass_chunk * pass_chunk);
    const int64_t max_passes =
        std::max<int64_t>(pass_chunk, static_cast<int64_t>(wave_sample_budget_bytes / sizeof(float4)) /
                                          (static_cast<int64_t>(padded_pixels_) * pass_chunk) * pass_chunk - pass_chunk);
    measured = std::min(measured, max_passes);
    const double samples = pixels * static_cast<double>(measured);
    const bool counting = counting_;
    counting_ = false;
    // Each candidate: the best of two measured launches, each after a one-chunk launch (the planner's probe) from a
    // fresh image
    const auto measure = [&](const tune_candidate& c) {
        apply(c);
        double best = 0;
        for (int k = 0; k < 2; ++k)
        {
            set_camera(camera_);
            launch(pass_chunk);
            const double seconds = launch(pass_chunk + measured);
            best = std::max(best, samples / std::max(seconds, 1e-9));
        }
        return best;
    };
    const tune_outcome o = coordinate_descent(tuned_, space, measure);
    counting_ = counting;
    tuning_.from_cache = 0;
    tuning_.trials = o.trials;
    tuning_.samples_per_second = o.best_speed;
    tuning_.default_samples_per_second = o.default_speed;
    apply(o.best);
    remember_tuning(tune_key(scene_->device(), view, scene_->quality()), o.best);
    set_camera(camera_);
    return tuning_;
}

cudaEvent_t* session::marks(size_t count)
{
    while (marks_.size() < count)
    {
        cudaEvent_t e = nullptr;
        check(cudaEventCreate(&e), "creating a CUDA event");
        marks_.push_back(e);
    }
    return marks_.data();
}

session::~session()
{
    for (cudaEvent_t e : marks_)
    {
        cudaEventDestroy(e);
    }
    wave_.reset(); // its arrays are freed on the stream, before it goes
    rgba_.release();
    partials_.release();
    sums_.release();
    counters_.release();
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

void session::set_camera(const rt_camera_desc& camera)
{
    if (camera.sampling != scene_->camera().sampling)
    {
        fail(RT_ERR_INVALID, "a new view must keep the scene's sampling strategy");
    }
    rt_scene_desc probe{};
    probe.camera = camera;
    probe.light_count = camera.sampling == RT_SAMPLING_LIGHTS || camera.sampling == RT_SAMPLING_MIXTURE ? 1 : 0;
    rt_light_desc dummy{};
    dummy.kind = RT_LIGHT_QUAD;
    probe.lights = &dummy;
    validate(probe);
    camera_ = camera;
    cam_ = to_camera(camera);
    cam_d_ = to_camera_d(camera);
    tiles_x_ = (camera.image_width + 7) / 8;
    const int tiles_y = (camera.image_height + 3) / 4;
    padded_pixels_ = tiles_x_ * tiles_y * 32;
    max_partial_entries_ = static_cast<int64_t>(partial_budget_bytes / (3 * sizeof(double)));
    const size_t pixels = static_cast<size_t>(camera.image_width) * static_cast<size_t>(camera.image_height);
    if (sums_.size() != pixels * 3)
    {
        sums_.allocate_async(pixels * 3, stream_); // a view of the same size keeps its sums' memory (cleared below)
    }
    check(cudaMemsetAsync(sums_.data(), 0, sums_.bytes(), stream_), "clearing the sums");
    check(cudaMemsetAsync(counters_.data(), 0, counters_.bytes(), stream_), "clearing the counters");
    check(cudaStreamSynchronize(stream_), "clearing the sums");
    passes_ = 0;
    kernel_seconds_ = 0;
    samples_per_second_ = 0;
    times_ = rt_kernel_times{};
}

int64_t session::plan(int64_t target, double budget_seconds) const
{
    const int64_t next_chunk = (passes_ / pass_chunk + 1) * pass_chunk;
    int64_t end;
    if (samples_per_second_ <= 0)
    {
        end = next_chunk; // the probe: one chunk
    }
    else
    {
        // As many whole chunks as fit the budget, at least one: a launch ends on a chunk boundary (or at the target),
        // so every chunk's partial is summed from the same samples in the same order however the launches fall
        const double pixels = static_cast<double>(camera_.image_width) * camera_.image_height;
        const double passes = std::floor(budget_seconds * samples_per_second_ / pixels);
        end = passes_ + static_cast<int64_t>(std::min(passes, 1e12));
        end = std::max(next_chunk, end / pass_chunk * pass_chunk);
    }
    // At most what the partials buffer holds (the wavefront: its samples buffer)
    const int64_t max_chunks =
        wavefront_ && !counting_
            ? std::max<int64_t>(1, static_cast<int64_t>(wave_sample_budget_bytes / sizeof(float4)) /
                                       (static_cast<int64_t>(padded_pixels_) * pass_chunk))
            : std::max<int64_t>(1, max_partial_entries_ / padded_pixels_);
    end = std::min(end, (passes_ / pass_chunk + max_chunks) * pass_chunk);
    return std::min(end, target);
}

double session::launch(int64_t end)
{
    const int64_t first_chunk = passes_ / pass_chunk;
    const int64_t chunks = (end + pass_chunk - 1) / pass_chunk - first_chunk;
    const bool wave = wavefront_ && !counting_;
    const size_t needed = static_cast<size_t>(chunks) * static_cast<size_t>(padded_pixels_) * 3;
    if (!wave && partials_.size() < needed)
    {
        partials_.allocate_async(needed, stream_);
    }
    launch_params p{};
    p.scene = scene_->view();
    p.cam = cam_;
    p.seed = options_.seed;
    p.pass_begin = passes_;
    p.pass_end = end;
    p.first_chunk = first_chunk;
    p.chunk = pass_chunk;
    p.chunks = static_cast<int32_t>(chunks);
    p.tiles_x = tiles_x_;
    p.padded_pixels = padded_pixels_;
    p.total_items = chunks * padded_pixels_;
    p.round_passes = camera_.sqrt_spp * camera_.sqrt_spp;
    p.job = 0;
    p.work_counter = counters_.data();
    p.partials = partials_.data();
    p.counters = counters_.data() + 1;

    reduce_params r{};
    r.partials = partials_.data();
    r.sums = sums_.data();
    r.width = camera_.image_width;
    r.height = camera_.image_height;
    r.tiles_x = tiles_x_;
    r.padded_pixels = padded_pixels_;
    r.chunks = p.chunks;

    check(cudaMemsetAsync(counters_.data(), 0, sizeof(unsigned long long), stream_), "resetting the work counter");
    wave_buffers b{};
    if (wave)
    {
        // allocated before the timing starts
        b = wave_->setup(static_cast<int64_t>(padded_pixels_) * (end - passes_), stream_);
    }
    check(cudaEventRecord(start_, stream_), "recording a CUDA event");
    int64_t steps = 0;
    cudaEvent_t* reduce_marks = timing_ ? marks(2) : nullptr;
    if (wave)
    {
        const bool quality = scene_->quality();
        steps = wave_->run(
            b, camera_.max_depth, stream_,
            [&](bool draining) {
                const cudaEvent_t* m = nullptr;
                if (timing_)
                {
                    m = marks(static_cast<size_t>(2 + 3 * (steps + 1))) + 2 + 3 * steps;
                }
                ++steps;
                return launch_wave_step(p, quality, b, shape_, stream_, m, draining);
            },
            counters_.data());
        last_kernel_launches_ = static_cast<int32_t>(2 * steps + 1);
        if (timing_)
        {
            reduce_marks = marks_.data();
            check(cudaEventRecord(reduce_marks[0], stream_), "recording a CUDA event");
        }
        check(launch_wave_reduce(r, b, p.pass_begin, p.pass_end, p.chunk, stream_), "launching the reduction");
    }
    else
    {
        cudaEvent_t* m = timing_ ? marks(3) : nullptr;
        if (f64_)
        {
            launch_params_f64 p64{};
            p64.scene = *scene_->view_f64();
            p64.cam = cam_d_;
            p64.seed = p.seed;
            p64.pass_begin = p.pass_begin;
            p64.pass_end = p.pass_end;
            p64.first_chunk = p.first_chunk;
            p64.chunk = p.chunk;
            p64.chunks = p.chunks;
            p64.tiles_x = p.tiles_x;
            p64.padded_pixels = p.padded_pixels;
            p64.total_items = p.total_items;
            p64.round_passes = p.round_passes;
            p64.work_counter = p.work_counter;
            p64.partials = p.partials;
            p64.counters = p.counters;
            check(launch_render_f64(p64, grid_, stream_), "launching the FP64 render kernel");
        }
        else
        {
            check(launch_render(p, scene_->quality(), counting_, grid_, stream_), "launching the render kernel");
        }
        if (m)
        {
            check(cudaEventRecord(m[2], stream_), "recording a CUDA event");
            reduce_marks = m + 2;
        }
        check(launch_reduce(r, stream_), "launching the reduction");
        last_kernel_launches_ = 2;
    }
    if (timing_)
    {
        check(cudaEventRecord(wave ? reduce_marks[1] : marks_[1], stream_), "recording a CUDA event");
    }
    check(cudaEventRecord(stop_, stream_), "recording a CUDA event");
    check(cudaEventSynchronize(stop_), "rendering on the GPU");
    if (timing_)
    {
        const auto elapsed = [](cudaEvent_t a, cudaEvent_t b) {
            float ms = 0;
            check(cudaEventElapsedTime(&ms, a, b), "timing a kernel");
            return ms / 1000.0;
        };
        if (wave)
        {
            for (int64_t k = 0; k < steps; ++k)
            {
                const cudaEvent_t* m = marks_.data() + 2 + 3 * k;
                times_.seconds[RT_KERNEL_SHADE] += elapsed(m[0], m[1]);
                times_.seconds[RT_KERNEL_TRACE] += elapsed(m[1], m[2]);
            }
            times_.launches[RT_KERNEL_SHADE] += steps;
            times_.launches[RT_KERNEL_TRACE] += steps;
            times_.seconds[RT_KERNEL_REDUCE] += elapsed(marks_[0], marks_[1]);
        }
        else
        {
            // marks: [0] unused, [1] after the reduction, [2] after the render kernel; the render starts at start_
            times_.seconds[RT_KERNEL_RENDER] += elapsed(start_, marks_[2]);
            ++times_.launches[RT_KERNEL_RENDER];
            times_.seconds[RT_KERNEL_REDUCE] += elapsed(marks_[2], marks_[1]);
        }
        ++times_.launches[RT_KERNEL_REDUCE];
    }
    float ms = 0;
    check(cudaEventElapsedTime(&ms, start_, stop_), "timing the GPU");
    const double seconds = std::max(1e-6, ms / 1000.0);
    const double samples = static_cast<double>(camera_.image_width) * camera_.image_height * static_cast<double>(end - passes_);
    samples_per_second_ = samples / seconds;
    passes_ = end;
    kernel_seconds_ += seconds;
    return seconds;
}

rt_render_report session::render_to(int64_t target)
{
    if (target < passes_)
    {
        fail(RT_ERR_INVALID, "the target is behind the image");
    }
    rt_render_report report{};
    if (camera_.max_depth == 0)
    {
        passes_ = target; // a path of no rays: every sample is 0, and no launch is needed
    }
    while (passes_ < target)
    {
        const double t = launch(plan(target, options_.launch_seconds));
        ++report.launches;
        report.kernel_launches += last_kernel_launches_;
        report.gpu_seconds += t;
        report.longest_launch_seconds = std::max(report.longest_launch_seconds, t);
    }
    report.state = state();
    return report;
}

rt_render_report session::render_for(double seconds, int64_t pass_limit)
{
    if (!(seconds >= 0 && seconds <= 3600))
    {
        fail(RT_ERR_INVALID, "seconds must be in [0, 3600]");
    }
    if (pass_limit < 0)
    {
        fail(RT_ERR_INVALID, "pass_limit must not be negative");
    }
    rt_render_report report{};
    if (camera_.max_depth == 0)
    {
        passes_ = std::max(passes_, std::min<int64_t>(pass_limit, passes_ + 1));
    }
    while (passes_ < pass_limit)
    {
        const double left = seconds - report.gpu_seconds;
        if (passes_ > 0 && report.launches > 0 && left < 0.25 * std::min(seconds, options_.launch_seconds))
        {
            break;
        }
        const double budget = std::max(1e-4, std::min(options_.launch_seconds, left));
        const double t = launch(plan(pass_limit, budget));
        ++report.launches;
        report.kernel_launches += last_kernel_launches_;
        report.gpu_seconds += t;
        report.longest_launch_seconds = std::max(report.longest_launch_seconds, t);
        if (report.gpu_seconds >= seconds && passes_ > 0)
        {
            break;
        }
    }
    report.state = state();
    return report;
}

void session::pixels(double* out, int64_t count) const
{
    const int64_t n = static_cast<int64_t>(camera_.image_width) * camera_.image_height * 3;
    if (count != n)
    {
        fail(RT_ERR_INVALID, "pixels: the buffer must hold width * height * 3 doubles");
    }
    if (passes_ == 0)
    {
        fail(RT_ERR_LOGIC, "pixels: the image has no complete pass");
    }
    check(cudaMemcpyAsync(out, sums_.data(), static_cast<size_t>(n) * sizeof(double), cudaMemcpyDeviceToHost, stream_),
          "copying the image");
    check(cudaStreamSynchronize(stream_), "copying the image");
    const double scale = 1.0 / static_cast<double>(passes_);
    for (int64_t i = 0; i < n; ++i)
    {
        out[i] *= scale;
    }
}

void session::display(const rt_display_options& options, uint8_t* rgba, int64_t byte_count)
{
    check_display(options);
    if (f64_ && options.tone_map != RT_TONE_BOOKS)
    {
        fail(RT_ERR_INVALID, "a tone map other than books is a new display transform, which works in float only");
    }
    const int64_t n = static_cast<int64_t>(camera_.image_width) * camera_.image_height * 4;
    if (byte_count != n)
    {
        fail(RT_ERR_INVALID, "display: the buffer must hold width * height * 4 bytes");
    }
    if (passes_ == 0)
    {
        fail(RT_ERR_LOGIC, "the image has no complete pass to show");
    }
    if (rgba_.size() < static_cast<size_t>(n))
    {
        rgba_.allocate_async(static_cast<size_t>(n), stream_);
    }
    // 1 / passes, as pixels() scales: a books byte equals the CPU writer's byte of the same pixel
    launch_display(sums_.data(), camera_.image_width, camera_.image_height, 1.0 / static_cast<double>(passes_), options,
                   rgba_.data(), stream_);
    check(cudaMemcpyAsync(rgba, rgba_.data(), static_cast<size_t>(n), cudaMemcpyDeviceToHost, stream_),
          "copying the display's bytes");
    check(cudaStreamSynchronize(stream_), "converting the image for the display");
}

uint64_t session::rays() const
{
    unsigned long long v = 0;
    check(cudaMemcpy(&v, counters_.data() + 1, sizeof(v), cudaMemcpyDeviceToHost), "reading the ray count");
    return v;
}

void session::fetch_counts(uint64_t out[4]) const
{
    unsigned long long v[4] = {};
    check(cudaMemcpy(v, counters_.data() + 3, sizeof(v), cudaMemcpyDeviceToHost), "reading the fetch counts");
    for (int i = 0; i < 4; ++i)
    {
        out[i] = v[i];
    }
}

uint64_t session::shadow_rays() const
{
    unsigned long long v = 0;
    check(cudaMemcpy(&v, counters_.data() + 2, sizeof(v), cudaMemcpyDeviceToHost), "reading the ray count");
    return v;
}

rt_kernel_info session::kernel() const
{
    kernel_attributes a{};
    if (wavefront_ && !counting_)
    {
        kernel_attributes shade{};
        check(wave_attributes(scene_->view(), scene_->quality(), shade, a, shape_.trace_min_blocks),
              "querying the wavefront kernels");
        a.blocks_per_sm = tuned_.trace_blocks_per_sm; // the trace kernel's launch, as the shape has it
    }
    else if (f64_)
    {
        check(render_f64_attributes(*scene_->view_f64(), a), "querying the FP64 render kernel");
    }
    else
    {
        check(render_attributes(scene_->view(), scene_->quality(), a), "querying the render kernel");
    }
    rt_kernel_info info{};
    const char* form = wavefront_ && !counting_ ? "wavefront" : "persistent";
    std::snprintf(info.name, sizeof(info.name), "%s %s", form,
                  f64_ ? "books fp64" : (scene_->quality() ? "nee-mis" : "books"));
    info.registers = a.registers;
    info.local_bytes = a.local_bytes;
    info.blocks_per_multiprocessor = a.blocks_per_sm;
    info.threads_per_block = a.threads_per_block;
    info.max_threads_per_multiprocessor = a.max_threads_per_sm;
    info.multiprocessors = a.multiprocessors;
    return info;
}
} // namespace rtb
