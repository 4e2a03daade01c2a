// The host runtime behind the C-ABI: errors, device memory, the resident scene and the session.
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "device_types.h"
#include "kernels.cuh"
#include "rt_b200.h"

namespace rtb
{
// An error with the status the C-ABI returns for it (the reference's exception classes, renderer.h:518-526)
struct rt_error : std::runtime_error
{
    rt_status status;
    rt_error(rt_status s, const std::string& message) : std::runtime_error(message), status(s) {}
};

[[noreturn]] void fail(rt_status status, const std::string& message);
void check(cudaError_t e, const char* what);
// Keeps a message for rt_last_error_message() on this thread
void remember_error(const char* message);

// The library's own stream on the current device (created once per device, non-blocking), from which arrays that
// belong to no session's or batch's stream (a scene's tables, counters) take their memory: the device's memory pool,
// which keeps what is freed. A synchronous cudaMalloc / cudaFree pair per array (a scene has about thirty) held the
// host for hundreds of milliseconds now and then on the B200 machines; the pool maps its memory once.
cudaStream_t allocation_stream();

// Device memory owned by one object, freed with it
template <class T>
class device_array
{
public:
    device_array() = default;
    explicit device_array(size_t count) { allocate(count); }
    ~device_array() { release(); }
    device_array(const device_array&) = delete;
    device_array& operator=(const device_array&) = delete;
    device_array(device_array&& o) noexcept
        : data_(o.data_), count_(o.count_), stream_(o.stream_), device_(o.device_)
    {
        o.data_ = nullptr;
        o.count_ = 0;
    }
    device_array& operator=(device_array&& o) noexcept
    {
        if (this != &o)
        {
            release();
            data_ = o.data_;
            count_ = o.count_;
            stream_ = o.stream_;
            device_ = o.device_;
            o.data_ = nullptr;
            o.count_ = 0;
        }
        return *this;
    }

    // Usable by any stream of the current device on return (as cudaMalloc's), from the memory pool
    void allocate(size_t count)
    {
        release();
        if (count > 0)
        {
            const cudaStream_t s = allocation_stream();
            check(cudaGetDevice(&device_), "querying the device");
            check(cudaMallocAsync(reinterpret_cast<void**>(&data_), count * sizeof(T), s), "allocating device memory");
            check(cudaStreamSynchronize(s), "allocating device memory");
        }
        count_ = count;
    }
    void upload(const std::vector<T>& host)
    {
        allocate(host.size());
        if (!host.empty())
        {
            check(cudaMemcpy(data_, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice), "copying to the device");
        }
    }
    // Stream-ordered, from the device's memory pool (no device-wide synchronisation; the pool keeps freed memory for
    // the next request): for arrays that come and go while kernels run, as a server's requests do. `stream` must
    // outlive the array.
    void allocate_async(size_t count, cudaStream_t stream)
    {
        release();
        if (count > 0)
        {
            check(cudaMallocAsync(reinterpret_cast<void**>(&data_), count * sizeof(T), stream),
                  "allocating device memory");
            stream_ = stream;
        }
        count_ = count;
    }
    void release()
    {
        if (data_)
        {
            if (stream_)
            {
                cudaFreeAsync(data_, stream_);
            }
            else
            {
                // as cudaFree: once the array's device has finished every kernel that may read it
                int current = 0;
                cudaGetDevice(&current);
                if (current != device_)
                {
                    cudaSetDevice(device_);
                }
                cudaDeviceSynchronize();
                cudaFreeAsync(data_, allocation_stream());
                if (current != device_)
                {
                    cudaSetDevice(current);
                }
            }
        }
        data_ = nullptr;
        count_ = 0;
        stream_ = nullptr;
    }
    T* data() const { return data_; }
    size_t size() const { return count_; }
    size_t bytes() const { return count_ * sizeof(T); }

private:
    T* data_ = nullptr;
    size_t count_ = 0;
    cudaStream_t stream_ = nullptr; // set when allocated stream-ordered on a caller's stream
    int device_ = 0;                // where allocate() took it
};

// The display transform (display.cu): the options' check (renderer.cu:1204-1220) and the kernel over an image's sums
// times `scale`, queued on `stream`
constexpr double max_exposure_stops = 24; // renderer.h:303
void check_display(const rt_display_options& options);
void launch_display(const double* sums, int width, int height, double scale, const rt_display_options& options,
                    uint8_t* rgba, cudaStream_t stream);
// The image files (image_io.cpp): PFM and PNG writers, the mean radiance
void save_image(const char* path, const double* pixels, int width, int height, const rt_display_options& options);
double mean_radiance(const double* pixels, int64_t pixel_count);
// A PNG's bytes already computed (8-bit RGBA, rows from the top) written as an RGB PNG
void save_png_rgba(const char* path, const uint8_t* rgba, int width, int height);

// Checks a scene's tables before anything is built (the reference's validate, renderer.cu:688-900); throws rt_error
void validate(const rt_scene_desc& desc);

// Whether the quads bound a convex shape (renderer.h:163-168 is_convex), the boundary a volume of smoke may have
bool is_convex(const rt_quad_desc* quads, int64_t count);

// The camera in the kernels' form: the pixel grid relative to the center subtracted in double (renderer.cu:512-532)
camera_params to_camera(const rt_camera_desc& desc);
camera_d to_camera_d(const rt_camera_desc& desc);

// A scene on the device: its BVH, primitives, materials, lights and lamps, uploaded once
class resident_scene
{
public:
    explicit resident_scene(const rt_scene_desc& desc);

    const scene_view& view() const { return view_; }
    const rt_camera_desc& camera() const { return camera_; }
    bool quality() const { return quality_; }
    const int32_t* prim_source() const { return prim_source_.data(); }
    const rt_scene_stats& stats() const { return stats_; }
    int device() const { return device_; }
    // The double tables for the books' integrator in FP64, made for the scenes it can render (no NEE/MIS, no
    // triangles); null otherwise
    const scene_view_f64* view_f64() const { return has_f64_ ? &view_f64_ : nullptr; }

private:
    int device_ = 0;
    rt_camera_desc camera_{};
    bool quality_ = false;
    scene_view view_{};
    bool has_f64_ = false;
    scene_view_f64 view_f64_{};
    device_array<sphere_d> spheres_d_;
    device_array<motion_d> sphere_motion_d_;
    device_array<frame_d> sphere_frames_d_;
    device_array<quad_d> quads_d_;
    device_array<material_d> materials_d_;
    device_array<light_d> lights_d_;
    device_array<texture_d> textures_d_;
    device_array<noise_d> noises_d_;
    device_array<medium_d> media_d_;
    device_array<quad_d> boundary_quads_d_;
    rt_scene_stats stats_{};
    device_array<bvh_node> nodes_;
    device_array<bvh4_node> wide_nodes_;
    device_array<sphere4> spheres_;
    device_array<quad12> quads_;
    device_array<triangle12> triangles_;
    device_array<int32_t> prim_material_;
    device_array<int32_t> prim_source_;
    device_array<material12> materials_;
    device_array<light24> lights_;
    device_array<emitter20> lamps_;
    device_array<int32_t> lamp_of_;
    device_array<env_texel> env_texels_;
    device_array<alias_bin> env_bins_;
    device_array<float> env_row_cos_;
    device_array<float4> sphere_motion_;
    device_array<sphere_frame> sphere_frames_;
    device_array<texture8> textures_;
    device_array<image_info> images_;
    device_array<float4> texels_;
    device_array<noise_table> noises_;
    device_array<medium16> media_;
    device_array<quad12> boundary_quads_;
};

// The environment map's tables (environment_table.cu:81-226 build_environment): texels with their densities Y/S,
// Vose's alias table over the cells (coins on the 2^-24 grid, error diffusion), the rows' cosines
struct environment_tables
{
    int width = 0, height = 0, log2_bins = 0;
    double total = 0;
    std::vector<env_texel> texels;
    std::vector<alias_bin> bins;
    std::vector<float> row_cos;
};
environment_tables build_environment(const rt_environment_desc& env);

// The device's memory pool keeps what is freed for the next stream-ordered allocation (a setting of this process's
// pool): the scratch that comes and goes with renders, views and requests is mapped once, not on every allocation
void retain_pool_memory();

// Page-locked host memory for what the host writes for kernels or reads back while they run (queue lengths, counters,
// job tables), from a process-wide cache: a block given back is kept for the next request of its size, never freed,
// because cudaFreeHost can hold the calling thread for hundreds of milliseconds (measured on the B200: 200-270 ms in
// some session teardowns, the end of a render() call)
void* acquire_pinned(size_t bytes);
void release_pinned(void* block, size_t bytes);

// The wavefront's host side: its buffers, sized to a launch's samples (slots: at most max_slots) and kept for the next,
// and the loop of steps, in groups of `group` with two groups in flight, until a step queues no ray
class wave_runner
{
public:
    wave_runner(int max_slots_, int group_);
    ~wave_runner();
    wave_runner(const wave_runner&) = delete;
    wave_runner& operator=(const wave_runner&) = delete;

    // Buffers from the device's memory pool, stream-ordered on `stream` (which must outlive the runner): a one-shot
    // render that needs them takes them from what earlier renders left in the pool
    wave_buffers setup(int64_t samples, cudaStream_t stream);
    // step() enqueues one step on `stream`; returns the steps run
    // The steps of one launch until a step queues nothing. step(draining) launches one; draining is true once the
    // host has seen every sample of the launch claimed (work_counter, when given, at sample_count or beyond): the
    // shade kernel then reads a slot's rows only if the slot still has work.
    int64_t run(const wave_buffers& b, int max_depth, cudaStream_t stream,
                const std::function<cudaError_t(bool draining)>& step,
                const unsigned long long* work_counter = nullptr);

    const int max_slots;
    const int group;

private:
    device_array<unsigned char> slots_;
    device_array<float4> query_o_;
    device_array<float4> query_d_;
    device_array<int4> query_meta_;
    device_array<int4> ext_result_;
    device_array<int32_t> shadow_result_;
    device_array<unsigned> control_;
    device_array<float4> samples_;
    unsigned* queued_ = nullptr; // pinned: the queue's length after each group of steps
    unsigned long long* claimed_ = nullptr; // pinned: the launch's work counter after each group
    cudaEvent_t done_[2] = {nullptr, nullptr};
};

// The wavefront's slots (paths in flight: 2^20 take 160 MB, and their queries 96 MB) and its steps per group between
// two looks at the queue's length. Measured on the B200 from 2^18 to 3 x 2^20 slots: the mesh gains up to 3 x 2^20
// (+11% from 2^20 to 1.5 x 2^20, +7.5% more to 3 x 2^20: a step's queries must outlast its slowest, longest walk), the
// bare flat scenes up to 1.5 x 2^20 (+3% on the glass Cornell box; the lamp-lit one loses 6% at 3 x 2^20), while the
// sphere trees and the textured scenes lose 5-7% past 2^20 (wave_slots_for). The batch engine's pool is the mesh's
// (its 64-job batch of sphere trees: +3.5% from 1.5 x 2^20 to 3 x 2^20).
#ifndef RTB_WAVE_SLOTS
#define RTB_WAVE_SLOTS (1 << 20)
#endif
#ifndef RTB_WAVE_SLOTS_LARGE
#define RTB_WAVE_SLOTS_LARGE (3 << 19)
#endif
#ifndef RTB_WAVE_SLOTS_MESH
#define RTB_WAVE_SLOTS_MESH (3 << 20)
#endif
#ifndef RTB_WAVE_GROUP
#define RTB_WAVE_GROUP 8
#endif
constexpr int wave_slots = RTB_WAVE_SLOTS / render_block * render_block;
constexpr int wave_slots_large = RTB_WAVE_SLOTS_LARGE / render_block * render_block;
constexpr int wave_slots_mesh = RTB_WAVE_SLOTS_MESH / render_block * render_block;
constexpr int wave_group = RTB_WAVE_GROUP;
// The pool for a scene: the largest for a scene with triangles, the larger one for a flat-searched one without
// textures, motion or smoke
inline int wave_slots_for(const scene_view& v)
{
    const bool triangles = v.prim_count > v.triangle_base;
    if (triangles)
    {
        return wave_slots_mesh;
    }
    return v.flat != 0 && !has_features(v) ? wave_slots_large : wave_slots;
}

// The wavefront's autotuner (tuner.cpp): a launch shape, the knobs' candidate values, and the search
struct tune_candidate
{
    int slots;
    int trace_blocks_per_sm;
    int shade_block;
    int trace_min_blocks;
};
struct tune_space
{
    std::vector<std::pair<int, int>> trace; // (register cap as min blocks, blocks per multiprocessor)
    std::vector<int> slots;
    std::vector<int> shade_blocks;
};
struct tune_outcome
{
    tune_candidate best;
    double best_speed;
    double default_speed;
    int trials;
};
tune_space default_tune_space(int max_trace_blocks, int max_trace_blocks_roomy);
tune_candidate default_candidate(int slots, int max_trace_blocks);
rt_tuning to_tuning(const tune_candidate& c);
tune_outcome coordinate_descent(const tune_candidate& start, const tune_space& space,
                                const std::function<double(const tune_candidate&)>& measure);
std::tuple<int, int, int, int, int, int, int> tune_key(int device, const scene_view& v, bool quality);
bool cached_tuning(const std::tuple<int, int, int, int, int, int, int>& key, tune_candidate& out);
void remember_tuning(const std::tuple<int, int, int, int, int, int, int>& key, const tune_candidate& c);
void forget_tunings();

// One view of a resident scene whose image gains passes on demand (renderer.h:591-673)
class session
{
public:
    session(std::shared_ptr<resident_scene> scene, const rt_session_options& options);
    ~session();
    session(const session&) = delete;
    session& operator=(const session&) = delete;

    void set_camera(const rt_camera_desc& camera);
    rt_accumulation state() const { return {passes_, 0, 0}; }
    rt_render_report render_to(int64_t target);
    rt_render_report render_for(double seconds, int64_t pass_limit);
    void pixels(double* out, int64_t count) const;
    uint64_t rays() const;
    uint64_t shadow_rays() const;
    double kernel_seconds() const { return kernel_seconds_; }
    rt_kernel_info kernel() const;
    const double* device_sums() const { return sums_.data(); }
    // The autotuner: short renders of this view under candidate launch shapes (the view must have no passes yet; it
    // starts over afterwards), the best shape kept for this session and remembered for its scene class
    rt_tuning autotune(int64_t trial_passes);
    rt_tuning tuning() const { return tuning_; }
    // A launch shape given by the caller (one an earlier autotune reported, kept across processes)
    void set_tuning(const rt_tuning& t);
    // Per-kernel timing (events around every kernel of every launch; slows launches a little): rt_kernel_times
    void set_timing(bool on) { timing_ = on; }
    rt_kernel_times kernel_times() const { return times_; }
    // session::display(options): the complete passes' bytes, 4 per pixel, into host memory
    void display(const rt_display_options& options, uint8_t* rgba, int64_t byte_count);
    int64_t passes() const { return passes_; }
    // The counting build: launches that also count node fetches and primitive tests (slower; for the roofline)
    void set_counting(bool on)
    {
        if (on && f64_)
        {
            fail(RT_ERR_LOGIC, "the counting build computes in float32");
        }
        counting_ = on;
    }
    void fetch_counts(uint64_t out[4]) const;
    const rt_camera_desc& camera() const { return camera_; }

private:
    std::shared_ptr<resident_scene> scene_;
    rt_session_options options_;
    rt_camera_desc camera_{};
    camera_params cam_{};
    camera_d cam_d_{};  // the same view in double, for an FP64 session
    bool f64_ = false;  // RT_FLOAT64: the books' integrator in double, persistent form
    cudaStream_t stream_ = nullptr;
    cudaEvent_t start_ = nullptr;
    cudaEvent_t stop_ = nullptr;
    device_array<double> sums_;
    device_array<double> partials_;
    device_array<unsigned long long> counters_; // [0] work, [1] rays, [2] shadow rays, [3..6] the counting build's
    device_array<uint8_t> rgba_;                 // the display's bytes, grown on demand
    bool counting_ = false;
    int64_t passes_ = 0;
    double kernel_seconds_ = 0;
    double samples_per_second_ = 0;
    int grid_ = 0;
    int tiles_x_ = 0;
    int padded_pixels_ = 0;
    int64_t max_partial_entries_ = 0;

    // The wavefront form (RT_FORM_WAVEFRONT, or AUTO on a tree-searched scene)
    bool wavefront_ = false;
    std::unique_ptr<wave_runner> wave_;
    int32_t last_kernel_launches_ = 0; // the last launch's kernels
    wave_shape shape_{};                // how a step is launched (the autotuner's choice or the defaults)
    tune_candidate tuned_{};
    rt_tuning tuning_{};
    int multiprocessors_ = 0;
    void apply(const tune_candidate& c);

    // Per-kernel timing: a pool of events, grown as launches need them
    bool timing_ = false;
    rt_kernel_times times_{};
    std::vector<cudaEvent_t> marks_;
    cudaEvent_t* marks(size_t count);

    // Renders passes [passes_, end) in one launch and its reduction; returns its GPU seconds
    double launch(int64_t end);

    int64_t plan(int64_t target, double budget_seconds) const;
};

#ifndef RTB_PASS_CHUNK
#define RTB_PASS_CHUNK 16
#endif
constexpr int pass_chunk = RTB_PASS_CHUNK; // passes per work item; chunk boundaries are absolute multiples of it
} // namespace rtb

// The C-ABI's opaque handles
struct rt_scene
{
    std::shared_ptr<rtb::resident_scene> scene;
};

struct rt_session
{
    std::unique_ptr<rtb::session> session;
};
