// Batched rendering: many jobs (requests) rendered together, one persistent launch per refinement step.
#pragma once

#include <chrono>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <vector>

#include "host.h"

namespace rtb
{
// The jobs of a batch, each a resident scene seen by its own camera, with its own sums, seed and passes. A step
// renders for each chosen job the passes from where it stands to a given end: the jobs of flat-searched scenes in one
// persistent launch of render_batch_kernel per group (captured once into a CUDA graph with the table's copies and
// replayed with new tables), the jobs of tree-searched scenes in the wavefront form, all of a group's jobs in one
// pool of slots, then one reduction of every job's chunk partials into its sums.
class batch_engine
{
public:
    // high_priority: its stream's kernels go ahead of other streams' (a server's first frames beside its continuous
    // wavefront)
    batch_engine(size_t partial_budget_bytes, bool use_graph, bool high_priority = false);
    ~batch_engine();
    batch_engine(const batch_engine&) = delete;
    batch_engine& operator=(const batch_engine&) = delete;

    // A new job; returns its handle. Its sums (24 bytes a pixel) are allocated here and stay resident until remove.
    int add(std::shared_ptr<resident_scene> scene, const rt_camera_desc& camera, uint64_t seed, uint32_t job_id);
    void remove(int handle);

    struct assignment
    {
        int handle;
        int64_t pass_end;
    };
    // One step; returns its GPU seconds. Jobs whose partials do not fit the arena this step are cut back to fewer
    // chunks (at least one each), so every assignment makes progress.
    double step(std::vector<assignment> work);

    // The wavefront's buffers for steps of up to `samples` samples and its kernels loaded now, not on first use
    void reserve_wavefront(int64_t samples);
    // The device's memory pool grown to `bytes` now (the jobs' sums come from it), so that admitting requests
    // maps no new memory
    void reserve_pool(size_t bytes);
    int64_t passes(int handle) const;
    void pixels(int handle, double* out, int64_t count);
    // The job's sums (width * height * 3 doubles) into device memory, complete on return
    void copy_sums(int handle, double* device_out);
    // The job's image through the display transform, 4 bytes per pixel into host memory
    void display(int handle, const rt_display_options& options, uint8_t* out, int64_t count);
    uint64_t rays(int handle) const;
    uint64_t shadow_rays(int handle) const;
    size_t job_bytes(const rt_camera_desc& camera) const;
    int64_t partial_entries() const { return max_partial_entries_; }
    int launches() const { return launches_; }
    int64_t last_samples() const { return last_samples_; } // pixel passes the last step rendered
    bool graph_used() const { return graph_exec_ != nullptr; }
    int grid() const { return grids_[persistent_groups - 1]; }
    // The chunks of [passes, pass_end) for a job of the given camera, and its padded pixel count
    static int64_t chunks_of(int64_t passes, int64_t pass_end);
    static int64_t padded_of(const rt_camera_desc& camera);

private:
    struct job
    {
        std::shared_ptr<resident_scene> scene;
        rt_camera_desc camera{};
        camera_params cam{};
        uint64_t seed = 0;
        uint32_t id = 0;
        device_array<double> sums;
        device_array<unsigned long long> counters; // [0] segments, [1] shadow rays
        int64_t passes = 0;
        int tiles_x = 0;
        int padded = 0;
    };
    std::map<int, std::unique_ptr<job>> jobs_;
    int next_handle_ = 0;
    bool use_graph_;
    int64_t max_partial_entries_;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t start_ = nullptr;
    cudaEvent_t stop_ = nullptr;
    int grids_[persistent_groups] = {}; // each persistent group's launch (batch_group)
    std::unique_ptr<wave_runner> wave_;  // the wavefront's groups (wave_batch_group), one after another
    int trace_grid_ = 0;
    device_array<double> arena_;
    device_array<batch_job> table_;
    device_array<batch_header> header_;
    device_array<unsigned long long> work_counter_;
    device_array<uint8_t> rgba_; // a job's display bytes, grown on demand
    batch_job* table_host_ = nullptr;   // pinned
    batch_header* header_host_ = nullptr;
    size_t capacity_ = 0;               // jobs the table (and the captured graph) hold
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
    int launches_ = 0;
    int64_t last_samples_ = 0;

    void ensure_capacity(size_t jobs, size_t partial_doubles);
    void capture();
    void release_graph();
};

// The server's continuous wavefront: one pool of path slots for the server's life, into which requests' samples
// are published in segments as they are scheduled (first frames at once, refinement while the unclaimed backlog is
// short), steps launched in groups two at a time, each finished segment reduced into its request's image (stream.cpp)
class stream_engine
{
public:
    stream_engine(int slots, int64_t value_capacity, int group_steps, double lookahead_seconds);
    ~stream_engine();
    stream_engine(const stream_engine&) = delete;
    stream_engine& operator=(const stream_engine&) = delete;

    // A request: its view of a resident scene, RNG seed and job field, and target passes. Its first pass is published
    // at the next advance, or, with first_pass_elsewhere, rendered by the caller into sums(handle) and handed over by
    // first_pass_done. Its sums and accumulator (48 bytes a pixel) stay resident until remove.
    int add(std::shared_ptr<resident_scene> scene, const rt_camera_desc& camera, uint64_t seed, uint32_t job_id,
            int64_t target, bool first_pass_elsewhere = false);
    double* sums(int handle) { return requests_.at(handle)->sums.data(); }
    // The request's first pass is in its sums (written and complete before the call): refinement may start
    void first_pass_done(int handle);
    // Stops publishing the request's samples, waits for those in flight and frees its memory
    void remove(int handle);
    // Runs groups of steps until at least `seconds` of GPU time have been read back (one group at least when there is
    // work); returns the GPU seconds read. A group may still be running on return.
    double advance(double seconds);
    bool has_work() const;
    // The device's memory pool grown to `bytes` now (the requests' sums come from it)
    void reserve_pool(size_t bytes);
    int64_t passes(int handle) const; // complete passes in the request's sums
    void pixels(int handle, double* out, int64_t count);
    void display(int handle, const rt_display_options& options, uint8_t* out, int64_t count);
    uint64_t rays(int handle) const;
    uint64_t shadow_rays(int handle) const;
    int64_t launches() const { return launches_; }
    double gpu_seconds() const { return gpu_seconds_; }
    int64_t groups() const { return groups_; }
    // the mean over groups of the slots that queued a ray in the group's last step, as a fraction of the pool
    double busy_slots() const { return groups_ > 0 ? busy_sum_ / static_cast<double>(groups_) : 0.0; }
    static size_t job_bytes(const rt_camera_desc& camera);

private:
    struct request
    {
        std::shared_ptr<resident_scene> scene;
        bool awaiting_first = false; // its first pass is rendered elsewhere and not yet handed over
        rt_camera_desc camera{};
        camera_params cam{};
        uint64_t seed = 0;
        uint32_t id = 0;
        int64_t target = 0;
        int tiles_x = 0;
        int64_t padded = 0;
        device_array<double> sums;
        device_array<double> acc; // the chunk accumulator: the passes since the sums' last addition
        device_array<unsigned long long> counters;
        int64_t published = 0; // its samples published, reduced (pass-major numbering)
        int64_t reduced = 0;
        int64_t passes = 0;
        bool cancelled = false;
        std::deque<int64_t> segments; // its segments in flight, oldest first
    };
    struct segment
    {
        int handle = -1; // the request; -1 once reduced
        bool finished = false;
        int64_t local_begin = 0;
        int64_t local_end = 0;
        int64_t global_begin = 0;
        int64_t value_offset = 0;
    };

    // What a group reads from the host when it starts: the published limit and the window of segments
    struct group_control
    {
        int64_t published;
        int32_t window_first;
        int32_t window_end;
    };

    int64_t value_room(int64_t count) const;
    cudaGraphExec_t group_graph(int k);
    int64_t publish(int handle, request& r, int64_t count);
    void schedule();
    void launch_group();
    double finish_group();
    bool reduce_finished(int group);
    static size_t readback_bytes();

    const int slot_count_;
    const int64_t value_capacity_;
    const int group_steps_;          // wavefront steps between two readings of the counts
    const double lookahead_seconds_; // the unclaimed backlog refinement keeps, in GPU time
    cudaStream_t stream_ = nullptr;
    cudaStream_t reduce_stream_ = nullptr;
    cudaEvent_t group_start_[2] = {};
    cudaEvent_t group_done_[2] = {};
    cudaEvent_t reduced_ = nullptr;
    device_array<unsigned char> slots_;
    device_array<float4> query_o_;
    device_array<float4> query_d_;
    device_array<int4> query_meta_;
    device_array<int4> ext_result_;
    device_array<int32_t> shadow_result_;
    device_array<unsigned> control_;
    device_array<unsigned long long> counters_;
    device_array<batch_job> table_;
    device_array<unsigned long long> done_;
    device_array<int64_t> starts_; // each ring entry's first sample
    device_array<float4> values_;
    device_array<stream_reduce_item> reduce_items_;
    device_array<uint8_t> rgba_;
    unsigned char* readback_ = nullptr; // pinned, one per group in flight
    group_control* staging_ = nullptr;  // pinned, one per group in flight
    cudaGraphExec_t graphs_[8] = {};    // (features, wide, group slot)
    std::vector<batch_job> table_host_;
    std::vector<segment> segments_;
    wave_buffers buffers_{};
    int trace_grid_ = 0;
    std::map<int, std::unique_ptr<request>> requests_;
    std::vector<int> fresh_; // requests whose first pass is not yet published
    int next_handle_ = 0;
    int64_t next_segment_ = 0;   // logical segment numbers: [oldest_segment_, next_segment_) hold table entries
    int64_t oldest_segment_ = 0;
    int live_segments_ = 0;      // published and not yet reduced
    int64_t published_ = 0;      // samples published
    int64_t taken_ = 0;          // samples surely taken by a slot
    int64_t value_head_ = 0;
    int64_t group_limit_[2] = {};    // each group in flight: the published limit it runs with
    int64_t group_segments_[2] = {}; // and the segments published before it
    int group_index_ = 0;
    int in_flight_ = 0;
    double claim_rate_ = 0;      // samples taken per GPU second, smoothed
    double group_seconds_ = 0;   // a group's GPU time, smoothed
    bool features_ = false;      // the kernels' variant: any scene with the second book's features
    bool wide_ = true;           // every scene's tree four wide
    unsigned long long last_progress_ = 0; // the claims and finished samples last read
    int stalled_groups_ = 0;               // groups read since they last changed
    int64_t launches_ = 0;
    double gpu_seconds_ = 0;
    int64_t groups_ = 0;
    double busy_sum_ = 0;
};

// The server of a stream of render requests: requests are admitted under an HBM budget, every
// step gives the newly admitted their first frame (one pass) before it refines the others, and a request is done when
// it reaches its target passes. Driven by the caller: submit between steps, step, poll, fetch. Its steps are batches
// of passes (batch_engine) or runs of the continuous wavefront (stream_engine).
class render_server
{
public:
    explicit render_server(const rt_server_options& options);

    int64_t submit(std::shared_ptr<resident_scene> scene, const rt_camera_desc& camera, uint64_t seed, int64_t target);
    rt_server_step_report step();
    rt_request_status poll(int64_t id) const;
    void fetch(int64_t id, double* pixels, int64_t count);
    void display(int64_t id, const rt_display_options& options, uint8_t* rgba, int64_t count);
    void cancel(int64_t id);
    rt_server_stats stats() const;

private:
    using clock = std::chrono::steady_clock;
    struct request
    {
        int64_t id;
        std::shared_ptr<resident_scene> scene;
        rt_camera_desc camera;
        uint64_t seed;
        int64_t target;
        int handle = -1;
        int first_handle = -1; // the continuous server: its first frame's job in the batch engine, until handed over
        int32_t state = RT_REQUEST_QUEUED;
        clock::time_point submitted;
        double first_frame_seconds = -1;
        double done_seconds = -1;
        size_t bytes = 0;
    };
    rt_server_options options_;
    std::unique_ptr<batch_engine> engine_;  // batched steps (the continuous server: its first frames)
    std::unique_ptr<stream_engine> stream_; // the continuous wavefront (refinement)
    std::map<int64_t, request> requests_;
    std::deque<int64_t> queue_;
    std::deque<int64_t> first_queue_; // the continuous server: admitted requests whose first frame is still to render
    uint64_t first_rays_ = 0;          // and the rays of the first frames it has handed over
    uint64_t first_shadow_rays_ = 0;
    // the estimated GPU time of a step of first frames (at least one frame a step)
    static constexpr double first_frame_seconds = 0.004;
    int64_t next_id_ = 1;
    size_t used_bytes_ = 0;
    std::map<const resident_scene*, double> cost_; // seconds per pixel pass, learned per scene
    double default_cost_ = 0;                      // the same over every scene, for a scene not seen yet
    rt_server_stats stats_{};

    int64_t passes_of(const request& r) const;
    rt_server_step_report step_continuous();
    void release(request& r);
    double cost_of(const resident_scene* scene) const;
    void learn_costs(const std::vector<std::pair<const resident_scene*, double>>& samples, double seconds);
};
} // namespace rtb

struct rt_server
{
    std::unique_ptr<rtb::render_server> server;
};
