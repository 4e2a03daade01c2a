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
    batch_engine(size_t partial_budget_bytes, bool use_graph);
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

// The server of a stream of render requests: requests are admitted under an HBM budget, every
// step gives the newly admitted their first frame (one pass) before it refines the others, and a request is done when
// it reaches its target passes. Driven by the caller: submit between steps, step, poll, fetch.
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
        int32_t state = RT_REQUEST_QUEUED;
        clock::time_point submitted;
        double first_frame_seconds = -1;
        double done_seconds = -1;
        size_t bytes = 0;
    };
    rt_server_options options_;
    batch_engine engine_;
    std::map<int64_t, request> requests_;
    std::deque<int64_t> queue_;
    int64_t next_id_ = 1;
    size_t used_bytes_ = 0;
    std::map<const resident_scene*, double> cost_; // seconds per pixel pass, learned per scene
    double default_cost_ = 0;                      // the same over every scene, for a scene not seen yet
    rt_server_stats stats_{};

    double cost_of(const resident_scene* scene) const;
    void learn_costs(const std::vector<std::pair<const resident_scene*, double>>& samples, double seconds);
};
} // namespace rtb

struct rt_server
{
    std::unique_ptr<rtb::render_server> server;
};
