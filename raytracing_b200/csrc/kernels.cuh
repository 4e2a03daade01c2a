// The launch interface between the host code (session.cpp) and the kernels (kernels.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "device_types.h"

namespace rtb
{
// One launch of the persistent render kernel: passes [pass_begin, pass_end) of every pixel of one view, cut into
// work items (pixel, chunk of passes). Chunks are aligned to absolute multiples of `chunk` passes, so an image of N
// passes is the same bit for bit however its passes were grouped into launches, as long as launches start and end
// on chunk boundaries.
struct launch_params
{
    scene_view scene;
    camera_params cam;
    uint64_t seed;          // round r of strata draws with seed + r * 2^32 (renderer.h:564-584)
    int64_t pass_begin;
    int64_t pass_end;
    int64_t first_chunk;    // pass_begin / chunk
    int32_t chunk;          // passes per work item
    int32_t chunks;         // work items per pixel in this launch
    int32_t tiles_x;        // the image in tiles of 8 x 4 pixels, a warp's worth
    int32_t padded_pixels;  // tiles * 32
    int64_t total_items;    // chunks * padded_pixels
    int32_t round_passes;   // sqrt_spp^2
    uint32_t job;           // a request's id in the RNG counter (0 for a plain render)
    unsigned long long* work_counter;
    double* partials;       // chunks * padded_pixels * 3
    unsigned long long* counters; // [0] path segments, [1] shadow rays; the counting build also [2] node fetches,
                                  // [3] sphere, [4] quad, [5] triangle tests
};

struct reduce_params
{
    const double* partials;
    double* sums;           // width * height * 3
    int32_t width, height;
    int32_t tiles_x;
    int32_t padded_pixels;
    int32_t chunks;
};

// One job of a batched launch: a resident scene's view, its camera, and the passes this step renders of it. Its work
// items are numbered from item_begin in the batch's item space, its pixels from pixel_begin in the batch's pixel
// space (for the reduction); partials is its own slice of the batch's partials arena. A job of a group the wavefront
// renders numbers its samples from sample_begin in its group's sample space.
struct alignas(16) batch_job
{
    scene_view scene;
    camera_params cam;
    uint64_t seed;
    int64_t pass_begin;
    int64_t pass_end;
    int64_t first_chunk;
    int64_t item_begin;
    int64_t pixel_begin;
    int64_t sample_begin;
    double* partials;
    double* sums;                 // width * height * 3, this job's
    unsigned long long* counters; // [0] segments, [1] shadow rays, this job's, accumulated
    int32_t chunk;
    int32_t chunks;
    int32_t tiles_x;
    int32_t padded_pixels;
    int32_t round_passes;
    int32_t quality;
    uint32_t job;                 // the RNG counter's job field
    int32_t pad0;
    // A stream run's segment (the server's continuous wavefront): its samples are [sample_begin, sample_begin +
    // pass-major count) of the run's sample space, numbered within the request from local_begin; their values go to
    // values[local - local_begin] and each finished one is counted in *done
    float4* values;
    unsigned long long* done;
    int64_t local_begin;
};

// Whether a scene has any of the second book's features (moving spheres, textures other than solid colors, smoke):
// its kernels are compiled with their code, the others without
inline bool has_features(const scene_view& s) { return s.has_motion != 0 || s.has_textures != 0 || s.medium_count > 0; }

// Whether a scene renders in the wavefront form unless a form is asked for: every tree-searched scene (its walks
// diverge: the mesh 3.2 times and the sphere scenes 1.2-2 times as fast as in the persistent kernel) and a
// flat-searched scene whose shading is heavy (lights or lamps, the second book's features, an environment: the glass
// Cornell box 10-16% faster, the marble spheres 55%); the bare small flat scenes (five spheres or five quads under
// the sky), whose paths are one or two cheap segments that cannot pay for the slots' traffic, stay in the persistent
// kernel (40% slower in the wavefront).
inline bool wavefront_suits(const scene_view& v)
{
    const bool heavy = v.light_count > 0 || v.lamp_count > 0 || has_features(v) || v.has_environment;
    return v.node_count > 0 && (v.flat == 0 || heavy);
}

// The jobs come in eight groups: the scenes of each search (flat, tree) without and with the second book's features,
// in each form. The first four are rendered each by its own launch of the persistent kernel compiled for it
// (batch_group), the other four each by its own run of the wavefront's steps (wave_batch_group); a scene takes the
// form wavefront_suits gives it, as a session's render of it does.
constexpr int persistent_groups = 4;
constexpr int batch_groups = 8;
RTB_HD constexpr int batch_group(bool flat, bool features) { return (flat ? 0 : 2) + (features ? 1 : 0); }
RTB_HD constexpr int wave_batch_group(bool flat, bool features) { return persistent_groups + batch_group(flat, features); }

struct batch_header
{
    int64_t total_pixels;
    int64_t group_items[batch_groups + 1]; // group g's items are [group_items[g], group_items[g + 1])
    int32_t group_jobs[batch_groups + 1];  // and its jobs [group_jobs[g], group_jobs[g + 1])
    int32_t job_count;
    int32_t pad0;
};

struct batch_params
{
    const batch_job* jobs;
    const batch_header* header;
    unsigned long long* work_counter; // one per group's launch
};

// The batch engine's groups of tree-searched jobs in the wavefront form: the jobs [job_first, job_end) of the table,
// their samples numbered from 0 (job j's from jobs[j].sample_begin) up to the wave_buffers' sample_count
struct wave_batch
{
    const batch_job* jobs;
    int32_t job_first;
    int32_t job_end;
    int64_t item_first; // the group's work items [item_first, item_end) in the batch's item space
    int64_t item_end;
    unsigned long long* work_counter; // the group's samples taken so far (zero at the start)
    // A stream run (the server's continuous wavefront; null in a batch's run): samples are claimed up to *published,
    // a claim beyond it waits in its slot until the host publishes that far; the jobs are segments in a ring of
    // job_mask + 1 entries, the window window[0] .. window[1] counted without wrapping (in device memory with the
    // limit, so that one captured graph of steps serves every group)
    const unsigned long long* published;
    int32_t job_mask;
    int32_t pad0;
    const int32_t* window;
    const int64_t* starts; // each ring entry's first sample (its sample_begin), compact for the claims' search
};

// The stream run's reduction: each item a segment's samples added, pixel by pixel in pass order, into its request's
// chunk accumulator, which goes into the request's sums at every chunk's end, after the first pass (the first frame)
// and at the target, as a session adds its chunk partials
struct stream_reduce_item
{
    const float4* values;
    double* sums;
    double* acc;
    int64_t local_begin; // the segment's samples [local_begin, local_end) of the request's pass-major numbering
    int64_t local_end;
    int64_t pixel_begin; // the item's pixels in the launch's pixel space
    int64_t target;
    int32_t padded_pixels;
    int32_t tiles_x;
    int32_t width;
    int32_t height;
    int32_t chunk;       // passes a chunk (16)
    int32_t pad0;
};
cudaError_t launch_stream_reduce(const stream_reduce_item* items, int32_t count, int64_t total_pixels,
                                 cudaStream_t stream);

// The kernels' static properties for kernel_info
struct kernel_attributes
{
    int registers;
    int local_bytes;
    int blocks_per_sm;
    int threads_per_block;
    int max_threads_per_sm;
    int multiprocessors;
};

constexpr int render_block = 128;

cudaError_t launch_render(const launch_params& p, bool quality, bool counting, int grid, cudaStream_t stream);
cudaError_t launch_reduce(const reduce_params& p, cudaStream_t stream);
// The batched step: the persistent kernel of groups [first_group, end_group) over their jobs' items (grids[g]
// blocks each), and the reduction of every job's pixels
cudaError_t launch_batch(const batch_params& p, const int* grids, int first_group, int end_group, cudaStream_t stream);
cudaError_t launch_batch_reduce(const batch_params& p, int grid, cudaStream_t stream);
cudaError_t batch_attributes(int group, kernel_attributes& out);
// The attributes of the render kernel that launch_render picks for the scene and integrator
cudaError_t render_attributes(const scene_view& scene, bool quality, kernel_attributes& out);

// The wavefront form of a launch, for scenes searched through the tree: `slot_count` resident paths, each the state a
// lane of the persistent kernel keeps in registers (its sample, path and pending shadow ray), advanced by steps of two
// kernels. The shade kernel (one thread per slot) takes the last step's hits, shades, stores finished samples, claims
// new ones and queues each slot's next ray and shadow ray; the trace kernel (persistent) walks the queued rays, each
// lane taking the next query as soon as its own is answered. A step that queues nothing ends the launch, and the
// reduction adds the samples into the sums chunk by chunk, in pass order.
struct wave_buffers
{
    void* slots;            // slot_count slots of wave_slot_bytes() each, cleared before a launch
    int32_t slot_count;     // a multiple of render_block
    float4* samples;        // sample_count: (pass - pass_begin) * padded_pixels + tile slot -> the sample's value
    int64_t sample_count;   // (pass_end - pass_begin) * padded_pixels
    float4* query_o;        // 2 * slot_count queries: origin, time
    float4* query_d;        // direction, t_max
    int4* query_meta;       // from, flags (1 inward, 2 shadow, 4 a camera ray to make; the job << 3), skip, slot
    int4* ext_result;       // per slot: the next ray's hit (id, t's bits, front)
    int32_t* shadow_result; // per slot: 1 if the shadow ray was blocked
    // [0] next rays and shadow rays the last shade step queued (from the bottom), [1] queries the trace kernel took,
    // [2] camera rays it queued (from the top down; tree-searched scenes only); [3] a stream run's error flag (a claim
    // outside the window of segments it was given), never cleared by a step
    unsigned* control;
    camera_params cam;      // a session's launch: its camera and RNG job field (a batch: each job's, in its table)
    uint32_t job;
    int32_t draining;       // every sample is claimed: the shade kernel reads a slot's rows only if it has work
};
size_t wave_slot_bytes();
// Every slot without a sample (its flags row zeroed), before a launch's first step
cudaError_t clear_wave_slots(const wave_buffers& b, cudaStream_t stream);
// How a session's wavefront step is launched (the autotuner's choice): the trace kernel's grid and register cap (its
// minimum resident blocks per multiprocessor: RTB_TRACE_MIN_BLOCKS or wave_trace_roomy_blocks), the shade kernel's
// block size (64 or 128 threads)
constexpr int wave_trace_roomy_blocks = 6;
#ifndef RTB_TRACE_MIN_BLOCKS_DEFAULT
#define RTB_TRACE_MIN_BLOCKS_DEFAULT 8
#endif
struct wave_shape
{
    int trace_grid;
    int shade_block;
    int trace_min_blocks;
};
// One step: clears the queue, the shade kernel over the slots, the trace kernel (shape.trace_grid blocks) over the queue
cudaError_t launch_wave_step(const launch_params& p, bool quality, const wave_buffers& b, const wave_shape& shape,
                             cudaStream_t stream, const cudaEvent_t* marks = nullptr, bool draining = false);
// The samples of passes [pass_begin, pass_end) into the sums (chunk partials in pass order, added in chunk order)
cudaError_t launch_wave_reduce(const reduce_params& r, const wave_buffers& b, int64_t pass_begin, int64_t pass_end,
                               int32_t chunk, cudaStream_t stream);
// The same for a group of batch jobs (flat: the group's scenes are searched flat; features: its kernels compile the
// second book's features; wide: every job's tree is four wide; quality: some job uses the NEE/MIS integrator, which
// the shade kernel then picks per job, where a group of books' jobs only gets a kernel without that code), and the
// group's samples into its jobs' chunk partials (then the batch's reduction adds them into the sums)
cudaError_t launch_wave_batch_step(const wave_batch& w, bool flat, bool features, bool wide, bool quality,
                                   const wave_buffers& b, int trace_grid, cudaStream_t stream,
                                   bool draining = false);
cudaError_t launch_wave_batch_partials(const wave_batch& w, const wave_buffers& b, cudaStream_t stream);
// Loads the batch wavefront's kernels (every variant) now, so that no step pays for loading them
cudaError_t preload_wave_batch();
// The shade kernel's and the trace kernel's attributes for the scene and integrator
// The shade kernel's and the session's trace kernel's attributes (the trace kernel of the scene's search, at the given
// register cap)
cudaError_t wave_attributes(const scene_view& scene, bool quality, kernel_attributes& shade, kernel_attributes& trace,
                            int trace_min_blocks = RTB_TRACE_MIN_BLOCKS_DEFAULT);

// The books' integrator in double (precision::float64; renderer.h:402-409, all_books_kernel<double>,
// renderer.cu:445-451): a persistent launch over the same (pixel, chunk) work items as launch_params' and into the
// same chunk partials, so launch_reduce adds them into the sums. Its own random numbers: 53-bit uniforms.
struct launch_params_f64
{
    scene_view_f64 scene;
    camera_d cam;
    uint64_t seed;
    int64_t pass_begin;
    int64_t pass_end;
    int64_t first_chunk;
    int32_t chunk;
    int32_t chunks;
    int32_t tiles_x;
    int32_t padded_pixels;
    int64_t total_items;
    int32_t round_passes;
    int32_t pad0;
    unsigned long long* work_counter;
    double* partials;
    unsigned long long* counters; // [0] path segments
};
cudaError_t launch_render_f64(const launch_params_f64& p, int grid, cudaStream_t stream);
cudaError_t render_f64_attributes(const scene_view_f64& scene, kernel_attributes& out);

// Parity hooks: closest hits of given rays (source ids through prim_source), and the camera rays of one pass
cudaError_t launch_closest_hits(const scene_view& s, const float* origins, const float* directions, int64_t count,
                                const int32_t* prim_source, int32_t* ids, float* ts, cudaStream_t stream);
cudaError_t launch_camera_rays(const camera_params& cam, uint64_t seed, int64_t pass, int32_t round_passes,
                               float* origins, float* directions, cudaStream_t stream);
} // namespace rtb
