// rt_render_passes_no_alloc: passes of a resident scene rendered into a caller-owned device buffer, with the render
// kernel's scratch (its work counter, ray counters and per-chunk partial sums) taken from a fixed array in this
// library's device image instead of from cudaMalloc.
//
// Who needs it: a program that owns every byte of device memory through its own pool (a renderer embedded in an
// engine or a server that reserves its HBM up front and hands out only pre-sized buffers), or one that renders from a
// thread that must not block on the allocator: cudaMalloc and cudaFree may synchronize the device and fragment the
// pool. Such a caller already has the scene resident and its output buffer allocated; this entry point adds nothing
// to the device's allocations.
//
// The scratch lives in a file-scope __device__ array. Every GPU that loads the library holds it until the process
// exits, and every call shares it: its contents are the last call's. Host code cannot use the array's name as a
// device address, so the first call on each device looks the address up with cudaGetSymbolAddress, with that device
// current, and passes it to the kernels. That first call also creates the device's stream for these calls (a
// non-blocking stream, so a call neither waits for nor holds up the caller's other streams; creating it allocates no
// device memory). Calls are synchronous: each waits for its own work on that stream before it returns. Two calls
// that overlap on the GPU (from two host threads) would race on the shared scratch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <string>

#include "host.h"
#include "kernels.cuh"
#include "rt_b200.h"

namespace
{
// 64 MiB: 256 bytes of counters, then the partials of up to (64 MiB - 256) / 24 = 2,796,192 (pixel, chunk) items
constexpr size_t scratch_bytes = size_t{64} << 20;
constexpr size_t counter_bytes = 256;
constexpr int64_t partial_entries = static_cast<int64_t>((scratch_bytes - counter_bytes) / (3 * sizeof(double)));

static __device__ __align__(256) unsigned char no_alloc_scratch[scratch_bytes];

constexpr int max_devices = 64;
std::mutex setup_mutex;
unsigned char* scratch_address[max_devices] = {};
cudaStream_t scratch_stream[max_devices] = {};

// The scratch's device address on `device` (current) and the device's stream for these calls: set up once per device
unsigned char* scratch_on(int device, cudaStream_t& stream)
{
    if (device < 0 || device >= max_devices)
    {
        rtb::fail(RT_ERR_RUNTIME, "device index out of range for the no-allocation scratch");
    }
    std::lock_guard<std::mutex> lock(setup_mutex);
    if (!scratch_address[device])
    {
        void* p = nullptr;
        rtb::check(cudaGetSymbolAddress(&p, no_alloc_scratch), "looking up the no-allocation scratch");
        cudaStream_t s = nullptr;
        rtb::check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "creating the no-allocation stream");
        scratch_stream[device] = s;
        scratch_address[device] = static_cast<unsigned char*>(p);
    }
    stream = scratch_stream[device];
    return scratch_address[device];
}
} // namespace

extern "C" rt_status rt_render_passes_no_alloc(rt_scene* scene, const rt_camera_desc* camera, uint64_t seed,
                                               int64_t pass_begin, int64_t pass_end, double* device_sums,
                                               uint64_t* rays, uint64_t* shadow_rays)
{
    try
    {
        if (!scene || !camera || !device_sums)
        {
            rtb::fail(RT_ERR_INVALID, "scene, camera and device_sums must not be null");
        }
        if (pass_begin < 0 || pass_end < pass_begin)
        {
            rtb::fail(RT_ERR_INVALID, "passes must satisfy 0 <= pass_begin <= pass_end");
        }
        const rtb::resident_scene& s = *scene->scene;
        if (camera->sampling != s.camera().sampling)
        {
            rtb::fail(RT_ERR_INVALID, "the camera must keep the scene's sampling strategy");
        }
        rt_scene_desc probe{};
        probe.camera = *camera;
        rt_light_desc dummy{};
        probe.lights = &dummy;
        probe.light_count = 1;
        rtb::validate(probe);
        const int tiles_x = (camera->image_width + 7) / 8;
        const int tiles_y = (camera->image_height + 3) / 4;
        const int64_t padded = int64_t{tiles_x} * tiles_y * 32;
        if (padded > partial_entries)
        {
            rtb::fail(RT_ERR_CAPACITY, "the image needs " + std::to_string(padded) +
                                           " partial slots per chunk; the no-allocation scratch holds " +
                                           std::to_string(partial_entries) + " (64 MiB)");
        }
        rtb::check(cudaSetDevice(s.device()), "selecting the scene's device");
        cudaStream_t stream = nullptr;
        unsigned char* scratch = scratch_on(s.device(), stream);
        auto* counters = reinterpret_cast<unsigned long long*>(scratch);
        auto* partials = reinterpret_cast<double*>(scratch + counter_bytes);
        rtb::kernel_attributes a{};
        rtb::check(rtb::render_attributes(s.view(), s.quality(), a), "querying the render kernel");
        const int grid = a.multiprocessors * (a.blocks_per_sm > 0 ? a.blocks_per_sm : 1);
        const int64_t max_chunks = partial_entries / padded;
        // The ray counters start at zero for this call; the work counter before every launch
        rtb::check(cudaMemsetAsync(counters, 0, counter_bytes, stream), "clearing the scratch counters");
        int64_t pass = pass_begin;
        while (pass < pass_end)
        {
            // Whole chunks, aligned as a session aligns them, so the sums equal a session's bit for bit
            const int64_t first_chunk = pass / rtb::pass_chunk;
            const int64_t end = std::min(pass_end, (first_chunk + max_chunks) * rtb::pass_chunk);
            const int64_t chunks = (end + rtb::pass_chunk - 1) / rtb::pass_chunk - first_chunk;
            rtb::launch_params p{};
            p.scene = s.view();
            p.cam = rtb::to_camera(*camera);
            p.seed = seed;
            p.pass_begin = pass;
            p.pass_end = end;
            p.first_chunk = first_chunk;
            p.chunk = rtb::pass_chunk;
            p.chunks = static_cast<int32_t>(chunks);
            p.tiles_x = tiles_x;
            p.padded_pixels = static_cast<int32_t>(padded);
            p.total_items = chunks * padded;
            p.round_passes = camera->sqrt_spp * camera->sqrt_spp;
            p.job = 0;
            p.work_counter = counters;
            p.partials = partials;
            p.counters = counters + 1;
            rtb::reduce_params r{};
            r.partials = partials;
            r.sums = device_sums;
            r.width = camera->image_width;
            r.height = camera->image_height;
            r.tiles_x = tiles_x;
            r.padded_pixels = static_cast<int32_t>(padded);
            r.chunks = p.chunks;
            rtb::check(cudaMemsetAsync(counters, 0, sizeof(unsigned long long), stream), "clearing the work counter");
            rtb::check(rtb::launch_render(p, s.quality(), false, grid, stream), "launching the render kernel");
            rtb::check(rtb::launch_reduce(r, stream), "launching the reduction");
            pass = end;
        }
        unsigned long long counts[2] = {};
        rtb::check(cudaMemcpyAsync(counts, counters + 1, sizeof(counts), cudaMemcpyDeviceToHost, stream),
                   "reading the ray counters");
        rtb::check(cudaStreamSynchronize(stream), "rendering on the GPU");
        if (rays)
        {
            *rays = counts[0];
        }
        if (shadow_rays)
        {
            *shadow_rays = counts[1];
        }
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
