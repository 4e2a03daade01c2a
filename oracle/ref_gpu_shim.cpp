// Test infrastructure, not product: C entry points into the reference's own CUDA renderer (its src/gpu sources,
// compiled unmodified into oracle/_ref by oracle/build_ref.py), so that tests and the bench can render a scene given
// as this library's C tables with the reference itself. It converts rt_scene_desc into the reference's gpu::scene_desc
// (src/gpu/renderer.h:381-395, member types 43-377), calls gpu::render (renderer.h:526) and copies the result out.
// Triangle meshes are refused: the reference renders them only through OptiX, which is absent here. A second entry
// point runs the reference's display transforms (display.cu, tonemap.cu) on given sums.
#include "renderer.h" // the reference's header, from its source tree

#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "display.cuh" // the reference's display transforms, from its source tree
#include "ref_scene_convert.h"
#include "tonemap.cuh"
#include "rt_b200.h"

namespace
{
using ref_convert::to_ref;

void copy_error(const char* what, char* error, int error_size)
{
    if (error && error_size > 0)
    {
        std::strncpy(error, what, static_cast<size_t>(error_size) - 1);
        error[error_size - 1] = '\0';
    }
}
} // namespace

extern "C" {

// What one reference render reports: render_result's counters (renderer.h:475-492) and its kernel's name
struct ref_gpu_result
{
    double seconds;
    double kernel_seconds;
    uint64_t rays;
    uint64_t shadow_rays;
    int32_t registers;
    int32_t blocks_per_multiprocessor;
    char kernel[32];
};

// Renders `scene` with the reference's gpu::render: `passes` passes (0: sqrt_spp^2) from `seed`, in float (fp64 = 0)
// or double (fp64 = 1); all_books = 1 forces the all-books kernel where the first-book kernel would run. Writes
// width * height * 3 doubles. Returns 0, or 1 with the reference's exception message in `error`.
int ref_gpu_render(const rt_scene_desc* scene, uint64_t seed, int64_t passes, int32_t fp64, int32_t all_books,
                   double* pixels, int64_t pixel_count, ref_gpu_result* result, char* error, int32_t error_size)
{
    try
    {
        if (scene->mesh_count > 0)
        {
            copy_error("the reference renders triangle meshes only through OptiX", error, error_size);
            return 1;
        }
        const gpu::scene_desc s = to_ref(*scene);
        gpu::render_options o;
        o.seed = seed;
        o.passes = passes;
        o.arithmetic = fp64 ? gpu::precision::float64 : gpu::precision::float32;
        o.all_books_kernel = all_books != 0;
        o.quality_kernel = scene->quality != 0;
        o.launch_seconds = 0.05;
        const gpu::render_result r = gpu::render(s, o);
        if (static_cast<int64_t>(r.pixels.size()) != pixel_count)
        {
            copy_error("the pixel buffer does not match the image", error, error_size);
            return 1;
        }
        std::memcpy(pixels, r.pixels.data(), r.pixels.size() * sizeof(double));
        if (result)
        {
            result->seconds = r.seconds;
            result->kernel_seconds = r.kernel_seconds;
            result->rays = r.rays;
            result->shadow_rays = r.shadow_rays;
            result->registers = r.kernel.registers;
            result->blocks_per_multiprocessor = r.kernel.blocks_per_multiprocessor;
            std::memset(result->kernel, 0, sizeof(result->kernel));
            std::strncpy(result->kernel, r.kernel.name.c_str(), sizeof(result->kernel) - 1);
        }
        return 0;
    }
    catch (const std::exception& e)
    {
        copy_error(e.what(), error, error_size);
        return 1;
    }
}
}

extern "C" {

// The reference's display transform (src/gpu/display.cu:26 rgba8_kernel for books, tonemap.cu:25 tone_map_kernel for
// the tone maps; both compiled -fmad=false) on given sums: width * height * 3 doubles in host memory, each channel's
// sum times `scale` (1 / passes) as session::display computes it for an image of complete passes
// (renderer.cu:1388-1470). op: 0 books, 1 none, 2 agx, 3 neutral (renderer.h:286-292); exposure in stops, turned
// into float(2^EV) as session::display does. Writes width * height * 4 bytes. Returns 0, or 1 with the message.
int ref_gpu_display_bytes(const double* sums, int32_t width, int32_t height, double scale, int32_t op, double exposure,
                          uint8_t* rgba, char* error, int32_t error_size)
{
    double* d_sums = nullptr;
    uint8_t* d_rgba = nullptr;
    try
    {
        const size_t pixels = static_cast<size_t>(width) * static_cast<size_t>(height);
        if (cudaMalloc(&d_sums, pixels * 3 * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&d_rgba, pixels * 4) != cudaSuccess)
        {
            throw std::runtime_error("allocating device memory");
        }
        if (cudaMemcpy(d_sums, sums, pixels * 3 * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        {
            throw std::runtime_error("copying the sums");
        }
        const auto tone = static_cast<gpu::tone_map>(op);
        if (tone == gpu::tone_map::books)
        {
            gpu::detail::to_rgba8(d_sums, width, 0, height, scale, d_rgba);
        }
        else
        {
            const auto exposure_scale = static_cast<float>(std::exp2(exposure));
            gpu::detail::to_rgba8_toned(d_sums, width, 0, height, scale, tone, exposure_scale, d_rgba);
        }
        if (cudaMemcpy(rgba, d_rgba, pixels * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        {
            throw std::runtime_error("copying the bytes");
        }
        cudaFree(d_sums);
        cudaFree(d_rgba);
        return 0;
    }
    catch (const std::exception& e)
    {
        cudaFree(d_sums);
        cudaFree(d_rgba);
        copy_error(e.what(), error, error_size);
        return 1;
    }
}
}
