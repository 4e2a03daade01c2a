// Test infrastructure, not product: C entry points that call the reference's gpu:: API (src/gpu/renderer.h) as its
// own programs do, on a build where that API is served by this library through the shim INTEGRATION.md documents
// (oracle/build_ref.py extracts the shim from INTEGRATION.md and links both into oracle/_ref/librenderer_b200.so).
// The scene goes in as this library's C tables and is converted into the reference's scene_desc first, so a test can
// compare gpu::render through the shim with rt_render on the same tables.
#include "renderer.h" // the reference's header, from its source tree

#include <cstdint>
#include <cstring>
#include <exception>

#include "ref_scene_convert.h"
#include "rt_b200.h"

namespace
{
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

// gpu::render(scene, options) with seed, passes and a display tone map (0 books .. 3 neutral, renderer.h:286-292):
// its pixels (width * height * 3 doubles), its rgba bytes (width * height * 4, filled only for a tone map other
// than books) and its ray count. Returns 0, or 1 with the exception's message.
int shim_render(const rt_scene_desc* scene, uint64_t seed, int64_t passes, int32_t tone, double exposure,
                double* pixels, uint8_t* rgba, uint64_t* rays, char* error, int32_t error_size)
{
    try
    {
        const gpu::scene_desc s = ref_convert::to_ref(*scene);
        gpu::render_options o;
        o.seed = seed;
        o.passes = passes;
        o.quality_kernel = scene->quality != 0;
        o.display.op = static_cast<gpu::tone_map>(tone);
        o.display.exposure = exposure;
        const gpu::render_result r = gpu::render(s, o);
        std::memcpy(pixels, r.pixels.data(), r.pixels.size() * sizeof(double));
        if (rgba && !r.rgba.empty())
        {
            std::memcpy(rgba, r.rgba.data(), r.rgba.size());
        }
        *rays = r.rays;
        return 0;
    }
    catch (const std::exception& e)
    {
        copy_error(e.what(), error, error_size);
        return 1;
    }
}

// gpu::render(scene, options) with options.arithmetic = precision::float64 (fp64 != 0) or float32: its pixels and
// ray count. Returns 0, or 1 with the exception's message.
int shim_render_precision(const rt_scene_desc* scene, uint64_t seed, int64_t passes, int32_t fp64, double* pixels,
                          uint64_t* rays, char* error, int32_t error_size)
{
    try
    {
        const gpu::scene_desc s = ref_convert::to_ref(*scene);
        gpu::render_options o;
        o.seed = seed;
        o.passes = passes;
        o.quality_kernel = scene->quality != 0;
        o.arithmetic = fp64 != 0 ? gpu::precision::float64 : gpu::precision::float32;
        const gpu::render_result r = gpu::render(s, o);
        std::memcpy(pixels, r.pixels.data(), r.pixels.size() * sizeof(double));
        *rays = r.rays;
        return 0;
    }
    catch (const std::exception& e)
    {
        copy_error(e.what(), error, error_size);
        return 1;
    }
}

// A gpu::session of the scene: render_to(passes), then pixels() and display(options) as the viewer calls them
int shim_session(const rt_scene_desc* scene, uint64_t seed, int64_t passes, int32_t tone, double exposure,
                 double* pixels, uint8_t* rgba, char* error, int32_t error_size)
{
    try
    {
        const gpu::scene_desc s = ref_convert::to_ref(*scene);
        gpu::session_options o;
        o.seed = seed;
        o.quality_kernel = scene->quality != 0;
        gpu::session view(s, o);
        view.render_to({passes, 0});
        const std::vector<double> p = view.pixels();
        std::memcpy(pixels, p.data(), p.size() * sizeof(double));
        gpu::display_options d;
        d.op = static_cast<gpu::tone_map>(tone);
        d.exposure = exposure;
        const std::span<const std::uint8_t> bytes = view.display(d);
        std::memcpy(rgba, bytes.data(), bytes.size());
        return 0;
    }
    catch (const std::exception& e)
    {
        copy_error(e.what(), error, error_size);
        return 1;
    }
}
}
