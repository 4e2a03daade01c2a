// The C-ABI (include/rt_b200.h): every entry point catches what the C++ runtime throws and returns its status, with
// the message kept per thread for rt_last_error_message().
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <new>
#include <string>
#include <vector>

#include "host.h"
#include "scene_store.h"

namespace
{
thread_local std::string last_error;

template <class F>
rt_status guarded(F&& f)
{
    try
    {
        last_error.clear();
        f();
        return RT_OK;
    }
    catch (const rtb::rt_error& e)
    {
        last_error = e.what();
        return e.status;
    }
    catch (const std::bad_alloc&)
    {
        last_error = "out of host memory";
        return RT_ERR_RUNTIME;
    }
    catch (const std::exception& e)
    {
        last_error = e.what();
        return RT_ERR_RUNTIME;
    }
    catch (...)
    {
        last_error = "unknown error";
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

rt_session_options session_options_of(const rt_render_options& o)
{
    rt_session_options s{};
    s.seed = o.seed;
    s.arithmetic = o.arithmetic;
    s.launch_seconds = o.launch_seconds > 0 ? o.launch_seconds : 0.05;
    return s;
}
} // namespace

void rtb::remember_error(const char* message) { last_error = message; }

extern "C" {

const char* rt_last_error_message(void) { return last_error.c_str(); }

int32_t rt_abi_version(void) { return RT_ABI_VERSION; }

rt_status rt_query_device(rt_device_info* info)
{
    return guarded([&] {
        need(info, "info");
        int count = 0;
        rtb::check(cudaGetDeviceCount(&count), "looking for a CUDA device");
        if (count == 0)
        {
            rtb::fail(RT_ERR_NO_DEVICE, "no CUDA device");
        }
        int device = 0;
        rtb::check(cudaGetDevice(&device), "selecting the CUDA device");
        cudaDeviceProp prop{};
        rtb::check(cudaGetDeviceProperties(&prop, device), "describing the CUDA device");
        rtb::check(cudaFree(nullptr), "starting CUDA");
        *info = rt_device_info{};
        std::snprintf(info->name, sizeof(info->name), "%s", prop.name);
        info->compute_capability_major = prop.major;
        info->compute_capability_minor = prop.minor;
        info->multiprocessors = prop.multiProcessorCount;
        info->memory_gib = static_cast<double>(prop.totalGlobalMem) / (1024.0 * 1024.0 * 1024.0);
        cudaRuntimeGetVersion(&info->runtime_version);
        cudaDriverGetVersion(&info->driver_version);
    });
}

rt_status rt_set_device(int32_t device)
{
    return guarded([&] { rtb::check(cudaSetDevice(device), "selecting the CUDA device"); });
}

rt_status rt_count_lamps(const rt_scene_desc* scene, int32_t* count)
{
    return guarded([&] {
        need(scene, "scene");
        need(count, "count");
        int32_t n = 0;
        const auto glows = [&](int32_t m) {
            return m >= 0 && m < scene->material_count && scene->materials[m].kind == RT_DIFFUSE_LIGHT &&
                   scene->materials[m].texture >= 0 && scene->materials[m].texture < scene->texture_count &&
                   scene->textures[scene->materials[m].texture].kind == RT_TEXTURE_SOLID;
        };
        for (int64_t i = 0; i < scene->sphere_count; ++i)
        {
            const rt_sphere_desc& s = scene->spheres[i];
            const bool still = s.displacement.x == 0 && s.displacement.y == 0 && s.displacement.z == 0;
            n += still && glows(s.material) ? 1 : 0;
        }
        for (int64_t i = 0; i < scene->quad_count; ++i)
        {
            n += glows(scene->quads[i].material) ? 1 : 0;
        }
        *count = n;
    });
}

rt_status rt_is_convex(const rt_quad_desc* quads, int64_t count, int32_t* convex)
{
    return guarded([&] {
        need(convex, "convex");
        if (count > 0)
        {
            need(quads, "quads");
        }
        *convex = rtb::is_convex(quads, count) ? 1 : 0;
    });
}

rt_status rt_scene_create(const rt_scene_desc* desc, rt_scene** scene)
{
    return guarded([&] {
        need(desc, "desc");
        need(scene, "scene");
        *scene = nullptr;
        auto s = std::make_unique<rt_scene>();
        s->scene = std::make_shared<rtb::resident_scene>(*desc);
        *scene = s.release();
    });
}

rt_status rt_scene_destroy(rt_scene* scene)
{
    return guarded([&] { delete scene; });
}

rt_status rt_scene_stats_get(const rt_scene* scene, rt_scene_stats* stats)
{
    return guarded([&] {
        need(scene, "scene");
        need(stats, "stats");
        *stats = scene->scene->stats();
    });
}

rt_status rt_session_create(rt_scene* scene, const rt_session_options* options, rt_session** session)
{
    return guarded([&] {
        need(scene, "scene");
        need(options, "options");
        need(session, "session");
        *session = nullptr;
        auto s = std::make_unique<rt_session>();
        s->session = std::make_unique<rtb::session>(scene->scene, *options);
        *session = s.release();
    });
}

rt_status rt_session_destroy(rt_session* session)
{
    return guarded([&] { delete session; });
}

rt_status rt_session_set_camera(rt_session* session, const rt_camera_desc* camera)
{
    return guarded([&] {
        need(session, "session");
        need(camera, "camera");
        session->session->set_camera(*camera);
    });
}

rt_status rt_session_state(const rt_session* session, rt_accumulation* state)
{
    return guarded([&] {
        need(session, "session");
        need(state, "state");
        *state = session->session->state();
    });
}

rt_status rt_session_render_to(rt_session* session, int64_t passes, rt_render_report* report)
{
    return guarded([&] {
        need(session, "session");
        const rt_render_report r = session->session->render_to(passes);
        if (report)
        {
            *report = r;
        }
    });
}

rt_status rt_session_render_for(rt_session* session, double seconds, int64_t pass_limit, rt_render_report* report)
{
    return guarded([&] {
        need(session, "session");
        const rt_render_report r = session->session->render_for(seconds, pass_limit);
        if (report)
        {
            *report = r;
        }
    });
}

rt_status rt_session_pixels(const rt_session* session, double* pixels, int64_t pixel_count)
{
    return guarded([&] {
        need(session, "session");
        need(pixels, "pixels");
        session->session->pixels(pixels, pixel_count);
    });
}

rt_status rt_session_counters(const rt_session* session, uint64_t* rays, uint64_t* shadow_rays,
                              double* kernel_seconds)
{
    return guarded([&] {
        need(session, "session");
        if (rays)
        {
            *rays = session->session->rays();
        }
        if (shadow_rays)
        {
            *shadow_rays = session->session->shadow_rays();
        }
        if (kernel_seconds)
        {
            *kernel_seconds = session->session->kernel_seconds();
        }
    });
}

rt_status rt_session_kernel(const rt_session* session, rt_kernel_info* info)
{
    return guarded([&] {
        need(session, "session");
        need(info, "info");
        *info = session->session->kernel();
    });
}

rt_status rt_session_device_sums(const rt_session* session, const double** sums, int64_t* passes)
{
    return guarded([&] {
        need(session, "session");
        need(sums, "sums");
        need(passes, "passes");
        *sums = session->session->device_sums();
        *passes = session->session->state().passes;
    });
}

rt_status rt_session_display(rt_session* session, const rt_display_options* options, uint8_t* rgba,
                             int64_t byte_count)
{
    return guarded([&] {
        need(session, "session");
        need(options, "options");
        need(rgba, "rgba");
        session->session->display(*options, rgba, byte_count);
    });
}

rt_status rt_display_device(const double* device_sums, int32_t width, int32_t height, int64_t passes,
                            const rt_display_options* options, uint8_t* device_rgba, void* stream)
{
    return guarded([&] {
        need(device_sums, "device_sums");
        need(options, "options");
        need(device_rgba, "device_rgba");
        if (width < 1 || height < 1)
        {
            rtb::fail(RT_ERR_INVALID, "an image is at least 1 x 1");
        }
        if (passes <= 0)
        {
            rtb::fail(RT_ERR_LOGIC, "the image has no complete pass to show");
        }
        rtb::launch_display(device_sums, width, height, 1.0 / static_cast<double>(passes), *options, device_rgba,
                            static_cast<cudaStream_t>(stream));
    });
}

rt_status rt_image_save(const char* path, const double* pixels, int32_t width, int32_t height,
                        const rt_display_options* options)
{
    return guarded([&] {
        need(path, "path");
        need(pixels, "pixels");
        const rt_display_options books{};
        rtb::save_image(path, pixels, width, height, options ? *options : books);
    });
}

rt_status rt_image_mean_radiance(const double* pixels, int32_t width, int32_t height, double* mean)
{
    return guarded([&] {
        need(pixels, "pixels");
        need(mean, "mean");
        if (width < 1 || height < 1)
        {
            rtb::fail(RT_ERR_INVALID, "an image is at least 1 x 1");
        }
        *mean = rtb::mean_radiance(pixels, static_cast<int64_t>(width) * height);
    });
}

rt_status rt_session_save(rt_session* session, const char* path, const rt_display_options* options)
{
    return guarded([&] {
        need(session, "session");
        need(path, "path");
        const rt_display_options books{};
        const rt_display_options& o = options ? *options : books;
        rtb::check_display(o);
        const rt_camera_desc& c = session->session->camera();
        const size_t n = static_cast<size_t>(c.image_width) * static_cast<size_t>(c.image_height);
        std::string name(path);
        std::string ext = name.size() >= 4 ? name.substr(name.size() - 4) : "";
        for (char& ch : ext)
        {
            ch = static_cast<char>(std::tolower(static_cast<unsigned char>(ch)));
        }
        if (ext == ".png")
        {
            // the bytes the session's display shows (the GPU's, for every tone map)
            std::vector<uint8_t> rgba(n * 4);
            session->session->display(o, rgba.data(), static_cast<int64_t>(rgba.size()));
            rtb::save_png_rgba(path, rgba.data(), c.image_width, c.image_height);
            return;
        }
        std::vector<double> pixels(n * 3);
        session->session->pixels(pixels.data(), static_cast<int64_t>(pixels.size()));
        rtb::save_image(path, pixels.data(), c.image_width, c.image_height, o);
    });
}

rt_status rt_session_mean_radiance(const rt_session* session, double* mean)
{
    return guarded([&] {
        need(session, "session");
        need(mean, "mean");
        const rt_camera_desc& c = session->session->camera();
        const size_t n = static_cast<size_t>(c.image_width) * static_cast<size_t>(c.image_height);
        std::vector<double> pixels(n * 3);
        session->session->pixels(pixels.data(), static_cast<int64_t>(pixels.size()));
        *mean = rtb::mean_radiance(pixels.data(), static_cast<int64_t>(n));
    });
}

rt_status rt_session_set_timing(rt_session* session, int32_t on)
{
    return guarded([&] {
        need(session, "session");
        session->session->set_timing(on != 0);
    });
}

rt_status rt_session_kernel_times(const rt_session* session, rt_kernel_times* times)
{
    return guarded([&] {
        need(session, "session");
        need(times, "times");
        *times = session->session->kernel_times();
    });
}

rt_status rt_session_autotune(rt_session* session, int64_t trial_passes, rt_tuning* result)
{
    return guarded([&] {
        need(session, "session");
        const rt_tuning t = session->session->autotune(trial_passes);
        if (result)
        {
            *result = t;
        }
    });
}

rt_status rt_session_set_tuning(rt_session* session, const rt_tuning* shape)
{
    return guarded([&] {
        need(session, "session");
        need(shape, "shape");
        session->session->set_tuning(*shape);
    });
}

rt_status rt_session_tuning(const rt_session* session, rt_tuning* current)
{
    return guarded([&] {
        need(session, "session");
        need(current, "current");
        *current = session->session->tuning();
    });
}

rt_status rt_session_set_counting(rt_session* session, int32_t on)
{
    return guarded([&] {
        need(session, "session");
        session->session->set_counting(on != 0);
    });
}

rt_status rt_session_fetch_counts(const rt_session* session, uint64_t counts[4])
{
    return guarded([&] {
        need(session, "session");
        need(counts, "counts");
        session->session->fetch_counts(counts);
    });
}

rt_status rt_render(const rt_scene_desc* scene, const rt_render_options* options, double* pixels,
                    int64_t pixel_count, rt_render_result* result)
{
    return guarded([&] {
        need(scene, "scene");
        need(options, "options");
        need(pixels, "pixels");
        if (options->passes < 0)
        {
            rtb::fail(RT_ERR_INVALID, "passes must not be negative");
        }
        const auto start = std::chrono::steady_clock::now();
        auto resident = std::make_shared<rtb::resident_scene>(*scene);
        rtb::session s(resident, session_options_of(*options));
        const int64_t passes = options->passes > 0
                                   ? options->passes
                                   : static_cast<int64_t>(scene->camera.sqrt_spp) * scene->camera.sqrt_spp;
        const rt_render_report report = s.render_to(passes);
        s.pixels(pixels, pixel_count);
        if (result)
        {
            *result = rt_render_result{};
            result->kernel_seconds = s.kernel_seconds();
            result->rays = s.rays();
            result->shadow_rays = s.shadow_rays();
            result->passes = passes;
            result->launches = report.launches;
            result->kernel_launches = report.kernel_launches;
            result->kernel = s.kernel();
            result->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
        }
    });
}

rt_status rt_scene_closest_hits(rt_scene* scene, const float* origins, const float* directions, int64_t count,
                                int32_t* ids, float* ts)
{
    return guarded([&] {
        need(scene, "scene");
        if (count <= 0)
        {
            return;
        }
        need(origins, "origins");
        need(directions, "directions");
        need(ids, "ids");
        need(ts, "ts");
        const size_t n = static_cast<size_t>(count);
        rtb::device_array<float> o(3 * n);
        rtb::device_array<float> d(3 * n);
        rtb::device_array<int32_t> id(n);
        rtb::device_array<float> t(n);
        rtb::check(cudaMemcpy(o.data(), origins, o.bytes(), cudaMemcpyHostToDevice), "copying rays");
        rtb::check(cudaMemcpy(d.data(), directions, d.bytes(), cudaMemcpyHostToDevice), "copying rays");
        rtb::check(rtb::launch_closest_hits(scene->scene->view(), o.data(), d.data(), count, scene->scene->prim_source(),
                                            id.data(), t.data(), nullptr),
                   "launching the closest-hit queries");
        rtb::check(cudaMemcpy(ids, id.data(), id.bytes(), cudaMemcpyDeviceToHost), "copying hits");
        rtb::check(cudaMemcpy(ts, t.data(), t.bytes(), cudaMemcpyDeviceToHost), "copying hits");
    });
}

rt_status rt_scene_camera_rays(rt_scene* scene, uint64_t seed, int64_t pass, float* origins, float* directions,
                               int64_t pixel_count)
{
    return guarded([&] {
        need(scene, "scene");
        need(origins, "origins");
        need(directions, "directions");
        const rt_camera_desc& c = scene->scene->camera();
        const int64_t n = static_cast<int64_t>(c.image_width) * c.image_height;
        if (pixel_count != n)
        {
            rtb::fail(RT_ERR_INVALID, "pixel_count must be width * height");
        }
        if (pass < 0)
        {
            rtb::fail(RT_ERR_INVALID, "pass must not be negative");
        }
        rtb::device_array<float> o(3 * static_cast<size_t>(n));
        rtb::device_array<float> d(3 * static_cast<size_t>(n));
        rtb::check(rtb::launch_camera_rays(rtb::to_camera(c), seed, pass, c.sqrt_spp * c.sqrt_spp, o.data(), d.data(),
                                           nullptr),
                   "launching the camera rays");
        rtb::check(cudaMemcpy(origins, o.data(), o.bytes(), cudaMemcpyDeviceToHost), "copying rays");
        rtb::check(cudaMemcpy(directions, d.data(), d.bytes(), cudaMemcpyDeviceToHost), "copying rays");
    });
}

rt_status rt_builtin_scene(const char* name, const rt_builtin_params* params, rt_owned_scene** scene)
{
    return guarded([&] {
        need(name, "name");
        need(scene, "scene");
        *scene = nullptr;
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
        auto owned = std::make_unique<rt_owned_scene>();
        std::string error;
        const rt_status s = rtb::build_builtin(name, p, owned->store, error);
        if (s != RT_OK)
        {
            rtb::fail(s, error);
        }
        *scene = owned.release();
    });
}

const rt_scene_desc* rt_owned_scene_desc(const rt_owned_scene* scene)
{
    return scene && scene->store ? &scene->store->desc : nullptr;
}

rt_status rt_owned_scene_destroy(rt_owned_scene* scene)
{
    return guarded([&] { delete scene; });
}

rt_status rt_scene_save(const rt_scene_desc* scene, const char* path)
{
    return guarded([&] {
        need(scene, "scene");
        need(path, "path");
        std::string error;
        const rt_status s = rtb::save_scene(*scene, path, error);
        if (s != RT_OK)
        {
            rtb::fail(s, error);
        }
    });
}

rt_status rt_scene_load(const char* path, rt_owned_scene** scene)
{
    return guarded([&] {
        need(path, "path");
        need(scene, "scene");
        *scene = nullptr;
        auto owned = std::make_unique<rt_owned_scene>();
        std::string error;
        const rt_status s = rtb::load_scene(path, owned->store, error);
        if (s != RT_OK)
        {
            rtb::fail(s, error);
        }
        *scene = owned.release();
    });
}
}
