// TEST INFRASTRUCTURE — the oracle's C entry points (liboracle.so), for tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg. Nothing in the product links or loads this library.
//
// oracle_render is the reference CPU renderer's camera::render (src/camera.ixx:204-272): worker threads take rows
// from an atomic counter, each row draws from its own std::mt19937_64 seeded with (seed << 32) | row, and each
// pixel adds its samples' without_nan colors. Passes beyond one round of k^2 strata are rendered round after round,
// round r drawing as seed + r (the GPU renderer's rounds, renderer.h:564-584, in the CPU's 32-bit seed).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <thread>
#include <vector>

#include "cpu_renderer.h"
#include "image_compare.h"
#include "quality_cpu.h"

namespace
{
thread_local char last_error[512] = "";

void set_error(const char* message)
{
    std::snprintf(last_error, sizeof(last_error), "%s", message);
}
} // namespace

extern "C" {

const char* oracle_last_error(void) { return last_error; }

typedef struct oracle_stats
{
    uint64_t rays;
    uint64_t shadow_rays;
    double seconds;
    int32_t threads;
    int32_t rows_rendered;
} oracle_stats;

// Renders passes [0, passes) of rows [row_begin, row_end) (row_end <= 0: to the bottom). pixels: width*height*3
// doubles, the mean of each pixel's samples (rows outside the range are left as they are).
int oracle_render(const rt_scene_desc* desc, uint64_t seed, int64_t passes, int32_t threads, int32_t row_begin,
                  int32_t row_end, double* pixels, oracle_stats* stats)
{
    oracle::scene s;
    const char* error = nullptr;
    if (!desc || !pixels || !oracle::make_scene(*desc, s, &error))
    {
        set_error(error ? error : "null argument");
        return 1;
    }
    const rt_camera_desc& c = s.camera;
    const int k = std::max(1, c.sqrt_spp);
    const int64_t round_passes = static_cast<int64_t>(k) * k;
    if (passes <= 0)
    {
        passes = round_passes;
    }
    const int height = c.image_height;
    const int width = c.image_width;
    if (row_end <= 0 || row_end > height)
    {
        row_end = height;
    }
    row_begin = std::max(0, row_begin);
    const bool quality = desc->quality != 0;
    const oracle::quality_scene q = oracle::make_quality(s, *desc);
    const unsigned thread_count = threads > 0 ? static_cast<unsigned>(threads)
                                              : std::max(1u, std::thread::hardware_concurrency());
    std::atomic<int> next_row{row_begin};
    std::atomic<uint64_t> rays{0};
    std::atomic<uint64_t> shadow_rays{0};
    const auto start = std::chrono::steady_clock::now();
    auto work = [&]() {
        oracle::counters n;
        oracle::rng g;
        std::vector<oracle::color> row(static_cast<size_t>(width));
        for (int j = next_row++; j < row_end; j = next_row++)
        {
            std::fill(row.begin(), row.end(), oracle::color{0, 0, 0});
            for (int64_t first = 0; first < passes; first += round_passes)
            {
                const int64_t round = first / round_passes;
                const int64_t count = std::min(round_passes, passes - first);
                const uint32_t round_seed = static_cast<uint32_t>(seed + static_cast<uint64_t>(round));
                g.seed((static_cast<uint64_t>(round_seed) << 32) | static_cast<uint64_t>(j));
                for (int i = 0; i < width; ++i)
                {
                    for (int64_t p = 0; p < count; ++p)
                    {
                        const int s_i = static_cast<int>(p % k);
                        const int s_j = static_cast<int>(p / k);
                        const oracle::ray r = oracle::get_ray(s, i, j, s_i, s_j, g);
                        const oracle::color sample = quality ? oracle::quality_sample(q, r, g, n)
                                                             : oracle::ray_color(s, r, c.max_depth, g, n);
                        row[static_cast<size_t>(i)] += oracle::without_nan(sample);
                    }
                }
            }
            const double scale = 1.0 / static_cast<double>(passes);
            for (int i = 0; i < width; ++i)
            {
                double* out = pixels + 3 * (static_cast<int64_t>(j) * width + i);
                out[0] = scale * row[static_cast<size_t>(i)].x;
                out[1] = scale * row[static_cast<size_t>(i)].y;
                out[2] = scale * row[static_cast<size_t>(i)].z;
            }
        }
        rays += n.rays;
        shadow_rays += n.shadow_rays;
    };
    std::vector<std::thread> workers;
    for (unsigned t = 0; t < thread_count; ++t)
    {
        workers.emplace_back(work);
    }
    for (std::thread& t : workers)
    {
        t.join();
    }
    if (stats)
    {
        stats->rays = rays.load();
        stats->shadow_rays = shadow_rays.load();
        stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
        stats->threads = static_cast<int32_t>(thread_count);
        stats->rows_rendered = row_end - row_begin;
    }
    return 0;
}

// The closest hit of each ray in double, in source index space (spheres, quads, triangles; -1 for a miss), over
// (0.001, inf): by the CPU's BVH (bvh.ixx) or by testing every primitive (hittable_list::hit) when brute_force != 0.
int oracle_closest_hits(const rt_scene_desc* desc, const double* origins, const double* directions, int64_t count,
                        int32_t brute_force, int32_t* ids, double* ts)
{
    oracle::scene s;
    const char* error = nullptr;
    if (!desc || !oracle::make_scene(*desc, s, &error))
    {
        set_error(error ? error : "null argument");
        return 1;
    }
    const unsigned thread_count = std::max(1u, std::thread::hardware_concurrency());
    std::atomic<int64_t> next{0};
    auto work = [&]() {
        constexpr int64_t chunk = 256;
        for (int64_t b = next.fetch_add(chunk); b < count; b = next.fetch_add(chunk))
        {
            for (int64_t i = b; i < std::min(count, b + chunk); ++i)
            {
                const oracle::ray r{{origins[3 * i], origins[3 * i + 1], origins[3 * i + 2]},
                                    {directions[3 * i], directions[3 * i + 1], directions[3 * i + 2]},
                                    0};
                const auto rec = brute_force ? s.geometry.hit_brute_force(r, oracle::interval{0.001, oracle::infinity})
                                             : s.geometry.hit(r, oracle::interval{0.001, oracle::infinity});
                ids[i] = rec ? rec->id : -1;
                ts[i] = rec ? rec->t : oracle::infinity;
            }
        }
    };
    std::vector<std::thread> workers;
    for (unsigned t = 0; t < thread_count; ++t)
    {
        workers.emplace_back(work);
    }
    for (std::thread& t : workers)
    {
        t.join();
    }
    return 0;
}

// For the first-hit test's tie rule: where, in double, each ray meets the primitive ids[i] (source index space) over
// (0.001, inf), or inf where it does not (or ids[i] < 0); a quad's or a triangle's barycentrics may lie `slack` outside
// their bounds (a float search's hit on the edge a neighbour shares). A mismatch between two searches is a tie when both
// primitives are met at the same distance within the stated relative tolerance (coplanar or touching faces: the
// reference's tracer-check class `ties`, tests/tracer_check_layout.h).
int oracle_hit_distances(const rt_scene_desc* desc, const double* origins, const double* directions, int64_t count,
                         const int32_t* ids, double slack, double* ts)
{
    oracle::scene s;
    const char* error = nullptr;
    if (!desc || !oracle::make_scene(*desc, s, &error))
    {
        set_error(error ? error : "null argument");
        return 1;
    }
    for (int64_t i = 0; i < count; ++i)
    {
        const oracle::ray r{{origins[3 * i], origins[3 * i + 1], origins[3 * i + 2]},
                            {directions[3 * i], directions[3 * i + 1], directions[3 * i + 2]},
                            0};
        const auto rec = s.geometry.hit_id(ids[i], r, oracle::interval{0.001, oracle::infinity}, slack);
        ts[i] = rec ? rec->t : oracle::infinity;
    }
    return 0;
}

int oracle_image_compare(const float* a, const float* b, int32_t width, int32_t height, int32_t tile_size,
                         oracle::compare_result* result)
{
    if (!a || !b || !result)
    {
        set_error("null argument");
        return 1;
    }
    *result = oracle::image_compare(a, b, width, height, tile_size);
    return 0;
}

// The thresholds ImageCompare uses for a given number of tested tiles (image_compare.cpp:442-458)
int oracle_thresholds(int32_t tested_tiles, double* whole_image, double* all_tiles, double* largest_tile,
                      int32_t* tiles_over_3)
{
    const oracle::thresholds t = oracle::alarm_thresholds(tested_tiles);
    *whole_image = t.whole_image;
    *all_tiles = t.all_tiles;
    *largest_tile = t.largest_tile;
    *tiles_over_3 = t.tiles_over_3;
    return 0;
}

int32_t oracle_sizeof_compare_result(void) { return static_cast<int32_t>(sizeof(oracle::compare_result)); }

// Turquin's energy table by the oracle's own quadrature: 32 x 32 doubles, [j * 32 + i] for r = j/31, sqrt(mu) = i/31
int oracle_ggx_energy_table(double* out)
{
    const std::vector<double> t = oracle::ggx_energy_table();
    std::copy(t.begin(), t.end(), out);
    return 0;
}
}
