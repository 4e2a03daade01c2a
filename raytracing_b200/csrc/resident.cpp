// A scene made resident on the device: checked, its BVH built, every table converted to the kernels' 16-byte-aligned
// form and copied once (the session constructor's first half in the reference, renderer.cu:1080-1199).
#include <algorithm>
#include <cmath>
#include <limits>
#include <string>

#include "bvh_builder.h"
#include "host.h"

namespace rtb
{
void fail(rt_status status, const std::string& message) { throw rt_error(status, message); }

void check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess)
    {
        const rt_status s =
            e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? RT_ERR_NO_DEVICE : RT_ERR_RUNTIME;
        fail(s, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

namespace
{
bool finite(const rt_vec3& v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }
rt_vec3 sub(rt_vec3 a, rt_vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
rt_vec3 cross(rt_vec3 u, rt_vec3 v) { return {u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x}; }
double dot(rt_vec3 a, rt_vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
rt_vec3 scale(double s, rt_vec3 v) { return {s * v.x, s * v.y, s * v.z}; }
f3 to_f3(rt_vec3 v) { return {static_cast<float>(v.x), static_cast<float>(v.y), static_cast<float>(v.z)}; }

std::string index_error(const char* table, int64_t i, const char* field, int64_t value)
{
    return std::string(table) + "[" + std::to_string(i) + "]." + field + " = " + std::to_string(value) +
           " is out of range";
}

// make_quad (quad.cuh:40-52): the normal and the dual basis in double, rounded once
quad12 make_quad(const rt_quad_desc& d)
{
    const rt_vec3 n = cross(d.u, d.v);
    const rt_vec3 normal = scale(1 / std::sqrt(dot(n, n)), n);
    const rt_vec3 w = scale(1 / dot(n, n), n);
    const rt_vec3 a = cross(d.v, w);
    const rt_vec3 b = cross(w, d.u);
    quad12 q{};
    q.qx = static_cast<float>(d.q.x);
    q.qy = static_cast<float>(d.q.y);
    q.qz = static_cast<float>(d.q.z);
    q.nx = static_cast<float>(normal.x);
    q.ny = static_cast<float>(normal.y);
    q.nz = static_cast<float>(normal.z);
    q.ax = static_cast<float>(a.x);
    q.ay = static_cast<float>(a.y);
    q.az = static_cast<float>(a.z);
    q.bx = static_cast<float>(b.x);
    q.by = static_cast<float>(b.y);
    q.bz = static_cast<float>(b.z);
    return q;
}

// The same quad in double, for the FP64 integrator
quad_d make_quad_d(const rt_quad_desc& d)
{
    const rt_vec3 n = cross(d.u, d.v);
    const rt_vec3 normal = scale(1 / std::sqrt(dot(n, n)), n);
    const rt_vec3 w = scale(1 / dot(n, n), n);
    const rt_vec3 a = cross(d.v, w);
    const rt_vec3 b = cross(w, d.u);
    return quad_d{{d.q.x, d.q.y, d.q.z}, {normal.x, normal.y, normal.z}, {a.x, a.y, a.z}, {b.x, b.y, b.z}};
}

// A scene of at most RTB_SMALL_SCENE primitives gets one leaf per primitive kind (a test of all of them beats a
// tree walk there, as the reference found for up to 8 shapes, renderer.cu:75-82); a larger scene of spheres and quads
// gets leaves of at most RTB_LEAF_SIZE
#ifndef RTB_SMALL_SCENE
#define RTB_SMALL_SCENE 16
#endif
#ifndef RTB_LEAF_SIZE
#define RTB_LEAF_SIZE 1
#endif
// and a scene with triangles leaves of at most RTB_TRIANGLE_LEAF (a triangle's test is cheap next to a node step)
#ifndef RTB_TRIANGLE_LEAF
#define RTB_TRIANGLE_LEAF 4
#endif
// A scene of at most RTB_FLAT_SCENE spheres and quads (no triangles) is searched without its tree: every primitive
// tested in turn, the same loop in every lane of a warp, where a tree walk splits the lanes up. Measured on the
// B200: the Cornell boxes (13-18 quads and spheres) and the five-sphere scene render 30-50% faster flat, while 20
// scattered spheres are as fast either way and 40 are 25% slower flat.
#ifndef RTB_FLAT_SCENE
#define RTB_FLAT_SCENE 24
#endif

// A sphere whose quadratic is solved in FP64: radius large next to the spacing of floats at its center, where the
// l-vector form's r^2 - |l|^2 is a difference of numbers near r^2 (the radius-1000 ground)
constexpr double fp64_radius = 128;

// quad_box (bvh.cuh:145-187): the corners widened by 1e-6 of the largest coordinate, and to 0.0001 at least
build_prim quad_prim(const rt_quad_desc& d, int32_t source)
{
    const rt_vec3 c[4] = {d.q,
                          {d.q.x + d.u.x, d.q.y + d.u.y, d.q.z + d.u.z},
                          {d.q.x + d.v.x, d.q.y + d.v.y, d.q.z + d.v.z},
                          {d.q.x + d.u.x + d.v.x, d.q.y + d.u.y + d.v.y, d.q.z + d.u.z + d.v.z}};
    build_prim p{};
    double largest = 0;
    for (int a = 0; a < 3; ++a)
    {
        p.lo[a] = std::numeric_limits<double>::infinity();
        p.hi[a] = -std::numeric_limits<double>::infinity();
    }
    for (const rt_vec3& v : c)
    {
        const double xyz[3] = {v.x, v.y, v.z};
        for (int a = 0; a < 3; ++a)
        {
            p.lo[a] = std::min(p.lo[a], xyz[a]);
            p.hi[a] = std::max(p.hi[a], xyz[a]);
            largest = std::max(largest, std::fabs(xyz[a]));
        }
    }
    const double margin = 1e-6 * (1 + largest);
    for (int a = 0; a < 3; ++a)
    {
        p.lo[a] -= margin;
        p.hi[a] += margin;
        if (p.hi[a] - p.lo[a] < 0.0001)
        {
            p.lo[a] -= 0.00005;
            p.hi[a] += 0.00005;
        }
    }
    p.kind = kind_quad;
    p.source = source;
    return p;
}
} // namespace

// renderer.h:163-168: for every quad, all the corners of all the quads lie on one side of its plane, or on it within
// 1e-9 of the largest coordinate
bool is_convex(const rt_quad_desc* quads, int64_t count)
{
    double largest = 0;
    std::vector<rt_vec3> corners;
    for (int64_t i = 0; i < count; ++i)
    {
        const rt_quad_desc& q = quads[i];
        const rt_vec3 c[4] = {q.q,
                              {q.q.x + q.u.x, q.q.y + q.u.y, q.q.z + q.u.z},
                              {q.q.x + q.v.x, q.q.y + q.v.y, q.q.z + q.v.z},
                              {q.q.x + q.u.x + q.v.x, q.q.y + q.u.y + q.v.y, q.q.z + q.u.z + q.v.z}};
        for (const rt_vec3& v : c)
        {
            corners.push_back(v);
            largest = std::fmax(largest, std::fmax(std::fabs(v.x), std::fmax(std::fabs(v.y), std::fabs(v.z))));
        }
    }
    const double tolerance = 1e-9 * std::fmax(1.0, largest);
    for (int64_t i = 0; i < count; ++i)
    {
        const rt_quad_desc& q = quads[i];
        const rt_vec3 n = cross(q.u, q.v);
        const double len = std::sqrt(dot(n, n));
        if (!(len > 0))
        {
            return false;
        }
        bool above = false;
        bool below = false;
        for (const rt_vec3& c : corners)
        {
            const double s = dot(sub(c, q.q), n) / len;
            above = above || s > tolerance;
            below = below || s < -tolerance;
        }
        if (above && below)
        {
            return false;
        }
    }
    return true;
}

void validate(const rt_scene_desc& d)
{
    const rt_camera_desc& c = d.camera;
    if (c.image_width < 1 || c.image_height < 1)
    {
        fail(RT_ERR_RUNTIME, "the camera's image must be at least 1 x 1 pixels");
    }
    if (static_cast<int64_t>(c.image_width) * c.image_height >= (int64_t{1} << 31))
    {
        fail(RT_ERR_RUNTIME, "the image has more than 2^31 pixels");
    }
    if (c.sqrt_spp < 1 || c.sqrt_spp > 46340)
    {
        fail(RT_ERR_RUNTIME, "camera.sqrt_spp must be in [1, 46340]");
    }
    if (c.max_depth < 0)
    {
        fail(RT_ERR_RUNTIME, "camera.max_depth must not be negative");
    }
    if (c.sampling < RT_SAMPLING_UNIFORM || c.sampling > RT_SAMPLING_MIXTURE)
    {
        fail(RT_ERR_RUNTIME, "camera.sampling is not a strategy");
    }
    if (!finite(c.center) || !finite(c.pixel00_loc) || !finite(c.pixel_delta_u) || !finite(c.pixel_delta_v) ||
        !finite(c.defocus_disk_u) || !finite(c.defocus_disk_v) || !finite(c.sky_bottom) || !finite(c.sky_top))
    {
        fail(RT_ERR_RUNTIME, "the camera has a coordinate that is not a finite number");
    }
    if ((d.sphere_count > 0 && !d.spheres) || (d.quad_count > 0 && !d.quads) ||
        (d.material_count > 0 && !d.materials) || (d.texture_count > 0 && !d.textures) ||
        (d.light_count > 0 && !d.lights) || (d.mesh_count > 0 && !d.meshes))
    {
        fail(RT_ERR_RUNTIME, "a table has a count but no data");
    }
    // Textures, images and Perlin tables (renderer.cu:688-760): a checker refers to textures before it, so walking a
    // chain of checkers ends; every index in range; pixels and gradients finite
    if ((d.image_count > 0 && !d.images) || (d.perlin_count > 0 && !d.perlins) || (d.medium_count > 0 && !d.media))
    {
        fail(RT_ERR_RUNTIME, "a table has a count but no data");
    }
    int64_t image_pixels = 0;
    for (int64_t i = 0; i < d.image_count; ++i)
    {
        const rt_image_desc& im = d.images[i];
        if (im.width < 1 || im.height < 1 || !im.rgb)
        {
            fail(RT_ERR_RUNTIME, "images[" + std::to_string(i) + "]: an image texture's pixels don't match its size");
        }
        const int64_t n = int64_t{im.width} * im.height;
        image_pixels += n;
        if (image_pixels >= (int64_t{1} << 31))
        {
            fail(RT_ERR_RUNTIME, "the images have too many pixels for the GPU renderer");
        }
        for (int64_t k = 0; k < 3 * n; ++k)
        {
            if (!std::isfinite(im.rgb[k]))
            {
                fail(RT_ERR_RUNTIME, "images[" + std::to_string(i) + "] has a pixel that is not a finite number");
            }
        }
    }
    for (int64_t i = 0; i < d.perlin_count; ++i)
    {
        const rt_perlin_desc& p = d.perlins[i];
        for (int k = 0; k < 256; ++k)
        {
            const int32_t perm[3] = {p.perm_x[k], p.perm_y[k], p.perm_z[k]};
            for (const int32_t v : perm)
            {
                if (v < 0 || v > 255)
                {
                    fail(RT_ERR_RUNTIME, "a Perlin permutation has an entry outside 0..255");
                }
            }
            if (!finite(p.random_vectors[k]))
            {
                fail(RT_ERR_RUNTIME, "perlins[" + std::to_string(i) + "] has a gradient that is not finite");
            }
        }
    }
    for (int64_t i = 0; i < d.texture_count; ++i)
    {
        const rt_texture_desc& t = d.textures[i];
        switch (t.kind)
        {
        case RT_TEXTURE_SOLID:
            if (!finite(t.rgb))
            {
                fail(RT_ERR_RUNTIME, "textures[" + std::to_string(i) + "] is not finite");
            }
            break;
        case RT_TEXTURE_CHECKER:
            if (t.even < 0 || t.even >= i || t.odd < 0 || t.odd >= i || !std::isfinite(t.inv_scale))
            {
                fail(RT_ERR_RUNTIME, "textures[" + std::to_string(i) +
                                         "]: a checker texture must refer to textures that come before it");
            }
            break;
        case RT_TEXTURE_IMAGE:
            if (t.image < 0 || t.image >= d.image_count)
            {
                fail(RT_ERR_RUNTIME, "textures[" + std::to_string(i) +
                                         "]: an image texture refers to an image that doesn't exist");
            }
            break;
        case RT_TEXTURE_NOISE:
            if (t.perlin < 0 || t.perlin >= d.perlin_count || !std::isfinite(t.scale))
            {
                fail(RT_ERR_RUNTIME, "textures[" + std::to_string(i) +
                                         "]: a marble texture refers to Perlin tables that don't exist");
            }
            break;
        default:
            fail(RT_ERR_RUNTIME, "textures[" + std::to_string(i) + "]: unknown texture kind");
        }
    }
    for (int64_t i = 0; i < d.material_count; ++i)
    {
        const rt_material_desc& m = d.materials[i];
        if (m.kind < RT_LAMBERTIAN || m.kind > RT_ISOTROPIC)
        {
            fail(RT_ERR_RUNTIME, "materials[" + std::to_string(i) + "] has no valid kind");
        }
        if (m.kind == RT_LAMBERTIAN || m.kind == RT_DIFFUSE_LIGHT || m.kind == RT_ISOTROPIC)
        {
            if (m.texture < 0 || m.texture >= d.texture_count)
            {
                fail(RT_ERR_RUNTIME, index_error("materials", i, "texture", m.texture));
            }
        }
        if (m.kind == RT_METAL && (!finite(m.albedo) || !(m.fuzz >= 0)))
        {
            fail(RT_ERR_RUNTIME, "materials[" + std::to_string(i) + "]: a metal needs a finite albedo and fuzz >= 0");
        }
        if (m.kind == RT_DIELECTRIC && !(m.refraction_index > 0 && std::isfinite(m.refraction_index)))
        {
            fail(RT_ERR_RUNTIME, "materials[" + std::to_string(i) + "]: refraction_index must be positive");
        }
    }
    for (int64_t i = 0; i < d.sphere_count; ++i)
    {
        const rt_sphere_desc& s = d.spheres[i];
        if (s.material < 0 || s.material >= d.material_count)
        {
            fail(RT_ERR_RUNTIME, index_error("spheres", i, "material", s.material));
        }
        if (!finite(s.center) || !(s.radius >= 0 && std::isfinite(s.radius)) || !finite(s.displacement) ||
            !std::isfinite(s.uv_cos) || !std::isfinite(s.uv_sin))
        {
            fail(RT_ERR_RUNTIME, "spheres[" + std::to_string(i) + "] is not a finite sphere");
        }
    }
    for (int64_t i = 0; i < d.quad_count; ++i)
    {
        const rt_quad_desc& q = d.quads[i];
        if (q.material < 0 || q.material >= d.material_count)
        {
            fail(RT_ERR_RUNTIME, index_error("quads", i, "material", q.material));
        }
        if (!finite(q.q) || !finite(q.u) || !finite(q.v))
        {
            fail(RT_ERR_RUNTIME, "quads[" + std::to_string(i) + "] is not finite");
        }
    }
    for (int64_t m = 0; m < d.mesh_count; ++m)
    {
        const rt_mesh_desc& mesh = d.meshes[m];
        if (mesh.material < 0 || mesh.material >= d.material_count)
        {
            fail(RT_ERR_RUNTIME, index_error("meshes", m, "material", mesh.material));
        }
        if ((mesh.triangle_count > 0 && (!mesh.indices || !mesh.positions)) || mesh.triangle_count < 0 ||
            mesh.vertex_count < 0)
        {
            fail(RT_ERR_RUNTIME, "meshes[" + std::to_string(m) + "] has a count but no data");
        }
        for (int64_t k = 0; k < mesh.triangle_count * 3; ++k)
        {
            if (mesh.indices[k] >= static_cast<uint64_t>(mesh.vertex_count))
            {
                fail(RT_ERR_RUNTIME, index_error("meshes.indices", k, "vertex", mesh.indices[k]));
            }
        }
    }
    if (d.medium_count > max_media)
    {
        fail(RT_ERR_UNSUPPORTED, "a scene may hold at most " + std::to_string(max_media) + " volumes of smoke");
    }
    for (int64_t i = 0; i < d.medium_count; ++i)
    {
        const rt_medium_desc& m = d.media[i];
        const std::string where = "media[" + std::to_string(i) + "]";
        if (m.material < 0 || m.material >= d.material_count || d.materials[m.material].kind != RT_ISOTROPIC)
        {
            fail(RT_ERR_RUNTIME, where + ": a volume of smoke must refer to an isotropic material");
        }
        if (!(m.neg_inv_density < 0 && std::isfinite(m.neg_inv_density)))
        {
            fail(RT_ERR_RUNTIME, where + ": a volume of smoke needs a finite density > 0 (neg_inv_density < 0)");
        }
        if (m.boundary == RT_BOUNDARY_SPHERE)
        {
            if (!finite(m.sphere.center) || !(m.sphere.radius > 0 && std::isfinite(m.sphere.radius)) ||
                !finite(m.sphere.displacement))
            {
                fail(RT_ERR_RUNTIME, where + ": its boundary is not a finite sphere");
            }
        }
        else if (m.boundary == RT_BOUNDARY_CONVEX_QUADS)
        {
            bool convex = m.quad_count > 0 && m.quads;
            for (int64_t k = 0; convex && k < m.quad_count; ++k)
            {
                convex = finite(m.quads[k].q) && finite(m.quads[k].u) && finite(m.quads[k].v);
            }
            if (!convex || !is_convex(m.quads, m.quad_count))
            {
                fail(RT_ERR_RUNTIME, where + ": a volume of smoke must be bounded by one sphere or by quads of a convex "
                                             "shape");
            }
        }
        else
        {
            fail(RT_ERR_RUNTIME, where + ": a volume of smoke must be bounded by one sphere or by quads of a convex shape");
        }
    }
    for (int64_t i = 0; i < d.light_count; ++i)
    {
        const rt_light_desc& l = d.lights[i];
        if (l.kind != RT_LIGHT_QUAD && l.kind != RT_LIGHT_SPHERE)
        {
            fail(RT_ERR_RUNTIME, "lights[" + std::to_string(i) + "] has no valid kind");
        }
        if (!(l.weight >= 0 && std::isfinite(l.weight)))
        {
            fail(RT_ERR_RUNTIME, "lights[" + std::to_string(i) + "].weight must be finite and >= 0");
        }
        if (l.kind == RT_LIGHT_SPHERE && !(l.radius > 0))
        {
            fail(RT_ERR_RUNTIME, "lights[" + std::to_string(i) + "] is a sphere without size");
        }
    }
    const bool aims = c.sampling == RT_SAMPLING_LIGHTS || c.sampling == RT_SAMPLING_MIXTURE;
    if (aims && d.light_count == 0)
    {
        fail(RT_ERR_RUNTIME, "the lights and mixture strategies need a lights list to aim at");
    }
    if (d.combination < RT_COMBINE_BSDF_ONLY || d.combination > RT_COMBINE_POWER_HEURISTIC)
    {
        fail(RT_ERR_RUNTIME, "combination is not a light combination");
    }
    if (d.quality && c.sampling != RT_SAMPLING_MATERIAL)
    {
        fail(RT_ERR_INVALID, "the NEE/MIS integrator samples as the material scatters: camera.sampling must be material");
    }
    if (d.microfacet_count != 0 && d.microfacet_count != d.material_count)
    {
        fail(RT_ERR_RUNTIME, "microfacets: none, or one per material");
    }
    bool side_entries = false;
    for (int64_t i = 0; i < d.microfacet_count; ++i)
    {
        const rt_microfacet_desc& f = d.microfacets[i];
        if (f.kind == RT_MICROFACET_NONE)
        {
            continue;
        }
        side_entries = true;
        const std::string where = "microfacets[" + std::to_string(i) + "]";
        if (f.kind != RT_MICROFACET_CONDUCTOR && f.kind != RT_MICROFACET_GLOSS)
        {
            fail(RT_ERR_RUNTIME, where + " has no valid kind");
        }
        if (!(f.roughness >= 0 && f.roughness <= 1))
        {
            fail(RT_ERR_RUNTIME, where + ".roughness must be in [0, 1]");
        }
        // renderer.h:249-261: a conductor completes a metal of fuzz 0, a coat a lambertian, whose alpha is >= 1e-3
        const rt_material_desc& m = d.materials[i];
        if (f.kind == RT_MICROFACET_CONDUCTOR && !(m.kind == RT_METAL && m.fuzz == 0))
        {
            fail(RT_ERR_RUNTIME, where + ": a conductor's material must be a metal of fuzz 0");
        }
        if (f.kind == RT_MICROFACET_GLOSS && (m.kind != RT_LAMBERTIAN || f.roughness * f.roughness < 1e-3))
        {
            fail(RT_ERR_RUNTIME, where + ": a coat's material must be a lambertian, with roughness^2 >= 1e-3");
        }
    }
    if (d.environment)
    {
        const rt_environment_desc& e = *d.environment;
        if (e.image.width < 1 || e.image.height < 1 || e.image.width > 2048 || e.image.height > 1024 || !e.image.rgb)
        {
            fail(RT_ERR_RUNTIME, "an environment map has 1x1 to 2048x1024 texels");
        }
        if (!std::isfinite(e.yaw_degrees) || !(std::isfinite(e.scale) && e.scale >= 0))
        {
            fail(RT_ERR_INVALID, "an environment map's yaw and scale must be finite, the scale >= 0");
        }
        const int64_t n = int64_t{e.image.width} * e.image.height * 3;
        for (int64_t k = 0; k < n; ++k)
        {
            if (!(std::isfinite(e.image.rgb[k]) && e.image.rgb[k] >= 0))
            {
                fail(RT_ERR_RUNTIME, "an environment map's texels must be finite and >= 0");
            }
        }
    }
    if ((side_entries || d.environment) && !d.quality)
    {
        fail(RT_ERR_INVALID, "GGX side entries and environment maps need the NEE/MIS integrator (quality)");
    }
}

camera_params to_camera(const rt_camera_desc& d)
{
    camera_params c{};
    c.width = d.image_width;
    c.height = d.image_height;
    c.sqrt_spp = d.sqrt_spp;
    c.max_depth = d.max_depth;
    c.recip_sqrt_spp = static_cast<float>(1.0 / d.sqrt_spp);
    c.center = to_f3(d.center);
    c.center_to_pixel00 = to_f3(sub(d.pixel00_loc, d.center));
    c.delta_u = to_f3(d.pixel_delta_u);
    c.delta_v = to_f3(d.pixel_delta_v);
    c.defocus = d.defocus;
    c.disk_u = to_f3(d.defocus_disk_u);
    c.disk_v = to_f3(d.defocus_disk_v);
    c.sky_bottom = to_f3(d.sky_bottom);
    c.sky_top = to_f3(d.sky_top);
    c.sampling = d.sampling;
    if (d.image_width > 0 && d.image_height > 0 && d.sqrt_spp > 0)
    {
        const auto tiles_x = static_cast<uint32_t>((d.image_width + 7) / 8);
        const auto tiles_y = static_cast<uint32_t>((d.image_height + 3) / 4);
        c.div_sqrt_spp = make_fast_divisor(static_cast<uint32_t>(d.sqrt_spp));
        c.div_round_passes = make_fast_divisor(static_cast<uint32_t>(d.sqrt_spp) * static_cast<uint32_t>(d.sqrt_spp));
        c.div_tiles_x = make_fast_divisor(tiles_x);
        c.div_padded = make_fast_divisor(tiles_x * tiles_y * 32u);
    }
    return c;
}

camera_d to_camera_d(const rt_camera_desc& d)
{
    const auto put = [](double* out, rt_vec3 v) {
        out[0] = v.x;
        out[1] = v.y;
        out[2] = v.z;
    };
    camera_d c{};
    c.width = d.image_width;
    c.height = d.image_height;
    c.sqrt_spp = d.sqrt_spp;
    c.max_depth = d.max_depth;
    c.recip_sqrt_spp = 1.0 / d.sqrt_spp;
    put(c.center, d.center);
    put(c.to_pixel00, sub(d.pixel00_loc, d.center));
    put(c.delta_u, d.pixel_delta_u);
    put(c.delta_v, d.pixel_delta_v);
    put(c.disk_u, d.defocus_disk_u);
    put(c.disk_v, d.defocus_disk_v);
    put(c.sky_bottom, d.sky_bottom);
    put(c.sky_top, d.sky_top);
    c.defocus = d.defocus;
    c.sampling = d.sampling;
    return c;
}

resident_scene::resident_scene(const rt_scene_desc& d)
{
    validate(d);
    check(cudaGetDevice(&device_), "selecting the CUDA device");
    camera_ = d.camera;
    quality_ = d.quality != 0;

    // The primitives' boxes for the builder
    std::vector<build_prim> prims;
    std::vector<sphere4> source_spheres;
    std::vector<float4> source_motion;
    std::vector<sphere_frame> source_frames;
    bool motion = false;
    for (int64_t i = 0; i < d.sphere_count; ++i)
    {
        const rt_sphere_desc& s = d.spheres[i];
        sphere4 v{static_cast<float>(s.center.x), static_cast<float>(s.center.y), static_cast<float>(s.center.z),
                  static_cast<float>(s.radius)};
        const float4 m = make_float4(static_cast<float>(s.displacement.x), static_cast<float>(s.displacement.y),
                                     static_cast<float>(s.displacement.z), 0.0f);
        motion = motion || m.x != 0.0f || m.y != 0.0f || m.z != 0.0f;
        // sphere_box (bvh.cuh:140-152): the float sphere's extent, each bound one double step outward; a moving
        // sphere's box holds it over the whole shutter (where it is at times 0 and 1)
        build_prim p{};
        const double c[3] = {v.cx, v.cy, v.cz};
        const double dm[3] = {m.x, m.y, m.z};
        for (int a = 0; a < 3; ++a)
        {
            const double lo = std::min(c[a], c[a] + dm[a]);
            const double hi = std::max(c[a], c[a] + dm[a]);
            p.lo[a] = std::nextafter(lo - static_cast<double>(v.r), -std::numeric_limits<double>::infinity());
            p.hi[a] = std::nextafter(hi + static_cast<double>(v.r), std::numeric_limits<double>::infinity());
        }
        p.kind = kind_sphere;
        p.source = static_cast<int32_t>(i);
        prims.push_back(p);
        if (s.radius >= fp64_radius)
        {
            v.r = -v.r;
        }
        source_spheres.push_back(v);
        source_motion.push_back(m);
        // The texture frame (sphere.cuh:119-168): the instances' turn, and for onto_sphere k = |c|^2 - r^2 and the
        // bound 2 r |c| below which its one Newton step helps
        const double cc = dot(s.center, s.center);
        source_frames.push_back({static_cast<float>(s.uv_cos), static_cast<float>(s.uv_sin),
                                 static_cast<float>(cc - s.radius * s.radius),
                                 static_cast<float>(2 * s.radius * std::sqrt(cc))});
    }
    std::vector<quad12> source_quads;
    for (int64_t i = 0; i < d.quad_count; ++i)
    {
        prims.push_back(quad_prim(d.quads[i], static_cast<int32_t>(i)));
        source_quads.push_back(make_quad(d.quads[i]));
    }
    std::vector<triangle12> source_triangles;
    std::vector<int32_t> triangle_material;
    for (int64_t m = 0; m < d.mesh_count; ++m)
    {
        const rt_mesh_desc& mesh = d.meshes[m];
        for (int64_t t = 0; t < mesh.triangle_count; ++t)
        {
            const float* a = mesh.positions + 3 * mesh.indices[3 * t];
            const float* b = mesh.positions + 3 * mesh.indices[3 * t + 1];
            const float* c = mesh.positions + 3 * mesh.indices[3 * t + 2];
            triangle12 tr{};
            tr.ax = a[0];
            tr.ay = a[1];
            tr.az = a[2];
            tr.bx = b[0];
            tr.by = b[1];
            tr.bz = b[2];
            tr.cx = c[0];
            tr.cy = c[1];
            tr.cz = c[2];
            build_prim p{};
            double largest = 0;
            for (int axis = 0; axis < 3; ++axis)
            {
                p.lo[axis] = std::min({static_cast<double>(a[axis]), static_cast<double>(b[axis]), static_cast<double>(c[axis])});
                p.hi[axis] = std::max({static_cast<double>(a[axis]), static_cast<double>(b[axis]), static_cast<double>(c[axis])});
                largest = std::max({largest, std::fabs(p.lo[axis]), std::fabs(p.hi[axis])});
            }
            const double margin = 1e-6 * (1 + largest);
            for (int axis = 0; axis < 3; ++axis)
            {
                p.lo[axis] -= margin;
                p.hi[axis] += margin;
            }
            p.kind = kind_triangle;
            p.source = static_cast<int32_t>(source_triangles.size());
            prims.push_back(p);
            source_triangles.push_back(tr);
            triangle_material.push_back(mesh.material);
        }
    }

    bvh_options options;
    options.max_leaf_size = prims.size() <= RTB_SMALL_SCENE ? max_leaf_size
                                                            : (source_triangles.empty() ? RTB_LEAF_SIZE : RTB_TRIANGLE_LEAF);
    const bvh_result tree = build_bvh(std::move(prims), options);

    // Each kind's array in leaf order; global ids: spheres, then quads, then triangles
    const auto S = static_cast<int32_t>(d.sphere_count);
    const auto Q = static_cast<int32_t>(d.quad_count);
    const auto T = static_cast<int32_t>(source_triangles.size());
    std::vector<sphere4> spheres(tree.order[kind_sphere].size());
    std::vector<float4> sphere_motion(motion ? spheres.size() : 0);
    std::vector<sphere_frame> sphere_frames(spheres.size());
    std::vector<quad12> quads(tree.order[kind_quad].size());
    std::vector<triangle12> triangles(tree.order[kind_triangle].size());
    std::vector<int32_t> prim_material(static_cast<size_t>(S + Q + T));
    std::vector<int32_t> prim_source(static_cast<size_t>(S + Q + T));
    std::vector<int32_t> sphere_gid(static_cast<size_t>(S));
    std::vector<int32_t> quad_gid(static_cast<size_t>(Q));
    for (size_t k = 0; k < spheres.size(); ++k)
    {
        const int32_t src = tree.order[kind_sphere][k];
        spheres[k] = source_spheres[static_cast<size_t>(src)];
        sphere_frames[k] = source_frames[static_cast<size_t>(src)];
        if (motion)
        {
            sphere_motion[k] = source_motion[static_cast<size_t>(src)];
        }
        prim_material[k] = d.spheres[src].material;
        prim_source[k] = src;
        sphere_gid[static_cast<size_t>(src)] = static_cast<int32_t>(k);
    }
    for (size_t k = 0; k < quads.size(); ++k)
    {
        const int32_t src = tree.order[kind_quad][k];
        quads[k] = source_quads[static_cast<size_t>(src)];
        prim_material[static_cast<size_t>(S) + k] = d.quads[src].material;
        prim_source[static_cast<size_t>(S) + k] = S + src;
        quad_gid[static_cast<size_t>(src)] = S + static_cast<int32_t>(k);
    }
    for (size_t k = 0; k < triangles.size(); ++k)
    {
        const int32_t src = tree.order[kind_triangle][k];
        triangles[k] = source_triangles[static_cast<size_t>(src)];
        prim_material[static_cast<size_t>(S + Q) + k] = triangle_material[static_cast<size_t>(src)];
        prim_source[static_cast<size_t>(S + Q) + k] = S + Q + src;
    }

    // Textures (texture.cuh): every texture as a record, an image's texels after the others', a marble's own noise
    // tables; a material whose texture is one solid color gets the color itself and no texture to read
    std::vector<texture8> textures;
    std::vector<image_info> images;
    std::vector<float4> texels;
    std::vector<noise_table> noises;
    for (int64_t i = 0; i < d.image_count; ++i)
    {
        const rt_image_desc& im = d.images[i];
        images.push_back({static_cast<int32_t>(texels.size()), im.width, im.height, 0});
        for (int64_t k = 0; k < int64_t{im.width} * im.height; ++k)
        {
            texels.push_back(make_float4(im.rgb[3 * k], im.rgb[3 * k + 1], im.rgb[3 * k + 2], 0.0f));
        }
    }
    for (int64_t i = 0; i < d.texture_count; ++i)
    {
        const rt_texture_desc& t = d.textures[i];
        texture8 v{};
        v.kind = t.kind;
        v.even = t.even;
        v.odd = t.odd;
        v.r = static_cast<float>(t.rgb.x);
        v.g = static_cast<float>(t.rgb.y);
        v.b = static_cast<float>(t.rgb.z);
        v.inv_scale = static_cast<float>(t.inv_scale);
        if (t.kind == RT_TEXTURE_IMAGE)
        {
            v.table = t.image;
        }
        else if (t.kind == RT_TEXTURE_NOISE)
        {
            v.table = static_cast<int32_t>(noises.size());
            noise_table n{};
            const rt_perlin_desc& p = d.perlins[t.perlin];
            for (int k = 0; k < 256; ++k)
            {
                n.gradients[k] = make_float4(static_cast<float>(p.random_vectors[k].x),
                                             static_cast<float>(p.random_vectors[k].y),
                                             static_cast<float>(p.random_vectors[k].z), 0.0f);
                n.perm_x[k] = static_cast<uint8_t>(p.perm_x[k]);
                n.perm_y[k] = static_cast<uint8_t>(p.perm_y[k]);
                n.perm_z[k] = static_cast<uint8_t>(p.perm_z[k]);
            }
            n.scale = static_cast<float>(t.scale);
            noises.push_back(n);
        }
        textures.push_back(v);
    }
    // What reading a texture needs of the hit: (u, v) for an image somewhere in its checkers' tree, the point for a
    // checker (moved onto a sphere exactly)
    const auto needs_of = [&](int32_t root) {
        int32_t needs = 0;
        std::vector<int32_t> pending{root};
        while (!pending.empty())
        {
            const rt_texture_desc& t = d.textures[pending.back()];
            pending.pop_back();
            if (t.kind == RT_TEXTURE_CHECKER)
            {
                needs |= texture_needs_point;
                pending.push_back(t.even);
                pending.push_back(t.odd);
            }
            needs |= t.kind == RT_TEXTURE_IMAGE ? texture_needs_uv : 0;
        }
        return needs;
    };

    // Materials: a solid texture becomes the material's color (renderer.cu:551-600)
    std::vector<material12> materials;
    for (int64_t i = 0; i < d.material_count; ++i)
    {
        const rt_material_desc& m = d.materials[i];
        material12 v{};
        v.kind = m.kind;
        v.texture = -1;
        const bool textured = m.kind == RT_LAMBERTIAN || m.kind == RT_DIFFUSE_LIGHT || m.kind == RT_ISOTROPIC;
        if (textured && d.textures[m.texture].kind != RT_TEXTURE_SOLID)
        {
            v.texture = m.texture;
            v.texture_needs = needs_of(m.texture);
        }
        const rt_vec3 color = textured ? d.textures[m.texture].rgb : m.albedo;
        v.r = static_cast<float>(color.x);
        v.g = static_cast<float>(color.y);
        v.b = static_cast<float>(color.z);
        v.fuzz = static_cast<float>(std::min(m.fuzz, 1.0));
        v.ior = static_cast<float>(m.refraction_index);
        if (i < d.microfacet_count)
        {
            v.lobe = d.microfacets[i].kind;
            v.roughness = static_cast<float>(d.microfacets[i].roughness);
            v.alpha = static_cast<float>(d.microfacets[i].roughness * d.microfacets[i].roughness);
        }
        materials.push_back(v);
    }

    // The books' lights list, with each light's twin (renderer.cu:968-1033): only the lights and mixture strategies
    // read it
    std::vector<light24> lights;
    if (d.camera.sampling == RT_SAMPLING_LIGHTS || d.camera.sampling == RT_SAMPLING_MIXTURE)
    {
        double cdf = 0;
        for (int64_t i = 0; i < d.light_count; ++i)
        {
            const rt_light_desc& l = d.lights[i];
            cdf += l.weight;
            light24 v{};
            v.twin = -1;
            if (l.kind == RT_LIGHT_QUAD)
            {
                v.quad = make_quad(l.quad);
                const rt_vec3 n = cross(l.quad.u, l.quad.v);
                v.ux = static_cast<float>(l.quad.u.x);
                v.uy = static_cast<float>(l.quad.u.y);
                v.uz = static_cast<float>(l.quad.u.z);
                v.area = static_cast<float>(std::sqrt(dot(n, n)));
                v.vx = static_cast<float>(l.quad.v.x);
                v.vy = static_cast<float>(l.quad.v.y);
                v.vz = static_cast<float>(l.quad.v.z);
                for (int64_t q = 0; q < d.quad_count; ++q)
                {
                    const rt_quad_desc& w = d.quads[q];
                    if (w.q.x == l.quad.q.x && w.q.y == l.quad.q.y && w.q.z == l.quad.q.z && w.u.x == l.quad.u.x &&
                        w.u.y == l.quad.u.y && w.u.z == l.quad.u.z && w.v.x == l.quad.v.x && w.v.y == l.quad.v.y &&
                        w.v.z == l.quad.v.z)
                    {
                        v.twin = quad_gid[static_cast<size_t>(q)];
                        break;
                    }
                }
            }
            else
            {
                v.cx = static_cast<float>(l.center.x);
                v.cy = static_cast<float>(l.center.y);
                v.cz = static_cast<float>(l.center.z);
                v.radius = static_cast<float>(l.radius);
                for (int64_t s = 0; s < d.sphere_count; ++s)
                {
                    const rt_sphere_desc& w = d.spheres[s];
                    if (w.center.x == l.center.x && w.center.y == l.center.y && w.center.z == l.center.z &&
                        w.radius == l.radius)
                    {
                        v.twin = sphere_gid[static_cast<size_t>(s)];
                        break;
                    }
                }
            }
            v.cdf = static_cast<float>(cdf);
            v.weight = static_cast<float>(l.weight);
            v.kind = l.kind;
            lights.push_back(v);
        }
    }

    // The NEE/MIS integrator's lamps: still spheres, then quads, glowing one solid color (lamp_table.cu)
    std::vector<emitter20> lamps;
    std::vector<int32_t> lamp_of(static_cast<size_t>(S + Q + T), -1);
    const auto glows = [&](int32_t material) {
        return d.materials[material].kind == RT_DIFFUSE_LIGHT &&
               d.textures[d.materials[material].texture].kind == RT_TEXTURE_SOLID;
    };
    const auto radiance = [&](int32_t material) { return d.textures[d.materials[material].texture].rgb; };
    for (int64_t i = 0; i < d.sphere_count; ++i)
    {
        const rt_sphere_desc& s = d.spheres[i];
        const bool still = s.displacement.x == 0 && s.displacement.y == 0 && s.displacement.z == 0;
        if (still && glows(s.material))
        {
            emitter20 e{};
            e.cx = static_cast<float>(s.center.x);
            e.cy = static_cast<float>(s.center.y);
            e.cz = static_cast<float>(s.center.z);
            e.size = static_cast<float>(s.radius);
            e.kind = RT_LIGHT_SPHERE;
            e.primitive = sphere_gid[static_cast<size_t>(i)];
            const rt_vec3 r = radiance(s.material);
            e.er = static_cast<float>(r.x);
            e.eg = static_cast<float>(r.y);
            e.eb = static_cast<float>(r.z);
            lamp_of[static_cast<size_t>(e.primitive)] = static_cast<int32_t>(lamps.size());
            lamps.push_back(e);
        }
    }
    for (int64_t i = 0; i < d.quad_count; ++i)
    {
        const rt_quad_desc& q = d.quads[i];
        if (glows(q.material))
        {
            const quad12 made = make_quad(q);
            const rt_vec3 n = cross(q.u, q.v);
            emitter20 e{};
            e.cx = static_cast<float>(q.q.x);
            e.cy = static_cast<float>(q.q.y);
            e.cz = static_cast<float>(q.q.z);
            e.size = static_cast<float>(std::sqrt(dot(n, n)));
            e.ux = static_cast<float>(q.u.x);
            e.uy = static_cast<float>(q.u.y);
            e.uz = static_cast<float>(q.u.z);
            e.kind = RT_LIGHT_QUAD;
            e.vx = static_cast<float>(q.v.x);
            e.vy = static_cast<float>(q.v.y);
            e.vz = static_cast<float>(q.v.z);
            e.primitive = quad_gid[static_cast<size_t>(i)];
            e.nx = made.nx;
            e.ny = made.ny;
            e.nz = made.nz;
            const rt_vec3 r = radiance(q.material);
            e.er = static_cast<float>(r.x);
            e.eg = static_cast<float>(r.y);
            e.eb = static_cast<float>(r.z);
            lamp_of[static_cast<size_t>(e.primitive)] = static_cast<int32_t>(lamps.size());
            lamps.push_back(e);
        }
    }

    // The environment map's tables (the NEE/MIS integrator's sky and light)
    environment_view env{};
    if (d.environment)
    {
        const environment_tables t = build_environment(*d.environment);
        env_texels_.upload(t.texels);
        env_bins_.upload(t.bins);
        env_row_cos_.upload(t.row_cos);
        env.texels = env_texels_.data();
        env.bins = env_bins_.data();
        env.row_cos = env_row_cos_.data();
        env.width = t.width;
        env.height = t.height;
        env.log2_bins = t.log2_bins;
        env.sampled = t.total > 0 ? 1 : 0;
        const double yaw = d.environment->yaw_degrees * 3.14159265358979323846 / 180;
        env.cos_yaw = static_cast<float>(std::cos(yaw));
        env.sin_yaw = static_cast<float>(std::sin(yaw));
        env.scale = static_cast<float>(d.environment->scale);
    }

    // Volumes of smoke (constant_medium.cuh): a box over the whole shutter, rounded outward, and the boundary
    std::vector<medium16> media;
    std::vector<quad12> boundary_quads;
    for (int64_t i = 0; i < d.medium_count; ++i)
    {
        const rt_medium_desc& m = d.media[i];
        medium16 v{};
        v.neg_inv_density = static_cast<float>(m.neg_inv_density);
        v.material = m.material;
        double lo[3] = {std::numeric_limits<double>::infinity(), std::numeric_limits<double>::infinity(),
                        std::numeric_limits<double>::infinity()};
        double hi[3] = {-lo[0], -lo[1], -lo[2]};
        if (m.boundary == RT_BOUNDARY_SPHERE)
        {
            const rt_sphere_desc& s = m.sphere;
            v.cx = static_cast<float>(s.center.x);
            v.cy = static_cast<float>(s.center.y);
            v.cz = static_cast<float>(s.center.z);
            v.radius = static_cast<float>(s.radius);
            v.dx = static_cast<float>(s.displacement.x);
            v.dy = static_cast<float>(s.displacement.y);
            v.dz = static_cast<float>(s.displacement.z);
            motion = motion || v.dx != 0.0f || v.dy != 0.0f || v.dz != 0.0f;
            const double c[3] = {s.center.x, s.center.y, s.center.z};
            const double dm[3] = {s.displacement.x, s.displacement.y, s.displacement.z};
            for (int a = 0; a < 3; ++a)
            {
                lo[a] = std::min(c[a], c[a] + dm[a]) - s.radius;
                hi[a] = std::max(c[a], c[a] + dm[a]) + s.radius;
            }
        }
        else
        {
            v.first_quad = static_cast<int32_t>(boundary_quads.size());
            v.quad_count = static_cast<int32_t>(m.quad_count);
            for (int64_t k = 0; k < m.quad_count; ++k)
            {
                boundary_quads.push_back(make_quad(m.quads[k]));
                const build_prim b = quad_prim(m.quads[k], 0);
                for (int a = 0; a < 3; ++a)
                {
                    lo[a] = std::min(lo[a], b.lo[a]);
                    hi[a] = std::max(hi[a], b.hi[a]);
                }
            }
        }
        v.lo_x = round_down(lo[0]);
        v.lo_y = round_down(lo[1]);
        v.lo_z = round_down(lo[2]);
        v.hi_x = round_up(hi[0]);
        v.hi_y = round_up(hi[1]);
        v.hi_z = round_up(hi[2]);
        media.push_back(v);
    }
    if (motion && sphere_motion.empty())
    {
        sphere_motion.assign(spheres.size(), make_float4(0.0f, 0.0f, 0.0f, 0.0f)); // a moving boundary alone moves
    }

    nodes_.upload(tree.nodes);
    // The tree four wide for the wavefront's walk, unless its depth would overflow that walk's stack
    if (!tree.nodes.empty())
    {
        std::vector<bvh4_node> wide;
        if (collapse_bvh4(tree.nodes, wide) <= max_wide_depth)
        {
            wide_nodes_.upload(wide);
        }
    }
    spheres_.upload(spheres);
    sphere_motion_.upload(sphere_motion);
    sphere_frames_.upload(sphere_frames);
    textures_.upload(textures);
    images_.upload(images);
    texels_.upload(texels);
    noises_.upload(noises);
    media_.upload(media);
    boundary_quads_.upload(boundary_quads);
    quads_.upload(quads);
    triangles_.upload(triangles);
    prim_material_.upload(prim_material);
    prim_source_.upload(prim_source);
    materials_.upload(materials);
    lights_.upload(lights);
    lamps_.upload(lamps);
    lamp_of_.upload(lamp_of);

    view_.nodes = nodes_.data();
    view_.wide_nodes = wide_nodes_.data();
    view_.spheres = spheres_.data();
    view_.quads = quads_.data();
    view_.triangles = triangles_.data();
    view_.quad_base = S;
    view_.triangle_base = S + Q;
    view_.node_count = static_cast<int32_t>(tree.nodes.size());
    view_.prim_count = S + Q + T;
    view_.prim_material = prim_material_.data();
    view_.materials = materials_.data();
    view_.lights = lights_.data();
    view_.light_count = static_cast<int32_t>(lights.size());
    view_.lamp_count = quality_ ? static_cast<int32_t>(lamps.size()) : 0;
    view_.lamps = lamps_.data();
    view_.lamp_of = lamp_of_.data();
    const size_t light_set = lamps.size() + (env.sampled ? 1 : 0);
    view_.light_pmf = light_set == 0 ? 0.0f : static_cast<float>(1.0 / static_cast<double>(light_set));
    view_.combination = quality_ ? d.combination : RT_COMBINE_BSDF_ONLY;
    view_.has_environment = d.environment ? 1 : 0;
    view_.flat = T == 0 && S + Q <= RTB_FLAT_SCENE ? 1 : 0;
    view_.env = env;
    view_.textures = textures_.data();
    view_.images = images_.data();
    view_.texels = texels_.data();
    view_.noises = noises_.data();
    view_.sphere_motion = sphere_motion_.data();
    view_.sphere_frames = sphere_frames_.data();
    view_.media = media_.data();
    view_.boundary_quads = boundary_quads_.data();
    view_.has_motion = motion ? 1 : 0;
    view_.has_textures = std::any_of(materials.begin(), materials.end(),
                                     [](const material12& m) { return m.texture >= 0; })
                             ? 1
                             : 0;
    view_.medium_count = static_cast<int32_t>(media.size());
    view_.medium_base = S + Q + T;

    // The double tables of the books' integrator in FP64 (precision::float64 renders the books' scenes only: the
    // NEE/MIS integrator and triangle meshes compute in float, renderer.cu:2064-2078), in the float tables' leaf order
    has_f64_ = !quality_ && T == 0;
    if (has_f64_)
    {
        std::vector<sphere_d> spheres_d(spheres.size());
        std::vector<motion_d> motion_d_rows(sphere_motion.empty() ? 0 : spheres.size());
        std::vector<frame_d> frames_d(spheres.size());
        // How far a double sphere can stand out of the box the builder made around its float copy (center, motion and
        // radius each rounded to float): the walk widens every node bound by twice that, and by a hair more for the
        // slab test's own rounding
        double stand_out = 0;
        double largest = 1;
        for (size_t k = 0; k < spheres.size(); ++k)
        {
            const int32_t src = tree.order[kind_sphere][k];
            const rt_sphere_desc& s = d.spheres[src];
            spheres_d[k] = {s.center.x, s.center.y, s.center.z, s.radius};
            if (!motion_d_rows.empty())
            {
                motion_d_rows[k] = {s.displacement.x, s.displacement.y, s.displacement.z, 0.0};
            }
            const double cc = dot(s.center, s.center);
            frames_d[k] = {s.uv_cos, s.uv_sin, cc - s.radius * s.radius, 2 * s.radius * std::sqrt(cc)};
            const sphere4& f = source_spheres[static_cast<size_t>(src)];
            const float4& fm = source_motion[static_cast<size_t>(src)];
            const double center_gap = std::max({std::fabs(f.cx - s.center.x), std::fabs(f.cy - s.center.y),
                                                std::fabs(f.cz - s.center.z)});
            const double motion_gap = std::max({std::fabs(fm.x - s.displacement.x), std::fabs(fm.y - s.displacement.y),
                                                std::fabs(fm.z - s.displacement.z)});
            stand_out = std::max(stand_out, center_gap + motion_gap + std::fabs(std::fabs(f.r) - s.radius));
            largest = std::max({largest, std::sqrt(cc) + s.radius + std::sqrt(dot(s.displacement, s.displacement))});
        }
        std::vector<quad_d> quads_d(quads.size());
        for (size_t k = 0; k < quads.size(); ++k)
        {
            const rt_quad_desc& q = d.quads[tree.order[kind_quad][k]];
            quads_d[k] = make_quad_d(q);
            largest = std::max({largest, std::fabs(q.q.x) + std::fabs(q.u.x) + std::fabs(q.v.x),
                                std::fabs(q.q.y) + std::fabs(q.u.y) + std::fabs(q.v.y),
                                std::fabs(q.q.z) + std::fabs(q.u.z) + std::fabs(q.v.z)});
        }
        std::vector<material_d> materials_d(materials.size());
        for (size_t i = 0; i < materials.size(); ++i)
        {
            const rt_material_desc& m = d.materials[i];
            const bool textured = m.kind == RT_LAMBERTIAN || m.kind == RT_DIFFUSE_LIGHT || m.kind == RT_ISOTROPIC;
            const rt_vec3 color = textured ? d.textures[m.texture].rgb : m.albedo;
            material_d& v = materials_d[i];
            v.r = color.x;
            v.g = color.y;
            v.b = color.z;
            v.fuzz = std::min(m.fuzz, 1.0);
            v.ior = m.refraction_index;
            v.kind = m.kind;
            v.texture = materials[i].texture;
            v.texture_needs = materials[i].texture_needs;
        }
        std::vector<texture_d> textures_d;
        std::vector<noise_d> noises_d;
        for (int64_t i = 0; i < d.texture_count; ++i)
        {
            const rt_texture_desc& t = d.textures[i];
            texture_d v{};
            v.kind = t.kind;
            v.even = t.even;
            v.odd = t.odd;
            v.table = textures[static_cast<size_t>(i)].table;
            v.r = t.rgb.x;
            v.g = t.rgb.y;
            v.b = t.rgb.z;
            v.inv_scale = t.inv_scale;
            if (t.kind == RT_TEXTURE_NOISE)
            {
                noise_d n{};
                const rt_perlin_desc& p = d.perlins[t.perlin];
                for (int k = 0; k < 256; ++k)
                {
                    n.gradients[k] = {p.random_vectors[k].x, p.random_vectors[k].y, p.random_vectors[k].z, 0.0};
                    n.perm_x[k] = static_cast<uint8_t>(p.perm_x[k]);
                    n.perm_y[k] = static_cast<uint8_t>(p.perm_y[k]);
                    n.perm_z[k] = static_cast<uint8_t>(p.perm_z[k]);
                }
                n.scale = t.scale;
                noises_d.push_back(n);
            }
            textures_d.push_back(v);
        }
        std::vector<light_d> lights_d(lights.size());
        double cdf = 0;
        for (size_t i = 0; i < lights.size(); ++i)
        {
            const rt_light_desc& l = d.lights[i];
            light_d& v = lights_d[i];
            cdf += l.weight;
            v.kind = l.kind;
            v.twin = lights[i].twin;
            v.weight = l.weight;
            v.cdf = cdf;
            if (l.kind == RT_LIGHT_QUAD)
            {
                v.quad = make_quad_d(l.quad);
                const rt_vec3 n = cross(l.quad.u, l.quad.v);
                v.area = std::sqrt(dot(n, n));
                v.u[0] = l.quad.u.x;
                v.u[1] = l.quad.u.y;
                v.u[2] = l.quad.u.z;
                v.v[0] = l.quad.v.x;
                v.v[1] = l.quad.v.y;
                v.v[2] = l.quad.v.z;
            }
            else
            {
                v.c[0] = l.center.x;
                v.c[1] = l.center.y;
                v.c[2] = l.center.z;
                v.radius = l.radius;
            }
        }
        std::vector<medium_d> media_d(media.size());
        std::vector<quad_d> boundary_d;
        for (size_t i = 0; i < media.size(); ++i)
        {
            const rt_medium_desc& m = d.media[i];
            medium_d& v = media_d[i];
            v.neg_inv_density = m.neg_inv_density;
            v.material = m.material;
            v.first_quad = static_cast<int32_t>(boundary_d.size());
            v.quad_count = media[i].quad_count;
            for (int a = 0; a < 3; ++a)
            {
                v.lo[a] = std::numeric_limits<double>::infinity();
                v.hi[a] = -std::numeric_limits<double>::infinity();
            }
            if (m.boundary == RT_BOUNDARY_SPHERE)
            {
                const rt_sphere_desc& s = m.sphere;
                const double c[3] = {s.center.x, s.center.y, s.center.z};
                const double dm[3] = {s.displacement.x, s.displacement.y, s.displacement.z};
                for (int a = 0; a < 3; ++a)
                {
                    v.c[a] = c[a];
                    v.dm[a] = dm[a];
                    v.lo[a] = std::min(c[a], c[a] + dm[a]) - s.radius;
                    v.hi[a] = std::max(c[a], c[a] + dm[a]) + s.radius;
                }
                v.radius = s.radius;
            }
            else
            {
                for (int64_t k = 0; k < m.quad_count; ++k)
                {
                    boundary_d.push_back(make_quad_d(m.quads[k]));
                    const build_prim b = quad_prim(m.quads[k], 0);
                    for (int a = 0; a < 3; ++a)
                    {
                        v.lo[a] = std::min(v.lo[a], b.lo[a]);
                        v.hi[a] = std::max(v.hi[a], b.hi[a]);
                    }
                }
            }
        }
        if (motion && motion_d_rows.empty())
        {
            motion_d_rows.assign(spheres.size(), d4{0.0, 0.0, 0.0, 0.0}); // a moving boundary alone moves
        }
        spheres_d_.upload(spheres_d);
        sphere_motion_d_.upload(motion_d_rows);
        sphere_frames_d_.upload(frames_d);
        quads_d_.upload(quads_d);
        materials_d_.upload(materials_d);
        lights_d_.upload(lights_d);
        textures_d_.upload(textures_d);
        noises_d_.upload(noises_d);
        media_d_.upload(media_d);
        boundary_quads_d_.upload(boundary_d);

        view_f64_.nodes = nodes_.data();
        view_f64_.spheres = spheres_d_.data();
        view_f64_.quads = quads_d_.data();
        view_f64_.prim_material = prim_material_.data();
        view_f64_.materials = materials_d_.data();
        view_f64_.lights = lights_d_.data();
        view_f64_.textures = textures_d_.data();
        view_f64_.images = images_.data();
        view_f64_.texels = texels_.data();
        view_f64_.noises = noises_d_.data();
        view_f64_.sphere_motion = sphere_motion_d_.data();
        view_f64_.sphere_frames = sphere_frames_d_.data();
        view_f64_.media = media_d_.data();
        view_f64_.boundary_quads = boundary_quads_d_.data();
        view_f64_.box_margin = 2 * stand_out + 1e-12 * largest;
        view_f64_.node_count = view_.node_count;
        view_f64_.flat = view_.flat;
        view_f64_.quad_base = S;
        view_f64_.prim_count = S + Q;
        view_f64_.light_count = static_cast<int32_t>(lights.size());
        view_f64_.has_motion = view_.has_motion;
        view_f64_.medium_count = view_.medium_count;
        view_f64_.medium_base = S + Q;
        view_f64_.has_textures = view_.has_textures;
    }

    stats_.spheres = S;
    stats_.quads = Q;
    stats_.triangles = T;
    stats_.nodes = static_cast<int64_t>(tree.nodes.size());
    stats_.leaves = tree.leaves;
    stats_.lamps = static_cast<int64_t>(lamps.size());
    stats_.lights = static_cast<int64_t>(lights.size());
    stats_.device_bytes = static_cast<int64_t>(nodes_.bytes() + spheres_.bytes() + quads_.bytes() + triangles_.bytes() +
                                               prim_material_.bytes() + prim_source_.bytes() + materials_.bytes() +
                                               lights_.bytes() + lamps_.bytes() + lamp_of_.bytes() +
                                               env_texels_.bytes() + env_bins_.bytes() + env_row_cos_.bytes() +
                                               sphere_motion_.bytes() + sphere_frames_.bytes() + textures_.bytes() +
                                               images_.bytes() + texels_.bytes() + noises_.bytes() + media_.bytes() +
                                               boundary_quads_.bytes() + spheres_d_.bytes() +
                                               sphere_motion_d_.bytes() + sphere_frames_d_.bytes() + quads_d_.bytes() +
                                               materials_d_.bytes() + lights_d_.bytes() + textures_d_.bytes() +
                                               noises_d_.bytes() + media_d_.bytes() + boundary_quads_d_.bytes());
    stats_.depth = tree.depth;
    stats_.max_leaf_size = options.max_leaf_size;
    stats_.flat = view_.flat;
}
} // namespace rtb
