// The books' integrator in double: the reference's precision::float64 (renderer.h:402-409), its all_books_kernel<double>
// and first_book_kernel<double> (renderer.cu:417-451), a mode "there to compare with" rather than a fast path.
//
// It renders what the reference renders in float64: the three books' scenes (spheres, moving spheres, quads, smoke,
// the solid, checker, image and marble textures) under the books' four strategies (camera.cuh:304-437, lights.cuh);
// the NEE/MIS integrator and triangle meshes compute in float only, there as here. Every number of a path is a
// double: rays, hits, normals, throughput, the random numbers (53-bit uniforms, as random_real<double> draws).
//
// The B200 form is the float kernel's: a persistent kernel whose lanes claim (pixel, chunk of 16 passes) work items by
// a warp ballot and one atomic a warp, regenerate paths as they end, and write each item's sum to its slot of the
// chunk partials, which the float path's reduction adds into the FP64 sums in chunk order. So the grouping of passes
// into launches does not change the image, as in float. The tree is the float tables' (its boxes rounded outward in
// float); a double primitive can stand out of its float box by the rounding of its float copy, so every node bound is
// widened by the scene's box_margin before the slab test, which keeps the walk conservative.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"
#include "philox.cuh"
#include "rt_b200.h"

namespace rtb
{
namespace
{
using v3 = double3;

__device__ __forceinline__ v3 operator+(v3 a, v3 b) { return make_double3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ v3 operator-(v3 a, v3 b) { return make_double3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ v3 operator-(v3 a) { return make_double3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ v3 operator*(double t, v3 v) { return make_double3(t * v.x, t * v.y, t * v.z); }
__device__ __forceinline__ v3 operator*(v3 a, v3 b) { return make_double3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double length_squared(v3 v) { return dot(v, v); }
__device__ __forceinline__ v3 unit_vector(v3 v) { return (1.0 / sqrt(length_squared(v))) * v; }
__device__ __forceinline__ v3 reflect(v3 v, v3 n) { return v - (2.0 * dot(v, n)) * n; }
__device__ __forceinline__ v3 refract(v3 uv, v3 n, double etai_over_etat) // vec3.cuh refract
{
    const double cos_theta = fmin(dot(-uv, n), 1.0);
    const v3 r_out_perp = etai_over_etat * (uv + cos_theta * n);
    const v3 r_out_parallel = -sqrt(fabs(1.0 - length_squared(r_out_perp))) * n;
    return r_out_perp + r_out_parallel;
}
__device__ __forceinline__ v3 vec(const double* p) { return make_double3(p[0], p[1], p[2]); }

constexpr double pi_d = 3.14159265358979323846;
constexpr double uniform_sphere_density = 1.0 / (4.0 * pi_d);
constexpr double infinity_d = __builtin_huge_val();
constexpr double t_min = 0.001;

// ---- random numbers: Philox4x32-10 on the float kernel's counter, 53 bits a uniform ----------------------------------
// 53 random bits as a double in [0, 1 - 2^-53], every value k / 2^53 exactly, as random_real<double> (random.cuh:79-93)
__device__ __forceinline__ double to_unit53(uint32_t hi, uint32_t lo)
{
    return static_cast<double>((static_cast<uint64_t>(hi >> 11) << 32) | lo) * 0x1p-53;
}

struct uniforms
{
    double x, y, z, w;
};

struct sampler
{
    uint2 key;
    uint32_t pixel;
    uint32_t pass;

    // Four uniforms for dimension block `block` of the vertex at depth `depth`: two Philox blocks, the counter of the
    // float kernel's draw and the same with the job word's top bit set (a plain render's job word is 0)
    __device__ __forceinline__ uniforms draw(int depth, int block) const
    {
        const uint32_t c = (static_cast<uint32_t>(depth) << 4) | static_cast<uint32_t>(block);
        const uint4 a = philox4x32_10(make_uint4(pixel, pass, c, 0u), key);
        const uint4 b = philox4x32_10(make_uint4(pixel, pass, c, 0x80000000u), key);
        return {to_unit53(a.x, a.y), to_unit53(a.z, a.w), to_unit53(b.x, b.y), to_unit53(b.z, b.w)};
    }
};

// The float kernel's dimension blocks: 0 the material's sample (at depth 0 the camera ray's), 1 the ray's time,
// 4-15 the free flights through the volumes of smoke, four volumes a block
constexpr int block_material = 0;
constexpr int block_time = 1;
constexpr int block_media = 4;

// ---- directions (random.cuh:95-140, material.cuh:55-64, pdf.cuh:21-26) -------------------------------------------
__device__ __forceinline__ v3 random_unit_vector(double u, double v)
{
    double s, c;
    sincospi(2.0 * v, &s, &c);
    const double r = 2.0 * sqrt(u * (1.0 - u));
    return make_double3(r * c, r * s, 1.0 - 2.0 * u);
}

__device__ __forceinline__ v3 random_cosine_direction(double r1, double r2)
{
    double s, c;
    sincospi(2.0 * r1, &s, &c);
    const double sin_theta = sqrt(r2);
    return make_double3(c * sin_theta, s * sin_theta, sqrt(1.0 - r2));
}

// v in a basis whose z axis is the unit vector n (Duff et al., "Building an Orthonormal Basis, Revisited", JCGT 2017)
__device__ __forceinline__ v3 around(v3 n, v3 v)
{
    const double sign = copysign(1.0, n.z);
    const double a = -1.0 / (sign + n.z);
    const double b = n.x * n.y * a;
    const v3 x_axis = make_double3(1.0 + sign * n.x * n.x * a, sign * b, -sign * n.x);
    const v3 y_axis = make_double3(b, sign + n.y * n.y * a, -n.y);
    return v.x * x_axis + v.y * y_axis + v.z * n;
}

__device__ __forceinline__ double cosine_density(v3 unit_normal, v3 direction)
{
    const double cosine = dot(unit_normal, direction) / sqrt(length_squared(direction));
    return cosine > 0.0 ? cosine / pi_d : 0.0;
}

// Schlick's reflectance (material.cuh:67-76)
__device__ __forceinline__ double reflectance(double cosine, double ri)
{
    double r0 = (1.0 - ri) / (1.0 + ri);
    r0 = r0 * r0;
    const double x = 1.0 - cosine;
    const double x2 = x * x;
    return r0 + (1.0 - r0) * (x2 * x2 * x);
}

// ---- primitive tests -----------------------------------------------------------------------------------------------
// 1 / x, never infinite (bvh.cuh:475-488): |x| below 2^-80 moves out to +-2^-80
__device__ __forceinline__ double safe_inverse(double x)
{
    const double tiny = 0x1p-80;
    return 1.0 / (fabs(x) > tiny ? x : copysign(tiny, x));
}

// The line's two roots with a sphere in the l-vector form (sphere.cuh:70-97): (h/a) -+ sqrt(r^2 - |l|^2)/sqrt(a), the
// three squares taken from r^2 by fused multiply-adds
__device__ __forceinline__ bool sphere_roots(const sphere_d& s, v3 o, v3 d, double inverse_a, double& near,
                                             double& far)
{
    const v3 oc = make_double3(s.x - o.x, s.y - o.y, s.z - o.z);
    const double h_over_a = dot(d, oc) * inverse_a;
    const v3 l = oc - h_over_a * d;
    const double disc = fma(-l.x, l.x, fma(-l.y, l.y, fma(-l.z, l.z, s.w * s.w)));
    if (disc < 0.0)
    {
        return false;
    }
    const double half_chord = sqrt(disc * inverse_a);
    near = h_over_a - half_chord;
    far = h_over_a + half_chord;
    return true;
}

// hit_sphere (sphere.cuh:99-117): the nearest root in (t_min, t_max); far_only for the sphere the ray leaves inward
__device__ __forceinline__ bool hit_sphere(const sphere_d& s, v3 o, v3 d, double inverse_a, double lo, double hi,
                                           bool far_only, double& t, bool& entering)
{
    double near, far;
    if (!sphere_roots(s, o, d, inverse_a, near, far))
    {
        return false;
    }
    t = near;
    entering = !far_only && t > lo;
    if (!entering)
    {
        t = far;
    }
    return lo < t && t < hi;
}

struct quad_v
{
    v3 q, n, a, b;
};

__device__ __forceinline__ quad_v load_quad(const quad_d& r)
{
    return {vec(r.q), vec(r.n), vec(r.a), vec(r.b)};
}

// hit_quad (quad.cuh:60-84): t in [lo, hi], alpha and beta in [0, 1], closed; NaNs fail every comparison
__device__ __forceinline__ bool hit_quad(const quad_v& s, v3 o, v3 d, double lo, double hi, double& t, bool& front)
{
    const double denominator = dot(s.n, d);
    if (!(fabs(denominator) >= 1e-8))
    {
        return false;
    }
    const v3 origin_to_q = s.q - o;
    t = dot(s.n, origin_to_q) / denominator;
    if (!(lo <= t && t <= hi))
    {
        return false;
    }
    const v3 p = t * d - origin_to_q;
    const double alpha = dot(p, s.a);
    const double beta = dot(p, s.b);
    if (!(0.0 <= alpha && alpha <= 1.0 && 0.0 <= beta && beta <= 1.0))
    {
        return false;
    }
    front = denominator < 0.0;
    return true;
}

struct hit_info
{
    int id; // global id, -1 for none
    double t;
    bool front;
};

// Sphere i (leaf order) where it is at the ray's time
__device__ __forceinline__ sphere_d sphere_at(const scene_view_f64& S, int i, double time)
{
    sphere_d s = S.spheres[i];
    if (S.has_motion)
    {
        const motion_d m = S.sphere_motion[i];
        s.x = fma(time, m.x, s.x);
        s.y = fma(time, m.y, s.y);
        s.z = fma(time, m.z, s.z);
    }
    return s;
}

// The leaf's primitives against the ray (spheres or quads: a float64 scene has no triangles), shrinking hit.t
__device__ __forceinline__ void test_leaf(const scene_view_f64& S, int link, v3 o, v3 d, double time,
                                          double inverse_a, int from, bool inward, hit_info& hit)
{
    const int kind = leaf_kind(link);
    const int count = leaf_count(link);
    const int start = leaf_start(link);
    if (kind == kind_sphere)
    {
        for (int i = start; i < start + count; ++i)
        {
            const bool own = i == from;
            if (own && !inward)
            {
                continue;
            }
            double t;
            bool entering;
            if (hit_sphere(sphere_at(S, i, time), o, d, inverse_a, t_min, hit.t, own, t, entering))
            {
                hit = {i, t, entering};
            }
        }
    }
    else
    {
        for (int i = start; i < start + count; ++i)
        {
            const int id = S.quad_base + i;
            if (id == from)
            {
                continue;
            }
            double t;
            bool front;
            if (hit_quad(load_quad(S.quads[i]), o, d, t_min, hit.t, t, front))
            {
                hit = {id, t, front};
            }
        }
    }
}

// The entry distance of the ray into a float box widened by `margin`, or +infinity if it misses it before `limit`
__device__ __forceinline__ double box_entry(float lo_x, float hi_x, float lo_y, float hi_y, float lo_z, float hi_z,
                                            double margin, v3 o, v3 inv, double limit)
{
    const double a0 = (static_cast<double>(lo_x) - margin - o.x) * inv.x;
    const double a1 = (static_cast<double>(hi_x) + margin - o.x) * inv.x;
    const double b0 = (static_cast<double>(lo_y) - margin - o.y) * inv.y;
    const double b1 = (static_cast<double>(hi_y) + margin - o.y) * inv.y;
    const double c0 = (static_cast<double>(lo_z) - margin - o.z) * inv.z;
    const double c1 = (static_cast<double>(hi_z) + margin - o.z) * inv.z;
    const double enter = fmax(fmax(fmin(a0, a1), fmin(b0, b1)), fmax(fmin(c0, c1), t_min));
    const double exit = fmin(fmin(fmax(a0, a1), fmax(b0, b1)), fmin(fmax(c0, c1), limit));
    return enter <= exit ? enter : infinity_d;
}

// The closest hit in (t_min, +inf) with the self-intersection rules of the primitive the ray leaves (bvh.cuh:539-575,
// 576-706): every primitive in turn for a flat scene, else a walk of the tree, nearer child first, with a stack of
// (node, entry distance) in local memory
__device__ hit_info closest_hit(const scene_view_f64& S, v3 o, v3 d, double time, int from, bool inward)
{
    hit_info hit{-1, infinity_d, false};
    if (S.node_count == 0)
    {
        return hit;
    }
    const double inverse_a = 1.0 / length_squared(d);
    if (S.flat)
    {
        for (int i = 0; i < S.quad_base; ++i)
        {
            const bool own = i == from;
            if (own && !inward)
            {
                continue;
            }
            double t;
            bool entering;
            if (hit_sphere(sphere_at(S, i, time), o, d, inverse_a, t_min, hit.t, own, t, entering))
            {
                hit = {i, t, entering};
            }
        }
        for (int i = 0; i < S.prim_count - S.quad_base; ++i)
        {
            const int id = S.quad_base + i;
            if (id == from)
            {
                continue;
            }
            double t;
            bool front;
            if (hit_quad(load_quad(S.quads[i]), o, d, t_min, hit.t, t, front))
            {
                hit = {id, t, front};
            }
        }
        return hit;
    }
    const v3 inv = make_double3(safe_inverse(d.x), safe_inverse(d.y), safe_inverse(d.z));
    const double m = S.box_margin;
    int links[max_bvh_depth];
    double entries[max_bvh_depth];
    int sp = 0;
    int link = 0;
    while (true)
    {
        if (link >= 0)
        {
            const bvh_node& n = S.nodes[link];
            const double e0 = box_entry(n.x[0], n.x[1], n.y[0], n.y[1], n.z[0], n.z[1], m, o, inv, hit.t);
            const double e1 = box_entry(n.x[2], n.x[3], n.y[2], n.y[3], n.z[2], n.z[3], m, o, inv, hit.t);
            const bool h0 = e0 != infinity_d;
            const bool h1 = e1 != infinity_d;
            if (h0 && h1)
            {
                const bool second_first = e1 < e0;
                link = second_first ? n.link[1] : n.link[0];
                links[sp] = second_first ? n.link[0] : n.link[1];
                entries[sp] = second_first ? e0 : e1;
                ++sp;
                continue;
            }
            if (h0 || h1)
            {
                link = h0 ? n.link[0] : n.link[1];
                continue;
            }
        }
        else
        {
            test_leaf(S, link, o, d, time, inverse_a, from, inward, hit);
        }
        // The next stack entry the ray enters before the closest hit so far
        link = traversal_done_link;
        while (sp > 0)
        {
            --sp;
            if (entries[sp] < hit.t)
            {
                link = links[sp];
                break;
            }
        }
        if (link == traversal_done_link)
        {
            return hit;
        }
    }
}

// ---- volumes of smoke (constant_medium.cuh:29-120, camera.cuh:259-284) -----------------------------------------------
// Where the ray's line crosses the medium's boundary: the sphere's roots where it is at the ray's time, kept if the
// chord is longer than 0.0001; or the nearest and the farthest plane of the boundary quads the line meets inside them
__device__ bool boundary_crossings(const scene_view_f64& S, const medium_d& m, v3 o, v3 d, double time,
                                   double inverse_a, double& t_in, double& t_out)
{
    if (m.quad_count == 0)
    {
        const sphere_d s{fma(time, m.dm[0], m.c[0]), fma(time, m.dm[1], m.c[1]), fma(time, m.dm[2], m.c[2]), m.radius};
        return sphere_roots(s, o, d, inverse_a, t_in, t_out) && t_out - t_in > 0.0001;
    }
    t_in = infinity_d;
    t_out = -infinity_d;
    for (int i = m.first_quad; i < m.first_quad + m.quad_count; ++i)
    {
        double t;
        bool front;
        if (hit_quad(load_quad(S.boundary_quads[i]), o, d, -infinity_d, infinity_d, t, front))
        {
            t_in = fmin(t_in, t);
            t_out = fmax(t_out, t);
        }
    }
    return t_out - t_in >= 0.0001;
}

// The stretch [t_in, t_out] of (t_min, t_max) inside the medium: its box first, then the boundary's crossings
__device__ bool medium_stretch(const scene_view_f64& S, const medium_d& m, v3 o, v3 d, double time, double inverse_a,
                               v3 inv, double t_max, double& t_in, double& t_out)
{
    const double a0 = (m.lo[0] - o.x) * inv.x, a1 = (m.hi[0] - o.x) * inv.x;
    const double b0 = (m.lo[1] - o.y) * inv.y, b1 = (m.hi[1] - o.y) * inv.y;
    const double c0 = (m.lo[2] - o.z) * inv.z, c1 = (m.hi[2] - o.z) * inv.z;
    const double enter = fmax(fmax(fmin(a0, a1), fmin(b0, b1)), fmax(fmin(c0, c1), t_min));
    const double exit = fmin(fmin(fmax(a0, a1), fmax(b0, b1)), fmin(fmax(c0, c1), t_max));
    if (!(enter <= exit))
    {
        return false;
    }
    double line_in, line_out;
    if (!boundary_crossings(S, m, o, d, time, inverse_a, line_in, line_out))
    {
        return false;
    }
    t_in = fmax(line_in, t_min);
    t_out = fmin(line_out, t_max);
    if (!(t_in < t_out))
    {
        return false;
    }
    t_in = fmax(t_in, 0.0);
    return true;
}

// A particle of smoke in front of the closest surface (closest_event, camera.cuh:259-284): each volume in turn against
// the closest event so far, a free flight of -log(u) / density from where the ray enters it
__device__ void media_event(const scene_view_f64& S, v3 o, v3 d, double time, const sampler& rng, int depth,
                            hit_info& hit)
{
    const double inverse_a = 1.0 / length_squared(d);
    const v3 inv = make_double3(safe_inverse(d.x), safe_inverse(d.y), safe_inverse(d.z));
    const double length = sqrt(length_squared(d));
    uniforms u{};
    for (int k = 0; k < S.medium_count; ++k)
    {
        if ((k & 3) == 0)
        {
            u = rng.draw(depth, block_media + (k >> 2));
        }
        const medium_d& m = S.media[k];
        double t_in, t_out;
        if (!medium_stretch(S, m, o, d, time, inverse_a, inv, hit.t, t_in, t_out))
        {
            continue;
        }
        const double uk = (k & 3) == 0 ? u.x : (k & 3) == 1 ? u.y : (k & 3) == 2 ? u.z : u.w;
        const double distance = m.neg_inv_density * log(uk);
        if (distance > (t_out - t_in) * length)
        {
            continue;
        }
        hit = {S.medium_base + k, t_in + distance / length, true};
    }
}

// ---- textures (texture.cuh, perlin.cuh) ---------------------------------------------------------------------------
// Perlin noise (perlin.ixx noise): Hermite-smoothed cell coordinates, the trilinear sum of the corners' gradient dot
// products; turbulence: 7 octaves, each at twice the frequency and half the weight, absolute value
__device__ double perlin_noise(const noise_d& n, v3 p)
{
    const double fx = floor(p.x), fy = floor(p.y), fz = floor(p.z);
    const int i = static_cast<int>(fx), j = static_cast<int>(fy), k = static_cast<int>(fz);
    const double u = p.x - fx, v = p.y - fy, w = p.z - fz;
    const double uu = u * u * (3.0 - 2.0 * u);
    const double vv = v * v * (3.0 - 2.0 * v);
    const double ww = w * w * (3.0 - 2.0 * w);
    double accum = 0.0;
    for (int di = 0; di < 2; ++di)
    {
        const int px = n.perm_x[(i + di) & 255];
        const double wx = di == 0 ? 1.0 - uu : uu;
        for (int dj = 0; dj < 2; ++dj)
        {
            const int py = n.perm_y[(j + dj) & 255];
            const double wy = dj == 0 ? 1.0 - vv : vv;
            for (int dk = 0; dk < 2; ++dk)
            {
                const int pz = n.perm_z[(k + dk) & 255];
                const double wz = dk == 0 ? 1.0 - ww : ww;
                const d4& g = n.gradients[px ^ py ^ pz];
                const double dot_g = g.x * (u - di) + g.y * (v - dj) + g.z * (w - dk);
                accum += wx * wy * wz * dot_g;
            }
        }
    }
    return accum;
}

__device__ double turbulence(const noise_d& n, v3 p)
{
    double accum = 0.0;
    double weight = 1.0;
    for (int layer = 0; layer < 7; ++layer)
    {
        accum += weight * perlin_noise(n, p);
        weight *= 0.5;
        p = 2.0 * p;
    }
    return fabs(accum);
}

// The texture's color at the hit (texture_value, texture.cuh:60-110): a checker walked down to its point's cube, an
// image read at (u, v) clamped with v flipped, a marble 0.5 (1 + sin(scale z + 10 turbulence(p)))
__device__ v3 texture_value(const scene_view_f64& S, int index, double u, double v, v3 p)
{
    texture_d t = S.textures[index];
    while (t.kind == RT_TEXTURE_CHECKER)
    {
        const int x = static_cast<int>(floor(t.inv_scale * p.x));
        const int y = static_cast<int>(floor(t.inv_scale * p.y));
        const int z = static_cast<int>(floor(t.inv_scale * p.z));
        t = S.textures[(x + y + z) % 2 == 0 ? t.even : t.odd];
    }
    if (t.kind == RT_TEXTURE_IMAGE)
    {
        const image_info im = S.images[t.table];
        const double cu = fmin(fmax(u, 0.0), 1.0);
        const double fv = 1.0 - fmin(fmax(v, 0.0), 1.0);
        const int column = static_cast<int>(cu * im.width);
        const int row = static_cast<int>(fv * im.height);
        const int i = column < im.width - 1 ? column : im.width - 1;
        const int j = row < im.height - 1 ? row : im.height - 1;
        const float4 c = S.texels[im.offset + j * im.width + i];
        return make_double3(c.x, c.y, c.z);
    }
    if (t.kind == RT_TEXTURE_NOISE)
    {
        const noise_d& n = S.noises[t.table];
        const double gray = 0.5 * (1.0 + sin(n.scale * p.z + 10.0 * turbulence(n, p)));
        return make_double3(gray, gray, gray);
    }
    return make_double3(t.r, t.g, t.b);
}

// ---- the books' lights list (lights.cuh:49-227) --------------------------------------------------------------------
__device__ __forceinline__ double one_minus_cos_theta_max(double radius, double distance_squared)
{
    const double sin_squared = radius * radius / distance_squared;
    return sin_squared / (1.0 + sqrt(1.0 - sin_squared));
}

__device__ double lights_pdf_value(const scene_view_f64& S, v3 origin, v3 direction, int from)
{
    double sum = 0.0;
    for (int k = 0; k < S.light_count; ++k)
    {
        const light_d& l = S.lights[k];
        const bool own = from >= 0 && l.twin == from;
        if (l.kind == RT_LIGHT_QUAD)
        {
            if (own)
            {
                continue; // a ray never hits the quad it leaves (the twin rule, lights.cuh:175-187)
            }
            double t;
            bool front;
            if (!hit_quad(load_quad(l.quad), origin, direction, t_min, infinity_d, t, front))
            {
                continue;
            }
            const double len2 = length_squared(direction);
            const double distance_squared = t * t * len2;
            const double cosine = fabs(dot(direction, vec(l.quad.n))) / sqrt(len2);
            sum += l.weight * (distance_squared / (cosine * l.area));
        }
        else
        {
            const v3 c = vec(l.c);
            const v3 to_center = c - origin;
            const double distance_squared = length_squared(to_center);
            if (distance_squared < l.radius * l.radius)
            {
                sum += l.weight * uniform_sphere_density;
                continue;
            }
            if (own && !(dot(direction, to_center) > 0.0))
            {
                continue;
            }
            double t;
            bool entering;
            if (!hit_sphere(sphere_d{c.x, c.y, c.z, l.radius}, origin, direction, 1.0 / length_squared(direction),
                            t_min, infinity_d, own, t, entering))
            {
                continue;
            }
            sum += l.weight * (1.0 / (2.0 * pi_d * one_minus_cos_theta_max(l.radius, distance_squared)));
        }
    }
    return sum;
}

// lights_random: the running sums pick a light with `pick`; (a, b) draw its point or direction
__device__ v3 lights_random(const scene_view_f64& S, v3 origin, double pick, double a, double b)
{
    int k = 0;
    while (k < S.light_count - 1 && !(pick < S.lights[k].cdf))
    {
        ++k;
    }
    const light_d& l = S.lights[k];
    if (l.kind == RT_LIGHT_QUAD)
    {
        return unit_vector((vec(l.quad.q) - origin) + a * vec(l.u) + b * vec(l.v));
    }
    const v3 to_center = vec(l.c) - origin;
    const double distance_squared = length_squared(to_center);
    if (distance_squared < l.radius * l.radius)
    {
        return random_unit_vector(a, b);
    }
    const double one_minus_cos_max = one_minus_cos_theta_max(l.radius, distance_squared);
    double s, c;
    sincospi(2.0 * a, &s, &c);
    const double one_minus_z = b * one_minus_cos_max;
    const double sin_theta = sqrt(one_minus_z * (2.0 - one_minus_z));
    return around((1.0 / sqrt(distance_squared)) * to_center,
                  make_double3(c * sin_theta, s * sin_theta, 1.0 - one_minus_z));
}

// ---- the camera (camera.cuh:53-107) ---------------------------------------------------------------------------------
__device__ __forceinline__ void camera_ray(const camera_d& cam, int i, int j, int s_i, int s_j, const uniforms& u,
                                           v3& origin, v3& direction)
{
    const double dx = (s_i + u.x) * cam.recip_sqrt_spp - 0.5;
    const double dy = (s_j + u.y) * cam.recip_sqrt_spp - 0.5;
    const v3 to_sample = vec(cam.to_pixel00) + (i + dx) * vec(cam.delta_u) + (j + dy) * vec(cam.delta_v);
    origin = vec(cam.center);
    direction = to_sample;
    if (cam.defocus)
    {
        const double r = sqrt(u.z);
        double s, c;
        sincospi(2.0 * u.w, &s, &c);
        const v3 lens = (r * c) * vec(cam.disk_u) + (r * s) * vec(cam.disk_v);
        origin = origin + lens;
        direction = to_sample - lens;
    }
}

__device__ __forceinline__ v3 sky(const camera_d& cam, v3 direction)
{
    const double a = 0.5 * (unit_vector(direction).y + 1.0);
    return (1.0 - a) * vec(cam.sky_bottom) + a * vec(cam.sky_top);
}

__device__ __forceinline__ double without_nan(double x) { return x == x ? x : 0.0; }

struct path_state
{
    v3 o, d;
    v3 throughput;
    int rays_left;
    int depth;
    int from;
    bool inward;
    double time;
};

struct surface
{
    v3 p;
    v3 outward;
    v3 normal;
    v3 color;
    int material;
    int from;
};

// A sphere point's texture coordinates (sphere.cuh:119-135): its outward normal turned back by the instances' turn,
// u from -x around y, v from the south pole
__device__ __forceinline__ void sphere_uv(v3 outward, const frame_d& f, double& u, double& v)
{
    const double nx = f.x * outward.x - f.y * outward.z;
    const double nz = f.y * outward.x + f.x * outward.z;
    const double phi = atan2(-nz, nx) + pi_d;
    const double theta = acos(fmin(fmax(-outward.y, -1.0), 1.0));
    u = phi / (2.0 * pi_d);
    v = theta / pi_d;
}

// The hit point moved onto the sphere by one Newton step, for a checker (onto_sphere, sphere.cuh:137-168): f = |p|^2
// - 2 p.c + k with k = |c|^2 - r^2 from the host, taken while its rounding bound stays below the frame's limit
__device__ __forceinline__ v3 onto_sphere(v3 p, v3 outward, const sphere_d& ball, const frame_d& f)
{
    const v3 c = make_double3(ball.x, ball.y, ball.z);
    const double p_p = dot(p, p);
    const double p_c = dot(p, c);
    if (!(p_p + 2.0 * fabs(p_c) + fabs(f.z) < f.w))
    {
        return p;
    }
    const double value = p_p - 2.0 * p_c + f.z;
    return p - (value / (2.0 * ball.w)) * outward;
}

// The hit as the shading needs it (surface_at, camera.cuh:171-253) and the material there with its color
__device__ surface surface_at(const scene_view_f64& S, const path_state& ps, const hit_info& h, material_d& m)
{
    surface s;
    s.from = h.id;
    double u = 0.0, v = 0.0;
    sphere_d ball{};
    bool on_sphere = false;
    if (h.id >= S.medium_base)
    {
        // A particle of smoke: any normal will do, the CPU's (1, 0, 0) and the front; no surface to leave
        s.p = ps.o + h.t * ps.d;
        s.outward = make_double3(1.0, 0.0, 0.0);
        s.normal = s.outward;
        s.material = S.media[h.id - S.medium_base].material;
        s.from = -1;
        m = S.materials[s.material];
    }
    else
    {
        s.material = S.prim_material[h.id];
        m = S.materials[s.material];
        if (h.id < S.quad_base)
        {
            ball = sphere_at(S, h.id, ps.time);
            on_sphere = true;
            s.p = ps.o + h.t * ps.d;
            s.outward = (1.0 / ball.w) * (s.p - make_double3(ball.x, ball.y, ball.z));
        }
        else
        {
            // The quad's point as the CPU computes it, t * d rounded, then the sum (camera.cuh:175-195 at_unfused)
            const quad_v q = load_quad(S.quads[h.id - S.quad_base]);
            s.p = make_double3(__dadd_rn(ps.o.x, __dmul_rn(h.t, ps.d.x)), __dadd_rn(ps.o.y, __dmul_rn(h.t, ps.d.y)),
                               __dadd_rn(ps.o.z, __dmul_rn(h.t, ps.d.z)));
            s.outward = q.n;
            if (m.texture >= 0 && (m.texture_needs & texture_needs_uv) != 0)
            {
                const v3 rel = h.t * ps.d - (q.q - ps.o);
                u = dot(rel, q.a);
                v = dot(rel, q.b);
            }
        }
        s.normal = h.front ? s.outward : -s.outward;
    }
    s.color = make_double3(m.r, m.g, m.b);
    if (m.texture >= 0)
    {
        v3 point = s.p;
        if (on_sphere && (m.texture_needs & (texture_needs_uv | texture_needs_point)) != 0)
        {
            const frame_d f = S.sphere_frames[h.id];
            if (m.texture_needs & texture_needs_uv)
            {
                sphere_uv(s.outward, f, u, v);
            }
            if (m.texture_needs & texture_needs_point)
            {
                point = onto_sphere(s.p, s.outward, ball, f);
            }
        }
        s.color = texture_value(S, m.texture, u, v, point);
    }
    return s;
}

// One segment of a books' path after its closest event (camera.cuh:364-437 trace_ray, diffuse_bounce 304-359,
// material.cuh:84-126 scatter): true when the sample is done, its value in `sample`
__device__ bool shade_books(const scene_view_f64& S, const camera_d& cam, const sampler& rng, path_state& ps,
                            const hit_info& h, v3& sample)
{
    const v3 black = make_double3(0.0, 0.0, 0.0);
    if (h.id < 0)
    {
        sample = ps.throughput * sky(cam, ps.d);
        return true;
    }
    material_d m;
    const surface s = surface_at(S, ps, h, m);
    const v3 albedo = s.color;
    v3 direction;
    if (m.kind == RT_DIFFUSE_LIGHT)
    {
        sample = h.front ? ps.throughput * albedo : black;
        return true;
    }
    const uniforms u = rng.draw(ps.depth, block_material);
    if (m.kind == RT_LAMBERTIAN || m.kind == RT_ISOTROPIC)
    {
        // A diffuse bounce: a matte surface, or a particle of smoke, which keeps its own density 1/(4 pi) except under
        // the lights strategy (isotropic::mixes_in_lights is false)
        const bool matte = m.kind == RT_LAMBERTIAN;
        int strategy = cam.sampling;
        if (!matte && strategy != RT_SAMPLING_LIGHTS)
        {
            strategy = RT_SAMPLING_MATERIAL;
        }
        if (strategy == RT_SAMPLING_MATERIAL)
        {
            direction = matte ? around(s.normal, random_cosine_direction(u.x, u.y)) : random_unit_vector(u.x, u.y);
            if (matte && !(dot(s.normal, direction) > 0.0))
            {
                sample = black;
                return true;
            }
            ps.throughput = ps.throughput * albedo;
        }
        else
        {
            bool toward_lights = strategy == RT_SAMPLING_LIGHTS;
            if (strategy == RT_SAMPLING_MIXTURE)
            {
                toward_lights = u.z < 0.5;
            }
            if (toward_lights)
            {
                direction = lights_random(S, s.p, u.w, u.x, u.y);
            }
            else
            {
                direction = strategy == RT_SAMPLING_UNIFORM ? random_unit_vector(u.x, u.y)
                                                            : around(s.normal, random_cosine_direction(u.x, u.y));
            }
            const double p_scatter = matte ? cosine_density(s.normal, direction) : uniform_sphere_density;
            double p = uniform_sphere_density;
            if (strategy != RT_SAMPLING_UNIFORM)
            {
                const double p_lights = lights_pdf_value(S, s.p, direction, s.from);
                p = strategy == RT_SAMPLING_LIGHTS ? p_lights : 0.5 * p_lights + 0.5 * p_scatter;
            }
            if (!(p > 0.0) || !(p_scatter > 0.0))
            {
                sample = black;
                return true;
            }
            ps.throughput = (p_scatter / p) * (ps.throughput * albedo);
        }
    }
    else if (m.kind == RT_METAL)
    {
        direction = unit_vector(reflect(ps.d, s.normal)) + m.fuzz * random_unit_vector(u.x, u.y);
        if (dot(direction, s.normal) <= 0.0)
        {
            sample = black;
            return true;
        }
        ps.throughput = ps.throughput * albedo;
    }
    else // dielectric
    {
        const double ri = h.front ? 1.0 / m.ior : m.ior;
        const v3 ud = unit_vector(ps.d);
        const double cos_theta = fmin(dot(-ud, s.normal), 1.0);
        const double sin_theta = sqrt(1.0 - cos_theta * cos_theta);
        const bool cannot_refract = ri * sin_theta > 1.0;
        direction = cannot_refract || reflectance(cos_theta, ri) > u.z ? reflect(ud, s.normal)
                                                                       : refract(ud, s.normal, ri);
    }
    if (--ps.rays_left == 0)
    {
        sample = black;
        return true;
    }
    ps.o = s.p;
    ps.d = direction;
    ps.from = s.from;
    ps.inward = dot(direction, s.outward) < 0.0;
    return false;
}

// The persistent launch: lanes claim (pixel, chunk) items by a warp ballot and one atomic a warp, as render_kernel does
// in float, trace one segment an iteration and start the next sample the moment one ends
__global__ void __launch_bounds__(render_block) render_f64_kernel(const __grid_constant__ launch_params_f64 P)
{
    __shared__ unsigned long long block_rays;
    if (threadIdx.x == 0)
    {
        block_rays = 0;
    }
    __syncthreads();

    const unsigned lane = threadIdx.x & 31u;
    const unsigned lanes_below = (1u << lane) - 1u;
    const camera_d& cam = P.cam;
    const scene_view_f64& S = P.scene;

    uint32_t rays = 0;
    bool need = true;
    bool start = false;
    int px = 0, py = 0;
    int64_t pass = 0, pass_end = 0;
    int64_t slot = 0;
    double acc_r = 0.0, acc_g = 0.0, acc_b = 0.0;
    sampler rng{};
    path_state ps{};

    while (true)
    {
        const unsigned active = __activemask();
        const unsigned needing = __ballot_sync(active, need);
        if (needing != 0u)
        {
            const int leader = __ffs(static_cast<int>(needing)) - 1;
            unsigned long long base = 0;
            if (static_cast<int>(lane) == leader)
            {
                base = atomicAdd(P.work_counter, static_cast<unsigned long long>(__popc(needing)));
            }
            base = __shfl_sync(active, base, leader);
            if (need)
            {
                const unsigned long long item = base + static_cast<unsigned long long>(__popc(needing & lanes_below));
                if (item >= static_cast<unsigned long long>(P.total_items))
                {
                    break;
                }
                const int64_t k = static_cast<int64_t>(item / static_cast<unsigned long long>(P.padded_pixels));
                const int q = static_cast<int>(item % static_cast<unsigned long long>(P.padded_pixels));
                const int tile = q >> 5;
                const int l = q & 31;
                px = (tile % P.tiles_x) * 8 + (l & 7);
                py = (tile / P.tiles_x) * 4 + (l >> 3);
                if (px >= cam.width || py >= cam.height)
                {
                    continue; // a lane of a tile over the image's edge
                }
                const int64_t chunk_first = (P.first_chunk + k) * P.chunk;
                pass = chunk_first > P.pass_begin ? chunk_first : P.pass_begin;
                const int64_t chunk_end = chunk_first + P.chunk;
                pass_end = chunk_end < P.pass_end ? chunk_end : P.pass_end;
                slot = k * P.padded_pixels + q;
                acc_r = acc_g = acc_b = 0.0;
                rng.pixel = static_cast<uint32_t>(py) * static_cast<uint32_t>(cam.width) + static_cast<uint32_t>(px);
                need = false;
                start = true;
            }
        }
        if (start)
        {
            // Pass n is pass n % k^2 of round n / k^2, whose numbers come from seed + round * 2^32
            const int64_t round = pass / P.round_passes;
            const int in_round = static_cast<int>(pass - round * P.round_passes);
            const uint64_t key = P.seed + (static_cast<uint64_t>(round) << 32);
            rng.key = make_uint2(static_cast<uint32_t>(key), static_cast<uint32_t>(key >> 32));
            rng.pass = static_cast<uint32_t>(in_round);
            camera_ray(cam, px, py, in_round % cam.sqrt_spp, in_round / cam.sqrt_spp, rng.draw(0, block_material),
                       ps.o, ps.d);
            ps.time = S.has_motion ? rng.draw(0, block_time).x : 0.0;
            ps.throughput = make_double3(1.0, 1.0, 1.0);
            ps.rays_left = cam.max_depth;
            ps.depth = 0;
            ps.from = -1;
            ps.inward = false;
            start = false;
        }

        hit_info h = closest_hit(S, ps.o, ps.d, ps.time, ps.from, ps.inward);
        ++rays;
        ++ps.depth;
        if (S.medium_count > 0)
        {
            media_event(S, ps.o, ps.d, ps.time, rng, ps.depth, h);
        }
        v3 sample;
        if (shade_books(S, cam, rng, ps, h, sample))
        {
            acc_r += without_nan(sample.x);
            acc_g += without_nan(sample.y);
            acc_b += without_nan(sample.z);
            if (++pass == pass_end)
            {
                double* out = P.partials + 3 * slot;
                out[0] = acc_r;
                out[1] = acc_g;
                out[2] = acc_b;
                need = true;
            }
            else
            {
                start = true;
            }
        }
    }
    atomicAdd(&block_rays, static_cast<unsigned long long>(rays));
    __syncthreads();
    if (threadIdx.x == 0)
    {
        atomicAdd(P.counters, block_rays);
    }
}
} // namespace

cudaError_t launch_render_f64(const launch_params_f64& p, int grid, cudaStream_t stream)
{
    render_f64_kernel<<<grid, render_block, 0, stream>>>(p);
    return cudaGetLastError();
}

cudaError_t render_f64_attributes(const scene_view_f64& scene, kernel_attributes& out)
{
    (void)scene;
    cudaFuncAttributes a{};
    cudaError_t e = cudaFuncGetAttributes(&a, render_f64_kernel);
    if (e != cudaSuccess)
    {
        return e;
    }
    int device = 0;
    e = cudaGetDevice(&device);
    if (e != cudaSuccess)
    {
        return e;
    }
    e = cudaDeviceGetAttribute(&out.multiprocessors, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess)
    {
        return e;
    }
    e = cudaDeviceGetAttribute(&out.max_threads_per_sm, cudaDevAttrMaxThreadsPerMultiProcessor, device);
    if (e != cudaSuccess)
    {
        return e;
    }
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&out.blocks_per_sm, render_f64_kernel, render_block, 0);
    out.registers = a.numRegs;
    out.local_bytes = static_cast<int>(a.localSizeBytes);
    out.threads_per_block = render_block;
    return e;
}
} // namespace rtb
