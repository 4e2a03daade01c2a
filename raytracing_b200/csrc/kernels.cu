// The path-tracing kernels for sm_100a.
//
// One persistent kernel renders a launch: a grid of (multiprocessors x resident blocks) threads, each of which takes
// work items (a pixel and a chunk of its passes) from a global counter, traces their samples one after another, and
// starts the next sample the moment one ends (path regeneration), so a warp's lanes stay busy however uneven the
// paths are. The lanes that need new work in an iteration claim it together: a ballot over the warp, one atomicAdd
// by its leader for the whole batch, and each lane's item from the prefix count of the ballot below it. Each item's
// sum goes to its own slot of a partials buffer, and a second kernel adds the slots to the pixels' sums in chunk
// order, so the image does not depend on which thread rendered what.
//
// The estimators are the reference's: the books' strategies (src/gpu/camera.cuh:304-437 diffuse_bounce, trace_ray;
// material.cuh:84-126 scatter; lights.cuh:49-227 the lights list) and the quality kernel's NEE with MIS
// (quality_path.cuh:61-188, light_sampler.cuh:40-103, lamps.cuh:81-146, mis.cuh:30-62). What differs is the B200 form:
// a 64-byte node holding both children's boxes, a flat search for small scenes, counter-based random numbers that
// depend only on (seed, pixel, pass, depth, dimension), work items instead of one thread per pixel, and FP64 only for
// a large sphere's quadratic and for the per-pixel sums.
#include <cuda_runtime.h>

#include <cstdint>

#include "ggx_energy_table.h"
#include "kernels.cuh"
#include "philox.cuh"
#include "rt_b200.h"

namespace rtb
{
namespace
{
// ---- float3 arithmetic --------------------------------------------------------------------------------------
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float t, float3 v) { return make_float3(t * v.x, t * v.y, t * v.z); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 u, float3 v)
{
    return make_float3(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x);
}
__device__ __forceinline__ float length_squared(float3 v) { return dot(v, v); }
__device__ __forceinline__ float3 unit_vector(float3 v) { return rsqrtf(length_squared(v)) * v; }
__device__ __forceinline__ float3 reflect(float3 v, float3 n) { return v - (2.0f * dot(v, n)) * n; }
__device__ __forceinline__ float3 refract(float3 uv, float3 n, float etai_over_etat) // vec3.cuh refract
{
    const float cos_theta = fminf(dot(-uv, n), 1.0f);
    const float3 perp = etai_over_etat * (uv + cos_theta * n);
    const float3 parallel = (-sqrtf(fabsf(1.0f - length_squared(perp)))) * n;
    return perp + parallel;
}
__device__ __forceinline__ float3 f3v(const f3& v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ float largest_channel(float3 c) { return fmaxf(fmaxf(c.x, c.y), c.z); }
constexpr float pi_f = 3.14159265358979323846f;
constexpr float inverse_pi_f = 0.318309886183790671538f;
constexpr float uniform_sphere_density = 0.0795774715459476678844f; // 1 / (4 pi)
constexpr float infinity_f = __builtin_huge_valf();

// ---- counter-based random numbers (philox.cuh) -------------------------------------------------------------------
// n / d by the divisor's multiplier (fast_divisor), for n < 2^32
__device__ __forceinline__ uint32_t quotient(uint32_t n, const fast_divisor& v)
{
    return v.magic != 0 ? static_cast<uint32_t>(__umul64hi(static_cast<unsigned long long>(n), v.magic)) : n;
}

// A pass's stratum within its round: column s_i = round_pass % sqrt_spp, row s_j = round_pass / sqrt_spp
__device__ __forceinline__ void stratum_of(const camera_params& cam, int round_pass, int& s_i, int& s_j)
{
    s_j = static_cast<int>(quotient(static_cast<uint32_t>(round_pass), cam.div_sqrt_spp));
    s_i = round_pass - s_j * cam.sqrt_spp;
}

// 24 random bits as a float in [0, 1 - 2^-24]: every value k / 2^24 exactly, as random_real<float> (random.cuh:79-93)
__device__ __forceinline__ float to_unit(uint32_t x) { return static_cast<float>(x >> 8) * 0x1p-24f; }

struct sampler
{
    uint2 key;
    uint32_t pixel;
    uint32_t pass;
    uint32_t job;

    // Four 32-bit numbers for dimension block `block` of the vertex at depth `depth` (0: the camera ray)
    __device__ __forceinline__ uint4 draw_bits(int depth, int block) const
    {
        return philox4x32_10(make_uint4(pixel, pass, (static_cast<uint32_t>(depth) << 4) | block, job), key);
    }

    // The same as uniform floats
    __device__ __forceinline__ float4 draw(int depth, int block) const
    {
        const uint4 r = draw_bits(depth, block);
        return make_float4(to_unit(r.x), to_unit(r.y), to_unit(r.z), to_unit(r.w));
    }
};

// The fixed dimension blocks of a vertex: block 0 the material's own sample (direction u0 u1, lobe or mixture
// choice u2, the lights list's pick u3; a books' vertex that aims at the lights list takes the point from u0 u1, which
// its direction then does not use, so a books' vertex draws one block), blocks 2-3 the NEE light sample (the pick, a
// lamp's point or the map's bin bits, coin and cell position), blocks 4-15 the free flights through the volumes of
// smoke, one number per volume. At depth 0, block 0 is the camera ray's (stratum jitter, lens) and block 1's first
// number the ray's time in a scene where something moves.
constexpr int block_material = 0;
constexpr int block_time = 1;
constexpr int block_nee = 2;

// ---- sampling of directions (random.cuh:95-140, material.cuh:55-64) --------------------------------------------
__device__ __forceinline__ float3 random_unit_vector(float u, float v)
{
    float s, c;
    sincospif(2.0f * v, &s, &c);
    const float r = 2.0f * sqrtf(u * (1.0f - u));
    return make_float3(r * c, r * s, 1.0f - 2.0f * u);
}

__device__ __forceinline__ float3 random_cosine_direction(float r1, float r2)
{
    float s, c;
    sincospif(2.0f * r1, &s, &c);
    const float sin_theta = sqrtf(r2);
    return make_float3(c * sin_theta, s * sin_theta, sqrtf(1.0f - r2));
}

// v given in a basis whose z axis is the unit vector n, in world coordinates: the branchless orthonormal basis of
// Duff, Burgess, Christensen, Hery, Kensler, Liani and Villemin, "Building an Orthonormal Basis, Revisited" (JCGT 2017)
__device__ __forceinline__ float3 around(float3 n, float3 v)
{
    const float sign = copysignf(1.0f, n.z);
    const float a = -1.0f / (sign + n.z);
    const float b = n.x * n.y * a;
    const float3 x_axis = make_float3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
    const float3 y_axis = make_float3(b, sign + n.y * n.y * a, -n.y);
    return v.x * x_axis + v.y * y_axis + v.z * n;
}

__device__ __forceinline__ float cosine_density(float3 unit_normal, float3 direction) // pdf.cuh:21-26
{
    const float cosine = dot(unit_normal, direction) * rsqrtf(length_squared(direction));
    return cosine > 0.0f ? cosine * inverse_pi_f : 0.0f;
}

// Schlick's reflectance (material.cuh:67-76)
__device__ __forceinline__ float reflectance(float cosine, float ri)
{
    float r0 = (1.0f - ri) / (1.0f + ri);
    r0 = r0 * r0;
    const float x = 1.0f - cosine;
    const float x2 = x * x;
    return r0 + (1.0f - r0) * (x2 * x2 * x);
}

// ---- primitive tests ------------------------------------------------------------------------------------------
// 1 / x, never infinite (bvh.cuh:475-488): |x| below 2^-80 moves out to +-2^-80
__device__ __forceinline__ float safe_inverse(float x)
{
    const float tiny = 0x1p-80f;
    return 1.0f / (fabsf(x) > tiny ? x : copysignf(tiny, x));
}

// The two roots of the line with a sphere, as (h/a) -+ sqrt(r^2 - |l|^2)/sqrt(a) with l the vector from the line's
// closest point to the center (sphere.cuh:70-97, after Haines et al., Ray Tracing Gems ch. 7): nothing larger than
// r^2 is subtracted, and the three squares go into r^2 through fused multiply-adds.
__device__ __forceinline__ bool sphere_roots(float4 s, float3 o, float3 d, float inverse_a, float& near, float& far)
{
    if (s.w >= 0.0f)
    {
        const float3 oc = make_float3(s.x - o.x, s.y - o.y, s.z - o.z);
        const float h_over_a = dot(d, oc) * inverse_a;
        const float3 l = oc - h_over_a * d;
        const float disc = fmaf(-l.x, l.x, fmaf(-l.y, l.y, fmaf(-l.z, l.z, s.w * s.w)));
        if (disc < 0.0f)
        {
            return false;
        }
        const float half_chord = sqrtf(disc * inverse_a);
        near = h_over_a - half_chord;
        far = h_over_a + half_chord;
        return true;
    }
    // A large sphere (negative radius): the same quadratic in FP64, where FP32's 24 bits cancel on its scale
    const double r = -static_cast<double>(s.w);
    const double ox = static_cast<double>(s.x) - o.x;
    const double oy = static_cast<double>(s.y) - o.y;
    const double oz = static_cast<double>(s.z) - o.z;
    const double dx = d.x, dy = d.y, dz = d.z;
    const double ia = 1.0 / (dx * dx + dy * dy + dz * dz);
    const double hoa = (dx * ox + dy * oy + dz * oz) * ia;
    const double lx = ox - hoa * dx, ly = oy - hoa * dy, lz = oz - hoa * dz;
    const double disc = fma(-lx, lx, fma(-ly, ly, fma(-lz, lz, r * r)));
    if (disc < 0.0)
    {
        return false;
    }
    const double half_chord = sqrt(disc * ia);
    near = static_cast<float>(hoa - half_chord);
    far = static_cast<float>(hoa + half_chord);
    return true;
}

// hit_sphere (sphere.cuh:99-117): the nearest root in (t_min, t_max); far_only for the sphere the ray leaves inward
__device__ __forceinline__ bool hit_sphere(float4 s, float3 o, float3 d, float inverse_a, float t_min, float t_max,
                                           bool far_only, float& t, bool& entering)
{
    float near, far;
    if (!sphere_roots(s, o, d, inverse_a, near, far))
    {
        return false;
    }
    t = near;
    entering = !far_only && t > t_min;
    if (!entering)
    {
        t = far;
    }
    return t_min < t && t < t_max;
}

struct quad_v
{
    float3 q, n, a, b;
};

__device__ __forceinline__ quad_v load_quad(const quad12* quads, int i)
{
    const float4* p = reinterpret_cast<const float4*>(quads + i);
    const float4 a = __ldg(p);
    const float4 b = __ldg(p + 1);
    const float4 c = __ldg(p + 2);
    return {make_float3(a.x, a.y, a.z), make_float3(a.w, b.x, b.y), make_float3(b.z, b.w, c.x),
            make_float3(c.y, c.z, c.w)};
}

// hit_quad (quad.cuh:60-84): t in [t_min, t_max] and alpha, beta in [0, 1], closed; the corner taken relative to the
// origin first. NaNs fail every comparison (a degenerate quad stays invisible).
__device__ __forceinline__ bool hit_quad(const quad_v& s, float3 o, float3 d, float t_min, float t_max, float& t,
                                         bool& front)
{
    const float denominator = dot(s.n, d);
    if (!(fabsf(denominator) >= 1e-8f))
    {
        return false;
    }
    const float3 origin_to_q = s.q - o;
    t = dot(s.n, origin_to_q) / denominator;
    if (!(t_min <= t && t <= t_max))
    {
        return false;
    }
    const float3 p = t * d - origin_to_q;
    const float alpha = dot(p, s.a);
    const float beta = dot(p, s.b);
    if (!(0.0f <= alpha && alpha <= 1.0f && 0.0f <= beta && beta <= 1.0f))
    {
        return false;
    }
    front = denominator < 0.0f;
    return true;
}

struct triangle_v
{
    float3 a, b, c;
};

__device__ __forceinline__ triangle_v load_triangle(const triangle12* tris, int i)
{
    const float4* p = reinterpret_cast<const float4*>(tris + i);
    const float4 a = __ldg(p);
    const float4 b = __ldg(p + 1);
    const float4 c = __ldg(p + 2);
    return {make_float3(a.x, a.y, a.z), make_float3(a.w, b.x, b.y), make_float3(b.z, b.w, c.x)};
}

__device__ __forceinline__ float axis_of(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// A ray's shear for the watertight triangle test: the axis along which the direction is largest (z after the
// permutation, the other two swapped when it points backwards so the winding is kept), and the shear that makes the
// direction (0, 0, 1). Computed once per leaf; the same floats for every triangle the ray meets.
struct ray_shear
{
    int kx, ky, kz;
    float sx, sy, sz;
};

__device__ __forceinline__ ray_shear shear_of(float3 d)
{
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    ray_shear r;
    r.kz = ax > ay ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    r.kx = r.kz == 2 ? 0 : r.kz + 1;
    r.ky = r.kx == 2 ? 0 : r.kx + 1;
    const float dz = axis_of(d, r.kz);
    if (dz < 0.0f)
    {
        const int k = r.kx;
        r.kx = r.ky;
        r.ky = k;
    }
    r.sz = 1.0f / dz;
    r.sx = axis_of(d, r.kx) * r.sz;
    r.sy = axis_of(d, r.ky) * r.sz;
    return r;
}

// The signed area of an edge seen along the sheared ray, rounded so that the same edge walked the other way by the
// neighbouring triangle gives exactly the opposite number (no fused multiply-add), and in double when it comes out 0
__device__ __forceinline__ float edge_function(float px, float py, float qx, float qy)
{
    const float e = __fsub_rn(__fmul_rn(px, qy), __fmul_rn(py, qx));
    if (e != 0.0f)
    {
        return e;
    }
    return static_cast<float>(static_cast<double>(px) * qy - static_cast<double>(py) * qx);
}

// The same test in double, for a ray whose float edge functions are too close to 0 to be sure of their signs: one
// grazing the triangle (its projection a sliver) or passing within rounding of an edge
__device__ __noinline__ bool hit_triangle_double(const triangle_v& tr, const ray_shear& r, float3 o, float3 d,
                                                 float t_min, float t_max, float& t, bool& front)
{
    const double ox = o.x, oy = o.y, oz = o.z;
    const double rel[3][3] = {{tr.a.x - ox, tr.a.y - oy, tr.a.z - oz},
                              {tr.b.x - ox, tr.b.y - oy, tr.b.z - oz},
                              {tr.c.x - ox, tr.c.y - oy, tr.c.z - oz}};
    const double dir[3] = {d.x, d.y, d.z};
    const double sz = 1.0 / dir[r.kz];
    const double sx = dir[r.kx] * sz, sy = dir[r.ky] * sz;
    double px[3], py[3], pz[3];
    for (int k = 0; k < 3; ++k)
    {
        pz[k] = rel[k][r.kz];
        px[k] = rel[k][r.kx] - sx * pz[k];
        py[k] = rel[k][r.ky] - sy * pz[k];
    }
    const double u = px[2] * py[1] - py[2] * px[1];
    const double v = px[0] * py[2] - py[0] * px[2];
    const double w = px[1] * py[0] - py[1] * px[0];
    if ((u < 0.0 || v < 0.0 || w < 0.0) && (u > 0.0 || v > 0.0 || w > 0.0))
    {
        return false;
    }
    const double det = u + v + w;
    if (det == 0.0)
    {
        return false;
    }
    const double tt = (u * pz[0] + v * pz[1] + w * pz[2]) * sz / det;
    t = static_cast<float>(tt);
    if (!(t_min < t && t < t_max))
    {
        return false;
    }
    front = dot(d, cross(tr.b - tr.a, tr.c - tr.a)) < 0.0f;
    return true;
}

__device__ __forceinline__ float max_abs(float3 v) { return fmaxf(fabsf(v.x), fmaxf(fabsf(v.y), fabsf(v.z))); }

// Woop, Benthin and Wald, "Watertight Ray/Triangle Intersection" (JCGT 2013): the triangle's vertices sheared into
// the ray's frame, the three edge functions of the origin's projection, all of one sign; so a ray through an edge or a
// vertex shared by triangles hits at least one of them, with no crack between (Möller-Trumbore in float lets such a
// ray through both, about 4 rays in a million on the 1.3M-triangle mesh). An edge function within its float rounding
// of 0 (a grazing ray, or one within rounding of an edge) sends the test to double. Barycentrics closed, t open. The
// front is the side (b - a) x (c - a) points to.
__device__ __forceinline__ bool hit_triangle(const triangle_v& tr, const ray_shear& r, float3 o, float3 d,
                                             float t_min, float t_max, float& t, bool& front)
{
    const float3 pa = tr.a - o, pb = tr.b - o, pc = tr.c - o;
    const float az = axis_of(pa, r.kz), bz = axis_of(pb, r.kz), cz = axis_of(pc, r.kz);
    const float ax = axis_of(pa, r.kx) - r.sx * az, ay = axis_of(pa, r.ky) - r.sy * az;
    const float bx = axis_of(pb, r.kx) - r.sx * bz, by = axis_of(pb, r.ky) - r.sy * bz;
    const float cx = axis_of(pc, r.kx) - r.sx * cz, cy = axis_of(pc, r.ky) - r.sy * cz;
    const float u = edge_function(cx, cy, bx, by);
    const float v = edge_function(ax, ay, cx, cy);
    const float w = edge_function(bx, by, ax, ay);
    // The edge functions' rounding: the shear's (a few units of the vertices' largest coordinate's last place) times
    // the projected coordinates' size, with a margin
    const float coords = fmaxf(max_abs(pa), fmaxf(max_abs(pb), max_abs(pc)));
    const float sheared = fmaxf(fmaxf(fmaxf(fabsf(ax), fabsf(ay)), fmaxf(fabsf(bx), fabsf(by))),
                                fmaxf(fabsf(cx), fabsf(cy)));
    const float rounding = 5e-7f * coords * sheared;
    if (fabsf(u) <= rounding || fabsf(v) <= rounding || fabsf(w) <= rounding)
    {
        return hit_triangle_double(tr, r, o, d, t_min, t_max, t, front);
    }
    if ((u < 0.0f || v < 0.0f || w < 0.0f) && (u > 0.0f || v > 0.0f || w > 0.0f))
    {
        return false;
    }
    const float det = u + v + w;
    if (det == 0.0f)
    {
        return false;
    }
    const float depth = u * (r.sz * az) + v * (r.sz * bz) + w * (r.sz * cz);
    t = depth / det;
    if (!(t_min < t && t < t_max))
    {
        return false;
    }
    front = dot(d, cross(tr.b - tr.a, tr.c - tr.a)) < 0.0f;
    return true;
}

// ---- traversal ------------------------------------------------------------------------------------------------
struct hit_info
{
    int id;     // global id, -1 for none
    float t;
    bool front; // the near root of a sphere, the front of a quad or a triangle
};

constexpr float t_min = 0.001f;

// What one traversal fetched, for the counting build (the roofline's algorithmic bytes); compiled away otherwise
struct fetch_counts
{
    uint32_t nodes = 0;
    uint32_t spheres = 0;
    uint32_t quads = 0;
    uint32_t triangles = 0;
};

// Sphere i (leaf order) where it is at the ray's time: its center moved by time * displacement in a scene where
// something moves (moving_sphere::at, sphere.cuh)
// FEATURES (here and below): the code of the second book's features (moving spheres, textures, smoke) is compiled in;
// the render kernels of scenes without them are compiled with FEATURES = false and keep none of its registers
template <bool FEATURES = true>
__device__ __forceinline__ float4 sphere_at(const scene_view& S, int i, float time)
{
    float4 s = __ldg(reinterpret_cast<const float4*>(S.spheres + i));
    if (FEATURES && S.has_motion)
    {
        const float4 m = __ldg(S.sphere_motion + i);
        s.x = fmaf(time, m.x, s.x);
        s.y = fmaf(time, m.y, s.y);
        s.z = fmaf(time, m.z, s.z);
    }
    return s;
}

// The leaf's primitives against the ray, shrinking hit.t; true at the first hit for a shadow ray (SHADOW, or `any`
// for a kernel that walks both kinds of ray)
template <bool SHADOW, bool COUNT, bool FEATURES>
__device__ __forceinline__ bool test_leaf(const scene_view& S, int link, float3 o, float3 d, float time,
                                          float inverse_a, int from, bool inward, int skip, hit_info& hit,
                                          fetch_counts* counts, bool any = false)
{
    const int kind = leaf_kind(link);
    const int count = leaf_count(link);
    const int start = leaf_start(link);
    if (COUNT)
    {
        (kind == kind_sphere ? counts->spheres : kind == kind_quad ? counts->quads : counts->triangles) += count;
    }
    if (kind == kind_sphere)
    {
        for (int i = start; i < start + count; ++i)
        {
            const int id = i; // spheres' global ids are their indices
            const bool own = id == from;
            if ((own && !inward) || id == skip)
            {
                continue;
            }
            const float4 s = sphere_at<FEATURES>(S, i, time);
            float t;
            bool entering;
            if (hit_sphere(s, o, d, inverse_a, t_min, hit.t, own, t, entering))
            {
                if (SHADOW || any)
                {
                    return true;
                }
                hit = {id, t, entering};
            }
        }
    }
    else if (kind == kind_quad)
    {
        for (int i = start; i < start + count; ++i)
        {
            const int id = S.quad_base + i;
            if (id == from || id == skip)
            {
                continue;
            }
            const quad_v q = load_quad(S.quads, i);
            float t;
            bool front;
            if (hit_quad(q, o, d, t_min, hit.t, t, front))
            {
                if (SHADOW || any)
                {
                    return true;
                }
                hit = {id, t, front};
            }
        }
    }
    else
    {
        const ray_shear shear = shear_of(d);
        for (int i = start; i < start + count; ++i)
        {
            const int id = S.triangle_base + i;
            if (id == from || id == skip)
            {
                continue;
            }
            const triangle_v tr = load_triangle(S.triangles, i);
            float t;
            bool front;
            if (hit_triangle(tr, shear, o, d, t_min, hit.t, t, front))
            {
                if (SHADOW || any)
                {
                    return true;
                }
                hit = {id, t, front};
            }
        }
    }
    return false;
}

// No more nodes to visit (a leaf link never takes this value: its kind field would be 3)
constexpr int traversal_done = traversal_done_link;

// The closest hit in (t_min, t_max) (SHADOW = false; the CPU's world.hit, bvh.cuh:576-706), or whether anything lies
// there (SHADOW = true; shadow.cuh:26-109 occluded, `skip` not tested). The self-intersection rules of the primitive
// the ray leaves, `from`: a quad or a triangle is never hit again (a line meets a plane once); a sphere left outward
// is never hit again, and left inward only at its far root (bvh.cuh:539-575).
//
// The loop is Aila and Laine's speculative while-while (HPG 2009): a lane descends through inner nodes, sets aside the
// first leaf it meets and keeps descending, and the warp leaves the node loop together once every lane holds a leaf;
// then the leaf loop tests them. Node steps and leaf tests so run with the warp's lanes side by side, where a single
// loop would run a node step for some lanes and a leaf test for the others one after the other.
//
// SEARCH: search_any follows the scene's `flat`; search_flat and search_tree compile one of the two searches alone
// (a kernel specialised for one of them keeps no code, registers or stack for the other).
constexpr int search_any = 0;
constexpr int search_flat = 1;
constexpr int search_tree = 2;

template <bool SHADOW, bool COUNT = false, int SEARCH = search_any, bool FEATURES = true>
__device__ __forceinline__ bool traverse(const scene_view& S, float3 o, float3 d, float time, float t_max, int from,
                                         bool inward, int skip, hit_info& hit, fetch_counts* counts = nullptr)
{
    hit.id = -1;
    hit.t = t_max;
    hit.front = false;
    if (S.node_count == 0)
    {
        return false;
    }
    const float inverse_a = 1.0f / length_squared(d);
    if (SEARCH == search_flat || (SEARCH == search_any && S.flat))
    {
        // A small scene of spheres and quads: every primitive tested in order, no tree. The warp's lanes run the same
        // loop over the same records (one broadcast load each), where a tree walk would split them up.
        for (int i = 0; i < S.quad_base; ++i)
        {
            const bool own = i == from;
            if ((own && !inward) || i == skip)
            {
                continue;
            }
            const float4 s = sphere_at<FEATURES>(S, i, time);
            float t;
            bool entering;
            if (hit_sphere(s, o, d, inverse_a, t_min, hit.t, own, t, entering))
            {
                if (SHADOW)
                {
                    return true;
                }
                hit = {i, t, entering};
            }
        }
        const int quads = S.triangle_base - S.quad_base;
        for (int i = 0; i < quads; ++i)
        {
            const int id = S.quad_base + i;
            if (id == from || id == skip)
            {
                continue;
            }
            float t;
            bool front;
            if (hit_quad(load_quad(S.quads, i), o, d, t_min, hit.t, t, front))
            {
                if (SHADOW)
                {
                    return true;
                }
                hit = {id, t, front};
            }
        }
        if (COUNT)
        {
            counts->spheres += S.quad_base;
            counts->quads += quads;
        }
        return hit.id >= 0;
    }
    const float3 inv = make_float3(safe_inverse(d.x), safe_inverse(d.y), safe_inverse(d.z));
    const float3 os = make_float3(o.x * inv.x, o.y * inv.y, o.z * inv.z);
    int2 stack[max_bvh_depth];
    int sp = 0;
    // The next stack entry the ray enters before the closest hit so far, or traversal_done
    const auto pop = [&]() -> int {
        while (sp > 0)
        {
            const int2 e = stack[--sp];
            if (SHADOW || __int_as_float(e.y) < hit.t)
            {
                return e.x;
            }
        }
        return traversal_done;
    };
    int link = 0;
    int leaf = 0; // a leaf set aside (leaf links are negative; 0: none)
    while (link != traversal_done)
    {
        while (link >= 0)
        {
            const float4* np = reinterpret_cast<const float4*>(S.nodes + link);
            const float4 nx = __ldg(np);
            const float4 ny = __ldg(np + 1);
            const float4 nz = __ldg(np + 2);
            const int2 nl = __ldg(reinterpret_cast<const int2*>(np + 3));
            if (COUNT)
            {
                ++counts->nodes;
            }
            const float a0 = fmaf(nx.x, inv.x, -os.x), a1 = fmaf(nx.y, inv.x, -os.x);
            const float b0 = fmaf(ny.x, inv.y, -os.y), b1 = fmaf(ny.y, inv.y, -os.y);
            const float c0 = fmaf(nz.x, inv.z, -os.z), c1 = fmaf(nz.y, inv.z, -os.z);
            const float enter0 = fmaxf(fmaxf(fminf(a0, a1), fminf(b0, b1)), fmaxf(fminf(c0, c1), t_min));
            const float exit0 = fminf(fminf(fmaxf(a0, a1), fmaxf(b0, b1)), fminf(fmaxf(c0, c1), hit.t));
            const float a2 = fmaf(nx.z, inv.x, -os.x), a3 = fmaf(nx.w, inv.x, -os.x);
            const float b2 = fmaf(ny.z, inv.y, -os.y), b3 = fmaf(ny.w, inv.y, -os.y);
            const float c2 = fmaf(nz.z, inv.z, -os.z), c3 = fmaf(nz.w, inv.z, -os.z);
            const float enter1 = fmaxf(fmaxf(fminf(a2, a3), fminf(b2, b3)), fmaxf(fminf(c2, c3), t_min));
            const float exit1 = fminf(fminf(fmaxf(a2, a3), fmaxf(b2, b3)), fminf(fmaxf(c2, c3), hit.t));
            const bool h0 = enter0 <= exit0;
            const bool h1 = enter1 <= exit1;
            if (h0 && h1)
            {
                const bool second_first = enter1 < enter0;
                link = second_first ? nl.y : nl.x;
                stack[sp++] = make_int2(second_first ? nl.x : nl.y, __float_as_int(second_first ? enter0 : enter1));
            }
            else if (h0 || h1)
            {
                link = h0 ? nl.x : nl.y;
            }
            else
            {
                link = pop();
            }
            // A leaf: set it aside and go on descending, unless one is already waiting
            if (link < 0 && link != traversal_done && leaf == 0)
            {
                leaf = link;
                link = pop();
            }
            if (!__any_sync(__activemask(), leaf == 0))
            {
                break; // every lane of the warp holds a leaf: test them together
            }
        }
        while (leaf < 0)
        {
            if (test_leaf<SHADOW, COUNT, FEATURES>(S, leaf, o, d, time, inverse_a, from, inward, skip, hit, counts))
            {
                return true;
            }
            leaf = 0;
            if (link < 0 && link != traversal_done)
            {
                leaf = link;
                link = pop();
            }
        }
    }
    return hit.id >= 0;
}

// ---- volumes of smoke (constant_medium.cuh:29-120, camera.cuh:259-284, shadow.cuh:129-165) -------------------------
constexpr int block_media = 4; // max_media volumes: one number each from blocks 4-15 of a vertex

// Where the ray's line crosses the medium's boundary: the sphere's two roots, the sphere where it is at the ray's time,
// kept only if the chord is longer than 0.0001; or the nearest and the farthest plane of the boundary quads the line
// meets inside them
__device__ bool boundary_crossings(const scene_view& S, const medium16& m, float3 o, float3 d, float time,
                                   float inverse_a, float& t_in, float& t_out)
{
    if (m.quad_count == 0)
    {
        const float4 s = make_float4(fmaf(time, m.dx, m.cx), fmaf(time, m.dy, m.cy), fmaf(time, m.dz, m.cz), m.radius);
        return sphere_roots(s, o, d, inverse_a, t_in, t_out) && t_out - t_in > 0.0001f;
    }
    t_in = infinity_f;
    t_out = -infinity_f;
    for (int i = m.first_quad; i < m.first_quad + m.quad_count; ++i)
    {
        float t;
        bool front;
        if (hit_quad(load_quad(S.boundary_quads, i), o, d, -infinity_f, infinity_f, t, front))
        {
            t_in = fminf(t_in, t);
            t_out = fmaxf(t_out, t);
        }
    }
    return t_out - t_in >= 0.0001f;
}

// The stretch [t_in, t_out] of (t_min, t_max) that lies inside the medium, or false: its box first (a ray that misses
// the box misses the volume), then the boundary's crossings
__device__ __forceinline__ bool medium_stretch(const scene_view& S, const medium16& m, float3 o, float3 d, float time,
                                               float inverse_a, float3 inv, float3 os, float t_max, float& t_in,
                                               float& t_out)
{
    const float a0 = fmaf(m.lo_x, inv.x, -os.x), a1 = fmaf(m.hi_x, inv.x, -os.x);
    const float b0 = fmaf(m.lo_y, inv.y, -os.y), b1 = fmaf(m.hi_y, inv.y, -os.y);
    const float c0 = fmaf(m.lo_z, inv.z, -os.z), c1 = fmaf(m.hi_z, inv.z, -os.z);
    const float enter = fmaxf(fmaxf(fminf(a0, a1), fminf(b0, b1)), fmaxf(fminf(c0, c1), t_min));
    const float exit = fminf(fminf(fmaxf(a0, a1), fmaxf(b0, b1)), fminf(fmaxf(c0, c1), t_max));
    if (!(enter <= exit))
    {
        return false;
    }
    float line_in, line_out;
    if (!boundary_crossings(S, m, o, d, time, inverse_a, line_in, line_out))
    {
        return false;
    }
    t_in = fmaxf(line_in, t_min);
    t_out = fminf(line_out, t_max);
    if (!(t_in < t_out))
    {
        return false;
    }
    t_in = fmaxf(t_in, 0.0f);
    return true;
}

// What the ray meets first: the closest surface `hit`, or a particle of smoke in front of it (closest_event,
// camera.cuh:259-284). Each volume, in the list's order, against the closest event so far: a free flight of
// -log(u) / density from where the ray enters it (medium_collision, constant_medium.cuh:86-120), u drawn from the
// vertex's media blocks.
// (Like transmittance and texture_value: only the kernels of scenes with these features call them, so they are
// inlined there; measured 5-10% faster on the second book's scenes than as calls.)
#define RTB_FEATURE_FUNCTION __device__ __forceinline__
RTB_FEATURE_FUNCTION void media_event(const scene_view& S, float3 o, float3 d, float time, const sampler& rng,
                                      int depth,
                            hit_info& hit)
{
    const float inverse_a = 1.0f / length_squared(d);
    const float3 inv = make_float3(safe_inverse(d.x), safe_inverse(d.y), safe_inverse(d.z));
    const float3 os = make_float3(o.x * inv.x, o.y * inv.y, o.z * inv.z);
    const float length = sqrtf(length_squared(d));
    float4 u = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (int k = 0; k < S.medium_count; ++k)
    {
        if ((k & 3) == 0)
        {
            u = rng.draw(depth, block_media + (k >> 2));
        }
        const medium16 m = S.media[k];
        float t_in, t_out;
        if (!medium_stretch(S, m, o, d, time, inverse_a, inv, os, hit.t, t_in, t_out))
        {
            continue;
        }
        const float uk = (k & 3) == 0 ? u.x : (k & 3) == 1 ? u.y : (k & 3) == 2 ? u.z : u.w;
        const float distance = m.neg_inv_density * logf(uk);
        if (distance > (t_out - t_in) * length)
        {
            continue; // through without meeting a particle
        }
        hit = {S.medium_base + k, t_in + distance / length, true};
    }
}

// The chance that (t_min, t_max) of the ray crosses every volume without meeting a particle: the expected value of
// media_event's free-flight test over exactly the stretch it would test (transmittance, shadow.cuh:129-165)
RTB_FEATURE_FUNCTION float transmittance(const scene_view& S, float3 o, float3 d, float time, float t_max)
{
    const float inverse_a = 1.0f / length_squared(d);
    const float3 inv = make_float3(safe_inverse(d.x), safe_inverse(d.y), safe_inverse(d.z));
    const float3 os = make_float3(o.x * inv.x, o.y * inv.y, o.z * inv.z);
    const float length = sqrtf(length_squared(d));
    float exponent = 0.0f;
    for (int k = 0; k < S.medium_count; ++k)
    {
        const medium16 m = S.media[k];
        float t_in, t_out;
        if (medium_stretch(S, m, o, d, time, inverse_a, inv, os, t_max, t_in, t_out))
        {
            exponent += (t_out - t_in) * length / m.neg_inv_density;
        }
    }
    return expf(exponent);
}

// ---- textures (texture.cuh, perlin.cuh: the books' solid, checker, image and marble textures) ------------------
// Perlin noise with Hermite smoothing of the cell's coordinates and the trilinear sum of the eight corners'
// gradient dot products (perlin.ixx noise); turbulence: 7 octaves of it, each at twice the frequency and half the
// weight, absolute value
__device__ float perlin_noise(const noise_table& n, float3 p)
{
    const float fx = floorf(p.x), fy = floorf(p.y), fz = floorf(p.z);
    const int i = static_cast<int>(fx), j = static_cast<int>(fy), k = static_cast<int>(fz);
    const float u = p.x - fx, v = p.y - fy, w = p.z - fz;
    const float uu = u * u * (3.0f - 2.0f * u);
    const float vv = v * v * (3.0f - 2.0f * v);
    const float ww = w * w * (3.0f - 2.0f * w);
    float accum = 0.0f;
#pragma unroll
    for (int di = 0; di < 2; ++di)
    {
        const int px = n.perm_x[(i + di) & 255];
        const float wx = di == 0 ? 1.0f - uu : uu;
#pragma unroll
        for (int dj = 0; dj < 2; ++dj)
        {
            const int py = n.perm_y[(j + dj) & 255];
            const float wy = dj == 0 ? 1.0f - vv : vv;
#pragma unroll
            for (int dk = 0; dk < 2; ++dk)
            {
                const int pz = n.perm_z[(k + dk) & 255];
                const float wz = dk == 0 ? 1.0f - ww : ww;
                const float4 g = n.gradients[px ^ py ^ pz];
                const float dot_g = g.x * (u - static_cast<float>(di)) + g.y * (v - static_cast<float>(dj)) +
                                    g.z * (w - static_cast<float>(dk));
                accum += wx * wy * wz * dot_g;
            }
        }
    }
    return accum;
}

__device__ float turbulence(const noise_table& n, float3 p)
{
    float accum = 0.0f;
    float weight = 1.0f;
    for (int layer = 0; layer < 7; ++layer)
    {
        accum += weight * perlin_noise(n, p);
        weight *= 0.5f;
        p = 2.0f * p;
    }
    return fabsf(accum);
}

// The texture's color at the hit (texture_value, texture.cuh:60-110): a checker is walked down to the texture of the
// point's cube (its textures come before it, so the walk ends); an image is read at (u, v) clamped to [0, 1], v
// flipped, the pixel they fall in; a marble is 0.5 (1 + sin(scale z + 10 turbulence(p))) in every channel
RTB_FEATURE_FUNCTION float3 texture_value(const scene_view& S, int index, float u, float v, float3 p)
{
    texture8 t = S.textures[index];
    while (t.kind == RT_TEXTURE_CHECKER)
    {
        const int x = static_cast<int>(floorf(t.inv_scale * p.x));
        const int y = static_cast<int>(floorf(t.inv_scale * p.y));
        const int z = static_cast<int>(floorf(t.inv_scale * p.z));
        t = S.textures[(x + y + z) % 2 == 0 ? t.even : t.odd];
    }
    if (t.kind == RT_TEXTURE_IMAGE)
    {
        const image_info im = S.images[t.table];
        const float cu = fminf(fmaxf(u, 0.0f), 1.0f);
        const float fv = 1.0f - fminf(fmaxf(v, 0.0f), 1.0f);
        const int column = static_cast<int>(cu * static_cast<float>(im.width));
        const int row = static_cast<int>(fv * static_cast<float>(im.height));
        const int i = column < im.width - 1 ? column : im.width - 1;
        const int j = row < im.height - 1 ? row : im.height - 1;
        const float4 c = __ldg(S.texels + im.offset + j * im.width + i);
        return make_float3(c.x, c.y, c.z);
    }
    if (t.kind == RT_TEXTURE_NOISE)
    {
        const noise_table& n = S.noises[t.table];
        const float gray = 0.5f * (1.0f + sinf(n.scale * p.z + 10.0f * turbulence(n, p)));
        return make_float3(gray, gray, gray);
    }
    return make_float3(t.r, t.g, t.b);
}

// ---- the books' lights list (lights.cuh:49-227) ---------------------------------------------------------------
__device__ __forceinline__ quad_v light_quad(const light24& l)
{
    return {make_float3(l.quad.qx, l.quad.qy, l.quad.qz), make_float3(l.quad.nx, l.quad.ny, l.quad.nz),
            make_float3(l.quad.ax, l.quad.ay, l.quad.az), make_float3(l.quad.bx, l.quad.by, l.quad.bz)};
}

__device__ __forceinline__ float one_minus_cos_theta_max(float radius, float distance_squared)
{
    const float sin_squared = radius * radius / distance_squared;
    return sin_squared / (1.0f + sqrtf(1.0f - sin_squared));
}

// |center - origin|^2 with its multiply-adds written out, so that the density and the sampler decide alike
__device__ __forceinline__ float sphere_distance_squared(float3 v)
{
    return fmaf(v.z, v.z, fmaf(v.x, v.x, __fmul_rn(v.y, v.y)));
}

__device__ float lights_pdf_value(const scene_view& S, float3 origin, float3 direction, int from)
{
    float sum = 0.0f;
    for (int k = 0; k < S.light_count; ++k)
    {
        const light24& l = S.lights[k];
        const bool own = from >= 0 && l.twin == from;
        if (l.kind == RT_LIGHT_QUAD)
        {
            if (own)
            {
                continue;
            }
            float t;
            bool front;
            if (!hit_quad(light_quad(l), origin, direction, t_min, infinity_f, t, front))
            {
                continue;
            }
            const float len2 = length_squared(direction);
            const float distance_squared = t * t * len2;
            const float3 n = make_float3(l.quad.nx, l.quad.ny, l.quad.nz);
            const float cosine = fabsf(dot(direction, n)) * rsqrtf(len2);
            sum += l.weight * (distance_squared / (cosine * l.area));
        }
        else
        {
            const float3 c = make_float3(l.cx, l.cy, l.cz);
            const float3 to_center = c - origin;
            const float distance_squared = sphere_distance_squared(to_center);
            if (distance_squared < l.radius * l.radius)
            {
                sum += l.weight * uniform_sphere_density;
                continue;
            }
            if (own && !(dot(direction, to_center) > 0.0f))
            {
                continue;
            }
            float t;
            bool entering;
            if (!hit_sphere(make_float4(c.x, c.y, c.z, l.radius), origin, direction, 1.0f / length_squared(direction),
                            t_min, infinity_f, own, t, entering))
            {
                continue;
            }
            sum += l.weight * (1.0f / (2.0f * pi_f * one_minus_cos_theta_max(l.radius, distance_squared)));
        }
    }
    return sum;
}

// lights_random: the running sums pick a light with `pick`; (a, b) draw its point or direction
__device__ float3 lights_random(const scene_view& S, float3 origin, float pick, float a, float b)
{
    int k = 0;
    while (k < S.light_count - 1 && !(pick < S.lights[k].cdf))
    {
        ++k;
    }
    const light24& l = S.lights[k];
    if (l.kind == RT_LIGHT_QUAD)
    {
        const float3 q = make_float3(l.quad.qx, l.quad.qy, l.quad.qz);
        return unit_vector((q - origin) + a * make_float3(l.ux, l.uy, l.uz) + b * make_float3(l.vx, l.vy, l.vz));
    }
    const float3 to_center = make_float3(l.cx, l.cy, l.cz) - origin;
    const float distance_squared = sphere_distance_squared(to_center);
    if (distance_squared < l.radius * l.radius)
    {
        return random_unit_vector(a, b);
    }
    const float one_minus_cos_max = one_minus_cos_theta_max(l.radius, distance_squared);
    float s, c;
    sincospif(2.0f * a, &s, &c);
    const float one_minus_z = b * one_minus_cos_max;
    const float sin_theta = sqrtf(one_minus_z * (2.0f - one_minus_z));
    return around(rsqrtf(distance_squared) * to_center,
                  make_float3(c * sin_theta, s * sin_theta, 1.0f - one_minus_z));
}

// ---- the NEE/MIS integrator's lamps and weights (lamps.cuh, light_sampler.cuh, mis.cuh) ------------------------
__device__ __forceinline__ float power_weight(float self, float other)
{
    if (!(self > 0.0f))
    {
        return 0.0f;
    }
    const float r = other / self;
    const float w = 1.0f / fmaf(r, r, 1.0f);
    return w == w ? w : 0.0f;
}

__device__ __forceinline__ float light_weight(int c, float p_light, float p_bsdf)
{
    return c == RT_COMBINE_POWER_HEURISTIC ? power_weight(p_light, p_bsdf) : 1.0f;
}

__device__ __forceinline__ float bsdf_weight(int c, float p_bsdf, float p_light)
{
    if (c == RT_COMBINE_BSDF_ONLY || !(p_bsdf > 0.0f) || !(p_light > 0.0f))
    {
        return 1.0f;
    }
    return c == RT_COMBINE_POWER_HEURISTIC ? power_weight(p_bsdf, p_light) : 0.0f;
}

struct lamp_sample
{
    float3 wi;
    float distance;
    float pdf;
};

// sample_lamp (lamps.cuh:81-131): two numbers; false for the back of a quad or a point inside a sphere
__device__ bool sample_lamp(const emitter20& e, float3 x, float a, float b, lamp_sample& out)
{
    const float3 corner = make_float3(e.cx, e.cy, e.cz);
    if (e.kind == RT_LIGHT_QUAD)
    {
        const float3 to = (corner - x) + a * make_float3(e.ux, e.uy, e.uz) + b * make_float3(e.vx, e.vy, e.vz);
        const float distance_squared = length_squared(to);
        const float inverse_distance = rsqrtf(distance_squared);
        out.wi = inverse_distance * to;
        out.distance = distance_squared * inverse_distance;
        const float cos_light = -dot(out.wi, make_float3(e.nx, e.ny, e.nz));
        if (!(cos_light > 0.0f))
        {
            return false;
        }
        out.pdf = distance_squared / (cos_light * e.size);
        return true;
    }
    const float3 to_center = corner - x;
    const float distance_squared = sphere_distance_squared(to_center);
    const float radius_squared = e.size * e.size;
    if (!(distance_squared > radius_squared))
    {
        return false;
    }
    const float one_minus_cos_max = one_minus_cos_theta_max(e.size, distance_squared);
    float s, c;
    sincospif(2.0f * a, &s, &c);
    const float one_minus_z = b * one_minus_cos_max;
    const float sin_squared = one_minus_z * (2.0f - one_minus_z);
    const float sin_theta = sqrtf(sin_squared);
    const float cos_theta = 1.0f - one_minus_z;
    const float inverse_distance = rsqrtf(distance_squared);
    out.wi = around(inverse_distance * to_center, make_float3(c * sin_theta, s * sin_theta, cos_theta));
    const float distance = distance_squared * inverse_distance;
    out.distance = distance * cos_theta - sqrtf(fmaxf(0.0f, fmaf(-distance_squared, sin_squared, radius_squared)));
    out.pdf = 1.0f / (2.0f * pi_f * one_minus_cos_max);
    return true;
}

// lamp_pdf (lamps.cuh:136-146), for a ray from x that hit lamp e at `distance`
__device__ float lamp_pdf(const emitter20& e, float3 x, float3 unit_dir, float distance)
{
    if (e.kind == RT_LIGHT_QUAD)
    {
        const float cos_light = -dot(unit_dir, make_float3(e.nx, e.ny, e.nz));
        return cos_light > 0.0f ? distance * distance / (cos_light * e.size) : 0.0f;
    }
    const float distance_squared = sphere_distance_squared(make_float3(e.cx, e.cy, e.cz) - x);
    return distance_squared > e.size * e.size
               ? 1.0f / (2.0f * pi_f * one_minus_cos_theta_max(e.size, distance_squared))
               : 0.0f;
}

// ---- the camera (camera.cuh:53-107) -----------------------------------------------------------------------------
__device__ __forceinline__ void camera_ray(const camera_params& cam, int i, int j, int s_i, int s_j, float4 u,
                                           float3& origin, float3& direction)
{
    const float dx = (static_cast<float>(s_i) + u.x) * cam.recip_sqrt_spp - 0.5f;
    const float dy = (static_cast<float>(s_j) + u.y) * cam.recip_sqrt_spp - 0.5f;
    const float3 to_sample = f3v(cam.center_to_pixel00) + (static_cast<float>(i) + dx) * f3v(cam.delta_u) +
                             (static_cast<float>(j) + dy) * f3v(cam.delta_v);
    origin = f3v(cam.center);
    direction = to_sample;
    if (cam.defocus)
    {
        // A uniform point of the unit disk: r = sqrt(u), angle 2 pi v (random.cuh:110-120)
        const float r = sqrtf(u.z);
        float s, c;
        sincospif(2.0f * u.w, &s, &c);
        const float3 lens = (r * c) * f3v(cam.disk_u) + (r * s) * f3v(cam.disk_v);
        origin = origin + lens;
        direction = to_sample - lens;
    }
}

__device__ __forceinline__ float3 sky(const camera_params& cam, float3 direction)
{
    const float a = 0.5f * (unit_vector(direction).y + 1.0f);
    return (1.0f - a) * f3v(cam.sky_bottom) + a * f3v(cam.sky_top);
}

__device__ __forceinline__ double without_nan(float x) { return static_cast<double>(x == x ? x : 0.0f); }

// ---- one path: its state between segments ----------------------------------------------------------------------
struct path_state
{
    float3 o, d;
    float3 throughput;
    float3 radiance; // the NEE/MIS integrator's light found so far
    float bsdf_pdf;  // the density of d at a vertex that took a light sample; 0 otherwise
    bool specular;   // d left the camera or a delta vertex: an escape sees the map filtered
    int rays_left;
    int depth;       // rays traced so far in this sample (the next vertex's depth in the RNG counter)
    int from;
    bool inward;
    float time;      // the moment in the shutter the sample's rays are at (0 in a scene where nothing moves)
};

// The hit as the shading needs it: point, outward normal, material, the hit's side
struct surface
{
    float3 p;
    float3 outward;
    float3 normal;
    float3 color; // the material's color here: its texture read at the hit, or its one solid color
    int material;
    int from;     // the next ray's `from`: the hit primitive, or -1 after a particle of smoke (which has no surface)
};

// The texture coordinates of a point of a sphere (sphere.cuh:119-135): the longitude and latitude of its outward
// normal turned back by the instances' turn, u from -x around y, v from the south pole
__device__ __forceinline__ void sphere_uv(float3 outward, const sphere_frame& f, float& u, float& v)
{
    const float nx = f.cos_theta * outward.x - f.sin_theta * outward.z;
    const float nz = f.sin_theta * outward.x + f.cos_theta * outward.z;
    const float phi = atan2f(-nz, nx) + pi_f;
    const float theta = acosf(fminf(fmaxf(-outward.y, -1.0f), 1.0f));
    u = phi * (0.5f * inverse_pi_f);
    v = theta * inverse_pi_f;
}

// The hit point moved onto the sphere by one Newton step along the outward normal, for a checker to read
// (onto_sphere, sphere.cuh:137-168): f = |p|^2 - 2 p.c + k with k = |c|^2 - r^2 from the host, taken only while its
// rounding bound stays below the frame's limit 2 r |c|
__device__ __forceinline__ float3 onto_sphere(float3 p, float3 outward, float4 ball, const sphere_frame& f)
{
    const float3 c = make_float3(ball.x, ball.y, ball.z);
    const float p_p = dot(p, p);
    const float p_c = dot(p, c);
    if (!(p_p + 2.0f * fabsf(p_c) + fabsf(f.k) < f.limit))
    {
        return p;
    }
    const float value = p_p - 2.0f * p_c + f.k;
    return p - (value / (2.0f * fabsf(ball.w))) * outward;
}

// The hit as the shading needs it (surface_at, camera.cuh:171-253), and the material there with its color
template <bool FEATURES = true>
__device__ __forceinline__ surface surface_at(const scene_view& S, const path_state& ps, const hit_info& h,
                                              material12& m)
{
    surface s;
    s.from = h.id;
    float u = 0.0f, v = 0.0f;
    float4 ball = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    bool on_sphere = false;
    if (FEATURES && h.id >= S.medium_base)
    {
        // A particle of smoke (constant_medium::hit): any normal and side will do, the CPU's (1, 0, 0) and the front
        s.p = ps.o + h.t * ps.d;
        s.outward = make_float3(1.0f, 0.0f, 0.0f);
        s.normal = s.outward;
        s.material = S.media[h.id - S.medium_base].material;
        s.from = -1;
        m = S.materials[s.material];
    }
    else
    {
        s.material = __ldg(S.prim_material + h.id);
        m = S.materials[s.material];
        if (h.id < S.quad_base)
        {
            ball = sphere_at<FEATURES>(S, h.id, ps.time);
            on_sphere = true;
            s.p = ps.o + h.t * ps.d;
            s.outward = (1.0f / fabsf(ball.w)) * (s.p - make_float3(ball.x, ball.y, ball.z));
        }
        else if (h.id < S.triangle_base)
        {
            // The quad's point as the CPU computes it, t * d rounded, then the sum (camera.cuh:175-195 at_unfused)
            const quad_v q = load_quad(S.quads, h.id - S.quad_base);
            s.p = make_float3(__fadd_rn(ps.o.x, __fmul_rn(h.t, ps.d.x)), __fadd_rn(ps.o.y, __fmul_rn(h.t, ps.d.y)),
                              __fadd_rn(ps.o.z, __fmul_rn(h.t, ps.d.z)));
            s.outward = q.n;
            if (FEATURES && m.texture >= 0 && (m.texture_needs & texture_needs_uv) != 0)
            {
                // quad_uv (quad.cuh:86-94): alpha and beta of the point, from hit_quad's expressions
                const float3 rel = h.t * ps.d - (q.q - ps.o);
                u = dot(rel, q.a);
                v = dot(rel, q.b);
            }
        }
        else
        {
            const triangle_v tr = load_triangle(S.triangles, h.id - S.triangle_base);
            s.p = ps.o + h.t * ps.d;
            s.outward = unit_vector(cross(tr.b - tr.a, tr.c - tr.a));
        }
        s.normal = h.front ? s.outward : -s.outward;
    }
    s.color = make_float3(m.r, m.g, m.b);
    if (FEATURES && m.texture >= 0)
    {
        float3 point = s.p;
        if (on_sphere && (m.texture_needs & (texture_needs_uv | texture_needs_point)) != 0)
        {
            const sphere_frame f = S.sphere_frames[h.id];
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

enum class step_result
{
    go_on,
    done,
};

// One segment of a books' path (camera.cuh:364-437 trace_ray with diffuse_bounce 304-359 and scatter
// material.cuh:84-126), after its closest hit
template <bool FEATURES = true>
__device__ __forceinline__ step_result shade_books(const scene_view& S, const camera_params& cam, const sampler& rng,
                                                   path_state& ps, const hit_info& h, float3& sample)
{
    if (h.id < 0)
    {
        sample = ps.throughput * sky(cam, ps.d);
        return step_result::done;
    }
    material12 m;
    const surface s = surface_at<FEATURES>(S, ps, h, m);
    const float3 albedo = s.color;
    float3 direction;
    if (m.kind == RT_DIFFUSE_LIGHT)
    {
        sample = h.front ? ps.throughput * albedo : make_float3(0.0f, 0.0f, 0.0f);
        return step_result::done;
    }
    const float4 u = rng.draw(ps.depth, block_material);
    if (m.kind == RT_LAMBERTIAN || m.kind == RT_ISOTROPIC)
    {
        // A diffuse bounce (diffuse_bounce, camera.cuh:300-359): a matte surface, or a particle of smoke, which keeps
        // its own density (1/(4 pi) everywhere) except under the lights strategy (isotropic::mixes_in_lights is false)
        const bool matte = m.kind == RT_LAMBERTIAN;
        int strategy = cam.sampling;
        if (!matte && strategy != RT_SAMPLING_LIGHTS)
        {
            strategy = RT_SAMPLING_MATERIAL;
        }
        if (strategy == RT_SAMPLING_MATERIAL)
        {
            direction = matte ? around(s.normal, random_cosine_direction(u.x, u.y)) : random_unit_vector(u.x, u.y);
            if (matte && !(dot(s.normal, direction) > 0.0f))
            {
                sample = make_float3(0.0f, 0.0f, 0.0f);
                return step_result::done;
            }
            ps.throughput = ps.throughput * albedo;
        }
        else
        {
            bool toward_lights = strategy == RT_SAMPLING_LIGHTS;
            if (strategy == RT_SAMPLING_MIXTURE)
            {
                toward_lights = u.z < 0.5f;
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
            const float p_scatter = matte ? cosine_density(s.normal, direction) : uniform_sphere_density;
            float p = uniform_sphere_density;
            if (strategy != RT_SAMPLING_UNIFORM)
            {
                const float p_lights = lights_pdf_value(S, s.p, direction, s.from);
                p = strategy == RT_SAMPLING_LIGHTS ? p_lights : 0.5f * p_lights + 0.5f * p_scatter;
            }
            if (!(p > 0.0f) || !(p_scatter > 0.0f))
            {
                sample = make_float3(0.0f, 0.0f, 0.0f);
                return step_result::done;
            }
            ps.throughput = (p_scatter / p) * (ps.throughput * albedo);
        }
    }
    else if (m.kind == RT_METAL)
    {
        direction = unit_vector(reflect(ps.d, s.normal)) + m.fuzz * random_unit_vector(u.x, u.y);
        if (dot(direction, s.normal) <= 0.0f)
        {
            sample = make_float3(0.0f, 0.0f, 0.0f);
            return step_result::done;
        }
        ps.throughput = ps.throughput * albedo;
    }
    else // dielectric
    {
        const float ri = h.front ? 1.0f / m.ior : m.ior;
        const float3 ud = unit_vector(ps.d);
        const float cos_theta = fminf(dot(-ud, s.normal), 1.0f);
        const float sin_theta = sqrtf(1.0f - cos_theta * cos_theta);
        const bool cannot_refract = ri * sin_theta > 1.0f;
        direction = cannot_refract || reflectance(cos_theta, ri) > u.z ? reflect(ud, s.normal)
                                                                       : refract(ud, s.normal, ri);
    }
    if (--ps.rays_left == 0)
    {
        sample = make_float3(0.0f, 0.0f, 0.0f);
        return step_result::done;
    }
    ps.o = s.p;
    ps.d = direction;
    ps.from = s.from;
    ps.inward = dot(direction, s.outward) < 0.0f;
    return step_result::go_on;
}

// ---- GGX (ggx.cuh: Walter et al. 2007, Heitz 2014 and 2018, Dupuy & Benyoub 2023, Turquin 2019) --------------
constexpr float min_ggx_alpha = 1e-3f; // below it, the perfect mirror with Schlick's F (ggx.cuh:37)

__constant__ float ggx_energy_table[32 * 32] = {RTB_GGX_ENERGY_TABLE};

__device__ __forceinline__ float smith_a(float c, float alpha2) { return sqrtf(fmaf(c * c, 1.0f - alpha2, alpha2)); }

// D(h) = alpha^2 / (pi (alpha^2 c^2 + sin^2)^2), sin^2 from |n x h|^2 (exact near the peak)
__device__ __forceinline__ float ggx_d(float3 n, float3 h, float alpha2)
{
    const float c = dot(n, h);
    if (!(c > 0.0f))
    {
        return 0.0f;
    }
    const float3 s = cross(n, h);
    const float d = fmaf(alpha2 * c, c, dot(s, s));
    return alpha2 * inverse_pi_f / (d * d);
}

__device__ __forceinline__ float3 schlick(float3 f0, float cosine)
{
    const float x = fmaxf(0.0f, 1.0f - cosine);
    const float x2 = x * x;
    const float x5 = x2 * x2 * x;
    return make_float3(fmaf(1.0f - f0.x, x5, f0.x), fmaf(1.0f - f0.y, x5, f0.y), fmaf(1.0f - f0.z, x5, f0.z));
}

// f * cos(theta_l) = F D cl / (2 (cl A_v + cv A_l)) and the visible-normal density D / (2 (cv + A_v))
__device__ float3 ggx_eval(float3 n, float3 v, float3 l, float alpha, float3 f0, float& pdf)
{
    pdf = 0.0f;
    const float cv = dot(n, v);
    const float cl = dot(n, l);
    const float3 sum = v + l;
    const float len2 = length_squared(sum);
    if (!(cv > 0.0f) || !(cl > 0.0f) || !(len2 > 0.0f))
    {
        return make_float3(0.0f, 0.0f, 0.0f);
    }
    const float3 h = rsqrtf(len2) * sum;
    const float alpha2 = alpha * alpha;
    const float d = ggx_d(n, h, alpha2);
    const float av = smith_a(cv, alpha2);
    const float al = smith_a(cl, alpha2);
    pdf = d / (2.0f * (cv + av));
    return (d * cl / (2.0f * (cl * av + cv * al))) * schlick(f0, dot(v, h));
}

// A direction by the visible normals with spherical caps: u1 the azimuth, u2 the height in the cap; weight
// F G2/G1 (at most F); false: absorbed
__device__ bool ggx_sample(float3 n, float3 v, float alpha, float3 f0, float u1, float u2, float3& l, float3& weight,
                           float& pdf)
{
    const float cv = dot(n, v);
    if (!(cv > 0.0f))
    {
        return false;
    }
    const float3 vs = unit_vector(alpha * (v - cv * n) + cv * n);
    const float zs = dot(n, vs);
    const float z = fmaf(1.0f - u2, 1.0f + zs, -zs);
    const float sin_theta = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    float s, c;
    sincospif(2.0f * u1, &s, &c);
    const float3 cap = around(n, make_float3(sin_theta * c, sin_theta * s, z));
    const float3 hs = cap + vs;
    const float hn = dot(n, hs);
    const float3 m = alpha * (hs - hn * n) + fmaxf(0.0f, hn) * n;
    const float m2 = length_squared(m);
    if (!(m2 > 0.0f))
    {
        return false;
    }
    const float3 h = rsqrtf(m2) * m;
    const float vh = dot(v, h);
    l = (2.0f * vh) * h - v;
    const float cl = dot(n, l);
    if (!(cl > 0.0f) || !(vh > 0.0f))
    {
        return false;
    }
    const float alpha2 = alpha * alpha;
    const float av = smith_a(cv, alpha2);
    const float al = smith_a(cl, alpha2);
    weight = (cl * (cv + av) / (cl * av + cv * al)) * schlick(f0, vh);
    pdf = ggx_d(n, h, alpha2) / (2.0f * (cv + av));
    return true;
}

// Turquin's factor 1 + F0 (1 - E) / E, E from the energy table (bilinear; nodes sqrt(mu) = i/31, r = j/31)
__device__ float3 ggx_compensation(float3 f0, float cos_v, float roughness)
{
    constexpr int last = 31;
    const float x = sqrtf(fminf(fmaxf(cos_v, 0.0f), 1.0f)) * static_cast<float>(last);
    const float y = fminf(fmaxf(roughness, 0.0f), 1.0f) * static_cast<float>(last);
    const int i = min(static_cast<int>(x), last - 1);
    const int j = min(static_cast<int>(y), last - 1);
    const float fx = x - static_cast<float>(i);
    const float fy = y - static_cast<float>(j);
    const float* row = ggx_energy_table + j * 32 + i;
    const float below = (1.0f - fx) * row[0] + fx * row[1];
    const float above = (1.0f - fx) * row[32] + fx * row[33];
    const float e = fminf((1.0f - fy) * below + fy * above, 1.0f);
    const float lost = (1.0f - e) / e;
    return make_float3(fmaf(f0.x, lost, 1.0f), fmaf(f0.y, lost, 1.0f), fmaf(f0.z, lost, 1.0f));
}

constexpr float gloss_coat_f0 = 0.04f;
constexpr float gloss_diffuse_scale = 0.37200738f; // 28 / (23 pi) * (1 - 0.04)

__device__ __forceinline__ float gloss_crossing(float c)
{
    const float x = 1.0f - 0.5f * c;
    const float x2 = x * x;
    return 1.0f - x2 * x2 * x;
}

// The coat over a matte base of color rho: GGX with F0 0.04 plus the coupled diffuse term; pdf the half-and-half
// mixture of the two lobes' densities
__device__ float3 gloss_eval(float3 n, float3 v, float3 l, float alpha, float3 rho, float& pdf)
{
    pdf = 0.0f;
    const float cv = dot(n, v);
    const float cl = dot(n, l);
    if (!(cv > 0.0f) || !(cl > 0.0f))
    {
        return make_float3(0.0f, 0.0f, 0.0f);
    }
    float coat_pdf;
    const float3 coat = ggx_eval(n, v, l, alpha, make_float3(gloss_coat_f0, gloss_coat_f0, gloss_coat_f0), coat_pdf);
    pdf = 0.5f * (coat_pdf + cl * inverse_pi_f);
    const float base = gloss_diffuse_scale * (gloss_crossing(cl) * gloss_crossing(cv)) * cl;
    return coat + base * rho;
}

// ---- the environment map (environment.cuh, background.cuh) ---------------------------------------------------
__device__ __forceinline__ float3 to_map(const environment_view& e, float3 d)
{
    return make_float3(e.cos_yaw * d.x + e.sin_yaw * d.z, d.y, -e.sin_yaw * d.x + e.cos_yaw * d.z);
}

__device__ __forceinline__ float3 from_map(const environment_view& e, float3 d)
{
    return make_float3(e.cos_yaw * d.x - e.sin_yaw * d.z, d.y, e.sin_yaw * d.x + e.cos_yaw * d.z);
}

// u = 0.5 + atan2(z, x) / (2 pi) across, t = atan2(sqrt(x^2 + z^2), y) / pi down: +y up, seen from inside
__device__ __forceinline__ void map_coordinates(float3 m, float& u, float& t)
{
    u = 0.5f + atan2f(m.z, m.x) * (0.5f * inverse_pi_f);
    t = atan2f(sqrtf(m.x * m.x + m.z * m.z), m.y) * inverse_pi_f;
}

__device__ __forceinline__ int clamp_index(int k, int n) { return k < 0 ? 0 : (k < n ? k : n - 1); }

// The one map from a direction to its cell, used by escapes and light samples alike
__device__ __forceinline__ int env_cell(const environment_view& e, float3 world)
{
    float u, t;
    map_coordinates(to_map(e, world), u, t);
    const int i = clamp_index(static_cast<int>(u * static_cast<float>(e.width)), e.width);
    const int j = clamp_index(static_cast<int>(t * static_cast<float>(e.height)), e.height);
    return j * e.width + i;
}

__device__ __forceinline__ float3 env_radiance(const environment_view& e, float3 dir, float& pdf)
{
    const env_texel texel = e.texels[env_cell(e, dir)];
    pdf = texel.pdf;
    return e.scale * make_float3(texel.r, texel.g, texel.b);
}

__device__ float3 env_radiance_filtered(const environment_view& e, float3 dir)
{
    float u, t;
    map_coordinates(to_map(e, dir), u, t);
    const float x = u * static_cast<float>(e.width) - 0.5f;
    const float y = t * static_cast<float>(e.height) - 0.5f;
    const float x0 = floorf(x);
    const float y0 = floorf(y);
    const float fx = x - x0;
    const float fy = y - y0;
    const int i = static_cast<int>(x0);
    const int i0 = i < 0 ? i + e.width : i;
    const int i1 = i0 + 1 < e.width ? i0 + 1 : 0;
    const int j = static_cast<int>(y0);
    const int j0 = clamp_index(j, e.height) * e.width;
    const int j1 = clamp_index(j + 1, e.height) * e.width;
    const auto texel = [&](int k) {
        const env_texel t4 = e.texels[k];
        return make_float3(t4.r, t4.g, t4.b);
    };
    const float3 a = texel(j0 + i0);
    const float3 b = texel(j0 + i1);
    const float3 c = texel(j1 + i0);
    const float3 d = texel(j1 + i1);
    const float3 top = a + fx * (b - a);
    const float3 bottom = c + fx * (d - c);
    return e.scale * (top + fy * (bottom - top));
}

// A cell from the alias table (the bin from the top bits of `bits`, then its coin), then a direction uniform over
// the cell's solid angle; the radiance and density of the cell the direction lands in
__device__ bool sample_environment(const environment_view& e, uint32_t bits, float coin, float s_theta, float s_phi,
                                   float3& wi, float3& le, float& pdf)
{
    const int bin = static_cast<int>(bits >> (32 - e.log2_bins));
    const alias_bin b = e.bins[bin];
    const int cell = coin < b.q ? bin : b.alias;
    const int j = cell / e.width;
    const int i = cell - j * e.width;
    const float top = e.row_cos[j];
    const float bottom = e.row_cos[j + 1];
    const float cos_theta = top - s_theta * (top - bottom);
    const float sin_theta = sqrtf(fmaxf(0.0f, (1.0f - cos_theta) * (1.0f + cos_theta)));
    float sp, cp;
    sincospif(2.0f * (static_cast<float>(i) + s_phi) / static_cast<float>(e.width) - 1.0f, &sp, &cp);
    wi = from_map(e, make_float3(sin_theta * cp, cos_theta, sin_theta * sp));
    le = env_radiance(e, wi, pdf);
    return pdf > 0.0f;
}

// ---- the NEE/MIS step (quality_path.cuh:83-188, bsdf.cuh:30-201, light_sampler.cuh:40-103) -------------------
enum lobe_id : int
{
    lobe_lambertian,
    lobe_isotropic,
    lobe_conductor,
    lobe_gloss,
    lobe_smooth_conductor, // from here on: delta lobes (no density)
    lobe_books_delta,
};

__device__ __forceinline__ int lobe_of(const material12& m)
{
    if (m.lobe == RT_MICROFACET_CONDUCTOR)
    {
        return m.alpha >= min_ggx_alpha ? lobe_conductor : lobe_smooth_conductor;
    }
    if (m.lobe == RT_MICROFACET_GLOSS)
    {
        return lobe_gloss;
    }
    return m.kind == RT_LAMBERTIAN ? lobe_lambertian : m.kind == RT_ISOTROPIC ? lobe_isotropic : lobe_books_delta;
}

// eval_bsdf: f * |cos| of a light sample's unit direction, and the lobe's density of it (0 for delta lobes)
__device__ float3 eval_lobe(int lobe, const material12& m, float3 albedo, float3 n, float3 wo, float3 wi, float& pdf)
{
    if (lobe == lobe_lambertian)
    {
        pdf = cosine_density(n, wi);
        return pdf * albedo;
    }
    if (lobe == lobe_isotropic)
    {
        pdf = uniform_sphere_density;
        return uniform_sphere_density * albedo;
    }
    if (lobe == lobe_conductor)
    {
        const float3 single = ggx_eval(n, wo, wi, m.alpha, albedo, pdf);
        return ggx_compensation(albedo, dot(n, wo), m.roughness) * single;
    }
    if (lobe == lobe_gloss)
    {
        return gloss_eval(n, wo, wi, m.alpha, albedo, pdf);
    }
    pdf = 0.0f;
    return make_float3(0.0f, 0.0f, 0.0f);
}

// A shadow ray handed back to the caller instead of traced (the wavefront's trace kernel walks it): the ray, and the
// light it brings to the path's radiance if nothing blocks it
struct shadow_query
{
    float3 o, d;
    float3 contribution;
    float t_max;
    int from;
    int skip;
    bool inward;
    bool lit;
};

// One segment of an NEE/MIS path after its closest hit; the shadow ray is traced here, or with DEFER handed back in
// `deferred` (lit set) with the path's radiance left without it: a `done` sample then is the radiance once the
// caller has added the light
template <bool COUNT, int SEARCH = search_any, bool FEATURES = true, bool DEFER = false>
__device__ __forceinline__ step_result shade_quality(const scene_view& S, const camera_params& cam,
                                                     const sampler& rng, path_state& ps, const hit_info& h,
                                                     float3& sample, uint32_t& shadow_rays, fetch_counts* counts,
                                                     shadow_query* deferred = nullptr)
{
    if (h.id < 0)
    {
        // The environment (filtered after the camera and delta vertices, the nearest texel with its density
        // otherwise), or the camera's sky
        if (!S.has_environment)
        {
            sample = ps.radiance + ps.throughput * sky(cam, ps.d);
            return step_result::done;
        }
        if (ps.specular)
        {
            sample = ps.radiance + ps.throughput * env_radiance_filtered(S.env, ps.d);
            return step_result::done;
        }
        float density;
        const float3 le = env_radiance(S.env, ps.d, density);
        const float p_light = S.env.sampled ? S.light_pmf * density : 0.0f;
        const float w = ps.bsdf_pdf > 0.0f ? bsdf_weight(S.combination, ps.bsdf_pdf, p_light) : 1.0f;
        sample = ps.radiance + w * (ps.throughput * le);
        return step_result::done;
    }
    material12 m;
    const surface s = surface_at<FEATURES>(S, ps, h, m);
    const float3 albedo = s.color;
    if (m.kind == RT_DIFFUSE_LIGHT)
    {
        float w = 1.0f;
        if (ps.bsdf_pdf > 0.0f)
        {
            const int k = S.lamp_count > 0 ? __ldg(S.lamp_of + h.id) : -1;
            float p_light = 0.0f;
            if (k >= 0)
            {
                const float distance = h.t * sqrtf(length_squared(ps.d));
                p_light = S.light_pmf * lamp_pdf(S.lamps[k], ps.o, unit_vector(ps.d), distance);
            }
            w = bsdf_weight(S.combination, ps.bsdf_pdf, p_light);
        }
        sample = ps.radiance + w * (h.front ? ps.throughput * albedo : make_float3(0.0f, 0.0f, 0.0f));
        return step_result::done;
    }
    const int lobe = lobe_of(m);
    const bool delta = lobe >= lobe_smooth_conductor;
    const float3 wo = -unit_vector(ps.d);
    const int lights = S.lamp_count + (S.env.sampled ? 1 : 0);
    const bool nee = S.combination != RT_COMBINE_BSDF_ONLY && ps.rays_left > 1 && !delta && lights > 0 &&
                     largest_channel(ps.throughput) > 0.0f;
    bool lit = false;
    float3 contribution = make_float3(0.0f, 0.0f, 0.0f);
    float3 light_dir = make_float3(0.0f, 0.0f, 0.0f);
    float light_distance = infinity_f;
    int skip = -1;
    if (nee)
    {
        // One number picks a light, the lamps first and the map last (light_sampler.cuh:40-75)
        const uint4 bits = rng.draw_bits(ps.depth, block_nee);
        const float pick = to_unit(bits.x);
        int k = static_cast<int>(pick * static_cast<float>(lights));
        k = k < lights ? k : lights - 1;
        bool drawn = false;
        float3 le;
        float p_light = 0.0f;
        if (k < S.lamp_count)
        {
            const emitter20 e = S.lamps[k];
            lamp_sample ls;
            if (sample_lamp(e, s.p, to_unit(bits.y), to_unit(bits.z), ls))
            {
                drawn = true;
                light_dir = ls.wi;
                light_distance = ls.distance;
                le = make_float3(e.er, e.eg, e.eb);
                p_light = S.light_pmf * ls.pdf;
                skip = e.primitive;
            }
        }
        else
        {
            float density;
            const float s_phi = rng.draw(ps.depth, block_nee + 1).x;
            if (sample_environment(S.env, bits.y, to_unit(bits.z), to_unit(bits.w), s_phi, light_dir, le, density))
            {
                drawn = true;
                p_light = S.light_pmf * density;
            }
        }
        if (drawn)
        {
            float p_bsdf;
            const float3 f = eval_lobe(lobe, m, albedo, s.normal, wo, light_dir, p_bsdf);
            if (p_light > 0.0f && largest_channel(f) > 0.0f)
            {
                contribution =
                    (light_weight(S.combination, p_light, p_bsdf) / p_light) * (ps.throughput * (f * le));
                const float sum = contribution.x + contribution.y + contribution.z;
                lit = sum > 0.0f && sum < infinity_f;
            }
        }
    }
    // The material's own sample: the path's next ray
    const float4 u = rng.draw(ps.depth, block_material);
    float3 wi = make_float3(0.0f, 0.0f, 0.0f);
    float3 weight = albedo;
    float pdf = 0.0f;
    bool scattered = true;
    if (lobe == lobe_lambertian)
    {
        wi = around(s.normal, random_cosine_direction(u.x, u.y));
        scattered = dot(s.normal, wi) > 0.0f;
        pdf = cosine_density(s.normal, wi);
    }
    else if (lobe == lobe_isotropic)
    {
        wi = random_unit_vector(u.x, u.y);
        pdf = uniform_sphere_density;
    }
    else if (lobe == lobe_conductor)
    {
        scattered = ggx_sample(s.normal, wo, m.alpha, albedo, u.x, u.y, wi, weight, pdf);
        if (scattered)
        {
            weight = weight * ggx_compensation(albedo, dot(s.normal, wo), m.roughness);
        }
    }
    else if (lobe == lobe_gloss)
    {
        // The coat or the base, half the time each, then the mixture's weight and density (ggx.cuh:300-324)
        if (u.z < 0.5f)
        {
            float3 coat_weight;
            float coat_pdf;
            scattered = ggx_sample(s.normal, wo, m.alpha, make_float3(gloss_coat_f0, gloss_coat_f0, gloss_coat_f0),
                                   u.x, u.y, wi, coat_weight, coat_pdf);
        }
        else
        {
            wi = around(s.normal, random_cosine_direction(u.x, u.y));
            scattered = dot(s.normal, wi) > 0.0f;
        }
        if (scattered)
        {
            const float3 f = gloss_eval(s.normal, wo, wi, m.alpha, albedo, pdf);
            scattered = pdf > 0.0f;
            weight = (1.0f / pdf) * f;
        }
    }
    else if (lobe == lobe_smooth_conductor)
    {
        // The mirror with Schlick's F: no random number (bsdf.cuh:153-166)
        scattered = dot(s.normal, wo) > 0.0f;
        wi = unit_vector(reflect(-wo, s.normal));
        weight = schlick(albedo, dot(s.normal, wo));
    }
    else if (m.kind == RT_METAL)
    {
        wi = unit_vector(reflect(ps.d, s.normal)) + m.fuzz * random_unit_vector(u.x, u.y);
        scattered = dot(wi, s.normal) > 0.0f;
    }
    else // dielectric
    {
        const float ri = h.front ? 1.0f / m.ior : m.ior;
        const float3 ud = unit_vector(ps.d);
        const float cos_theta = fminf(dot(-ud, s.normal), 1.0f);
        const float sin_theta = sqrtf(1.0f - cos_theta * cos_theta);
        wi = ri * sin_theta > 1.0f || reflectance(cos_theta, ri) > u.z ? reflect(ud, s.normal)
                                                                       : refract(ud, s.normal, ri);
        weight = make_float3(1.0f, 1.0f, 1.0f);
    }
    if (DEFER)
    {
        deferred->lit = lit;
        if (lit)
        {
            ++shadow_rays;
            *deferred = {s.p, light_dir, contribution, light_distance, s.from, skip, dot(light_dir, s.outward) < 0.0f,
                         true};
        }
    }
    else if (lit)
    {
        ++shadow_rays;
        hit_info blocker;
        const bool blocked = traverse<true, COUNT, SEARCH, FEATURES>(
            S, s.p, light_dir, ps.time, light_distance, s.from, dot(light_dir, s.outward) < 0.0f, skip, blocker, counts);
        if (!blocked)
        {
            // through smoke, the light arrives with the chance of crossing it (its expected value, not a draw)
            const float through =
                FEATURES && S.medium_count > 0 ? transmittance(S, s.p, light_dir, ps.time, light_distance) : 1.0f;
            ps.radiance = ps.radiance + through * contribution;
        }
    }
    if (!scattered)
    {
        sample = ps.radiance;
        return step_result::done;
    }
    ps.throughput = ps.throughput * weight;
    ps.bsdf_pdf = nee ? pdf : 0.0f;
    ps.specular = delta;
    if (S.combination != RT_COMBINE_BSDF_ONLY && ps.throughput.x == 0.0f && ps.throughput.y == 0.0f &&
        ps.throughput.z == 0.0f)
    {
        sample = ps.radiance;
        return step_result::done;
    }
    if (--ps.rays_left == 0)
    {
        sample = ps.radiance;
        return step_result::done;
    }
    ps.o = s.p;
    ps.d = wi;
    ps.from = s.from;
    ps.inward = dot(wi, s.outward) < 0.0f;
    return step_result::go_on;
}

// ---- the persistent render kernel ------------------------------------------------------------------------------
// The render kernel's resident blocks per multiprocessor, which caps its registers: the books' integrator at 64 (8
// blocks of 128 threads measured fastest against 5 and 6 blocks, for the latency they hide), the NEE/MIS integrator,
// whose GGX and environment code spills heavily at 64, at 80 (6 blocks); with the flat search (no tree stack) both
// at 72 (7 blocks), measured fastest against 5, 6 and 8 on the Cornell boxes
#ifndef RTB_MIN_BLOCKS
#define RTB_MIN_BLOCKS 8
#endif
#ifndef RTB_MIN_BLOCKS_QUALITY
#define RTB_MIN_BLOCKS_QUALITY 6
#endif
#ifndef RTB_MIN_BLOCKS_FLAT
#define RTB_MIN_BLOCKS_FLAT 7
#endif
#ifndef RTB_MIN_BLOCKS_QUALITY_FLAT
#define RTB_MIN_BLOCKS_QUALITY_FLAT 7
#endif
// The kernels of scenes with the second book's features (textures, motion, smoke): 96 registers (5 blocks), measured
// fastest against 72 and 80 on the final, smoke, perlin and light scenes (their textures and free flights spill)
#ifndef RTB_MIN_BLOCKS_FEATURES
#define RTB_MIN_BLOCKS_FEATURES 5 // 0: as the kernel without the features
#endif

// Where sample number `local` of a launch (or of a batch job) lies: pass-major, then the pixels in 8x4 tiles (a
// warp's worth); x may fall past the image's right edge or y past its bottom in the last tiles
struct sample_place
{
    int64_t pass;
    int x, y;
};

// (uses the camera's divisors: cam.div_padded and cam.div_tiles_x; a number of 2^32 or more, which only a served
// request's numbering reaches, takes the 64-bit division)
__device__ __forceinline__ sample_place place_of(int64_t local, const camera_params& cam, int64_t pass_begin)
{
    const uint32_t padded = cam.div_padded.d;
    int64_t j;
    int q;
    if (local < (int64_t{1} << 32))
    {
        const auto n = static_cast<uint32_t>(local);
        const uint32_t jj = quotient(n, cam.div_padded);
        j = jj;
        q = static_cast<int>(n - jj * padded);
    }
    else
    {
        j = local / padded;
        q = static_cast<int>(local - j * padded);
    }
    const int tile = q >> 5;
    const int l = q & 31;
    const auto ty = static_cast<int>(quotient(static_cast<uint32_t>(tile), cam.div_tiles_x));
    const int tx = tile - ty * static_cast<int>(cam.div_tiles_x.d);
    return {pass_begin + j, tx * 8 + (l & 7), ty * 4 + (l >> 3)};
}

// A pass's round of strata and its pass within the round (cam.div_round_passes)
__device__ __forceinline__ int64_t round_of(int64_t pass, const camera_params& cam)
{
    return pass < (int64_t{1} << 32) ? static_cast<int64_t>(quotient(static_cast<uint32_t>(pass), cam.div_round_passes))
                                     : pass / static_cast<int64_t>(cam.div_round_passes.d);
}

// A sample's random-number stream: its pixel, its pass within its round of strata, and the round's key
// (seed + round * 2^32), as the persistent kernel sets them when it starts the sample
__device__ __forceinline__ int sample_rng(const sample_place& at, const camera_params& cam, uint64_t seed, sampler& rng)
{
    const int64_t round = round_of(at.pass, cam);
    const int round_pass = static_cast<int>(at.pass - round * static_cast<int64_t>(cam.div_round_passes.d));
    const uint64_t key = seed + (static_cast<uint64_t>(round) << 32);
    rng.key = make_uint2(static_cast<uint32_t>(key), static_cast<uint32_t>(key >> 32));
    rng.pass = static_cast<uint32_t>(round_pass);
    rng.pixel = static_cast<uint32_t>(at.y) * static_cast<uint32_t>(cam.width) + static_cast<uint32_t>(at.x);
    return round_pass;
}

template <bool QUALITY, bool FLAT, bool FEATURES>
constexpr int render_min_blocks()
{
    if (FEATURES && RTB_MIN_BLOCKS_FEATURES > 0)
    {
        return RTB_MIN_BLOCKS_FEATURES;
    }
    return QUALITY ? (FLAT ? RTB_MIN_BLOCKS_QUALITY_FLAT : RTB_MIN_BLOCKS_QUALITY)
                   : (FLAT ? RTB_MIN_BLOCKS_FLAT : RTB_MIN_BLOCKS);
}

// FEATURES: the scene has moving spheres, textures other than solid colors, or smoke (the counting build always
// compiles them in)
template <bool QUALITY, bool COUNT, bool FLAT, bool FEATURES>
__global__ void __launch_bounds__(render_block, render_min_blocks<QUALITY, FLAT, FEATURES>())
    render_kernel(const __grid_constant__ launch_params P)
{
    __shared__ unsigned long long block_rays;
    __shared__ unsigned long long block_shadow_rays;
    if (threadIdx.x == 0)
    {
        block_rays = 0;
        block_shadow_rays = 0;
    }
    __syncthreads();

    const unsigned lane = threadIdx.x & 31u;
    const unsigned lanes_below = (1u << lane) - 1u;
    const camera_params& cam = P.cam;

    uint32_t rays = 0;
    uint32_t shadow_rays = 0;
    fetch_counts counts;
    bool need = true;
    bool start = false;
    int px = 0, py = 0;
    int64_t pass = 0, pass_end = 0;
    int64_t slot = 0;
    double acc_r = 0.0, acc_g = 0.0, acc_b = 0.0;
    sampler rng{};
    rng.job = P.job;
    path_state ps{};

    while (true)
    {
        // Claim work for the lanes that need it: one atomic per warp
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
                    break; // no work left for this lane
                }
                const sample_place at = place_of(static_cast<int64_t>(item), cam, 0);
                const int64_t k = at.pass; // the item's chunk within the launch
                const int q = static_cast<int>(static_cast<int64_t>(item) - k * P.padded_pixels);
                px = at.x;
                py = at.y;
                if (px >= cam.width || py >= cam.height)
                {
                    continue; // a lane of a tile that hangs over the image's edge: nothing to render
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
            // A new sample: pass n is pass n % k^2 of round n / k^2, whose numbers come from seed + round * 2^32
            const int64_t round = round_of(pass, cam);
            const int in_round = static_cast<int>(pass - round * P.round_passes);
            const uint64_t key = P.seed + (static_cast<uint64_t>(round) << 32);
            rng.key = make_uint2(static_cast<uint32_t>(key), static_cast<uint32_t>(key >> 32));
            rng.pass = static_cast<uint32_t>(in_round);
            const float4 u = rng.draw(0, 0);
            int s_i, s_j;
            stratum_of(cam, in_round, s_i, s_j);
            camera_ray(cam, px, py, s_i, s_j, u, ps.o, ps.d);
            // the moment in the shutter, in a scene where something moves (camera.ixx get_ray's ray time)
            ps.time = FEATURES && P.scene.has_motion ? rng.draw(0, block_time).x : 0.0f;
            ps.throughput = make_float3(1.0f, 1.0f, 1.0f);
            ps.radiance = make_float3(0.0f, 0.0f, 0.0f);
            ps.bsdf_pdf = 0.0f;
            ps.specular = true;
            ps.rays_left = cam.max_depth;
            ps.depth = 0;
            ps.from = -1;
            ps.inward = false;
            start = false;
        }

        // One segment: the closest event (a surface, or a particle of smoke before it), then the vertex's shading
        constexpr int search = FLAT ? search_flat : search_tree;
        hit_info h;
        traverse<false, COUNT, search, FEATURES>(P.scene, ps.o, ps.d, ps.time, infinity_f, ps.from, ps.inward, -1,
                                                 h, &counts);
        ++rays;
        ++ps.depth;
        if (FEATURES && P.scene.medium_count > 0)
        {
            media_event(P.scene, ps.o, ps.d, ps.time, rng, ps.depth, h);
        }
        float3 sample;
        const step_result r =
            QUALITY ? shade_quality<COUNT, search, FEATURES>(P.scene, cam, rng, ps, h, sample, shadow_rays, &counts)
                    : shade_books<FEATURES>(P.scene, cam, rng, ps, h, sample);
        if (r == step_result::done)
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
    if (COUNT)
    {
        atomicAdd(P.counters + 2, static_cast<unsigned long long>(counts.nodes));
        atomicAdd(P.counters + 3, static_cast<unsigned long long>(counts.spheres));
        atomicAdd(P.counters + 4, static_cast<unsigned long long>(counts.quads));
        atomicAdd(P.counters + 5, static_cast<unsigned long long>(counts.triangles));
    }
    atomicAdd(&block_rays, static_cast<unsigned long long>(rays));
    if (QUALITY)
    {
        atomicAdd(&block_shadow_rays, static_cast<unsigned long long>(shadow_rays));
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        atomicAdd(P.counters, block_rays);
        if (QUALITY)
        {
            atomicAdd(P.counters + 1, block_shadow_rays);
        }
    }
}

// Adds each pixel's chunk partials to its sums, in chunk order (the sums are plain doubles in HBM, 24 bytes a pixel)
__global__ void reduce_kernel(const reduce_params P)
{
    const int x = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    const int y = static_cast<int>(blockIdx.y);
    if (x >= P.width || y >= P.height)
    {
        return;
    }
    const int q = ((y >> 2) * P.tiles_x + (x >> 3)) * 32 + ((y & 3) << 3) + (x & 7);
    double* sum = P.sums + 3 * (static_cast<int64_t>(y) * P.width + x);
    double r = sum[0], g = sum[1], b = sum[2];
    for (int k = 0; k < P.chunks; ++k)
    {
        const double* part = P.partials + 3 * (static_cast<int64_t>(k) * P.padded_pixels + q);
        r += part[0];
        g += part[1];
        b += part[2];
    }
    sum[0] = r;
    sum[1] = g;
    sum[2] = b;
}

// ---- batched launches: many jobs (requests), each its own scene, camera and passes, in one persistent kernel ------

// The job of jobs [first, end) whose range of the batch's item (or pixel) space holds `index`: a binary search over
// the jobs' starts
constexpr int job_items = 0;   // find_job by item_begin
constexpr int job_pixels = 1;  // by pixel_begin
constexpr int job_samples = 2; // by sample_begin (a wavefront group's sample space)

template <int SPACE>
__device__ __forceinline__ int find_job(const batch_job* jobs, int first, int end, int64_t index, int mask = 0)
{
    int lo = first;
    int hi = end - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        const batch_job& j = jobs[mask != 0 ? (mid & mask) : mid]; // a stream run's ring: [first, end) unwrapped
        const int64_t begin = SPACE == job_pixels    ? j.pixel_begin
                              : SPACE == job_samples ? j.sample_begin
                                                     : j.item_begin;
        if (begin <= index)
        {
            lo = mid;
        }
        else
        {
            hi = mid - 1;
        }
    }
    return lo;
}

// The same loop as render_kernel, with the job of each work item looked up in the job table: the jobs' items follow
// each other in one item space, so the persistent threads pull work from every job at once, and a small job's tail
// fills with another's work. Each job may use either integrator. The jobs of flat scenes come first in the table and
// the item space, and each search has its own launch (FLAT: items [0, flat_items) of jobs [0, flat_jobs); otherwise
// the rest), compiled as render_kernel's for that search, so a job renders the same bits as its plain render.
template <bool FLAT, bool FEATURES>
__global__ void __launch_bounds__(render_block, render_min_blocks<true, FLAT, FEATURES>())
    render_batch_kernel(const batch_params P)
{
    constexpr int search = FLAT ? search_flat : search_tree;
    constexpr int group = batch_group(FLAT, FEATURES);
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lanes_below = (1u << lane) - 1u;
    const int64_t item_begin = P.header->group_items[group];
    const int64_t total_items = P.header->group_items[group + 1];
    const int job_first = P.header->group_jobs[group];
    const int job_end = P.header->group_jobs[group + 1];
    unsigned long long* const work_counter = P.work_counter + group;

    uint32_t rays = 0;
    uint32_t shadow_rays = 0;
    bool need = true;
    bool start = false;
    int px = 0, py = 0;
    int64_t pass = 0, pass_end = 0;
    int64_t slot = 0;
    double acc_r = 0.0, acc_g = 0.0, acc_b = 0.0;
    const batch_job* J = nullptr;
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
                base = atomicAdd(work_counter, static_cast<unsigned long long>(__popc(needing)));
            }
            base = __shfl_sync(active, base, leader);
            if (need)
            {
                const auto item = item_begin + static_cast<int64_t>(base + __popc(needing & lanes_below));
                if (item >= total_items)
                {
                    break;
                }
                J = P.jobs + find_job<job_items>(P.jobs, job_first, job_end, item);
                const int64_t local = item - J->item_begin;
                const sample_place at = place_of(local, J->cam, 0);
                const int64_t k = at.pass; // the item's chunk within the step
                const int q = static_cast<int>(local - k * J->padded_pixels);
                px = at.x;
                py = at.y;
                if (px >= J->cam.width || py >= J->cam.height)
                {
                    continue;
                }
                const int64_t chunk_first = (J->first_chunk + k) * J->chunk;
                pass = chunk_first > J->pass_begin ? chunk_first : J->pass_begin;
                const int64_t chunk_end = chunk_first + J->chunk;
                pass_end = chunk_end < J->pass_end ? chunk_end : J->pass_end;
                slot = k * J->padded_pixels + q;
                acc_r = acc_g = acc_b = 0.0;
                rng.pixel = static_cast<uint32_t>(py) * static_cast<uint32_t>(J->cam.width) + static_cast<uint32_t>(px);
                rng.job = J->job;
                rays = 0;
                shadow_rays = 0;
                need = false;
                start = true;
            }
        }
        const camera_params& cam = J->cam;
        if (start)
        {
            const int64_t round = round_of(pass, cam);
            const int in_round = static_cast<int>(pass - round * J->round_passes);
            const uint64_t key = J->seed + (static_cast<uint64_t>(round) << 32);
            rng.key = make_uint2(static_cast<uint32_t>(key), static_cast<uint32_t>(key >> 32));
            rng.pass = static_cast<uint32_t>(in_round);
            const float4 u = rng.draw(0, 0);
            int s_i, s_j;
            stratum_of(cam, in_round, s_i, s_j);
            camera_ray(cam, px, py, s_i, s_j, u, ps.o, ps.d);
            ps.time = FEATURES && J->scene.has_motion ? rng.draw(0, block_time).x : 0.0f;
            ps.throughput = make_float3(1.0f, 1.0f, 1.0f);
            ps.radiance = make_float3(0.0f, 0.0f, 0.0f);
            ps.bsdf_pdf = 0.0f;
            ps.specular = true;
            ps.rays_left = cam.max_depth;
            ps.depth = 0;
            ps.from = -1;
            ps.inward = false;
            start = false;
        }
        hit_info h;
        traverse<false, false, search, FEATURES>(J->scene, ps.o, ps.d, ps.time, infinity_f, ps.from, ps.inward, -1,
                                                 h);
        ++rays;
        ++ps.depth;
        if (FEATURES && J->scene.medium_count > 0)
        {
            media_event(J->scene, ps.o, ps.d, ps.time, rng, ps.depth, h);
        }
        float3 sample;
        const step_result r =
            J->quality
                ? shade_quality<false, search, FEATURES>(J->scene, cam, rng, ps, h, sample, shadow_rays, nullptr)
                : shade_books<FEATURES>(J->scene, cam, rng, ps, h, sample);
        if (r == step_result::done)
        {
            acc_r += without_nan(sample.x);
            acc_g += without_nan(sample.y);
            acc_b += without_nan(sample.z);
            if (++pass == pass_end)
            {
                double* out = J->partials + 3 * slot;
                out[0] = acc_r;
                out[1] = acc_g;
                out[2] = acc_b;
                atomicAdd(J->counters, static_cast<unsigned long long>(rays));
                if (shadow_rays)
                {
                    atomicAdd(J->counters + 1, static_cast<unsigned long long>(shadow_rays));
                }
                need = true;
            }
            else
            {
                start = true;
            }
        }
    }
}

// Every job's pixels, in one grid-stride pass: each pixel's chunk partials added to its job's sums in chunk order
__global__ void reduce_batch_kernel(const batch_params P)
{
    const int64_t total = P.header->total_pixels;
    const int job_count = P.header->job_count;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    {
        const batch_job& J = P.jobs[find_job<job_pixels>(P.jobs, 0, job_count, i)];
        const int64_t local = i - J.pixel_begin;
        const int y = static_cast<int>(local / J.cam.width);
        const int x = static_cast<int>(local - static_cast<int64_t>(y) * J.cam.width);
        const int q = ((y >> 2) * J.tiles_x + (x >> 3)) * 32 + ((y & 3) << 3) + (x & 7);
        double* sum = J.sums + 3 * local;
        double r = sum[0], g = sum[1], b = sum[2];
        for (int k = 0; k < J.chunks; ++k)
        {
            const double* part = J.partials + 3 * (static_cast<int64_t>(k) * J.padded_pixels + q);
            r += part[0];
            g += part[1];
            b += part[2];
        }
        sum[0] = r;
        sum[1] = g;
        sum[2] = b;
    }
}

__global__ void closest_hits_kernel(const scene_view S, const float* origins, const float* directions, int64_t count,
                                    const int32_t* prim_source, int32_t* ids, float* ts)
{
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count)
    {
        return;
    }
    const float3 o = make_float3(origins[3 * i], origins[3 * i + 1], origins[3 * i + 2]);
    const float3 d = make_float3(directions[3 * i], directions[3 * i + 1], directions[3 * i + 2]);
    hit_info h;
    traverse<false>(S, o, d, 0.0f, infinity_f, -1, false, -1, h);
    ids[i] = h.id >= 0 ? prim_source[h.id] : -1;
    ts[i] = h.id >= 0 ? h.t : infinity_f;
}

__global__ void camera_rays_kernel(const camera_params cam, uint64_t seed, int64_t pass, int32_t round_passes,
                                   float* origins, float* directions)
{
    const int x = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    const int y = static_cast<int>(blockIdx.y);
    if (x >= cam.width || y >= cam.height)
    {
        return;
    }
    const int64_t round = pass / round_passes;
    const int in_round = static_cast<int>(pass - round * round_passes);
    const uint64_t key = seed + (static_cast<uint64_t>(round) << 32);
    sampler rng{make_uint2(static_cast<uint32_t>(key), static_cast<uint32_t>(key >> 32)),
                static_cast<uint32_t>(y) * static_cast<uint32_t>(cam.width) + static_cast<uint32_t>(x),
                static_cast<uint32_t>(in_round), 0u};
    float3 o, d;
    camera_ray(cam, x, y, in_round % cam.sqrt_spp, in_round / cam.sqrt_spp, rng.draw(0, 0), o, d);
    const int64_t i = static_cast<int64_t>(y) * cam.width + x;
    origins[3 * i] = o.x;
    origins[3 * i + 1] = o.y;
    origins[3 * i + 2] = o.z;
    directions[3 * i] = d.x;
    directions[3 * i + 1] = d.y;
    directions[3 * i + 2] = d.z;
}

// ---- the wavefront form: resident path slots, a shade kernel and a trace kernel ----------------------------------
// In the persistent kernel a warp walks the tree for all its lanes' rays together, and a lane whose ray left the
// scene at the root waits for the lane whose ray goes deepest: on the mesh and the sphere grids a walk step runs with
// 4 to 10 of 32 lanes. Here the walk is a kernel of its own whose lanes take a new ray as soon as theirs is answered
// (Aila and Laine's persistent while-while with replacement of finished rays, HPG 2009 and its 2012 addendum), and the
// paths between walks live in HBM as slots. A slot goes through the same steps, in the same order and with the same
// arithmetic, as a persistent kernel's lane: the images are the persistent kernel's.
constexpr uint32_t wave_exhausted = 1u; // no work item left for the slot
constexpr uint32_t wave_ext = 2u;       // the path's next ray is queued (its hit comes back in ext_result)
constexpr uint32_t wave_shadow = 4u;    // a shadow ray is queued (blocked or not comes back in shadow_result)
constexpr uint32_t wave_finish = 8u;    // the sample ended at the shadow ray's vertex: it completes once the ray is in

// A slot in HBM, structure of arrays: five float4 rows of the path and its sample, three of its pending shadow ray,
// each row slot_count long, so that a warp's loads and stores of a row are 512 contiguous bytes. Rows: the ray's
// origin and time; its direction and the last BSDF density; the throughput and the radiance's red; the radiance's
// green and blue, the primitive the ray leaves and the rays left; the depth, the flags, the sample's number and the
// job. The sample's pass, pixel and random-number key are not stored: they follow from its number (sample_rng).
constexpr int wave_rows = 5;
constexpr int wave_shadow_rows = 3;
constexpr int wave_flags_row = 4; // depth, flags, sample, job: a slot whose row is zero has no sample
// A query's flags (its meta's second word): 1 the ray starts inside the surface it leaves, 2 a shadow ray, 4 a new
// sample's camera ray still to be made (a primary query); the job above them (<< 3)
constexpr int wave_query_primary = 4;
constexpr uint32_t wave_specular = 1u << 8;
constexpr uint32_t wave_inward = 1u << 9;
constexpr uint32_t wave_reserved = 1u << 10; // a stream run's slot holds a claim beyond what is published (its number
                                             // in the flags row's last two words) and waits for it

constexpr unsigned full_warp = 0xffffffffu;

// The slots, queries, answers and samples pass through L2 once per step: loaded and stored evict-first (.cs), so that
// they do not push the tree and the primitives, which every walk reads, out of L2
#ifndef RTB_WAVE_STREAMING
#define RTB_WAVE_STREAMING 1
#endif
template <class T>
__device__ __forceinline__ T stream_load(const T* p)
{
#if RTB_WAVE_STREAMING
    return __ldcs(p);
#else
    return *p;
#endif
}
template <class T>
__device__ __forceinline__ void stream_store(T* p, T v)
{
#if RTB_WAVE_STREAMING
    __stcs(p, v);
#else
    *p = v;
#endif
}

// The shade kernel's resident blocks per multiprocessor: 0 takes the persistent kernel's for the integrator
#ifndef RTB_WAVE_SHADE_MIN_BLOCKS
#define RTB_WAVE_SHADE_MIN_BLOCKS 0
#endif
template <bool QUALITY, bool FEATURES>
constexpr int wave_shade_min_blocks()
{
    return RTB_WAVE_SHADE_MIN_BLOCKS > 0 ? RTB_WAVE_SHADE_MIN_BLOCKS : render_min_blocks<QUALITY, false, FEATURES>();
}


// A slot's step: the last walk's answers, the shading, the sample's end, a new sample, the next rays queued.
// BATCH: the slots render the samples of a group of batch jobs (W), each slot its job's scene, camera and integrator
// (with QUALITY each job's own, picked at run time; without, a group of books' jobs only, compiled without the NEE/MIS
// code); otherwise the launch's one view (P). A batch kernel keeps the NEE/MIS kernels' register budget either way:
// at the books' tighter one its per-job loads spill.
// Every load of the slot's rows and answer is issued at the start, before any of them is needed, so the step waits
// for one round trip to memory, not one for the flags and another for what they say to read.
template <bool QUALITY, bool FEATURES, bool BATCH>
__global__ void __launch_bounds__(render_block, wave_shade_min_blocks<QUALITY || BATCH, FEATURES>())
    wave_shade_kernel(const __grid_constant__ launch_params P, const __grid_constant__ wave_buffers B,
                      const __grid_constant__ wave_batch W)
{
    const int n = B.slot_count;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lanes_below = (1u << lane) - 1u;
    float4* rows = static_cast<float4*>(B.slots);
    float4* shadow_rows = rows + static_cast<int64_t>(wave_rows) * n;
    const int own = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    // The slot's rows and its answer: all loads issued together while samples are left to claim (nearly every slot
    // has work); once every sample is claimed (the drain) the flags first, and the rest only for a slot with work
    float4 r0, r1, r2, r3;
    int4 r5, answer; // r5: the flags row
    // Compact slots, in a session's launch of a scene without the second book's features (nothing moves, so no time;
    // no job; the rays left are max_depth - depth): the depth and the six flags in one word of the flags row, which
    // also holds the sample's number, the primitive left and one more value. The books' paths carry no NEE radiance
    // or density: three rows, (origin, throughput x), (direction, throughput y), flags row (..., throughput z). The
    // NEE/MIS paths: four, (origin, NEE density), (direction, radiance r), (throughput, radiance g), flags row (...,
    // radiance b). A camera ray the trace kernel writes into rows 0 and 1 leaves their last words 0: no density, no
    // radiance. Row 3 (and for the books row 2) is neither read nor written.
    constexpr bool compact_slots = !BATCH && !FEATURES;
    constexpr bool books_slots = compact_slots && !QUALITY;
    int compact_from = -1;
    float compact_last = 0.0f; // the flags row's last word: throughput z (books) or radiance b (NEE/MIS)
    const auto load_flags = [&] {
        r5 = stream_load(reinterpret_cast<const int4*>(rows) + wave_flags_row * n + own);
        if constexpr (compact_slots)
        {
            // into the five-row form's (depth, flags, sample, job)
            const auto w = static_cast<uint32_t>(r5.x);
            compact_from = r5.z;
            compact_last = __int_as_float(r5.w);
            const uint32_t f = ((w & 1u) ? wave_ext : 0u) | ((w & 2u) ? wave_exhausted : 0u) |
                               ((w & 4u) ? wave_inward : 0u) | ((w & 8u) ? wave_specular : 0u) |
                               ((w & 16u) ? wave_shadow : 0u) | ((w & 32u) ? wave_finish : 0u);
            r5 = make_int4(static_cast<int>(w >> 6), static_cast<int>(f), r5.y, 0);
        }
    };
    const auto load_rest = [&] {
        r0 = stream_load(rows + own);
        r1 = stream_load(rows + n + own);
        if constexpr (!books_slots)
        {
            r2 = stream_load(rows + 2 * n + own);
        }
        if constexpr (!compact_slots)
        {
            r3 = stream_load(rows + 3 * n + own);
        }
        answer = stream_load(B.ext_result + own);
    };
    if (!B.draining)
    {
        load_rest();
        load_flags();
    }
    else
    {
        load_flags();
        if ((static_cast<uint32_t>(r5.y) & wave_exhausted) == 0u)
        {
            load_rest();
        }
        else
        {
            r0 = r1 = r2 = r3 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            answer = make_int4(0, 0, 0, 0);
        }
    }
    const int i = own; // the slot this thread shades
    uint32_t flags = static_cast<uint32_t>(r5.y);
    uint32_t shadow_rays = 0; // counted where the walks are (the trace kernel), or as queued (BATCH)
    // Samples may be claimed below `limit`: the launch's count, or what a stream run's host has published
    const bool stream_run = BATCH && W.published != nullptr;
    const unsigned long long limit =
        stream_run ? __ldcg(W.published) : static_cast<unsigned long long>(B.sample_count);
    const int2 window =
        stream_run ? __ldcg(reinterpret_cast<const int2*>(W.window)) : make_int2(W.job_first, W.job_end);
    // a warp whose slots have all run out of work has nothing left to do in this launch
    if (!__all_sync(full_warp, (flags & wave_exhausted) != 0u))
    {
        const bool live = (flags & wave_exhausted) == 0u;
        // the slot's job: its scene, camera and numbers (a session's launch: the launch's own)
        int job = BATCH && (flags & wave_reserved) == 0u ? r5.w : 0;
        const batch_job* J = BATCH ? W.jobs + job : nullptr;
        const auto scene = [&]() -> const scene_view& {
            if constexpr (BATCH)
            {
                return J->scene;
            }
            else
            {
                return P.scene;
            }
        };
        const auto camera = [&]() -> const camera_params& {
            if constexpr (BATCH)
            {
                return J->cam;
            }
            else
            {
                return P.cam;
            }
        };
        const auto quality = [&]() -> bool {
            if constexpr (BATCH)
            {
                return QUALITY && J->quality != 0; // a group of books' jobs only: no NEE/MIS code
            }
            else
            {
                return QUALITY;
            }
        };
        path_state ps;
        sampler rng;
        shadow_query sq;
        int64_t sample_index = 0, pass = 0;
        int px = 0, py = 0; // the pixel of a sample claimed in this step (a slot's camera ray needs no more)
        bool need = false;
        bool start = false;
        bool ready = false;             // a stream run's reservation the host has since published
        unsigned long long reserved = 0;
        int finished_job = -1;          // a stream run's segment whose sample this slot finished
        bool primary = false; // a new sample whose camera ray the trace kernel makes (wave_camera_query)
        int round_pass = 0;   // its pass within its round of strata
        rng.job = BATCH ? J->job : P.job;
        if (live)
        {
            ps.o = make_float3(r0.x, r0.y, r0.z);
            ps.time = r0.w;
            ps.d = make_float3(r1.x, r1.y, r1.z);
            ps.depth = r5.x;
            if constexpr (books_slots)
            {
                ps.time = 0.0f;
                ps.throughput = make_float3(r0.w, r1.w, compact_last);
                ps.bsdf_pdf = 0.0f;
                ps.radiance = make_float3(0.0f, 0.0f, 0.0f);
                ps.from = compact_from;
                ps.rays_left = camera().max_depth - ps.depth;
            }
            else if constexpr (compact_slots)
            {
                ps.time = 0.0f;
                ps.bsdf_pdf = r0.w;
                ps.throughput = make_float3(r2.x, r2.y, r2.z);
                ps.radiance = make_float3(r1.w, r2.w, compact_last);
                ps.from = compact_from;
                ps.rays_left = camera().max_depth - ps.depth;
            }
            else
            {
                ps.throughput = make_float3(r2.x, r2.y, r2.z);
                ps.bsdf_pdf = r1.w;
                ps.radiance = make_float3(r2.w, r3.x, r3.y);
                ps.from = __float_as_int(r3.z);
                ps.rays_left = __float_as_int(r3.w);
            }
            ps.specular = (flags & wave_specular) != 0u;
            ps.inward = (flags & wave_inward) != 0u;
            sample_index = static_cast<int64_t>(static_cast<uint32_t>(r5.z));
            if (flags & (wave_ext | wave_shadow | wave_finish))
            {
                // the sample's stream, from its number
                const int64_t local = sample_index + (BATCH ? J->local_begin : 0);
                const sample_place at = place_of(local, camera(), BATCH ? J->pass_begin : P.pass_begin);
                sample_rng(at, camera(), BATCH ? J->seed : P.seed, rng);
            }
            bool finished = false;
            float3 sample = make_float3(0.0f, 0.0f, 0.0f);
            if (flags & wave_shadow)
            {
                if (stream_load(B.shadow_result + i) == 0)
                {
                    const float4 q0 = stream_load(shadow_rows + i);
                    const float4 q1 = stream_load(shadow_rows + n + i);
                    const int4 q2 = stream_load(reinterpret_cast<const int4*>(shadow_rows) + 2 * n + i);
                    const float3 contribution = make_float3(q1.w, __int_as_float(q2.x), __int_as_float(q2.y));
                    // through smoke, the light arrives with the chance of crossing it (its expected value)
                    const float through =
                        FEATURES && scene().medium_count > 0
                            ? transmittance(scene(), make_float3(q0.x, q0.y, q0.z), make_float3(q1.x, q1.y, q1.z),
                                            ps.time, q0.w)
                            : 1.0f;
                    ps.radiance = ps.radiance + through * contribution;
                }
                flags &= ~wave_shadow;
            }
            if (flags & wave_finish)
            {
                sample = ps.radiance;
                finished = true;
                flags &= ~wave_finish;
            }
            else if (flags & wave_ext)
            {
                const int4 r = answer;
                hit_info h;
                h.id = r.x;
                h.t = __int_as_float(r.y);
                h.front = r.z != 0;
                ++ps.depth;
                if (FEATURES && scene().medium_count > 0)
                {
                    media_event(scene(), ps.o, ps.d, ps.time, rng, ps.depth, h);
                }
                step_result res;
                if (quality())
                {
                    sq.lit = false; // a vertex that ends the path before its light sample queues no shadow ray
                    res = shade_quality<false, search_tree, FEATURES, true>(scene(), camera(), rng, ps, h, sample,
                                                                            shadow_rays, nullptr, &sq);
                    if (sq.lit)
                    {
                        flags |= wave_shadow;
                    }
                }
                else
                {
                    res = shade_books<FEATURES>(scene(), camera(), rng, ps, h, sample);
                }
                if (res == step_result::done)
                {
                    flags &= ~wave_ext;
                    if (flags & wave_shadow)
                    {
                        flags |= wave_finish; // the sample's value waits for its last shadow ray
                    }
                    else
                    {
                        finished = true;
                    }
                }
            }
            else if (BATCH && (flags & wave_reserved))
            {
                // a stream run's claim made before the host published it: taken below once it has
                const unsigned long long held =
                    static_cast<unsigned long long>(static_cast<uint32_t>(r5.z)) |
                    (static_cast<unsigned long long>(static_cast<uint32_t>(r5.w)) << 32);
                if (held < limit)
                {
                    reserved = held;
                    ready = true;
                }
                else
                {
                    sample_index = static_cast<uint32_t>(held);
                    job = static_cast<int>(held >> 32);
                }
            }
            else
            {
                need = true; // a slot without a sample
            }
            if (finished)
            {
                // the sample's value, added into its chunk's partial in pass order by the reduction
                const float4 value = make_float4(sample.x, sample.y, sample.z, 0.0f);
                if (stream_run)
                {
                    stream_store(J->values + sample_index, value);
                    finished_job = job; // counted below, one atomic per segment per warp
                }
                else
                {
                    stream_store(B.samples + (BATCH ? J->sample_begin : 0) + sample_index, value);
                }
                need = true;
            }
        }
        if (stream_run)
        {
            // the warp's finished samples counted per segment: the host reduces a segment once all are in
            const unsigned peers = __match_any_sync(full_warp, finished_job);
            if (finished_job >= 0 && (peers & lanes_below) == 0u)
            {
                atomicAdd(W.jobs[finished_job].done, static_cast<unsigned long long>(__popc(peers)));
            }
        }
        // A stream run's segment (logical number) holding sample s: `hint` first (a warp's claims are consecutive
        // numbers, nearly always in its leader's segment), else a binary search over the ring of segment starts
        const auto find_segment = [&](int64_t s, int hint) -> int {
            const int mask = W.job_mask;
            if (hint >= window.x && hint < window.y && W.starts[hint & mask] <= s &&
                (hint + 1 >= window.y || s < W.starts[(hint + 1) & mask]))
            {
                return hint;
            }
            int lo = window.x, hi = window.y - 1;
            while (lo < hi)
            {
                const int mid = (lo + hi + 1) >> 1;
                if (W.starts[mid & mask] <= s)
                {
                    lo = mid;
                }
                else
                {
                    hi = mid - 1;
                }
            }
            return lo;
        };
        // Sample s taken by this slot: its job, its pixel and pass (false for a lane of a tile over the image's edge,
        // which claims again; in a stream run it counts as done, having no value to wait for)
        const auto take = [&](unsigned long long s, int hint) -> bool {
            int k = 0;
            if constexpr (BATCH)
            {
                k = stream_run ? (find_segment(static_cast<int64_t>(s), hint) & W.job_mask)
                               : find_job<job_samples>(W.jobs, window.x, window.y, static_cast<int64_t>(s));
            }
            const batch_job* K = BATCH ? W.jobs + k : nullptr;
            const camera_params& c = BATCH ? K->cam : P.cam;
            const int64_t index = static_cast<int64_t>(s) - (BATCH ? K->sample_begin : 0);
            if (stream_run && index < 0)
            {
                // below the window the host gave: a sample no entry holds; reported, never written
                atomicOr(B.control + 3, 1u);
                return false;
            }
            const sample_place at = place_of(index + (BATCH ? K->local_begin : 0), c, BATCH ? K->pass_begin : P.pass_begin);
            if (!(at.x < c.width && at.y < c.height))
            {
                if (stream_run)
                {
                    atomicAdd(K->done, 1ull);
                }
                return false;
            }
            px = at.x;
            py = at.y;
            job = k;
            J = K;
            sample_index = index;
            pass = at.pass;
            rng.job = BATCH ? K->job : P.job;
            start = true;
            return true;
        };
        if (ready)
        {
            flags &= ~wave_reserved;
            need = !take(reserved, -1);
        }
        // Samples for the slots that need one, a pass of the image after another (of each job after another): one
        // atomic per warp. In a stream run a claim beyond what is published waits in the slot (wave_reserved).
        while (true)
        {
            const unsigned needing = __ballot_sync(full_warp, need);
            if (needing == 0u)
            {
                break;
            }
            const int leader = __ffs(static_cast<int>(needing)) - 1;
            unsigned long long base = 0;
            if (static_cast<int>(lane) == leader)
            {
                base = atomicAdd(BATCH ? W.work_counter : P.work_counter,
                                 static_cast<unsigned long long>(__popc(needing)));
            }
            base = __shfl_sync(full_warp, base, leader);
            int hint = -1;
            if (stream_run)
            {
                if (static_cast<int>(lane) == leader && base < limit)
                {
                    hint = find_segment(static_cast<int64_t>(base), -1);
                }
                hint = __shfl_sync(full_warp, hint, leader);
            }
            if (need)
            {
                const unsigned long long s = base + static_cast<unsigned long long>(__popc(needing & lanes_below));
                if (s >= limit)
                {
                    if (stream_run)
                    {
                        flags |= wave_reserved;
                        sample_index = static_cast<uint32_t>(s);
                        job = static_cast<int>(s >> 32);
                    }
                    else
                    {
                        flags |= wave_exhausted;
                    }
                    need = false;
                }
                else
                {
                    need = !take(s, hint);
                }
            }
        }
        if (start)
        {
            // A new sample, as the persistent kernel starts one
            const camera_params& cam = camera();
            round_pass = sample_rng({pass, px, py}, cam, BATCH ? J->seed : P.seed, rng);
            // Under a tree walk and the heavier shading (NEE/MIS, the second book's features) the trace kernel makes
            // the camera ray, a warp's 32 at once, instead of this warp for its few new samples: the mesh +3.6%, the
            // second book's final scene +3.7%. The books' plain sphere scenes (-2%) and the flat searches (-3% to
            // -7%: their trace kernel's tail grows by it) make their own here.
            primary = (quality() || FEATURES) && scene().flat == 0;
            if (!primary)
            {
                const float4 u = rng.draw(0, 0);
                int s_i, s_j;
                stratum_of(cam, round_pass, s_i, s_j);
                camera_ray(cam, px, py, s_i, s_j, u, ps.o, ps.d);
                ps.time = FEATURES && scene().has_motion ? rng.draw(0, block_time).x : 0.0f;
            }
            ps.throughput = make_float3(1.0f, 1.0f, 1.0f);
            ps.radiance = make_float3(0.0f, 0.0f, 0.0f);
            ps.bsdf_pdf = 0.0f;
            ps.specular = true;
            ps.rays_left = cam.max_depth;
            ps.depth = 0;
            ps.from = -1;
            ps.inward = false;
            flags |= wave_ext;
        }
        // The slot's queries: one atomic per warp for its next rays and its shadow rays from the bottom of the queue,
        // one for its new samples' camera rays (primary queries) from the top down
        const bool ext = (flags & wave_ext) != 0u && !primary;
        const bool shadow = QUALITY && (flags & wave_shadow) != 0u;
        const unsigned ext_lanes = __ballot_sync(full_warp, ext);
        const unsigned shadow_lanes = __ballot_sync(full_warp, shadow);
        const unsigned primary_lanes = __ballot_sync(full_warp, primary);
        const int queued = __popc(ext_lanes) + __popc(shadow_lanes);
        if constexpr (BATCH)
        {
            // each job's segments and shadow rays, counted as queued: one atomic per job of the warp
            const bool any = ext || shadow || primary;
            const unsigned peers = __match_any_sync(full_warp, any ? job : -1);
            if (any && static_cast<int>(lane) == __ffs(static_cast<int>(peers)) - 1)
            {
                const unsigned e = __popc(peers & (ext_lanes | primary_lanes)), sh = __popc(peers & shadow_lanes);
                if (e)
                {
                    atomicAdd(J->counters, static_cast<unsigned long long>(e));
                }
                if (sh)
                {
                    atomicAdd(J->counters + 1, static_cast<unsigned long long>(sh));
                }
            }
        }
        if (queued > 0)
        {
            unsigned base = 0;
            if (lane == 0u)
            {
                base = atomicAdd(B.control, static_cast<unsigned>(queued));
            }
            base = __shfl_sync(full_warp, base, 0);
            if (ext)
            {
                const unsigned q = base + static_cast<unsigned>(__popc(ext_lanes & lanes_below));
                stream_store(B.query_o + q, make_float4(ps.o.x, ps.o.y, ps.o.z, ps.time));
                stream_store(B.query_d + q, make_float4(ps.d.x, ps.d.y, ps.d.z, infinity_f));
                stream_store(B.query_meta + q, make_int4(ps.from, (ps.inward ? 1 : 0) | (job << 3), -1, i));
            }
            if (shadow)
            {
                const unsigned q = base + static_cast<unsigned>(__popc(ext_lanes)) +
                                   static_cast<unsigned>(__popc(shadow_lanes & lanes_below));
                stream_store(B.query_o + q, make_float4(sq.o.x, sq.o.y, sq.o.z, ps.time));
                stream_store(B.query_d + q, make_float4(sq.d.x, sq.d.y, sq.d.z, sq.t_max));
                stream_store(B.query_meta + q, make_int4(sq.from, (sq.inward ? 1 : 0) | 2 | (job << 3), sq.skip, i));
                // what the next step needs of it: the light it brings and, through smoke, its segment
                stream_store(shadow_rows + i, make_float4(sq.o.x, sq.o.y, sq.o.z, sq.t_max));
                stream_store(shadow_rows + n + i, make_float4(sq.d.x, sq.d.y, sq.d.z, sq.contribution.x));
                stream_store(reinterpret_cast<int4*>(shadow_rows) + 2 * n + i,
                             make_int4(__float_as_int(sq.contribution.y), __float_as_int(sq.contribution.z), 0, 0));
            }
        }
        if (primary_lanes != 0u)
        {
            const int leader = __ffs(static_cast<int>(primary_lanes)) - 1;
            unsigned base = 0;
            if (static_cast<int>(lane) == leader)
            {
                base = atomicAdd(B.control + 2, static_cast<unsigned>(__popc(primary_lanes)));
            }
            base = __shfl_sync(full_warp, base, leader);
            if (primary)
            {
                // the pixel, the pass in its round and the RNG's key: what the camera ray is made of
                const unsigned q = 2u * static_cast<unsigned>(n) - 1u -
                                   (base + static_cast<unsigned>(__popc(primary_lanes & lanes_below)));
                stream_store(B.query_o + q, make_float4(__int_as_float(px), __int_as_float(py),
                                                        __int_as_float(round_pass), 0.0f));
                stream_store(B.query_d + q, make_float4(__uint_as_float(rng.key.x), __uint_as_float(rng.key.y), 0.0f,
                                                        infinity_f));
                stream_store(B.query_meta + q, make_int4(-1, wave_query_primary | (job << 3), -1, i));
            }
        }
        if (live)
        {
            flags = (flags & ~(wave_specular | wave_inward)) | (ps.specular ? wave_specular : 0u) |
                    (ps.inward ? wave_inward : 0u);
            // the compact forms' flags word: depth << 6 and the six flags
            const auto compact_word = [&](int depth) {
                return static_cast<int>((static_cast<uint32_t>(depth) << 6) | ((flags & wave_ext) ? 1u : 0u) |
                                        ((flags & wave_exhausted) ? 2u : 0u) | ((flags & wave_inward) ? 4u : 0u) |
                                        ((flags & wave_specular) ? 8u : 0u) | ((flags & wave_shadow) ? 16u : 0u) |
                                        ((flags & wave_finish) ? 32u : 0u));
            };
            if (flags & wave_exhausted)
            {
                stream_store(reinterpret_cast<int4*>(rows) + wave_flags_row * n + i,
                             compact_slots ? make_int4(compact_word(0), 0, 0, 0)
                                           : make_int4(0, static_cast<int>(flags), 0, 0));
            }
            else if constexpr (books_slots)
            {
                stream_store(rows + i, make_float4(ps.o.x, ps.o.y, ps.o.z, ps.throughput.x));
                stream_store(rows + n + i, make_float4(ps.d.x, ps.d.y, ps.d.z, ps.throughput.y));
                stream_store(reinterpret_cast<int4*>(rows) + wave_flags_row * n + i,
                             make_int4(compact_word(ps.depth), static_cast<int>(static_cast<uint32_t>(sample_index)),
                                       ps.from, __float_as_int(ps.throughput.z)));
            }
            else if constexpr (compact_slots)
            {
                stream_store(rows + i, make_float4(ps.o.x, ps.o.y, ps.o.z, ps.bsdf_pdf));
                stream_store(rows + n + i, make_float4(ps.d.x, ps.d.y, ps.d.z, ps.radiance.x));
                stream_store(rows + 2 * n + i,
                             make_float4(ps.throughput.x, ps.throughput.y, ps.throughput.z, ps.radiance.y));
                stream_store(reinterpret_cast<int4*>(rows) + wave_flags_row * n + i,
                             make_int4(compact_word(ps.depth), static_cast<int>(static_cast<uint32_t>(sample_index)),
                                       ps.from, __float_as_int(ps.radiance.z)));
            }
            else
            {
                stream_store(rows + i, make_float4(ps.o.x, ps.o.y, ps.o.z, ps.time));
                stream_store(rows + n + i, make_float4(ps.d.x, ps.d.y, ps.d.z, ps.bsdf_pdf));
                stream_store(rows + 2 * n + i,
                             make_float4(ps.throughput.x, ps.throughput.y, ps.throughput.z, ps.radiance.x));
                stream_store(rows + 3 * n + i, make_float4(ps.radiance.y, ps.radiance.z, __int_as_float(ps.from),
                                                           __int_as_float(ps.rays_left)));
                stream_store(reinterpret_cast<int4*>(rows) + wave_flags_row * n + i,
                             make_int4(ps.depth, static_cast<int>(flags), static_cast<int>(static_cast<uint32_t>(
                                                                              sample_index)),
                                       job));
            }
        }
    }
}

// The query at position q of the queue: the shade step's next rays and shadow rays fill it from the bottom (`lower`
// of them), its new samples' camera rays from the top down. A primary query (pixel, pass in its round, the RNG's key) is
// made into its camera ray here, the persistent kernel's start of a sample with the same random numbers, and the ray
// goes into its slot's first two rows, which the shade step that meets its hit reads.
template <bool FEATURES, bool BATCH>
__device__ __forceinline__ void wave_camera_query(const wave_buffers& B, const wave_batch& W, const scene_view& S0,
                                                  unsigned q, unsigned lower, float4& qo, float4& qd, int4& qm)
{
    const unsigned k = q < lower ? q : 2u * static_cast<unsigned>(B.slot_count) - 1u - (q - lower);
    qo = stream_load(B.query_o + k);
    qd = stream_load(B.query_d + k);
    qm = stream_load(B.query_meta + k);
    if (qm.y & wave_query_primary)
    {
        const batch_job* J = BATCH ? W.jobs + (qm.y >> 3) : nullptr;
        const camera_params& cam = BATCH ? J->cam : B.cam;
        const scene_view& S = BATCH ? J->scene : S0;
        const int px = __float_as_int(qo.x), py = __float_as_int(qo.y), round_pass = __float_as_int(qo.z);
        sampler rng;
        rng.key = make_uint2(__float_as_uint(qd.x), __float_as_uint(qd.y));
        rng.pixel = static_cast<uint32_t>(py) * static_cast<uint32_t>(cam.width) + static_cast<uint32_t>(px);
        rng.pass = static_cast<uint32_t>(round_pass);
        rng.job = BATCH ? J->job : B.job;
        float3 o, d;
        int s_i, s_j;
        stratum_of(cam, round_pass, s_i, s_j);
        camera_ray(cam, px, py, s_i, s_j, rng.draw(0, 0), o, d);
        const float time = FEATURES && S.has_motion ? rng.draw(0, block_time).x : 0.0f;
        float4* rows = static_cast<float4*>(B.slots);
        stream_store(rows + qm.w, make_float4(o.x, o.y, o.z, time));
        stream_store(rows + B.slot_count + qm.w, make_float4(d.x, d.y, d.z, 0.0f)); // bsdf_pdf 0 at the camera
        qo = make_float4(o.x, o.y, o.z, time);
        qd = make_float4(d.x, d.y, d.z, infinity_f);
        qm.y &= ~wave_query_primary;
    }
}

template <bool FEATURES>
__device__ __forceinline__ void flat_search(const scene_view& S, float3 o, float3 d, float time, int from, bool inward,
                                            int skip, bool any, hit_info& hit);
// The same, called rather than inlined: a walk compiled with the flat search inlined beside its own leaf tests rounds
// differently (the shared tests are contracted differently), and the walk must give a session's hits bit for bit
template <bool FEATURES>
__device__ __noinline__ void flat_search_call(const scene_view& S, float3 o, float3 d, float time, int from,
                                              bool inward, int skip, bool any, hit_info& hit);

// The trace kernel's resident blocks per multiprocessor (64 registers at 8) and the number of lanes still walking
// under which a warp stops to give its idle lanes new queries (the addendum's 20 of 32)
#ifndef RTB_TRACE_MIN_BLOCKS
#define RTB_TRACE_MIN_BLOCKS RTB_TRACE_MIN_BLOCKS_DEFAULT
#endif
#ifndef RTB_REFILL_LANES
#define RTB_REFILL_LANES 20
#endif

// The queued queries' walks through the tree: closest hits for the paths' next rays, any hit for shadow rays (the
// persistent kernel's traverse, the same leaf tests and self-intersection rules). WIDE: the tree four wide, a node's
// hit children visited nearest first (a four-key sorting network); otherwise the binary tree in the persistent
// kernel's node order. BATCH: each query walks its own job's scene (the job in its flags); otherwise the launch's
// scene S0. The walks are counted into `counters` when it is given.
template <bool FEATURES, bool BATCH, bool WIDE, int MINB = RTB_TRACE_MIN_BLOCKS>
__global__ void __launch_bounds__(render_block, MINB)
    wave_trace_kernel(const __grid_constant__ scene_view S0, const __grid_constant__ wave_buffers B,
                      const __grid_constant__ wave_batch W, unsigned long long* counters)
{
    __shared__ unsigned block_walks[2]; // the block's closest-hit and shadow queries: the path segments and shadow rays
    if (threadIdx.x < 2)
    {
        block_walks[threadIdx.x] = 0;
    }
    __syncthreads();
    const unsigned lower = B.control[0];
    const unsigned count = lower + B.control[2];
    unsigned walks[2] = {0, 0};
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lanes_below = (1u << lane) - 1u;
    int2 stack[WIDE ? wide_stack : max_bvh_depth];
    int sp = 0;
    int link = traversal_done;
    int leaf = 0;
    bool has_query = false;
    bool drained = false; // the warp found the queue empty: no idle lane can take a query any more
    float3 o = make_float3(0.0f, 0.0f, 0.0f);
    float3 d = o, inv = o, os = o;
    float time = 0.0f;
    float inverse_a = 0.0f;
    int from = -1, skip = -1, slot = 0;
    bool inward = false, shadow = false;
    hit_info hit{-1, 0.0f, false};
    // the scene the lane's query walks: its job's, or the launch's (a __grid_constant__ parameter, read in place)
    const scene_view* job_scene = BATCH ? &W.jobs[W.job_first].scene : &S0;
    const auto scene = [&]() -> const scene_view& { return *job_scene; };
    // the lane's tree, read from its scene once a query (a batch's scene is in global memory, where every read of it
    // in the walk would wait on L1 behind the stack's stores)
    const bvh_node* tree_nodes = scene().nodes;
    const bvh4_node* tree_wide = scene().wide_nodes;
    const auto pop = [&]() -> int {
        while (sp > 0)
        {
            const int2 e = stack[--sp];
            if (shadow || __int_as_float(e.y) < hit.t)
            {
                return e.x;
            }
        }
        return traversal_done;
    };
    // Warp-synchronous: every lane runs every loop, with nothing to do once its query is answered and the queue is
    // empty, so that each ballot sees the whole warp and the refill rule holds as written
    while (true)
    {
        const bool answered = has_query && link == traversal_done && leaf == 0;
        if (answered)
        {
            if (shadow)
            {
                stream_store(B.shadow_result + slot, hit.id >= 0 ? 1 : 0);
            }
            else
            {
                stream_store(B.ext_result + slot, make_int4(hit.id, __float_as_int(hit.t), hit.front ? 1 : 0, 0));
            }
            has_query = false;
        }
        // New queries for the idle lanes: one atomic per warp
        const unsigned idle = __ballot_sync(full_warp, !has_query);
        if (idle != 0u && !drained)
        {
            const int leader = __ffs(static_cast<int>(idle)) - 1;
            unsigned base = 0;
            if (static_cast<int>(lane) == leader)
            {
                base = atomicAdd(B.control + 1, static_cast<unsigned>(__popc(idle)));
            }
            base = __shfl_sync(full_warp, base, leader);
            drained = base + static_cast<unsigned>(__popc(idle)) >= count;
            const unsigned q = base + static_cast<unsigned>(__popc(idle & lanes_below));
            if (!has_query && q < count)
            {
                float4 qo, qd;
                int4 qm;
                wave_camera_query<FEATURES, BATCH>(B, W, S0, q, lower, qo, qd, qm);
                o = make_float3(qo.x, qo.y, qo.z);
                time = qo.w;
                d = make_float3(qd.x, qd.y, qd.z);
                hit.id = -1;
                hit.t = qd.w;
                hit.front = false;
                from = qm.x;
                inward = (qm.y & 1) != 0;
                shadow = (qm.y & 2) != 0;
                skip = qm.z;
                slot = qm.w;
                if constexpr (BATCH)
                {
                    job_scene = &W.jobs[qm.y >> 3].scene;
                    tree_nodes = scene().nodes;
                    tree_wide = scene().wide_nodes;
                }
                ++walks[shadow ? 1 : 0];
                inverse_a = 1.0f / length_squared(d);
                inv = make_float3(safe_inverse(d.x), safe_inverse(d.y), safe_inverse(d.z));
                os = make_float3(o.x * inv.x, o.y * inv.y, o.z * inv.z);
                sp = 0;
                leaf = 0;
                link = scene().node_count == 0 ? traversal_done : 0;
                has_query = true;
                if (BATCH && scene().flat != 0)
                {
                    // a flat-searched scene beside tree-searched ones (a stream run): its query answered here by the
                    // flat search, the same hits its session's flat trace kernel finds
                    flat_search_call<FEATURES>(scene(), o, d, time, from, inward, skip, shadow, hit);
                    link = traversal_done;
                }
            }
        }
        if (__ballot_sync(full_warp, has_query) == 0u)
        {
            break; // the queue is empty and every lane's query answered
        }
        // The walks, until fewer than RTB_REFILL_LANES lanes are still walking (or none, once the queue is empty)
        while (true)
        {
            // inner nodes: a lane descends, setting aside the first leaf it meets, until every descending lane holds one
            while (true)
            {
                const bool descending = has_query && link >= 0;
                if (!__any_sync(full_warp, descending))
                {
                    break;
                }
                if (WIDE && descending)
                {
                    const float4* np = reinterpret_cast<const float4*>(tree_wide + link);
                    const float4 lx = __ldg(np), hx = __ldg(np + 1);
                    const float4 ly = __ldg(np + 2), hy = __ldg(np + 3);
                    const float4 lz = __ldg(np + 4), hz = __ldg(np + 5);
                    const int4 nl = __ldg(reinterpret_cast<const int4*>(np + 6));
                    // each child's entry distance, or infinity where the ray misses it (or the slot is unused)
                    const auto entry = [&](float lox, float hix, float loy, float hiy, float loz, float hiz,
                                           int child) -> float {
                        const float a0 = fmaf(lox, inv.x, -os.x), a1 = fmaf(hix, inv.x, -os.x);
                        const float b0 = fmaf(loy, inv.y, -os.y), b1 = fmaf(hiy, inv.y, -os.y);
                        const float c0 = fmaf(loz, inv.z, -os.z), c1 = fmaf(hiz, inv.z, -os.z);
                        const float enter = fmaxf(fmaxf(fminf(a0, a1), fminf(b0, b1)), fmaxf(fminf(c0, c1), t_min));
                        const float exit = fminf(fminf(fmaxf(a0, a1), fmaxf(b0, b1)), fminf(fmaxf(c0, c1), hit.t));
                        return enter <= exit && child != traversal_done ? enter : infinity_f;
                    };
                    float k0 = entry(lx.x, hx.x, ly.x, hy.x, lz.x, hz.x, nl.x);
                    float k1 = entry(lx.y, hx.y, ly.y, hy.y, lz.y, hz.y, nl.y);
                    float k2 = entry(lx.z, hx.z, ly.z, hy.z, lz.z, hz.z, nl.z);
                    float k3 = entry(lx.w, hx.w, ly.w, hy.w, lz.w, hz.w, nl.w);
                    int l0 = nl.x, l1 = nl.y, l2 = nl.z, l3 = nl.w;
                    const auto order = [](float& ka, int& la, float& kb, int& lb) {
                        if (kb < ka)
                        {
                            const float k = ka;
                            ka = kb;
                            kb = k;
                            const int l = la;
                            la = lb;
                            lb = l;
                        }
                    };
                    order(k0, l0, k1, l1);
                    order(k2, l2, k3, l3);
                    order(k0, l0, k2, l2);
                    order(k1, l1, k3, l3);
                    order(k1, l1, k2, l2);
                    if (k0 == infinity_f)
                    {
                        link = pop();
                    }
                    else
                    {
                        // the far ones wait on the stack, farthest deepest; the nearest is next
                        if (k3 != infinity_f)
                        {
                            stack[sp++] = make_int2(l3, __float_as_int(k3));
                        }
                        if (k2 != infinity_f)
                        {
                            stack[sp++] = make_int2(l2, __float_as_int(k2));
                        }
                        if (k1 != infinity_f)
                        {
                            stack[sp++] = make_int2(l1, __float_as_int(k1));
                        }
                        link = l0;
                    }
                    if (link < 0 && link != traversal_done && leaf == 0)
                    {
                        leaf = link;
                        link = pop();
                    }
                }
                else if (descending)
                {
                    const float4* np = reinterpret_cast<const float4*>(tree_nodes + link);
                    const float4 nx = __ldg(np);
                    const float4 ny = __ldg(np + 1);
                    const float4 nz = __ldg(np + 2);
                    const int2 nl = __ldg(reinterpret_cast<const int2*>(np + 3));
                    const float a0 = fmaf(nx.x, inv.x, -os.x), a1 = fmaf(nx.y, inv.x, -os.x);
                    const float b0 = fmaf(ny.x, inv.y, -os.y), b1 = fmaf(ny.y, inv.y, -os.y);
                    const float c0 = fmaf(nz.x, inv.z, -os.z), c1 = fmaf(nz.y, inv.z, -os.z);
                    const float enter0 = fmaxf(fmaxf(fminf(a0, a1), fminf(b0, b1)), fmaxf(fminf(c0, c1), t_min));
                    const float exit0 = fminf(fminf(fmaxf(a0, a1), fmaxf(b0, b1)), fminf(fmaxf(c0, c1), hit.t));
                    const float a2 = fmaf(nx.z, inv.x, -os.x), a3 = fmaf(nx.w, inv.x, -os.x);
                    const float b2 = fmaf(ny.z, inv.y, -os.y), b3 = fmaf(ny.w, inv.y, -os.y);
                    const float c2 = fmaf(nz.z, inv.z, -os.z), c3 = fmaf(nz.w, inv.z, -os.z);
                    const float enter1 = fmaxf(fmaxf(fminf(a2, a3), fminf(b2, b3)), fmaxf(fminf(c2, c3), t_min));
                    const float exit1 = fminf(fminf(fmaxf(a2, a3), fmaxf(b2, b3)), fminf(fmaxf(c2, c3), hit.t));
                    const bool h0 = enter0 <= exit0;
                    const bool h1 = enter1 <= exit1;
                    if (h0 && h1)
                    {
                        const bool second_first = enter1 < enter0;
                        link = second_first ? nl.y : nl.x;
                        stack[sp++] =
                            make_int2(second_first ? nl.x : nl.y, __float_as_int(second_first ? enter0 : enter1));
                    }
                    else if (h0 || h1)
                    {
                        link = h0 ? nl.x : nl.y;
                    }
                    else
                    {
                        link = pop();
                    }
                    if (link < 0 && link != traversal_done && leaf == 0)
                    {
                        leaf = link;
                        link = pop();
                    }
                }
                if (!__any_sync(full_warp, has_query && link >= 0 && leaf == 0))
                {
                    break; // every lane still descending holds a leaf: test them together
                }
            }
            // leaves
            while (true)
            {
                const bool testing = has_query && leaf < 0;
                if (!__any_sync(full_warp, testing))
                {
                    break;
                }
                if (testing)
                {
                    if (test_leaf<false, false, FEATURES>(scene(), leaf, o, d, time, inverse_a, from, inward, skip,
                                                          hit, nullptr, shadow))
                    {
                        hit.id = 1; // a shadow ray's blocker: answered
                        leaf = 0;
                        link = traversal_done;
                    }
                    else
                    {
                        leaf = 0;
                        if (link < 0 && link != traversal_done)
                        {
                            leaf = link;
                            link = pop();
                        }
                    }
                }
            }
            const unsigned walking = __ballot_sync(full_warp, has_query && !(link == traversal_done && leaf == 0));
            if (walking == 0u || (!drained && __popc(walking) < RTB_REFILL_LANES))
            {
                break;
            }
        }
    }
    atomicAdd(&block_walks[0], walks[0]);
    atomicAdd(&block_walks[1], walks[1]);
    __syncthreads();
    if (counters != nullptr && threadIdx.x < 2 && block_walks[threadIdx.x] != 0u)
    {
        atomicAdd(counters + threadIdx.x, static_cast<unsigned long long>(block_walks[threadIdx.x]));
    }
}

// A flat-searched scene's query in the wavefront: every sphere, then every quad, in order (the persistent kernel's
// flat search, the same tests and self-intersection rules); `any` (a shadow ray) stops at the first hit
template <bool FEATURES>
__device__ __forceinline__ void flat_search(const scene_view& S, float3 o, float3 d, float time, int from, bool inward,
                                            int skip, bool any, hit_info& hit)
{
    const float inverse_a = 1.0f / length_squared(d);
    for (int i = 0; i < S.quad_base; ++i)
    {
        const bool own = i == from;
        if ((own && !inward) || i == skip)
        {
            continue;
        }
        const float4 s = sphere_at<FEATURES>(S, i, time);
        float t;
        bool entering;
        if (hit_sphere(s, o, d, inverse_a, t_min, hit.t, own, t, entering))
        {
            hit = {i, t, entering};
            if (any)
            {
                return;
            }
        }
    }
    const int quads = S.triangle_base - S.quad_base;
    for (int i = 0; i < quads; ++i)
    {
        const int id = S.quad_base + i;
        if (id == from || id == skip)
        {
            continue;
        }
        float t;
        bool front;
        if (hit_quad(load_quad(S.quads, i), o, d, t_min, hit.t, t, front))
        {
            hit = {id, t, front};
            if (any)
            {
                return;
            }
        }
    }
}

template <bool FEATURES>
__device__ __noinline__ void flat_search_call(const scene_view& S, float3 o, float3 d, float time, int from,
                                              bool inward, int skip, bool any, hit_info& hit)
{
    flat_search<FEATURES>(S, o, d, time, from, inward, skip, any, hit);
}

// The queued queries of a flat-searched scene: one query per thread at a time (grid-stride), every lane the same
// loop over the same records, no tree, no stack, no refill. BATCH: each query searches its job's scene (W's table; a
// warp's lanes may loop over different scenes), its walks counted where the shade kernel queued it.
template <bool FEATURES, bool BATCH, int MINB = RTB_TRACE_MIN_BLOCKS>
__global__ void __launch_bounds__(render_block, MINB)
    wave_flat_trace_kernel(const __grid_constant__ scene_view S, const __grid_constant__ wave_buffers B,
                           const __grid_constant__ wave_batch W, unsigned long long* counters)
{
    __shared__ unsigned block_walks[2];
    if (threadIdx.x < 2)
    {
        block_walks[threadIdx.x] = 0;
    }
    __syncthreads();
    const unsigned count = B.control[0];
    unsigned walks[2] = {0, 0};
    for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x)
    {
        const float4 qo = stream_load(B.query_o + q);
        const float4 qd = stream_load(B.query_d + q);
        const int4 qm = stream_load(B.query_meta + q);
        const bool shadow = (qm.y & 2) != 0;
        hit_info hit{-1, qd.w, false};
        const scene_view* scene = &S;
        if constexpr (BATCH)
        {
            scene = &W.jobs[qm.y >> 3].scene;
        }
        flat_search<FEATURES>(*scene, make_float3(qo.x, qo.y, qo.z), make_float3(qd.x, qd.y, qd.z), qo.w, qm.x,
                              (qm.y & 1) != 0, qm.z, shadow, hit);
        if (shadow)
        {
            stream_store(B.shadow_result + qm.w, hit.id >= 0 ? 1 : 0);
        }
        else
        {
            stream_store(B.ext_result + qm.w, make_int4(hit.id, __float_as_int(hit.t), hit.front ? 1 : 0, 0));
        }
        ++walks[shadow ? 1 : 0];
    }
    atomicAdd(&block_walks[0], walks[0]);
    atomicAdd(&block_walks[1], walks[1]);
    __syncthreads();
    if (counters != nullptr && threadIdx.x < 2 && block_walks[threadIdx.x] != 0u)
    {
        atomicAdd(counters + threadIdx.x, static_cast<unsigned long long>(block_walks[threadIdx.x]));
    }
}

// The wavefront's samples into the image's sums: each chunk's samples added in pass order into its partial, the
// partials in chunk order into the sums, as the persistent kernel's lanes and reduce_kernel add them
__global__ void wave_reduce_kernel(const reduce_params R, const float4* samples, int64_t pass_begin, int64_t pass_end,
                                   int32_t chunk)
{
    const int x = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    const int y = static_cast<int>(blockIdx.y);
    if (x >= R.width || y >= R.height)
    {
        return;
    }
    const int q = ((y >> 2) * R.tiles_x + (x >> 3)) * 32 + ((y & 3) << 3) + (x & 7);
    double* sum = R.sums + 3 * (static_cast<int64_t>(y) * R.width + x);
    double r = sum[0], g = sum[1], b = sum[2];
    int64_t pass = pass_begin;
    while (pass < pass_end)
    {
        const int64_t chunk_end = (pass / chunk + 1) * chunk;
        const int64_t end = chunk_end < pass_end ? chunk_end : pass_end;
        double pr = 0.0, pg = 0.0, pb = 0.0;
        for (; pass < end; ++pass)
        {
            const float4 s = samples[(pass - pass_begin) * R.padded_pixels + q];
            pr += without_nan(s.x);
            pg += without_nan(s.y);
            pb += without_nan(s.z);
        }
        r += pr;
        g += pg;
        b += pb;
    }
    sum[0] = r;
    sum[1] = g;
    sum[2] = b;
}

// A stream run's finished segments into their requests' images (stream_reduce_item): one thread per pixel of an
// item; the segment's samples of that pixel, pass after pass, into the request's chunk accumulator, which goes into
// the sums after a chunk's last pass, after the first pass (the first frame) and at the target. A pixel's passes
// arrive in order (the host reduces a request's segments one after another), so a pixel's sums are the session's
// chunk partials added in chunk order, up to the first frame's split of the first chunk.
__global__ void stream_reduce_kernel(const stream_reduce_item* items, int32_t count, int64_t total_pixels)
{
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total_pixels;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    {
        int lo = 0, hi = count - 1;
        while (lo < hi)
        {
            const int mid = (lo + hi + 1) >> 1;
            if (items[mid].pixel_begin <= i)
            {
                lo = mid;
            }
            else
            {
                hi = mid - 1;
            }
        }
        const stream_reduce_item& it = items[lo];
        const int64_t pixel = i - it.pixel_begin;
        const int y = static_cast<int>(pixel / it.width);
        const int x = static_cast<int>(pixel - static_cast<int64_t>(y) * it.width);
        const int q = ((y >> 2) * it.tiles_x + (x >> 3)) * 32 + ((y & 3) << 3) + (x & 7);
        // the passes whose sample of this pixel lies in [local_begin, local_end)
        const int64_t padded = it.padded_pixels;
        int64_t pass = (it.local_begin - q + padded - 1) / padded;
        pass = pass < 0 ? 0 : pass;
        double* acc = it.acc + 3 * pixel;
        double* sum = it.sums + 3 * pixel;
        double ar = acc[0], ag = acc[1], ab = acc[2];
        for (int64_t local = pass * padded + q; local < it.local_end; local += padded, ++pass)
        {
            const float4 v = it.values[local - it.local_begin];
            ar += without_nan(v.x);
            ag += without_nan(v.y);
            ab += without_nan(v.z);
            const int64_t done = pass + 1;
            if (done % it.chunk == 0 || done == 1 || done == it.target)
            {
                sum[0] += ar;
                sum[1] += ag;
                sum[2] += ab;
                ar = ag = ab = 0.0;
            }
        }
        acc[0] = ar;
        acc[1] = ag;
        acc[2] = ab;
    }
}


// A wavefront group's samples into its jobs' chunk partials, laid out as the persistent batch kernel writes them: each
// work item (chunk, pixel) the sum of its passes' samples in pass order; items of pixels over the image's edge skipped
__global__ void wave_batch_partials_kernel(const wave_batch W, const float4* samples)
{
    for (int64_t i = W.item_first + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < W.item_end;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    {
        const batch_job& J = W.jobs[find_job<job_items>(W.jobs, W.job_first, W.job_end, i)];
        const int64_t local = i - J.item_begin;
        const int64_t k = local / J.padded_pixels;
        const int q = static_cast<int>(local - k * J.padded_pixels);
        const int tile = q >> 5;
        const int l = q & 31;
        if ((tile % J.tiles_x) * 8 + (l & 7) >= J.cam.width || (tile / J.tiles_x) * 4 + (l >> 3) >= J.cam.height)
        {
            continue;
        }
        const int64_t chunk_first = (J.first_chunk + k) * J.chunk;
        const int64_t begin = chunk_first > J.pass_begin ? chunk_first : J.pass_begin;
        const int64_t end = chunk_first + J.chunk < J.pass_end ? chunk_first + J.chunk : J.pass_end;
        double r = 0.0, g = 0.0, b = 0.0;
        for (int64_t pass = begin; pass < end; ++pass)
        {
            const float4 s = samples[J.sample_begin + (pass - J.pass_begin) * J.padded_pixels + q];
            r += without_nan(s.x);
            g += without_nan(s.y);
            b += without_nan(s.z);
        }
        double* out = J.partials + 3 * local;
        out[0] = r;
        out[1] = g;
        out[2] = b;
    }
}
} // namespace

namespace
{
using render_function = void (*)(launch_params);

template <bool QUALITY, bool FLAT>
render_function render_kernel_of(bool counting, bool features)
{
    if (counting)
    {
        return render_kernel<QUALITY, true, FLAT, true>;
    }
    return features ? render_kernel<QUALITY, false, FLAT, true> : render_kernel<QUALITY, false, FLAT, false>;
}

// The render kernel for an integrator, the counting build or not, a flat or a tree search, and a scene with or
// without the second book's features
render_function render_kernel_for(bool quality, bool counting, bool flat, bool features)
{
    if (quality)
    {
        return flat ? render_kernel_of<true, true>(counting, features)
                    : render_kernel_of<true, false>(counting, features);
    }
    return flat ? render_kernel_of<false, true>(counting, features) : render_kernel_of<false, false>(counting, features);
}
} // namespace

cudaError_t launch_render(const launch_params& p, bool quality, bool counting, int grid, cudaStream_t stream)
{
    render_kernel_for(quality, counting, p.scene.flat != 0, has_features(p.scene))<<<grid, render_block, 0, stream>>>(
        p);
    return cudaGetLastError();
}

namespace
{
using batch_function = void (*)(batch_params);

batch_function batch_kernel_of(int group)
{
    switch (group)
    {
    case 0:
        return render_batch_kernel<true, false>;
    case 1:
        return render_batch_kernel<true, true>;
    case 2:
        return render_batch_kernel<false, false>;
    default:
        return render_batch_kernel<false, true>;
    }
}
} // namespace

cudaError_t launch_batch(const batch_params& p, const int* grids, int first_group, int end_group, cudaStream_t stream)
{
    for (int g = first_group; g < end_group; ++g)
    {
        batch_kernel_of(g)<<<grids[g], render_block, 0, stream>>>(p);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess)
        {
            return e;
        }
    }
    return cudaSuccess;
}

cudaError_t launch_batch_reduce(const batch_params& p, int grid, cudaStream_t stream)
{
    reduce_batch_kernel<<<grid, 256, 0, stream>>>(p);
    return cudaGetLastError();
}

namespace
{
// A kernel's registers, local memory and resident blocks, and the device's multiprocessors (two attribute queries:
// cudaGetDeviceProperties would fill every field of the device's description, a cost each session paid)
template <class Kernel>
cudaError_t attributes_of(Kernel kernel, kernel_attributes& out)
{
    cudaFuncAttributes a{};
    cudaError_t e = cudaFuncGetAttributes(&a, kernel);
    int device = 0;
    if (e == cudaSuccess)
    {
        e = cudaGetDevice(&device);
    }
    int blocks = 0;
    if (e == cudaSuccess)
    {
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, render_block, 0);
    }
    int multiprocessors = 0;
    int max_threads = 0;
    if (e == cudaSuccess)
    {
        e = cudaDeviceGetAttribute(&multiprocessors, cudaDevAttrMultiProcessorCount, device);
    }
    if (e == cudaSuccess)
    {
        e = cudaDeviceGetAttribute(&max_threads, cudaDevAttrMaxThreadsPerMultiProcessor, device);
    }
    if (e != cudaSuccess)
    {
        return e;
    }
    out.registers = a.numRegs;
    out.local_bytes = static_cast<int>(a.localSizeBytes);
    out.blocks_per_sm = blocks;
    out.threads_per_block = render_block;
    out.max_threads_per_sm = max_threads;
    out.multiprocessors = multiprocessors;
    return cudaSuccess;
}
} // namespace

cudaError_t batch_attributes(int group, kernel_attributes& out) { return attributes_of(batch_kernel_of(group), out); }

cudaError_t launch_reduce(const reduce_params& p, cudaStream_t stream)
{
    const dim3 block(128, 1);
    const dim3 grid(static_cast<unsigned>((p.width + 127) / 128), static_cast<unsigned>(p.height));
    reduce_kernel<<<grid, block, 0, stream>>>(p);
    return cudaGetLastError();
}

cudaError_t render_attributes(const scene_view& scene, bool quality, kernel_attributes& out)
{
    return attributes_of(render_kernel_for(quality, false, scene.flat != 0, has_features(scene)), out);
}

cudaError_t launch_closest_hits(const scene_view& s, const float* origins, const float* directions, int64_t count,
                                const int32_t* prim_source, int32_t* ids, float* ts, cudaStream_t stream)
{
    if (count <= 0)
    {
        return cudaSuccess;
    }
    const int block = 128;
    const auto grid = static_cast<unsigned>((count + block - 1) / block);
    closest_hits_kernel<<<grid, block, 0, stream>>>(s, origins, directions, count, prim_source, ids, ts);
    return cudaGetLastError();
}

size_t wave_slot_bytes() { return (wave_rows + wave_shadow_rows) * sizeof(float4); }

cudaError_t clear_wave_slots(const wave_buffers& b, cudaStream_t stream)
{
    // the other rows are written when a slot's first sample starts
    return cudaMemsetAsync(static_cast<float4*>(b.slots) + int64_t{wave_flags_row} * b.slot_count, 0,
                           static_cast<size_t>(b.slot_count) * sizeof(float4), stream);
}

namespace
{
using wave_shade_function = void (*)(launch_params, wave_buffers, wave_batch);
using wave_trace_function = void (*)(scene_view, wave_buffers, wave_batch, unsigned long long*);

template <bool BATCH>
wave_trace_function wave_trace_variant(bool features, bool wide)
{
    if (wide)
    {
        return features ? wave_trace_kernel<true, BATCH, true> : wave_trace_kernel<false, BATCH, true>;
    }
    return features ? wave_trace_kernel<true, BATCH, false> : wave_trace_kernel<false, BATCH, false>;
}

wave_shade_function wave_shade_of(bool quality, bool features)
{
    if (quality)
    {
        return features ? wave_shade_kernel<true, true, false> : wave_shade_kernel<true, false, false>;
    }
    return features ? wave_shade_kernel<false, true, false> : wave_shade_kernel<false, false, false>;
}

// A session's walk at one of the register caps the autotuner chooses between: the default blocks per multiprocessor
// (64 registers a thread at 8 blocks of 128) or fewer blocks with more registers (80 at 6)
wave_trace_function wave_trace_of(bool features, bool wide, int min_blocks = RTB_TRACE_MIN_BLOCKS)
{
    if (min_blocks == wave_trace_roomy_blocks)
    {
        if (wide)
        {
            return features ? wave_trace_kernel<true, false, true, wave_trace_roomy_blocks>
                            : wave_trace_kernel<false, false, true, wave_trace_roomy_blocks>;
        }
        return features ? wave_trace_kernel<true, false, false, wave_trace_roomy_blocks>
                        : wave_trace_kernel<false, false, false, wave_trace_roomy_blocks>;
    }
    return wave_trace_variant<false>(features, wide);
}

template <bool BATCH>
wave_trace_function wave_flat_trace_of(bool features, int min_blocks = RTB_TRACE_MIN_BLOCKS)
{
    if (!BATCH && min_blocks == wave_trace_roomy_blocks)
    {
        return features ? wave_flat_trace_kernel<true, false, wave_trace_roomy_blocks>
                        : wave_flat_trace_kernel<false, false, wave_trace_roomy_blocks>;
    }
    return features ? wave_flat_trace_kernel<true, BATCH> : wave_flat_trace_kernel<false, BATCH>;
}
} // namespace

// marks (when given): three events recorded before the shade kernel, between the two kernels and after the trace
// kernel, for per-kernel timing
cudaError_t launch_wave_step(const launch_params& p, bool quality, const wave_buffers& slots, const wave_shape& shape,
                             cudaStream_t stream, const cudaEvent_t* marks, bool draining)
{
    const int trace_grid = shape.trace_grid;
    const int shade_block = shape.shade_block > 0 ? shape.shade_block : render_block;
    wave_buffers b = slots; // with the launch's camera and RNG job, for the camera rays the trace kernel makes
    b.cam = p.cam;
    b.job = p.job;
    b.draining = draining ? 1 : 0;
    cudaError_t e = cudaMemsetAsync(b.control, 0, 3 * sizeof(unsigned), stream);
    if (e != cudaSuccess)
    {
        return e;
    }
    const bool features = has_features(p.scene);
    if (marks)
    {
        cudaEventRecord(marks[0], stream);
    }
    wave_shade_of(quality, features)<<<b.slot_count / shade_block, shade_block, 0, stream>>>(p, b, wave_batch{});
    e = cudaGetLastError();
    if (e != cudaSuccess)
    {
        return e;
    }
    if (marks)
    {
        cudaEventRecord(marks[1], stream);
    }
    if (p.scene.flat != 0)
    {
        wave_flat_trace_of<false>(features, shape.trace_min_blocks)<<<trace_grid, render_block, 0, stream>>>(
            p.scene, b, wave_batch{}, p.counters);
    }
    else
    {
        wave_trace_of(features, p.scene.wide_nodes != nullptr, shape.trace_min_blocks)<<<trace_grid, render_block, 0,
                                                                                          stream>>>(
            p.scene, b, wave_batch{}, p.counters);
    }
    e = cudaGetLastError();
    if (marks && e == cudaSuccess)
    {
        cudaEventRecord(marks[2], stream);
    }
    return e;
}

cudaError_t launch_wave_batch_step(const wave_batch& w, bool flat, bool features, bool wide, bool quality,
                                   const wave_buffers& b, int trace_grid, cudaStream_t stream, bool draining)
{
    cudaError_t e = cudaMemsetAsync(b.control, 0, 3 * sizeof(unsigned), stream);
    if (e != cudaSuccess)
    {
        return e;
    }
    const launch_params none{};
    const auto shade = quality ? (features ? wave_shade_kernel<true, true, true> : wave_shade_kernel<true, false, true>)
                               : (features ? wave_shade_kernel<false, true, true> : wave_shade_kernel<false, false, true>);
    wave_buffers bd = b;
    bd.draining = draining ? 1 : 0;
    shade<<<b.slot_count / render_block, render_block, 0, stream>>>(none, bd, w);
    e = cudaGetLastError();
    if (e != cudaSuccess)
    {
        return e;
    }
    const wave_trace_function trace = flat ? wave_flat_trace_of<true>(features) : wave_trace_variant<true>(features, wide);
    trace<<<trace_grid, render_block, 0, stream>>>(scene_view{}, bd, w, nullptr);
    return cudaGetLastError();
}

cudaError_t preload_wave_batch()
{
    cudaFuncAttributes a{};
    const void* kernels[] = {reinterpret_cast<const void*>(wave_shade_kernel<false, false, true>),
                             reinterpret_cast<const void*>(wave_shade_kernel<false, true, true>),
                             reinterpret_cast<const void*>(wave_shade_kernel<true, false, true>),
                             reinterpret_cast<const void*>(wave_shade_kernel<true, true, true>),
                             reinterpret_cast<const void*>(wave_trace_variant<true>(false, false)),
                             reinterpret_cast<const void*>(wave_trace_variant<true>(false, true)),
                             reinterpret_cast<const void*>(wave_trace_variant<true>(true, false)),
                             reinterpret_cast<const void*>(wave_trace_variant<true>(true, true)),
                             reinterpret_cast<const void*>(wave_flat_trace_of<true>(false)),
                             reinterpret_cast<const void*>(wave_flat_trace_of<true>(true)),
                             reinterpret_cast<const void*>(wave_batch_partials_kernel)};
    for (const void* k : kernels)
    {
        const cudaError_t e = cudaFuncGetAttributes(&a, k);
        if (e != cudaSuccess)
        {
            return e;
        }
    }
    return cudaSuccess;
}

cudaError_t launch_stream_reduce(const stream_reduce_item* items, int32_t count, int64_t total_pixels,
                                 cudaStream_t stream)
{
    if (count <= 0 || total_pixels <= 0)
    {
        return cudaSuccess;
    }
    const int64_t wanted = (total_pixels + 255) / 256;
    const int64_t blocks = wanted < 148 * 16 ? wanted : 148 * 16;
    stream_reduce_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(items, count, total_pixels);
    return cudaGetLastError();
}

cudaError_t launch_wave_batch_partials(const wave_batch& w, const wave_buffers& b, cudaStream_t stream)
{
    if (w.item_end <= w.item_first)
    {
        return cudaSuccess;
    }
    const int64_t blocks = std::min<int64_t>((w.item_end - w.item_first + 255) / 256, 148 * 16);
    wave_batch_partials_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(w, b.samples);
    return cudaGetLastError();
}

cudaError_t launch_wave_reduce(const reduce_params& r, const wave_buffers& b, int64_t pass_begin, int64_t pass_end,
                               int32_t chunk, cudaStream_t stream)
{
    const dim3 block(128, 1);
    const dim3 grid(static_cast<unsigned>((r.width + 127) / 128), static_cast<unsigned>(r.height));
    wave_reduce_kernel<<<grid, block, 0, stream>>>(r, b.samples, pass_begin, pass_end, chunk);
    return cudaGetLastError();
}

cudaError_t wave_attributes(const scene_view& scene, bool quality, kernel_attributes& shade, kernel_attributes& trace,
                            int trace_min_blocks)
{
    const bool features = has_features(scene);
    const cudaError_t e = attributes_of(wave_shade_of(quality, features), shade);
    if (e != cudaSuccess)
    {
        return e;
    }
    // the session's trace kernel of the scene's search at the given register cap
    if (scene.flat != 0)
    {
        return attributes_of(wave_flat_trace_of<false>(features, trace_min_blocks), trace);
    }
    return attributes_of(wave_trace_of(features, scene.wide_nodes != nullptr, trace_min_blocks), trace);
}

cudaError_t launch_camera_rays(const camera_params& cam, uint64_t seed, int64_t pass, int32_t round_passes,
                               float* origins, float* directions, cudaStream_t stream)
{
    const dim3 block(128, 1);
    const dim3 grid(static_cast<unsigned>((cam.width + 127) / 128), static_cast<unsigned>(cam.height));
    camera_rays_kernel<<<grid, block, 0, stream>>>(cam, seed, pass, round_passes, origins, directions);
    return cudaGetLastError();
}
} // namespace rtb
