// TEST INFRASTRUCTURE — the CPU oracle. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
// as the checker and the CPU baseline; the product path never links or calls it.
//
// A restatement, in double precision and header form, of the reference's CPU ray tracer: the C++23 modules of src/
// (vec3.ixx, random.ixx, interval.ixx, onb.ixx, aabb.ixx, bvh.ixx, hittable.ixx, sphere.ixx, quad.ixx, material.ixx,
// pdf.ixx, camera.ixx), which MSVC builds with `import std;` and GCC cannot. The algorithms are the reference's, step
// for step; what changes is only the form: headers instead of modules, a flat scene table in (the rt_scene_desc that
// every renderer here is fed) instead of the scene's object graph, and std::thread workers instead of std::jthread.
// Every function names the reference lines it follows.
#pragma once

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <limits>
#include <memory>
#include <numbers>
#include <optional>
#include <random>
#include <span>
#include <thread>
#include <vector>

#include "rt_b200.h"

namespace oracle
{
constexpr double infinity = std::numeric_limits<double>::infinity();

// ---- vec3.ixx ------------------------------------------------------------------------------------------------
struct vec3
{
    double x = 0, y = 0, z = 0;
    vec3 operator-() const { return {-x, -y, -z}; }
    vec3& operator+=(const vec3& v)
    {
        x += v.x;
        y += v.y;
        z += v.z;
        return *this;
    }
    double length_squared() const { return x * x + y * y + z * z; }
    double length() const { return std::sqrt(length_squared()); }
};
using point3 = vec3;
using color = vec3;
inline vec3 operator+(const vec3& u, const vec3& v) { return {u.x + v.x, u.y + v.y, u.z + v.z}; }
inline vec3 operator-(const vec3& u, const vec3& v) { return {u.x - v.x, u.y - v.y, u.z - v.z}; }
inline vec3 operator*(const vec3& u, const vec3& v) { return {u.x * v.x, u.y * v.y, u.z * v.z}; }
inline vec3 operator*(double t, const vec3& v) { return {t * v.x, t * v.y, t * v.z}; }
inline vec3 operator*(const vec3& v, double t) { return t * v; }
inline vec3 operator/(const vec3& v, double t) { return (1 / t) * v; }
inline double dot(const vec3& u, const vec3& v) { return u.x * v.x + u.y * v.y + u.z * v.z; }
inline vec3 cross(const vec3& u, const vec3& v)
{
    return {u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x};
}
inline vec3 unit_vector(const vec3& v) { return v / v.length(); }
inline vec3 reflect(const vec3& v, const vec3& n) { return v - 2 * dot(v, n) * n; }
inline vec3 refract(const vec3& uv, const vec3& n, double etai_over_etat) // vec3.ixx:93-99
{
    const double cos_theta = std::fmin(dot(-uv, n), 1.0);
    const vec3 r_out_perp = etai_over_etat * (uv + cos_theta * n);
    const vec3 r_out_parallel = -std::sqrt(std::fabs(1.0 - r_out_perp.length_squared())) * n;
    return r_out_perp + r_out_parallel;
}
inline vec3 from(const rt_vec3& v) { return {v.x, v.y, v.z}; }

// ---- random.ixx: a per-thread std::mt19937_64 and uniform_real_distribution ----------------------------------
struct rng
{
    std::mt19937_64 engine;
    void seed(uint64_t s) { engine.seed(s); }
    double next() { return std::uniform_real_distribution<double>(0.0, 1.0)(engine); }
    double next(double lo, double hi) { return lo + (hi - lo) * next(); }
    int next_int(int lo, int hi) { return static_cast<int>(next(lo, hi + 1)); } // random.ixx:33-36
};

inline vec3 random_in_unit_disk(rng& g) // vec3.ixx:77-87: rejection
{
    while (true)
    {
        const double x = g.next(-1, 1);
        const double y = g.next(-1, 1);
        const vec3 p{x, y, 0};
        if (p.length_squared() < 1)
        {
            return p;
        }
    }
}

inline vec3 random_unit_vector(rng& g) // vec3.ixx:105-117: rejection in the cube
{
    while (true)
    {
        const double x = g.next(-1, 1);
        const double y = g.next(-1, 1);
        const double z = g.next(-1, 1);
        const vec3 p{x, y, z};
        const double lensq = p.length_squared();
        if (1e-160 < lensq && lensq <= 1)
        {
            return p / std::sqrt(lensq);
        }
    }
}

inline vec3 random_cosine_direction(rng& g) // vec3.ixx:124-132
{
    const double r1 = g.next();
    const double r2 = g.next();
    const double phi = 2 * std::numbers::pi * r1;
    return {std::cos(phi) * std::sqrt(r2), std::sin(phi) * std::sqrt(r2), std::sqrt(1 - r2)};
}

// ---- onb.ixx -------------------------------------------------------------------------------------------------
struct onb
{
    vec3 u, v, w;
    explicit onb(const vec3& unit_w) : w(unit_w) // onb.ixx:17-30
    {
        const vec3 a = std::fabs(w.x) > 0.9 ? vec3{0, 1, 0} : vec3{1, 0, 0};
        v = unit_vector(cross(w, a));
        u = cross(v, w);
    }
    vec3 transform(const vec3& a) const { return a.x * u + a.y * v + a.z * w; }
};

// ---- interval.ixx, ray.ixx, aabb.ixx -------------------------------------------------------------------------
struct interval
{
    double min = +infinity, max = -infinity;
    double size() const { return max - min; }
    bool contains(double x) const { return min <= x && x <= max; }
    bool surrounds(double x) const { return min < x && x < max; }
    interval expand(double delta) const { return {min - delta / 2, max + delta / 2}; }
};
inline interval enclose(const interval& a, const interval& b) { return {std::min(a.min, b.min), std::max(a.max, b.max)}; }

struct ray
{
    point3 origin;
    vec3 direction;
    double time = 0;
    point3 at(double t) const { return origin + t * direction; }
};

struct aabb
{
    interval x, y, z;
    static interval axis_span(double a, double b) // aabb.ixx:50-55
    {
        constexpr double min_size = 0.0001;
        const interval span{std::min(a, b), std::max(a, b)};
        return span.size() < min_size ? span.expand(min_size) : span;
    }
    static aabb from_corners(const point3& a, const point3& b)
    {
        return {axis_span(a.x, b.x), axis_span(a.y, b.y), axis_span(a.z, b.z)};
    }
    const interval& axis_interval(int axis) const { return axis == 0 ? x : axis == 1 ? y : z; }
    int longest_axis() const // aabb.ixx:22-29
    {
        if (x.size() > y.size())
        {
            return x.size() > z.size() ? 0 : 2;
        }
        return y.size() > z.size() ? 1 : 2;
    }
    static bool hit_slab(const interval& slab, double origin, double direction, interval& ray_t) // aabb.ixx:59-71
    {
        const double inverse = 1.0 / direction;
        double t0 = (slab.min - origin) * inverse;
        double t1 = (slab.max - origin) * inverse;
        if (t0 > t1)
        {
            std::swap(t0, t1);
        }
        ray_t.min = std::max(ray_t.min, t0);
        ray_t.max = std::min(ray_t.max, t1);
        return ray_t.min < ray_t.max;
    }
    bool hit(const ray& r, interval ray_t) const
    {
        return hit_slab(x, r.origin.x, r.direction.x, ray_t) && hit_slab(y, r.origin.y, r.direction.y, ray_t) &&
               hit_slab(z, r.origin.z, r.direction.z, ray_t);
    }
};
inline aabb enclose(const aabb& a, const aabb& b) { return {enclose(a.x, b.x), enclose(a.y, b.y), enclose(a.z, b.z)}; }

// ---- hittable.ixx: the hit record ------------------------------------------------------------------------------
struct hit_record
{
    point3 p;
    vec3 normal;
    int material = -1;
    int id = -1;    // the primitive in source index space: spheres, then quads, then triangles
    double t = 0;
    double u = 0, v = 0;
    bool front_face = false;
    color color_at; // the material's color at the hit (its texture there), filled by scene::closest_event
    void set_face_normal(const ray& r, const vec3& outward)
    {
        front_face = dot(r.direction, outward) < 0;
        normal = front_face ? outward : -outward;
    }
};

// ---- sphere.ixx ----------------------------------------------------------------------------------------------
struct sphere
{
    ray center; // center_.at(time): start + time * displacement
    double radius = 0;
    int material = -1;
    int id = -1;
    aabb bbox;
    double uv_cos = 1, uv_sin = 0; // the turn of the rotate_y instances around it, for its texture coordinates

    sphere(const point3& c1, const point3& c2, double r, int mat, int ident)
        : center{c1, c2 - c1}, radius(std::fmax(0.0, r)), material(mat), id(ident)
    {
        const vec3 rv{radius, radius, radius};
        bbox = enclose(aabb::from_corners(center.at(0) - rv, center.at(0) + rv),
                       aabb::from_corners(center.at(1) - rv, center.at(1) + rv));
    }

    std::optional<hit_record> hit(const ray& r, interval ray_t) const // sphere.ixx:43-92
    {
        const point3 c = center.at(r.time);
        const vec3 oc = c - r.origin;
        const double a = r.direction.length_squared();
        const double h = dot(r.direction, oc);
        const double cc = oc.length_squared() - radius * radius;
        const double discriminant = h * h - a * cc;
        if (discriminant < 0)
        {
            return std::nullopt;
        }
        const double sqrtd = std::sqrt(discriminant);
        double root = (h - sqrtd) / a;
        if (!ray_t.surrounds(root))
        {
            root = (h + sqrtd) / a;
            if (!ray_t.surrounds(root))
            {
                return std::nullopt;
            }
        }
        hit_record rec;
        rec.t = root;
        rec.p = r.at(rec.t);
        const vec3 outward = (rec.p - c) / radius;
        rec.set_face_normal(r, outward);
        rec.material = material;
        rec.id = id;
        // get_sphere_uv of the normal in the sphere's own coordinates (turned back by its rotate_y instances)
        const vec3 n{uv_cos * outward.x - uv_sin * outward.z, outward.y, uv_sin * outward.x + uv_cos * outward.z};
        const double phi = std::atan2(-n.z, n.x) + std::numbers::pi;
        const double theta = std::acos(std::clamp(-n.y, -1.0, 1.0));
        rec.u = phi / (2 * std::numbers::pi);
        rec.v = theta / std::numbers::pi;
        return rec;
    }

    // sphere.ixx:101-151: one minus cos theta_max in the digit-keeping form, and the light-sampling density
    double one_minus_cos_theta_max(double distance_squared) const
    {
        const double sin_squared = radius * radius / distance_squared;
        return sin_squared / (1 + std::sqrt(1 - sin_squared));
    }
    double pdf_value(const point3& origin, const vec3& direction) const
    {
        const double distance_squared = (center.at(0) - origin).length_squared();
        if (distance_squared < radius * radius)
        {
            return 1 / (4 * std::numbers::pi);
        }
        if (!hit(ray{origin, direction}, interval{0.001, infinity}))
        {
            return 0;
        }
        return 1 / (2 * std::numbers::pi * one_minus_cos_theta_max(distance_squared));
    }
    vec3 random(const point3& origin, rng& g) const
    {
        const vec3 to_center = center.at(0) - origin;
        const double distance_squared = to_center.length_squared();
        if (distance_squared < radius * radius)
        {
            return random_unit_vector(g);
        }
        const onb uvw{unit_vector(to_center)};
        const double one_minus_cos_max = one_minus_cos_theta_max(distance_squared);
        const double r1 = g.next();
        const double r2 = g.next();
        const double phi = 2 * std::numbers::pi * r1;
        const double one_minus_z = r2 * one_minus_cos_max;
        const double sin_theta = std::sqrt(one_minus_z * (2 - one_minus_z));
        return uvw.transform({std::cos(phi) * sin_theta, std::sin(phi) * sin_theta, 1 - one_minus_z});
    }
};

// ---- quad.ixx ------------------------------------------------------------------------------------------------
struct quad
{
    point3 q;
    vec3 u, v;
    int material = -1;
    int id = -1;
    vec3 normal;
    double d = 0;
    vec3 w;
    double area = 0;
    aabb bbox;

    quad(const point3& q0, const vec3& u0, const vec3& v0, int mat, int ident) // quad.ixx:17-31
        : q(q0), u(u0), v(v0), material(mat), id(ident)
    {
        const vec3 n = cross(u, v);
        normal = unit_vector(n);
        d = dot(normal, q);
        w = n / dot(n, n);
        area = n.length();
        bbox = enclose(aabb::from_corners(q, q + u + v), aabb::from_corners(q + u, q + v));
    }

    // slack (the first-hit test's tie rule only): alpha and beta accepted that far outside [0, 1]
    std::optional<hit_record> hit(const ray& r, interval ray_t, double slack = 0) const // quad.ixx:68-106
    {
        const double denom = dot(normal, r.direction);
        if (std::fabs(denom) < 1e-8)
        {
            return std::nullopt;
        }
        const double t = (d - dot(normal, r.origin)) / denom;
        if (!ray_t.contains(t))
        {
            return std::nullopt;
        }
        const point3 intersection = r.at(t);
        const vec3 p = intersection - q;
        const double alpha = dot(w, cross(p, v));
        const double beta = dot(w, cross(u, p));
        const interval unit{-slack, 1 + slack};
        if (!unit.contains(alpha) || !unit.contains(beta))
        {
            return std::nullopt;
        }
        hit_record rec;
        rec.t = t;
        rec.p = intersection;
        rec.material = material;
        rec.id = id;
        rec.set_face_normal(r, normal);
        rec.u = alpha;
        rec.v = beta;
        return rec;
    }

    double pdf_value(const point3& origin, const vec3& direction) const // quad.ixx:44-57
    {
        const auto rec = hit(ray{origin, direction}, interval{0.001, infinity});
        if (!rec)
        {
            return 0;
        }
        const double distance_squared = rec->t * rec->t * direction.length_squared();
        const double cosine = std::fabs(dot(direction, normal)) / direction.length();
        return distance_squared / (cosine * area);
    }

    vec3 random(const point3& origin, rng& g) const // quad.ixx:60-65
    {
        const double a = g.next();
        const double b = g.next();
        return unit_vector(q + a * u + b * v - origin);
    }
};

// A triangle (the displaced icosphere's; the reference traces meshes only through OptiX). Möller–Trumbore in double,
// closed barycentric bounds, outward normal e1 x e2 (counter-clockwise seen from the front).
struct triangle
{
    point3 a, b, c;
    int material = -1;
    int id = -1;
    aabb bbox;
    triangle(const point3& a0, const point3& b0, const point3& c0, int mat, int ident)
        : a(a0), b(b0), c(c0), material(mat), id(ident)
    {
        const point3 lo{std::min({a.x, b.x, c.x}), std::min({a.y, b.y, c.y}), std::min({a.z, b.z, c.z})};
        const point3 hi{std::max({a.x, b.x, c.x}), std::max({a.y, b.y, c.y}), std::max({a.z, b.z, c.z})};
        bbox = aabb::from_corners(lo, hi);
    }
    // slack (the first-hit test's tie rule only): barycentrics accepted that far outside the triangle
    std::optional<hit_record> hit(const ray& r, interval ray_t, double slack = 0) const
    {
        const vec3 e1 = b - a;
        const vec3 e2 = c - a;
        const vec3 pv = cross(r.direction, e2);
        const double det = dot(e1, pv);
        if (std::fabs(det) < 1e-300)
        {
            return std::nullopt;
        }
        const double inv = 1 / det;
        const vec3 tv = r.origin - a;
        const double beta = dot(tv, pv) * inv;
        if (beta < -slack || beta > 1 + slack)
        {
            return std::nullopt;
        }
        const vec3 qv = cross(tv, e1);
        const double gamma = dot(r.direction, qv) * inv;
        if (gamma < -slack || beta + gamma > 1 + slack)
        {
            return std::nullopt;
        }
        const double t = dot(e2, qv) * inv;
        if (!ray_t.surrounds(t))
        {
            return std::nullopt;
        }
        hit_record rec;
        rec.t = t;
        rec.p = r.at(t);
        rec.material = material;
        rec.id = id;
        rec.set_face_normal(r, unit_vector(cross(e1, e2)));
        rec.u = beta;
        rec.v = gamma;
        return rec;
    }
};

// ---- the world: the flat primitives, and bvh.ixx's tree over them -----------------------------------------------
struct primitive
{
    int kind; // 0 sphere, 1 quad, 2 triangle
    int index;
};

class world
{
public:
    std::vector<sphere> spheres;
    std::vector<quad> quads;
    std::vector<triangle> triangles;

    aabb box_of(const primitive& p) const
    {
        return p.kind == 0 ? spheres[p.index].bbox : p.kind == 1 ? quads[p.index].bbox : triangles[p.index].bbox;
    }

    std::optional<hit_record> hit_primitive(const primitive& p, const ray& r, interval t) const
    {
        return p.kind == 0 ? spheres[p.index].hit(r, t) : p.kind == 1 ? quads[p.index].hit(r, t)
                                                                         : triangles[p.index].hit(r, t);
    }

    // bvh.ixx:53-84: an object-median split on the longest axis of the common box, sorted by the boxes' min there
    void build()
    {
        std::vector<primitive> prims;
        for (int i = 0; i < static_cast<int>(spheres.size()); ++i)
        {
            prims.push_back({0, i});
        }
        for (int i = 0; i < static_cast<int>(quads.size()); ++i)
        {
            prims.push_back({1, i});
        }
        for (int i = 0; i < static_cast<int>(triangles.size()); ++i)
        {
            prims.push_back({2, i});
        }
        nodes_.clear();
        if (!prims.empty())
        {
            nodes_.reserve(prims.size() * 2);
            root_ = build(prims, 0, prims.size());
        }
    }

    std::optional<hit_record> hit(const ray& r, interval t) const // bvh_node::hit, bvh.ixx:26-37
    {
        if (nodes_.empty())
        {
            return std::nullopt;
        }
        return hit_node(root_, r, t, -1);
    }

    // The same search with the primitive `skip` left out (the lamp a shadow ray aims at, shadow.cuh:26-109)
    std::optional<hit_record> hit_except(const ray& r, interval t, int skip) const
    {
        if (nodes_.empty())
        {
            return std::nullopt;
        }
        return hit_node(root_, r, t, skip);
    }

    // Primitive `id` alone (source index space: spheres, then quads, then triangles), for the first-hit test's tie
    // rule: where it is hit along the ray in double, if at all
    std::optional<hit_record> hit_id(int id, const ray& r, interval t, double slack = 0) const
    {
        const auto n_spheres = static_cast<int>(spheres.size());
        const auto n_quads = static_cast<int>(quads.size());
        if (id < 0)
        {
            return std::nullopt;
        }
        if (id < n_spheres)
        {
            return spheres[static_cast<size_t>(id)].hit(r, t);
        }
        if (id < n_spheres + n_quads)
        {
            return quads[static_cast<size_t>(id - n_spheres)].hit(r, t, slack);
        }
        const auto k = static_cast<size_t>(id - n_spheres - n_quads);
        return k < triangles.size() ? triangles[k].hit(r, t, slack) : std::nullopt;
    }

    // The closest hit by testing every primitive in turn (hittable_list::hit, hittable.ixx:170-183): the brute-force
    // check the first-hit parity test compares against
    std::optional<hit_record> hit_brute_force(const ray& r, interval t) const
    {
        std::optional<hit_record> closest;
        const auto visit = [&](const std::optional<hit_record>& rec) {
            if (rec)
            {
                t.max = rec->t;
                closest = rec;
            }
        };
        for (const sphere& s : spheres)
        {
            visit(s.hit(r, t));
        }
        for (const quad& q : quads)
        {
            visit(q.hit(r, t));
        }
        for (const triangle& tr : triangles)
        {
            visit(tr.hit(r, t));
        }
        return closest;
    }

private:
    struct node
    {
        aabb box;
        int left = -1, right = -1; // node indices, or -1
        primitive leaf{-1, -1};    // kind -1: an inner node
    };
    std::vector<node> nodes_;
    int root_ = 0;

    int build(std::vector<primitive>& prims, size_t begin, size_t end)
    {
        const int index = static_cast<int>(nodes_.size());
        nodes_.push_back({});
        if (end - begin == 1)
        {
            nodes_[index].leaf = prims[begin];
            nodes_[index].box = box_of(prims[begin]);
            return index;
        }
        aabb box;
        for (size_t i = begin; i < end; ++i)
        {
            box = enclose(box, box_of(prims[i]));
        }
        const int axis = box.longest_axis();
        std::sort(prims.begin() + static_cast<std::ptrdiff_t>(begin), prims.begin() + static_cast<std::ptrdiff_t>(end),
                  [&](const primitive& a, const primitive& b) {
                      return box_of(a).axis_interval(axis).min < box_of(b).axis_interval(axis).min;
                  });
        const size_t middle = begin + (end - begin) / 2;
        const int left = build(prims, begin, middle);
        const int right = build(prims, middle, end);
        nodes_[index].left = left;
        nodes_[index].right = right;
        nodes_[index].box = enclose(nodes_[left].box, nodes_[right].box);
        return index;
    }

    std::optional<hit_record> hit_node(int index, const ray& r, interval t, int skip) const
    {
        const node& n = nodes_[index];
        if (n.leaf.kind >= 0)
        {
            auto rec = hit_primitive(n.leaf, r, t);
            if (rec && rec->id == skip)
            {
                return std::nullopt;
            }
            return rec;
        }
        if (!n.box.hit(r, t))
        {
            return std::nullopt;
        }
        const auto hit_left = hit_node(n.left, r, t, skip);
        const auto hit_right = hit_node(n.right, r, interval{t.min, hit_left ? hit_left->t : t.max}, skip);
        return hit_right ? hit_right : hit_left;
    }
};

// ---- materials: material.ixx -----------------------------------------------------------------------------------
struct material
{
    int kind = RT_LAMBERTIAN;
    color albedo;            // lambertian, diffuse_light, isotropic: the solid texture's color; metal: its albedo
    int texture = -1;        // lambertian, diffuse_light, isotropic: its texture when it is not one solid color
    double fuzz = 0;
    double refraction_index = 1;
    int lobe = RT_MICROFACET_NONE; // the quality integrator's GGX side entry (renderer.h:249-261)
    double roughness = 0;
    double alpha = 0;              // r^2, rounded to float as the GPU's
};

// ---- texture.ixx and perlin.ixx: solid, checker, image and marble textures, in double ----------------------------
struct perlin_table
{
    std::array<vec3, 256> gradients;
    std::array<int, 256> perm_x, perm_y, perm_z;

    double noise(const point3& p) const // perlin.ixx noise: Hermite-smoothed trilinear sum of gradient dot products
    {
        const double fx = std::floor(p.x), fy = std::floor(p.y), fz = std::floor(p.z);
        const double u = p.x - fx, v = p.y - fy, w = p.z - fz;
        const int i = static_cast<int>(fx), j = static_cast<int>(fy), k = static_cast<int>(fz);
        const double uu = u * u * (3 - 2 * u), vv = v * v * (3 - 2 * v), ww = w * w * (3 - 2 * w);
        double accum = 0;
        for (int di = 0; di < 2; ++di)
        {
            for (int dj = 0; dj < 2; ++dj)
            {
                for (int dk = 0; dk < 2; ++dk)
                {
                    const vec3& g = gradients[static_cast<size_t>(perm_x[(i + di) & 255] ^ perm_y[(j + dj) & 255] ^
                                                                  perm_z[(k + dk) & 255])];
                    const vec3 offset{u - di, v - dj, w - dk};
                    accum += (di * uu + (1 - di) * (1 - uu)) * (dj * vv + (1 - dj) * (1 - vv)) *
                             (dk * ww + (1 - dk) * (1 - ww)) * dot(g, offset);
                }
            }
        }
        return accum;
    }

    double turbulence(point3 p, int depth) const // perlin.ixx turb
    {
        double accum = 0;
        double weight = 1;
        for (int layer = 0; layer < depth; ++layer)
        {
            accum += weight * noise(p);
            weight *= 0.5;
            p = 2 * p;
        }
        return std::fabs(accum);
    }
};

struct image_texture_data
{
    int width = 0, height = 0;
    std::vector<float> rgb; // rows from the top
};

struct texture
{
    int kind = RT_TEXTURE_SOLID;
    color rgb;
    double inv_scale = 1;
    int even = -1, odd = -1, image = -1, perlin = -1;
    double scale = 1;
};

struct texture_set
{
    std::vector<texture> textures;
    std::vector<image_texture_data> images;
    std::vector<perlin_table> perlins;

    // texture::value at (u, v) and the point p (texture.ixx): a checker picks its texture by the parity of p's cube,
    // an image the pixel (u, v) falls in (clamped, v flipped), a marble 0.5 (1 + sin(scale z + 10 turb(p)))
    color value(int index, double u, double v, const point3& p) const
    {
        const texture& t = textures[static_cast<size_t>(index)];
        switch (t.kind)
        {
        case RT_TEXTURE_CHECKER:
        {
            const int x = static_cast<int>(std::floor(t.inv_scale * p.x));
            const int y = static_cast<int>(std::floor(t.inv_scale * p.y));
            const int z = static_cast<int>(std::floor(t.inv_scale * p.z));
            return value((x + y + z) % 2 == 0 ? t.even : t.odd, u, v, p);
        }
        case RT_TEXTURE_IMAGE:
        {
            const image_texture_data& im = images[static_cast<size_t>(t.image)];
            const double cu = std::clamp(u, 0.0, 1.0);
            const double cv = 1.0 - std::clamp(v, 0.0, 1.0);
            const int i = std::min(static_cast<int>(cu * im.width), im.width - 1);
            const int j = std::min(static_cast<int>(cv * im.height), im.height - 1);
            const float* px = im.rgb.data() + 3 * (static_cast<size_t>(j) * im.width + i);
            return {px[0], px[1], px[2]};
        }
        case RT_TEXTURE_NOISE:
        {
            const double gray =
                0.5 * (1 + std::sin(t.scale * p.z + 10 * perlins[static_cast<size_t>(t.perlin)].turbulence(p, 7)));
            return {gray, gray, gray};
        }
        default:
            return t.rgb;
        }
    }
};

// ---- constant_medium.ixx: a volume of smoke of constant density inside a boundary --------------------------------
struct medium
{
    std::unique_ptr<sphere> ball;  // the boundary: a sphere, or
    std::vector<quad> faces;       // the quads of a convex shape
    double neg_inv_density = 0;
    int material = -1;

    // The boundary's nearest hit in t (the quads' nearest one, as a hittable_list of them)
    std::optional<hit_record> boundary_hit(const ray& r, interval t) const
    {
        if (ball)
        {
            return ball->hit(r, t);
        }
        std::optional<hit_record> closest;
        for (const quad& q : faces)
        {
            if (auto rec = q.hit(r, t))
            {
                t.max = rec->t;
                closest = rec;
            }
        }
        return closest;
    }

    // The stretch of ray_t inside the volume (constant_medium.ixx:35-62): the boundary's first hit anywhere on the line
    // and its next one 0.0001 beyond, clamped to ray_t
    bool stretch(const ray& r, interval ray_t, double& t_in, double& t_out) const
    {
        const auto rec1 = boundary_hit(r, interval{-infinity, infinity});
        if (!rec1)
        {
            return false;
        }
        const auto rec2 = boundary_hit(r, interval{rec1->t + 0.0001, infinity});
        if (!rec2)
        {
            return false;
        }
        t_in = std::max(rec1->t, ray_t.min);
        t_out = std::min(rec2->t, ray_t.max);
        if (t_in >= t_out)
        {
            return false;
        }
        t_in = std::max(t_in, 0.0);
        return true;
    }

    // constant_medium::hit: a particle met after an exponential free flight, or nothing
    std::optional<double> hit(const ray& r, interval ray_t, rng& g) const
    {
        double t_in, t_out;
        if (!stretch(r, ray_t, t_in, t_out))
        {
            return std::nullopt;
        }
        const double length = r.direction.length();
        const double distance_inside = (t_out - t_in) * length;
        const double hit_distance = neg_inv_density * std::log(g.next());
        if (hit_distance > distance_inside)
        {
            return std::nullopt;
        }
        return t_in + hit_distance / length;
    }
};

inline double reflectance(double cosine, double refraction_index) // material.ixx:101-107 (Schlick)
{
    double r0 = (1 - refraction_index) / (1 + refraction_index);
    r0 = r0 * r0;
    return r0 + (1 - r0) * std::pow(1 - cosine, 5);
}

// ---- the lights list (hittable_list::pdf_value and random, hittable.ixx:146-168) --------------------------------
struct light_entry
{
    int kind; // RT_LIGHT_*
    std::unique_ptr<quad> q;
    std::unique_ptr<sphere> s;
    double weight = 0;
    double cdf = 0;
};

struct scene
{
    world geometry;
    std::vector<material> materials;
    std::vector<light_entry> lights;
    texture_set textures;
    std::vector<medium> media;
    rt_camera_desc camera{};
    int sampling = RT_SAMPLING_MATERIAL;
    color sky_bottom, sky_top;

    // What the ray meets first: the closest surface, or a particle of smoke before it (the CPU's world.hit over a list
    // that holds the volumes; each volume tested against the closest event so far), with the material's color there
    // in rec.color_at. A particle's record: normal (1, 0, 0), the front, id -1.
    std::optional<hit_record> closest_event(const ray& r, rng& g) const
    {
        auto rec = geometry.hit(r, interval{0.001, infinity});
        for (const medium& m : media)
        {
            if (const auto t = m.hit(r, interval{0.001, rec ? rec->t : infinity}, g))
            {
                hit_record particle;
                particle.t = *t;
                particle.p = r.at(*t);
                particle.normal = {1, 0, 0};
                particle.front_face = true;
                particle.material = m.material;
                particle.id = -1;
                rec = particle;
            }
        }
        if (rec)
        {
            const material& mm = materials[static_cast<size_t>(rec->material)];
            rec->color_at = mm.texture >= 0 ? textures.value(mm.texture, rec->u, rec->v, rec->p) : mm.albedo;
        }
        return rec;
    }

    // The chance that (0.001, t_max) of r crosses every volume without meeting a particle: exp(-sum density * length)
    double transmittance(const ray& r, double t_max) const
    {
        double exponent = 0;
        for (const medium& m : media)
        {
            double t_in, t_out;
            if (m.stretch(r, interval{0.001, t_max}, t_in, t_out))
            {
                exponent += (t_out - t_in) * r.direction.length() / m.neg_inv_density;
            }
        }
        return std::exp(exponent);
    }

    double lights_pdf_value(const point3& origin, const vec3& direction) const
    {
        double sum = 0;
        for (const light_entry& l : lights)
        {
            sum += l.weight * (l.kind == RT_LIGHT_QUAD ? l.q->pdf_value(origin, direction)
                                                       : l.s->pdf_value(origin, direction));
        }
        return sum;
    }

    vec3 lights_random(const point3& origin, rng& g) const
    {
        // random_int(0, n - 1) for a flat list of equal weights; the running sums of the weights for nested lists
        const double xi = g.next();
        size_t k = 0;
        while (k + 1 < lights.size() && !(xi < lights[k].cdf))
        {
            ++k;
        }
        const light_entry& l = lights[k];
        return l.kind == RT_LIGHT_QUAD ? l.q->random(origin, g) : l.s->random(origin, g);
    }

    color sky(const vec3& direction) const // camera.ixx:18-28 sky::in_direction
    {
        const double a = 0.5 * (unit_vector(direction).y + 1.0);
        return (1.0 - a) * sky_bottom + a * sky_top;
    }
};

// Builds the oracle's scene from the flat tables. Tables it cannot render are reported through `error`.
inline bool make_scene(const rt_scene_desc& d, scene& s, const char** error)
{
    for (int64_t i = 0; i < d.image_count; ++i)
    {
        const rt_image_desc& im = d.images[i];
        image_texture_data data;
        data.width = im.width;
        data.height = im.height;
        data.rgb.assign(im.rgb, im.rgb + static_cast<size_t>(im.width) * static_cast<size_t>(im.height) * 3);
        s.textures.images.push_back(std::move(data));
    }
    for (int64_t i = 0; i < d.perlin_count; ++i)
    {
        perlin_table p;
        for (int k = 0; k < 256; ++k)
        {
            p.gradients[static_cast<size_t>(k)] = from(d.perlins[i].random_vectors[k]);
            p.perm_x[static_cast<size_t>(k)] = d.perlins[i].perm_x[k];
            p.perm_y[static_cast<size_t>(k)] = d.perlins[i].perm_y[k];
            p.perm_z[static_cast<size_t>(k)] = d.perlins[i].perm_z[k];
        }
        s.textures.perlins.push_back(p);
    }
    for (int64_t i = 0; i < d.texture_count; ++i)
    {
        const rt_texture_desc& t = d.textures[i];
        texture tt;
        tt.kind = t.kind;
        tt.rgb = from(t.rgb);
        tt.inv_scale = t.inv_scale;
        tt.even = t.even;
        tt.odd = t.odd;
        tt.image = t.image;
        tt.perlin = t.perlin;
        tt.scale = t.scale;
        s.textures.textures.push_back(tt);
    }
    for (int64_t i = 0; i < d.material_count; ++i)
    {
        const rt_material_desc& m = d.materials[i];
        material mm;
        mm.kind = m.kind;
        mm.fuzz = std::min(m.fuzz, 1.0);
        mm.refraction_index = m.refraction_index;
        if (i < d.microfacet_count)
        {
            mm.lobe = d.microfacets[i].kind;
            mm.roughness = d.microfacets[i].roughness;
            mm.alpha = static_cast<float>(d.microfacets[i].roughness * d.microfacets[i].roughness);
        }
        if (m.kind == RT_METAL)
        {
            mm.albedo = from(m.albedo);
        }
        else if (m.kind != RT_DIELECTRIC)
        {
            if (m.texture < 0 || m.texture >= d.texture_count)
            {
                *error = "a material refers to a texture that doesn't exist";
                return false;
            }
            mm.albedo = from(d.textures[m.texture].rgb);
            mm.texture = d.textures[m.texture].kind == RT_TEXTURE_SOLID ? -1 : m.texture;
        }
        s.materials.push_back(mm);
    }
    int id = 0;
    for (int64_t i = 0; i < d.sphere_count; ++i)
    {
        const rt_sphere_desc& sp = d.spheres[i];
        const point3 c = from(sp.center);
        s.geometry.spheres.emplace_back(c, c + from(sp.displacement), sp.radius, sp.material, id++);
        s.geometry.spheres.back().uv_cos = sp.uv_cos;
        s.geometry.spheres.back().uv_sin = sp.uv_sin;
    }
    for (int64_t i = 0; i < d.quad_count; ++i)
    {
        const rt_quad_desc& q = d.quads[i];
        s.geometry.quads.emplace_back(from(q.q), from(q.u), from(q.v), q.material, id++);
    }
    for (int64_t m = 0; m < d.mesh_count; ++m)
    {
        const rt_mesh_desc& mesh = d.meshes[m];
        for (int64_t t = 0; t < mesh.triangle_count; ++t)
        {
            const auto vertex = [&](uint32_t k) {
                return point3{mesh.positions[3 * k], mesh.positions[3 * k + 1], mesh.positions[3 * k + 2]};
            };
            s.geometry.triangles.emplace_back(vertex(mesh.indices[3 * t]), vertex(mesh.indices[3 * t + 1]),
                                              vertex(mesh.indices[3 * t + 2]), mesh.material, id++);
        }
    }
    for (int64_t i = 0; i < d.medium_count; ++i)
    {
        const rt_medium_desc& md = d.media[i];
        medium m;
        m.neg_inv_density = md.neg_inv_density;
        m.material = md.material;
        if (md.boundary == RT_BOUNDARY_SPHERE)
        {
            const point3 c = from(md.sphere.center);
            m.ball = std::make_unique<sphere>(c, c + from(md.sphere.displacement), md.sphere.radius, -1, -1);
        }
        else
        {
            for (int64_t k = 0; k < md.quad_count; ++k)
            {
                m.faces.emplace_back(from(md.quads[k].q), from(md.quads[k].u), from(md.quads[k].v), -1, -1);
            }
        }
        s.media.push_back(std::move(m));
    }
    double cdf = 0;
    for (int64_t i = 0; i < d.light_count; ++i)
    {
        const rt_light_desc& l = d.lights[i];
        light_entry e;
        e.kind = l.kind;
        e.weight = l.weight;
        cdf += l.weight;
        e.cdf = cdf;
        if (l.kind == RT_LIGHT_QUAD)
        {
            e.q = std::make_unique<quad>(from(l.quad.q), from(l.quad.u), from(l.quad.v), -1, -1);
        }
        else
        {
            const point3 c = from(l.center);
            e.s = std::make_unique<sphere>(c, c, l.radius, -1, -1);
        }
        s.lights.push_back(std::move(e));
    }
    s.camera = d.camera;
    s.sampling = d.camera.sampling;
    const bool aims = s.sampling == RT_SAMPLING_LIGHTS || s.sampling == RT_SAMPLING_MIXTURE;
    if (aims && s.lights.empty())
    {
        s.sampling = RT_SAMPLING_MATERIAL; // camera.ixx:56-62 effective_sampling
    }
    s.sky_bottom = from(d.camera.sky_bottom);
    s.sky_top = from(d.camera.sky_top);
    s.geometry.build();
    return true;
}

// ---- camera.ixx: get_ray and ray_color ----------------------------------------------------------------------
inline double cosine_density(const vec3& unit_normal, const vec3& direction) // pdf.ixx:22-26
{
    const double cosine = dot(unit_normal, unit_vector(direction));
    return cosine > 0 ? cosine / std::numbers::pi : 0.0;
}
constexpr double uniform_sphere_density = 1 / (4 * std::numbers::pi);

struct counters
{
    uint64_t rays = 0;
    uint64_t shadow_rays = 0;
};

// camera.ixx:303-336 get_ray with sample_square_stratified and defocus_disk_sample
inline ray get_ray(const scene& s, int i, int j, int s_i, int s_j, rng& g)
{
    const rt_camera_desc& c = s.camera;
    const double recip = 1.0 / c.sqrt_spp;
    const double px = (s_i + g.next()) * recip - 0.5;
    const double py = (s_j + g.next()) * recip - 0.5;
    const point3 pixel_sample = from(c.pixel00_loc) + ((i + px) * from(c.pixel_delta_u)) +
                                ((j + py) * from(c.pixel_delta_v));
    point3 origin = from(c.center);
    if (c.defocus)
    {
        const vec3 p = random_in_unit_disk(g);
        origin = from(c.center) + p.x * from(c.defocus_disk_u) + p.y * from(c.defocus_disk_v);
    }
    const double time = g.next();
    return ray{origin, pixel_sample - origin, time};
}

// camera.ixx:355-452 ray_color: the recursive estimator of the books' strategies
inline color ray_color(const scene& s, const ray& r, int depth, rng& g, counters& n)
{
    if (depth <= 0)
    {
        return {0, 0, 0};
    }
    const auto rec = s.closest_event(r, g);
    ++n.rays;
    if (!rec)
    {
        return s.sky(r.direction);
    }
    const material& m = s.materials[static_cast<size_t>(rec->material)];
    // material::emitted: a lamp glows on its front side only (material.ixx:125-128), its texture's color there
    const color emitted = m.kind == RT_DIFFUSE_LIGHT && rec->front_face ? rec->color_at : color{0, 0, 0};
    switch (m.kind)
    {
    case RT_DIFFUSE_LIGHT:
        return emitted;
    case RT_METAL: // material.ixx:45-56
    {
        const vec3 reflected = unit_vector(reflect(r.direction, rec->normal)) + m.fuzz * random_unit_vector(g);
        if (dot(reflected, rec->normal) <= 0)
        {
            return emitted;
        }
        return emitted + m.albedo * ray_color(s, ray{rec->p, reflected, r.time}, depth - 1, g, n);
    }
    case RT_DIELECTRIC: // material.ixx:72-93
    {
        const double ri = rec->front_face ? (1.0 / m.refraction_index) : m.refraction_index;
        const vec3 unit_direction = unit_vector(r.direction);
        const double cos_theta = std::fmin(dot(-unit_direction, rec->normal), 1.0);
        const double sin_theta = std::sqrt(1.0 - cos_theta * cos_theta);
        const bool cannot_refract = ri * sin_theta > 1.0;
        const vec3 direction = cannot_refract || reflectance(cos_theta, ri) > g.next()
                                   ? reflect(unit_direction, rec->normal)
                                   : refract(unit_direction, rec->normal, ri);
        return emitted + color{1, 1, 1} * ray_color(s, ray{rec->p, direction, r.time}, depth - 1, g, n);
    }
    default:
        break;
    }
    // A diffuse bounce: lambertian (cosine_pdf) or isotropic (sphere_pdf), drawn by the camera's strategy
    const bool matte = m.kind == RT_LAMBERTIAN;
    const onb uvw{rec->normal};
    const auto own_generate = [&]() { return matte ? uvw.transform(random_cosine_direction(g)) : random_unit_vector(g); };
    const auto own_value = [&](const vec3& d) { return matte ? cosine_density(rec->normal, d) : uniform_sphere_density; };
    const auto scattering_pdf = [&](const vec3& d) {
        return matte ? cosine_density(rec->normal, d) : uniform_sphere_density;
    };
    const auto finish = [&](const vec3& direction, double pdf_value) -> color {
        const double sp = scattering_pdf(direction);
        if (!(pdf_value > 0) || !(sp > 0))
        {
            return {0, 0, 0};
        }
        return rec->color_at * (sp / pdf_value) * ray_color(s, ray{rec->p, direction, r.time}, depth - 1, g, n);
    };
    int strategy = s.sampling;
    if (strategy == RT_SAMPLING_MIXTURE && !matte)
    {
        strategy = RT_SAMPLING_MATERIAL; // isotropic::mixes_in_lights is false
    }
    switch (strategy)
    {
    case RT_SAMPLING_UNIFORM:
    {
        const vec3 d = random_unit_vector(g);
        return emitted + finish(d, uniform_sphere_density);
    }
    case RT_SAMPLING_MATERIAL:
    {
        const vec3 d = own_generate();
        return emitted + finish(d, own_value(d));
    }
    case RT_SAMPLING_LIGHTS:
    {
        const vec3 d = s.lights_random(rec->p, g);
        return emitted + finish(d, s.lights_pdf_value(rec->p, d));
    }
    default: // mixture_pdf{hittable_pdf{lights, p}, material}: pdf.ixx:104-121
    {
        const vec3 d = g.next() < 0.5 ? s.lights_random(rec->p, g) : own_generate();
        const double p = 0.5 * s.lights_pdf_value(rec->p, d) + 0.5 * own_value(d);
        return emitted + finish(d, p);
    }
    }
}

inline color without_nan(const color& c) // camera.ixx:338-347
{
    return {std::isnan(c.x) ? 0.0 : c.x, std::isnan(c.y) ? 0.0 : c.y, std::isnan(c.z) ? 0.0 : c.z};
}
} // namespace oracle
