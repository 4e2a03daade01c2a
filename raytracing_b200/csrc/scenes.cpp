// Built-in scenes, restated from the reference's scene code (src/scenes.ixx:79-518 and src/gpu_scenes.ixx) and
// flattened the way its GPU translator flattens a CPU world (src/gpu_scene.ixx:89-168 placement, 670-745 lights):
// instances are baked into world coordinates, the lights list is flattened with weights 1/n multiplied down nested
// lists, and the camera is the frame the CPU's camera computes from its settings (src/camera.ixx:138-182).
//
// The scenes' random content is drawn once here, with std::mt19937_64 default-seeded as the CPU program's main thread
// is (src/random.ixx:9-25, scenes.ixx:74-76) and std::uniform_real_distribution: that is implementation-defined
// across standard libraries, so the cover scene built here is libstdc++'s, and every renderer (the oracle, the
// reference's own GPU build, this one) is fed the same serialized tables.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numbers>
#include <random>
#include <string>
#include <unordered_map>

#include "scene_store.h"

namespace rtb
{
namespace
{
rt_vec3 v3(double x, double y, double z) { return {x, y, z}; }
rt_vec3 add(rt_vec3 a, rt_vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
rt_vec3 sub(rt_vec3 a, rt_vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
rt_vec3 mul(double t, rt_vec3 v) { return {t * v.x, t * v.y, t * v.z}; }
rt_vec3 hadamard(rt_vec3 a, rt_vec3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
rt_vec3 divide(rt_vec3 v, double t) { return mul(1 / t, v); } // vec3.ixx: v / t = (1 / t) * v
double dot(rt_vec3 a, rt_vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
rt_vec3 cross(rt_vec3 u, rt_vec3 v)
{
    return {u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x};
}
double length(rt_vec3 v) { return std::sqrt(dot(v, v)); }
rt_vec3 unit_vector(rt_vec3 v) { return divide(v, length(v)); }
double degrees_to_radians(double d) { return d * std::numbers::pi / 180.0; }

// The main thread's generator of the CPU program (random.ixx:9-25): default-constructed, never reseeded while scenes
// are built. scene_seed != 0 reseeds it, for the batched jobs' cover variants that each have their own seed.
class scene_random
{
public:
    explicit scene_random(uint64_t seed)
    {
        if (seed != 0)
        {
            engine_.seed(seed);
        }
    }
    double next() { return std::uniform_real_distribution<double>(0.0, 1.0)(engine_); }
    double next(double lo, double hi) { return lo + (hi - lo) * next(); }
    rt_vec3 vec() // vec3::random(): brace-initialized, so drawn x, y, z in order
    {
        const double x = next();
        const double y = next();
        const double z = next();
        return {x, y, z};
    }
    rt_vec3 vec(double lo, double hi)
    {
        const double x = next(lo, hi);
        const double y = next(lo, hi);
        const double z = next(lo, hi);
        return {x, y, z};
    }

private:
    std::mt19937_64 engine_;
};

// gpu_scene.ixx:89-130 placement: a turn about y (rotate_y::to_world), then a shift
struct placement
{
    double cos_theta = 1;
    double sin_theta = 0;
    rt_vec3 offset{0, 0, 0};

    rt_vec3 turn(rt_vec3 v) const
    {
        return {cos_theta * v.x + sin_theta * v.z, v.y, -sin_theta * v.x + cos_theta * v.z};
    }
    rt_vec3 place(rt_vec3 p) const { return add(turn(p), offset); }
    placement translated(rt_vec3 by) const { return {cos_theta, sin_theta, place(by)}; }
    placement rotated_y(double degrees) const
    {
        const double s = std::sin(degrees_to_radians(degrees));
        const double c = std::cos(degrees_to_radians(degrees));
        return {cos_theta * c - sin_theta * s, sin_theta * c + cos_theta * s, offset};
    }
};

// quad.ixx:118-140 box(): six faces whose u x v points out of the box
void box_faces(rt_vec3 a, rt_vec3 b, std::vector<rt_quad_desc>& out, int material, const placement& where)
{
    const rt_vec3 mn{std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)};
    const rt_vec3 mx{std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)};
    const rt_vec3 dx{mx.x - mn.x, 0, 0};
    const rt_vec3 dy{0, mx.y - mn.y, 0};
    const rt_vec3 dz{0, 0, mx.z - mn.z};
    const rt_vec3 neg_dx = mul(-1, dx);
    const rt_vec3 neg_dz = mul(-1, dz);
    const rt_vec3 faces[6][3] = {
        {{mn.x, mn.y, mx.z}, dx, dy},     // front (z = max)
        {{mx.x, mn.y, mx.z}, neg_dz, dy}, // right (x = max)
        {{mx.x, mn.y, mn.z}, neg_dx, dy}, // back (z = min)
        {{mn.x, mn.y, mn.z}, dz, dy},     // left (x = min)
        {{mn.x, mx.y, mx.z}, dx, neg_dz}, // top (y = max)
        {{mn.x, mn.y, mn.z}, dx, dz},     // bottom (y = min)
    };
    for (const auto& f : faces)
    {
        rt_quad_desc q{};
        q.q = where.place(f[0]);
        q.u = where.turn(f[1]);
        q.v = where.turn(f[2]);
        q.material = material;
        out.push_back(q);
    }
}

rt_quad_desc make_quad(rt_vec3 q, rt_vec3 u, rt_vec3 v, int material)
{
    rt_quad_desc d{};
    d.q = q;
    d.u = u;
    d.v = v;
    d.material = material;
    return d;
}

rt_sphere_desc make_sphere(rt_vec3 center, double radius, int material)
{
    rt_sphere_desc s{};
    s.center = center;
    s.radius = std::fmax(0.0, radius);
    s.material = material;
    s.uv_cos = 1;
    s.uv_sin = 0;
    return s;
}

rt_light_desc quad_light(const rt_quad_desc& q, double weight)
{
    rt_light_desc l{};
    l.kind = RT_LIGHT_QUAD;
    l.quad = q;
    l.quad.material = 0;
    l.weight = weight;
    return l;
}

rt_light_desc sphere_light(rt_vec3 center, double radius, double weight)
{
    rt_light_desc l{};
    l.kind = RT_LIGHT_SPHERE;
    l.center = center;
    l.radius = radius;
    l.weight = weight;
    return l;
}

// camera.ixx:23-31 daylight_sky
constexpr rt_vec3 daylight_bottom{1.0, 1.0, 1.0};
constexpr rt_vec3 daylight_top{0.5, 0.7, 1.0};

// scenes.ixx:130-142 cover_camera
camera_settings cover_camera()
{
    camera_settings c;
    c.aspect_ratio = 16.0 / 9.0;
    c.image_width = 1920;
    c.samples_per_pixel = 500;
    c.max_depth = 50;
    c.vfov = 20;
    c.lookfrom = v3(13, 2, 3);
    c.lookat = v3(0, 0, 0);
    c.defocus_angle = 0.6;
    c.focus_dist = 10.0;
    c.sky_bottom = daylight_bottom;
    c.sky_top = daylight_top;
    return c;
}

// scenes.ixx:348-357 cornell_camera
camera_settings cornell_camera()
{
    camera_settings c;
    c.aspect_ratio = 1.0;
    c.image_width = 1080;
    c.samples_per_pixel = 1000;
    c.max_depth = 50;
    c.vfov = 40;
    c.lookfrom = v3(278, 278, -800);
    c.lookat = v3(278, 278, 0);
    return c;
}

// texture.ixx checker_texture(scale, even, odd): the cubes of side `scale`, two solid colors
int checker_texture(scene_store& s, double scale, rt_vec3 even, rt_vec3 odd)
{
    const int e = s.add_solid_texture(even);
    const int o = s.add_solid_texture(odd);
    rt_texture_desc t{};
    t.kind = RT_TEXTURE_CHECKER;
    t.even = e;
    t.odd = o;
    t.image = t.perlin = -1;
    t.inv_scale = 1.0 / scale;
    t.scale = 1;
    s.textures.push_back(t);
    return static_cast<int>(s.textures.size()) - 1;
}

// A material that reads a texture (lambertian, diffuse_light or isotropic)
int textured(scene_store& s, int kind, int texture)
{
    rt_material_desc m{};
    m.kind = kind;
    m.texture = texture;
    m.refraction_index = 1;
    return s.add_material(m);
}

// constant_medium(boundary, density, albedo): a volume of smoke, its phase function an isotropic material
void add_medium(scene_store& s, const rt_sphere_desc* ball, const std::vector<rt_quad_desc>* faces, double density,
                rt_vec3 albedo)
{
    medium_store m;
    m.desc.material = textured(s, RT_ISOTROPIC, s.add_solid_texture(albedo));
    m.desc.neg_inv_density = -1.0 / density;
    if (ball)
    {
        m.desc.boundary = RT_BOUNDARY_SPHERE;
        m.desc.sphere = *ball;
    }
    else
    {
        m.desc.boundary = RT_BOUNDARY_CONVEX_QUADS;
        m.quads = *faces;
    }
    s.media.push_back(std::move(m));
}

// scenes.ixx:79-127 random_spheres(bouncing): the first book's cover. grid_half: the grid runs a, b in [-grid_half,
// grid_half) (11 in the book); the small spheres keep the book's placement and material draws. bouncing: the second
// book's variant, a checker floor and matte spheres that jump by up to 0.5 while the shutter is open.
void cover_world(scene_store& s, scene_random& rng, int grid_half, bool bouncing = false)
{
    const int ground = bouncing ? textured(s, RT_LAMBERTIAN, checker_texture(s, 0.32, v3(0.2, 0.3, 0.1),
                                                                             v3(0.9, 0.9, 0.9)))
                                : s.lambertian(v3(0.5, 0.5, 0.5));
    s.spheres.push_back(make_sphere(v3(0, -1000, 0), 1000, ground));
    for (int a = -grid_half; a < grid_half; ++a)
    {
        for (int b = -grid_half; b < grid_half; ++b)
        {
            const double choose_mat = rng.next();
            const double cx = a + 0.9 * rng.next();
            const double cz = b + 0.9 * rng.next();
            const rt_vec3 center{cx, 0.2, cz};
            if (length(sub(center, v3(4, 0.2, 0))) <= 0.9)
            {
                continue;
            }
            int material;
            rt_vec3 jump{0, 0, 0};
            if (choose_mat < 0.8)
            {
                const rt_vec3 c1 = rng.vec();
                const rt_vec3 c2 = rng.vec();
                material = s.lambertian(hadamard(c1, c2));
                if (bouncing)
                {
                    jump = v3(0, rng.next(0, 0.5), 0);
                }
            }
            else if (choose_mat < 0.95)
            {
                const rt_vec3 albedo = rng.vec(0.5, 1);
                material = s.metal(albedo, rng.next(0, 0.5));
            }
            else
            {
                material = s.dielectric(1.5);
            }
            rt_sphere_desc ball = make_sphere(center, 0.2, material);
            ball.displacement = jump;
            s.spheres.push_back(ball);
        }
    }
    s.spheres.push_back(make_sphere(v3(0, 1, 0), 1.0, s.dielectric(1.5)));
    s.spheres.push_back(make_sphere(v3(-4, 1, 0), 1.0, s.lambertian(v3(0.4, 0.2, 0.1))));
    s.spheres.push_back(make_sphere(v3(4, 1, 0), 1.0, s.metal(v3(0.7, 0.6, 0.5), 0.0)));
}

// scenes.ixx:294-305 add_cornell_walls
void cornell_walls(scene_store& s)
{
    const int red = s.lambertian(v3(0.65, 0.05, 0.05));
    const int white = s.lambertian(v3(0.73, 0.73, 0.73));
    const int green = s.lambertian(v3(0.12, 0.45, 0.15));
    s.quads.push_back(make_quad(v3(555, 0, 0), v3(0, 555, 0), v3(0, 0, 555), green));
    s.quads.push_back(make_quad(v3(0, 0, 0), v3(0, 555, 0), v3(0, 0, 555), red));
    s.quads.push_back(make_quad(v3(0, 0, 0), v3(555, 0, 0), v3(0, 0, 555), white));
    s.quads.push_back(make_quad(v3(555, 555, 555), v3(-555, 0, 0), v3(0, 0, -555), white));
    s.quads.push_back(make_quad(v3(0, 0, 555), v3(555, 0, 0), v3(0, 555, 0), white));
}

// scenes.ixx:331-335 cornell_lamp
rt_quad_desc cornell_lamp(int material)
{
    return make_quad(v3(343, 554, 332), v3(-130, 0, 0), v3(0, 0, -105), material);
}

// scenes.ixx:310-322 tall_block / short_block: box, rotate_y, translate
void tall_block(scene_store& s, int material)
{
    const placement where = placement{}.translated(v3(265, 0, 295)).rotated_y(15);
    box_faces(v3(0, 0, 0), v3(165, 330, 165), s.quads, material, where);
}

void short_block(scene_store& s, int material)
{
    const placement where = placement{}.translated(v3(130, 0, 65)).rotated_y(-18);
    box_faces(v3(0, 0, 0), v3(165, 165, 165), s.quads, material, where);
}

// perlin.ixx: 256 random unit gradients and three Fisher-Yates permutations of 0..255, drawn from the scene's
// generator in that order; noise() blends the 8 lattice corners' dot products with Hermite weights; turbulence() sums
// `depth` octaves, each twice as fine and half as strong, and takes the absolute value
class perlin_noise
{
public:
    explicit perlin_noise(scene_random& rng)
    {
        for (rt_vec3& v : gradients_)
        {
            v = unit_vector(rng.vec(-1, 1));
        }
        permute(perm_x_, rng);
        permute(perm_y_, rng);
        permute(perm_z_, rng);
    }

    double noise(rt_vec3 p) const
    {
        const double fx = std::floor(p.x), fy = std::floor(p.y), fz = std::floor(p.z);
        const int i = static_cast<int>(fx), j = static_cast<int>(fy), k = static_cast<int>(fz);
        const double u = p.x - fx, v = p.y - fy, w = p.z - fz;
        const double uu = u * u * (3 - 2 * u), vv = v * v * (3 - 2 * v), ww = w * w * (3 - 2 * w);
        double accum = 0;
        for (int di = 0; di < 2; ++di)
        {
            for (int dj = 0; dj < 2; ++dj)
            {
                for (int dk = 0; dk < 2; ++dk)
                {
                    const rt_vec3& g = gradients_[static_cast<size_t>(perm_x_[(i + di) & 255] ^ perm_y_[(j + dj) & 255] ^
                                                                      perm_z_[(k + dk) & 255])];
                    const rt_vec3 offset{u - di, v - dj, w - dk};
                    accum += (di * uu + (1 - di) * (1 - uu)) * (dj * vv + (1 - dj) * (1 - vv)) *
                             (dk * ww + (1 - dk) * (1 - ww)) * dot(g, offset);
                }
            }
        }
        return accum;
    }

    double turbulence(rt_vec3 p, int depth) const
    {
        double accum = 0;
        double weight = 1;
        for (int layer = 0; layer < depth; ++layer)
        {
            accum += weight * noise(p);
            weight *= 0.5;
            p = mul(2, p);
        }
        return std::fabs(accum);
    }

    // The tables as a scene's perlin_desc (renderer.h:85-93)
    rt_perlin_desc desc() const
    {
        rt_perlin_desc d{};
        for (size_t k = 0; k < 256; ++k)
        {
            d.random_vectors[k] = gradients_[k];
            d.perm_x[k] = perm_x_[k];
            d.perm_y[k] = perm_y_[k];
            d.perm_z[k] = perm_z_[k];
        }
        return d;
    }

private:
    std::array<rt_vec3, 256> gradients_;
    std::array<int, 256> perm_x_, perm_y_, perm_z_;

    static void permute(std::array<int, 256>& perm, scene_random& rng)
    {
        for (int i = 0; i < 256; ++i)
        {
            perm[static_cast<size_t>(i)] = i;
        }
        for (int i = 255; i > 0; --i)
        {
            const int target = static_cast<int>(rng.next(0, i + 1)); // random_int(0, i)
            std::swap(perm[static_cast<size_t>(i)], perm[static_cast<size_t>(target)]);
        }
    }
};

// texture.ixx noise_texture(scale): a marble of its own Perlin tables, drawn from the scene's generator here
int noise_texture(scene_store& s, scene_random& rng, double scale)
{
    const perlin_noise noise(rng);
    s.perlins.push_back(noise.desc());
    rt_texture_desc t{};
    t.kind = RT_TEXTURE_NOISE;
    t.even = t.odd = t.image = -1;
    t.perlin = static_cast<int>(s.perlins.size()) - 1;
    t.inv_scale = 1;
    t.scale = scale;
    s.textures.push_back(t);
    return static_cast<int>(s.textures.size()) - 1;
}

// An image texture of a synthetic planet, `width` x width/2, linear colors: oceans and continents from a turbulence
// field over the sphere, ice towards the poles. It stands in for the reference's assets/earthmap.jpg (a photograph
// this project does not ship): the same kind of texture and the same lookups.
int planet_texture(scene_store& s, scene_random& rng, int width)
{
    const int height = width / 2;
    const perlin_noise noise(rng);
    std::vector<float> rgb(static_cast<size_t>(width) * height * 3);
    for (int j = 0; j < height; ++j)
    {
        for (int i = 0; i < width; ++i)
        {
            const double phi = 2 * std::numbers::pi * (i + 0.5) / width;
            const double theta = std::numbers::pi * (j + 0.5) / height;
            const rt_vec3 n{std::sin(theta) * std::cos(phi), std::cos(theta), std::sin(theta) * std::sin(phi)};
            const double land = noise.turbulence(mul(3, n), 5);
            const bool ice = std::fabs(n.y) > 0.85;
            const rt_vec3 c = ice ? v3(0.85, 0.88, 0.9) : land > 0.35 ? v3(0.25 + 0.3 * land, 0.35, 0.12)
                                                                      : v3(0.02, 0.08, 0.25 + 0.3 * land);
            float* out = rgb.data() + 3 * (static_cast<size_t>(j) * width + i);
            out[0] = static_cast<float>(c.x);
            out[1] = static_cast<float>(c.y);
            out[2] = static_cast<float>(c.z);
        }
    }
    rt_image_desc im{};
    im.width = width;
    im.height = height;
    s.images.push_back(im);
    s.image_pixels.push_back(std::move(rgb));
    rt_texture_desc t{};
    t.kind = RT_TEXTURE_IMAGE;
    t.even = t.odd = t.perlin = -1;
    t.image = static_cast<int>(s.images.size()) - 1;
    t.inv_scale = 1;
    t.scale = 1;
    s.textures.push_back(t);
    return static_cast<int>(s.textures.size()) - 1;
}

// meshes.ixx:159-230 icosphere(level): the icosahedron, its faces turned counter-clockwise seen from outside, each
// triangle cut into four `level` times with the edge midpoints pushed onto the unit sphere (shared between the two
// triangles of an edge): V = 10 * 4^k + 2 vertices and T = 20 * 4^k triangles
void icosphere(int level, std::vector<rt_vec3>& points, std::vector<std::array<uint32_t, 3>>& faces)
{
    const double phi = (1 + std::sqrt(5.0)) / 2;
    points = {{-1, phi, 0}, {1, phi, 0},  {-1, -phi, 0}, {1, -phi, 0}, {0, -1, phi},  {0, 1, phi},
              {0, -1, -phi}, {0, 1, -phi}, {phi, 0, -1},  {phi, 0, 1},  {-phi, 0, -1}, {-phi, 0, 1}};
    for (rt_vec3& p : points)
    {
        p = unit_vector(p);
    }
    faces = {{0, 11, 5}, {0, 5, 1},  {0, 1, 7},   {0, 7, 10}, {0, 10, 11}, {1, 5, 9},  {5, 11, 4},
             {11, 10, 2}, {10, 7, 6}, {7, 1, 8},   {3, 9, 4},  {3, 4, 2},   {3, 2, 6},  {3, 6, 8},
             {3, 8, 9},  {4, 9, 5},  {2, 4, 11},  {6, 2, 10}, {8, 6, 7},   {9, 8, 1}};
    for (auto& f : faces)
    {
        if (dot(cross(sub(points[f[1]], points[f[0]]), sub(points[f[2]], points[f[0]])), points[f[0]]) < 0)
        {
            std::swap(f[1], f[2]);
        }
    }
    for (int k = 0; k < level; ++k)
    {
        std::unordered_map<uint64_t, uint32_t> midpoints;
        midpoints.reserve(faces.size() * 3 / 2);
        const auto midpoint = [&](uint32_t a, uint32_t b) {
            const uint64_t key = (uint64_t{std::min(a, b)} << 32) | std::max(a, b);
            const auto [it, added] = midpoints.try_emplace(key, static_cast<uint32_t>(points.size()));
            if (added)
            {
                points.push_back(unit_vector(add(points[a], points[b])));
            }
            return it->second;
        };
        std::vector<std::array<uint32_t, 3>> finer;
        finer.reserve(faces.size() * 4);
        for (const auto& f : faces)
        {
            const uint32_t ab = midpoint(f[0], f[1]);
            const uint32_t bc = midpoint(f[1], f[2]);
            const uint32_t ca = midpoint(f[2], f[0]);
            finer.push_back({f[0], ab, ca});
            finer.push_back({f[1], bc, ab});
            finer.push_back({f[2], ca, bc});
            finer.push_back({ab, bc, ca});
        }
        faces = std::move(finer);
    }
}

// A synthetic equirectangular sky, +y up, row 0 at the top: the daylight gradient of camera.ixx:21-31 by the
// direction's height, plus a sun disc of angular diameter sun_degrees at radiance sun_radiance, its coverage of each
// texel measured by 8 x 8 sub-samples (so the sun's light is spread over the texels it really covers)
void sky_with_sun(int width, int height, rt_vec3 sun_dir, double sun_degrees, double sun_radiance,
                  std::vector<float>& rgb)
{
    rgb.assign(static_cast<size_t>(width) * height * 3, 0.0f);
    const double cos_sun = std::cos(degrees_to_radians(sun_degrees / 2));
    const auto direction = [&](double u, double t) {
        const double ph = 2 * std::numbers::pi * (u - 0.5);
        const double th = std::numbers::pi * t;
        return rt_vec3{std::sin(th) * std::cos(ph), std::cos(th), std::sin(th) * std::sin(ph)};
    };
    // the texel size in angle, to find the texels near the sun
    const double texel_radians = std::numbers::pi / height;
    for (int j = 0; j < height; ++j)
    {
        for (int i = 0; i < width; ++i)
        {
            const rt_vec3 d = direction((i + 0.5) / width, (j + 0.5) / height);
            const double a = 0.5 * (d.y + 1.0);
            float* out = rgb.data() + 3 * (static_cast<size_t>(j) * width + i);
            out[0] = static_cast<float>((1 - a) * 1.0 + a * 0.5);
            out[1] = static_cast<float>((1 - a) * 1.0 + a * 0.7);
            out[2] = static_cast<float>((1 - a) * 1.0 + a * 1.0);
            if (std::acos(std::clamp(dot(d, sun_dir), -1.0, 1.0)) > degrees_to_radians(sun_degrees) + 4 * texel_radians)
            {
                continue;
            }
            int inside = 0;
            for (int sj = 0; sj < 8; ++sj)
            {
                for (int si = 0; si < 8; ++si)
                {
                    const rt_vec3 s = direction((i + (si + 0.5) / 8) / width, (j + (sj + 0.5) / 8) / height);
                    inside += dot(s, sun_dir) >= cos_sun ? 1 : 0;
                }
            }
            const auto sun = static_cast<float>(sun_radiance * inside / 64.0);
            out[0] += sun;
            out[1] += sun;
            out[2] += sun;
        }
    }
}

// Applies the overrides of rt_builtin_params to the scene's camera settings and computes the frame
void set_camera(scene_store& s, camera_settings c, const rt_builtin_params& p, bool has_lights)
{
    if (p.image_width > 0)
    {
        c.image_width = p.image_width;
    }
    if (p.samples_per_pixel > 0)
    {
        c.samples_per_pixel = p.samples_per_pixel;
    }
    if (p.max_depth > 0)
    {
        c.max_depth = p.max_depth;
    }
    if (p.sampling >= 0)
    {
        c.sampling = p.sampling;
    }
    if (p.orbit != 0)
    {
        // A random orbit camera for served requests: the look-at point fixed, the distance kept
        const rt_vec3 to = sub(c.lookfrom, c.lookat);
        const double r = length(to);
        const double az = degrees_to_radians(p.orbit_azimuth);
        const double el = degrees_to_radians(p.orbit_elevation);
        c.lookfrom = add(c.lookat, v3(r * std::cos(el) * std::sin(az), r * std::sin(el), r * std::cos(el) * std::cos(az)));
    }
    // camera.ixx:56-62 effective_sampling: lights and mixture need a lights list
    const bool aims = c.sampling == RT_SAMPLING_LIGHTS || c.sampling == RT_SAMPLING_MIXTURE;
    if (aims && !has_lights)
    {
        c.sampling = RT_SAMPLING_MATERIAL;
    }
    s.camera = camera_frame(c, p.image_height);
}
} // namespace

int scene_store::add_solid_texture(rt_vec3 rgb)
{
    rt_texture_desc t{};
    t.kind = RT_TEXTURE_SOLID;
    t.even = t.odd = t.image = t.perlin = -1;
    t.rgb = rgb;
    t.inv_scale = 1;
    t.scale = 1;
    textures.push_back(t);
    return static_cast<int>(textures.size()) - 1;
}

int scene_store::lambertian(rt_vec3 albedo)
{
    rt_material_desc m{};
    m.kind = RT_LAMBERTIAN;
    m.texture = add_solid_texture(albedo);
    m.refraction_index = 1;
    return add_material(m);
}

int scene_store::metal(rt_vec3 albedo, double fuzz)
{
    rt_material_desc m{};
    m.kind = RT_METAL;
    m.texture = -1;
    m.albedo = albedo;
    m.fuzz = std::min(fuzz, 1.0); // material.ixx:44 caps it
    m.refraction_index = 1;
    return add_material(m);
}

int scene_store::dielectric(double refraction_index)
{
    rt_material_desc m{};
    m.kind = RT_DIELECTRIC;
    m.texture = -1;
    m.refraction_index = refraction_index;
    return add_material(m);
}

int scene_store::diffuse_light(rt_vec3 emit)
{
    rt_material_desc m{};
    m.kind = RT_DIFFUSE_LIGHT;
    m.texture = add_solid_texture(emit);
    m.refraction_index = 1;
    return add_material(m);
}

const rt_scene_desc& scene_store::finish()
{
    desc = rt_scene_desc{};
    desc.spheres = spheres.data();
    desc.sphere_count = static_cast<int64_t>(spheres.size());
    desc.materials = materials.data();
    desc.material_count = static_cast<int64_t>(materials.size());
    desc.camera = camera;
    desc.textures = textures.data();
    desc.texture_count = static_cast<int64_t>(textures.size());
    for (size_t i = 0; i < images.size(); ++i)
    {
        images[i].rgb = image_pixels[i].data();
    }
    desc.images = images.data();
    desc.image_count = static_cast<int64_t>(images.size());
    desc.perlins = perlins.data();
    desc.perlin_count = static_cast<int64_t>(perlins.size());
    desc.quads = quads.data();
    desc.quad_count = static_cast<int64_t>(quads.size());
    media_desc.clear();
    for (medium_store& m : media)
    {
        m.desc.quads = m.quads.data();
        m.desc.quad_count = static_cast<int64_t>(m.quads.size());
        media_desc.push_back(m.desc);
    }
    desc.media = media_desc.data();
    desc.medium_count = static_cast<int64_t>(media_desc.size());
    desc.lights = lights.data();
    desc.light_count = static_cast<int64_t>(lights.size());
    desc.combination = combination;
    desc.quality = quality;
    desc.microfacets = microfacets.data();
    desc.microfacet_count = static_cast<int64_t>(microfacets.size());
    if (has_environment)
    {
        environment.image.rgb = environment_pixels.data();
        desc.environment = &environment;
    }
    mesh_desc.clear();
    for (const mesh_store& m : meshes)
    {
        rt_mesh_desc d{};
        d.positions = m.positions.data();
        d.vertex_count = static_cast<int64_t>(m.positions.size() / 3);
        d.indices = m.indices.data();
        d.triangle_count = static_cast<int64_t>(m.indices.size() / 3);
        d.material = m.material;
        mesh_desc.push_back(d);
    }
    desc.meshes = mesh_desc.data();
    desc.mesh_count = static_cast<int64_t>(mesh_desc.size());
    return desc;
}

std::unique_ptr<scene_store> scene_store::copy_of(const rt_scene_desc& d)
{
    auto s = std::make_unique<scene_store>();
    s->spheres.assign(d.spheres, d.spheres + d.sphere_count);
    s->materials.assign(d.materials, d.materials + d.material_count);
    s->camera = d.camera;
    s->textures.assign(d.textures, d.textures + d.texture_count);
    for (int64_t i = 0; i < d.image_count; ++i)
    {
        const rt_image_desc& im = d.images[i];
        s->images.push_back(im);
        s->image_pixels.emplace_back(im.rgb, im.rgb + static_cast<size_t>(im.width) * im.height * 3);
    }
    s->perlins.assign(d.perlins, d.perlins + d.perlin_count);
    s->quads.assign(d.quads, d.quads + d.quad_count);
    for (int64_t i = 0; i < d.medium_count; ++i)
    {
        medium_store m;
        m.desc = d.media[i];
        m.quads.assign(d.media[i].quads, d.media[i].quads + d.media[i].quad_count);
        s->media.push_back(std::move(m));
    }
    s->lights.assign(d.lights, d.lights + d.light_count);
    s->combination = d.combination;
    s->quality = d.quality;
    s->microfacets.assign(d.microfacets, d.microfacets + d.microfacet_count);
    if (d.environment)
    {
        s->has_environment = true;
        s->environment = *d.environment;
        const rt_image_desc& im = d.environment->image;
        s->environment_pixels.assign(im.rgb, im.rgb + static_cast<size_t>(im.width) * im.height * 3);
    }
    for (int64_t i = 0; i < d.mesh_count; ++i)
    {
        mesh_store m;
        m.positions.assign(d.meshes[i].positions, d.meshes[i].positions + d.meshes[i].vertex_count * 3);
        m.indices.assign(d.meshes[i].indices, d.meshes[i].indices + d.meshes[i].triangle_count * 3);
        m.material = d.meshes[i].material;
        s->meshes.push_back(std::move(m));
    }
    s->finish();
    return s;
}

// camera.ixx:138-182: the viewport on the focus plane, the pixel grid and the lens disk
rt_camera_desc camera_frame(const camera_settings& s, int height_override)
{
    rt_camera_desc c{};
    c.image_width = s.image_width;
    c.image_height =
        height_override > 0 ? height_override : std::max(1, static_cast<int>(s.image_width / s.aspect_ratio));
    c.sqrt_spp = std::max(1, static_cast<int>(std::lround(std::sqrt(s.samples_per_pixel))));
    c.max_depth = s.max_depth;
    c.center = s.lookfrom;
    const double h = std::tan(degrees_to_radians(s.vfov) / 2);
    const double viewport_height = 2 * h * s.focus_dist;
    const double viewport_width = viewport_height * (static_cast<double>(c.image_width) / c.image_height);
    const rt_vec3 w = unit_vector(sub(s.lookfrom, s.lookat));
    const rt_vec3 u = unit_vector(cross(s.vup, w));
    const rt_vec3 v = cross(w, u);
    const rt_vec3 viewport_u = mul(viewport_width, u);
    const rt_vec3 viewport_v = mul(viewport_height, mul(-1, v));
    c.pixel_delta_u = divide(viewport_u, c.image_width);
    c.pixel_delta_v = divide(viewport_v, c.image_height);
    const rt_vec3 upper_left =
        sub(sub(sub(c.center, mul(s.focus_dist, w)), divide(viewport_u, 2)), divide(viewport_v, 2));
    c.pixel00_loc = add(upper_left, mul(0.5, add(c.pixel_delta_u, c.pixel_delta_v)));
    const double defocus_radius = s.focus_dist * std::tan(degrees_to_radians(s.defocus_angle / 2));
    c.defocus = s.defocus_angle > 0 ? 1 : 0;
    c.defocus_disk_u = mul(defocus_radius, u);
    c.defocus_disk_v = mul(defocus_radius, v);
    c.sky_bottom = s.sky_bottom;
    c.sky_top = s.sky_top;
    c.sampling = s.sampling;
    return c;
}

rt_status build_builtin(const std::string& name, const rt_builtin_params& p, std::unique_ptr<scene_store>& out,
                        std::string& error)
{
    auto s = std::make_unique<scene_store>();
    scene_random rng(p.scene_seed);
    if (name == "weekend")
    {
        cover_world(*s, rng, 11);
        set_camera(*s, cover_camera(), p, false);
    }
    else if (name.rfind("cover-", 0) == 0 || name == "cover")
    {
        // A cover variant of about N random spheres (a square grid of side round(sqrt(N)) centered like the book's
        // 22 x 22), the camera pulled back in proportion to the grid
        int n = p.sphere_count > 0 ? p.sphere_count : 484;
        if (name.size() > 6)
        {
            n = std::atoi(name.c_str() + 6);
        }
        if (n < 1 || n > 4000000)
        {
            error = "cover-N: N must be in [1, 4000000]";
            return RT_ERR_INVALID;
        }
        const int side = std::max(2, static_cast<int>(std::lround(std::sqrt(static_cast<double>(n)))));
        const int half = (side + 1) / 2;
        cover_world(*s, rng, half);
        camera_settings c = cover_camera();
        const double scale = std::max(1.0, half / 11.0);
        c.lookfrom = mul(scale, c.lookfrom);
        c.focus_dist = 10.0 * scale;
        set_camera(*s, c, p, false);
    }
    else if (name == "materials")
    {
        // scenes.ixx:149-171
        const int ground = s->lambertian(v3(0.8, 0.8, 0.0));
        const int center = s->lambertian(v3(0.1, 0.2, 0.5));
        const int left = s->dielectric(1.50);
        const int bubble = s->dielectric(1.00 / 1.50);
        const int right = s->metal(v3(0.8, 0.6, 0.2), 1.0);
        s->spheres.push_back(make_sphere(v3(0.0, -100.5, -1.0), 100.0, ground));
        s->spheres.push_back(make_sphere(v3(0.0, 0.0, -1.2), 0.5, center));
        s->spheres.push_back(make_sphere(v3(-1.0, 0.0, -1.0), 0.5, left));
        s->spheres.push_back(make_sphere(v3(-1.0, 0.0, -1.0), 0.4, bubble));
        s->spheres.push_back(make_sphere(v3(1.0, 0.0, -1.0), 0.5, right));
        camera_settings c = cover_camera();
        c.lookfrom = v3(-2, 2, 1);
        c.lookat = v3(0, 0, -1);
        c.defocus_angle = 10.0;
        c.focus_dist = 3.4;
        set_camera(*s, c, p, false);
    }
    else if (name == "quads")
    {
        // scenes.ixx:224-249
        const int left_red = s->lambertian(v3(1.0, 0.2, 0.2));
        const int back_green = s->lambertian(v3(0.2, 1.0, 0.2));
        const int right_blue = s->lambertian(v3(0.2, 0.2, 1.0));
        const int upper_orange = s->lambertian(v3(1.0, 0.5, 0.0));
        const int lower_teal = s->lambertian(v3(0.2, 0.8, 0.8));
        s->quads.push_back(make_quad(v3(-3, -2, 5), v3(0, 0, -4), v3(0, 4, 0), left_red));
        s->quads.push_back(make_quad(v3(-2, -2, 0), v3(4, 0, 0), v3(0, 4, 0), back_green));
        s->quads.push_back(make_quad(v3(3, -2, 1), v3(0, 0, 4), v3(0, 4, 0), right_blue));
        s->quads.push_back(make_quad(v3(-2, 3, 1), v3(4, 0, 0), v3(0, 0, 4), upper_orange));
        s->quads.push_back(make_quad(v3(-2, -3, 5), v3(4, 0, 0), v3(0, 0, -4), lower_teal));
        camera_settings c;
        c.aspect_ratio = 1.0;
        c.image_width = 1080;
        c.samples_per_pixel = 500;
        c.max_depth = 50;
        c.vfov = 80;
        c.lookfrom = v3(0, 0, 9);
        c.lookat = v3(0, 0, 0);
        c.sky_bottom = daylight_bottom;
        c.sky_top = daylight_top;
        set_camera(*s, c, p, false);
    }
    else if (name == "cornell")
    {
        // scenes.ixx:360-374: two white blocks, the lamp in the lights list
        cornell_walls(*s);
        s->quads.push_back(cornell_lamp(s->diffuse_light(v3(15, 15, 15))));
        const int white = s->lambertian(v3(0.73, 0.73, 0.73));
        tall_block(*s, white);
        short_block(*s, white);
        s->lights.push_back(quad_light(cornell_lamp(0), 1.0));
        set_camera(*s, cornell_camera(), p, true);
    }
    else if (name == "glass" || name == "cornell-mis")
    {
        // scenes.ixx:484-501: the Cornell box with a glass ball instead of the short block; the lights list holds
        // the lamp and the ball (weights 1/2 each, hittable_list::random)
        cornell_walls(*s);
        s->quads.push_back(cornell_lamp(s->diffuse_light(v3(15, 15, 15))));
        tall_block(*s, s->lambertian(v3(0.73, 0.73, 0.73)));
        s->spheres.push_back(make_sphere(v3(190, 90, 190), 90, s->dielectric(1.5)));
        s->lights.push_back(quad_light(cornell_lamp(0), 0.5));
        s->lights.push_back(sphere_light(v3(190, 90, 190), 90, 0.5));
        rt_builtin_params q = p;
        if (name == "cornell-mis")
        {
            // The quality integrator's -p mis: light samples at every vertex, power-heuristic MIS; its light set is
            // the lamps (lamps.cuh:1-8: the ball doesn't glow), and its strategy is the material's
            s->quality = 1;
            s->combination = RT_COMBINE_POWER_HEURISTIC;
            q.sampling = RT_SAMPLING_MATERIAL;
        }
        set_camera(*s, cornell_camera(), q, true);
    }
    else if (name == "bouncing")
    {
        // scenes.ixx:176-181: the cover with a checker floor and bouncing matte spheres (motion blur)
        cover_world(*s, rng, 11, true);
        set_camera(*s, cover_camera(), p, false);
    }
    else if (name == "checker")
    {
        // scenes.ixx:184-196: two huge spheres with one solid checker texture
        const int checker = textured(*s, RT_LAMBERTIAN, checker_texture(*s, 0.32, v3(0.2, 0.3, 0.1), v3(0.9, 0.9, 0.9)));
        s->spheres.push_back(make_sphere(v3(0, -10, 0), 10, checker));
        s->spheres.push_back(make_sphere(v3(0, 10, 0), 10, checker));
        camera_settings c = cover_camera();
        c.defocus_angle = 0;
        set_camera(*s, c, p, false);
    }
    else if (name == "earth")
    {
        // scenes.ixx:199-209: an image wrapped around a sphere (a synthetic planet: see planet_texture)
        const int surface = textured(*s, RT_LAMBERTIAN, planet_texture(*s, rng, p.env_width > 0 ? p.env_width : 512));
        s->spheres.push_back(make_sphere(v3(0, 0, 0), 2, surface));
        camera_settings c = cover_camera();
        c.lookfrom = v3(0, 0, 12);
        c.defocus_angle = 0;
        set_camera(*s, c, p, false);
    }
    else if (name == "perlin" || name == "light")
    {
        // scenes.ixx:212-222 perlin_spheres: marble spheres (one noise texture of scale 4 for both); light
        // (scenes.ixx:255-292): the same in the dark, lit by a glowing sphere and a glowing quad, both in the lights
        // list (quad first)
        const int marble = textured(*s, RT_LAMBERTIAN, noise_texture(*s, rng, 4));
        s->spheres.push_back(make_sphere(v3(0, -1000, 0), 1000, marble));
        s->spheres.push_back(make_sphere(v3(0, 2, 0), 2, marble));
        camera_settings c = cover_camera();
        c.defocus_angle = 0;
        bool has_lights = false;
        if (name == "light")
        {
            const int lamp = s->diffuse_light(v3(4, 4, 4));
            s->spheres.push_back(make_sphere(v3(0, 7, 0), 2, lamp));
            const rt_quad_desc quad_lamp = make_quad(v3(3, 1, -2), v3(2, 0, 0), v3(0, 2, 0), lamp);
            s->quads.push_back(quad_lamp);
            s->lights.push_back(quad_light(quad_lamp, 0.5));
            s->lights.push_back(sphere_light(v3(0, 7, 0), 2, 0.5));
            has_lights = true;
            c = camera_settings{};
            c.aspect_ratio = 16.0 / 9.0;
            c.image_width = 1920;
            c.samples_per_pixel = 1000;
            c.max_depth = 50;
            c.vfov = 20;
            c.lookfrom = v3(26, 3, 6);
            c.lookat = v3(0, 2, 0);
        }
        set_camera(*s, c, p, has_lights);
    }
    else if (name == "smoke")
    {
        // scenes.ixx:359-377: the Cornell box with blocks of black and white smoke (density 0.01) and a bigger,
        // dimmer lamp
        cornell_walls(*s);
        const rt_quad_desc lamp = make_quad(v3(113, 554, 127), v3(330, 0, 0), v3(0, 0, 305), 0);
        rt_quad_desc glowing = lamp;
        glowing.material = s->diffuse_light(v3(7, 7, 7));
        s->quads.push_back(glowing);
        std::vector<rt_quad_desc> tall;
        box_faces(v3(0, 0, 0), v3(165, 330, 165), tall, 0, placement{}.translated(v3(265, 0, 295)).rotated_y(15));
        std::vector<rt_quad_desc> small;
        box_faces(v3(0, 0, 0), v3(165, 165, 165), small, 0, placement{}.translated(v3(130, 0, 65)).rotated_y(-18));
        add_medium(*s, nullptr, &tall, 0.01, v3(0, 0, 0));
        add_medium(*s, nullptr, &small, 0.01, v3(1, 1, 1));
        s->lights.push_back(quad_light(lamp, 1.0));
        set_camera(*s, cornell_camera(), p, true);
    }
    else if (name == "final")
    {
        // scenes.ixx:380-461: the second book's final scene, its instances baked into world coordinates
        const int ground = s->lambertian(v3(0.48, 0.83, 0.53));
        for (int i = 0; i < 20; ++i)
        {
            for (int j = 0; j < 20; ++j)
            {
                const double w = 100.0;
                const rt_vec3 corner0{-1000.0 + i * w, 0.0, -1000.0 + j * w};
                const rt_vec3 corner1{corner0.x + w, rng.next(1, 101), corner0.z + w};
                box_faces(corner0, corner1, s->quads, ground, placement{});
            }
        }
        const rt_quad_desc lamp = make_quad(v3(123, 554, 147), v3(300, 0, 0), v3(0, 0, 265), 0);
        rt_quad_desc glowing = lamp;
        glowing.material = s->diffuse_light(v3(7, 7, 7));
        s->quads.push_back(glowing);
        rt_sphere_desc moving = make_sphere(v3(400, 400, 200), 50, s->lambertian(v3(0.7, 0.3, 0.1)));
        moving.displacement = v3(30, 0, 0);
        s->spheres.push_back(moving);
        s->spheres.push_back(make_sphere(v3(260, 150, 45), 50, s->dielectric(1.5)));
        s->spheres.push_back(make_sphere(v3(0, 150, 145), 50, s->metal(v3(0.8, 0.8, 0.9), 1.0)));
        const int glass = s->dielectric(1.5);
        const rt_sphere_desc boundary = make_sphere(v3(360, 150, 145), 70, glass);
        s->spheres.push_back(boundary);
        add_medium(*s, &boundary, nullptr, 0.2, v3(0.2, 0.4, 0.9));
        const rt_sphere_desc haze = make_sphere(v3(0, 0, 0), 5000, glass);
        add_medium(*s, &haze, nullptr, 0.0001, v3(1, 1, 1));
        const int earth = textured(*s, RT_LAMBERTIAN, planet_texture(*s, rng, p.env_width > 0 ? p.env_width : 512));
        s->spheres.push_back(make_sphere(v3(400, 200, 400), 100, earth));
        const int marble = textured(*s, RT_LAMBERTIAN, noise_texture(*s, rng, 0.2));
        s->spheres.push_back(make_sphere(v3(220, 280, 300), 80, marble));
        // A cloud of 1000 white balls in a 165^3 cube, turned 15 degrees about y and moved: the turn is kept for the
        // balls' texture coordinates
        const int white = s->lambertian(v3(0.73, 0.73, 0.73));
        const placement cloud = placement{}.translated(v3(-100, 270, 395)).rotated_y(15);
        for (int k = 0; k < 1000; ++k)
        {
            rt_sphere_desc ball = make_sphere(cloud.place(rng.vec(0, 165)), 10, white);
            ball.uv_cos = cloud.cos_theta;
            ball.uv_sin = cloud.sin_theta;
            s->spheres.push_back(ball);
        }
        s->lights.push_back(quad_light(lamp, 1.0));
        camera_settings c;
        c.aspect_ratio = 1.0;
        c.image_width = 1080;
        c.samples_per_pixel = 1000;
        c.max_depth = 40;
        c.vfov = 40;
        c.lookfrom = v3(478, 278, -600);
        c.lookat = v3(278, 278, 0);
        set_camera(*s, c, p, true);
    }
    else if (name == "aluminum")
    {
        // scenes.ixx:464-478: the Cornell box with a tall block of polished aluminum
        cornell_walls(*s);
        s->quads.push_back(cornell_lamp(s->diffuse_light(v3(15, 15, 15))));
        tall_block(*s, s->metal(v3(0.8, 0.85, 0.88), 0.0));
        short_block(*s, s->lambertian(v3(0.73, 0.73, 0.73)));
        s->lights.push_back(quad_light(cornell_lamp(0), 1.0));
        set_camera(*s, cornell_camera(), p, true);
    }
    else if (name == "feature-furnace")
    {
        // The white furnace with the second book's features in it: a moving sphere with a white-on-white checker, a
        // quad with an all-white image, a sphere and a box of white smoke. Every bounce keeps all of the light and
        // every path ends in the white sky, so every pixel is exactly 1 under the material's own sampling, whatever
        // the motion, the textures' lookups and the free flights do.
        const int checker = textured(*s, RT_LAMBERTIAN, checker_texture(*s, 0.25, v3(1, 1, 1), v3(1, 1, 1)));
        rt_sphere_desc ball = make_sphere(v3(0, 0, 0), 1.0, checker);
        ball.displacement = v3(0.4, 0.1, 0);
        s->spheres.push_back(ball);
        rt_image_desc im{};
        im.width = 4;
        im.height = 2;
        s->images.push_back(im);
        s->image_pixels.emplace_back(4 * 2 * 3, 1.0f);
        rt_texture_desc image{};
        image.kind = RT_TEXTURE_IMAGE;
        image.even = image.odd = image.perlin = -1;
        image.image = 0;
        image.inv_scale = 1;
        image.scale = 1;
        s->textures.push_back(image);
        s->quads.push_back(make_quad(v3(-2, -1.5, -1), v3(4, 0, 0), v3(0, 0, 2),
                                     textured(*s, RT_LAMBERTIAN, static_cast<int>(s->textures.size()) - 1)));
        // (the volumes stay clear of the sphere: smoke inside an opaque surface would trap its paths)
        const rt_sphere_desc fog = make_sphere(v3(2.1, 0.7, -0.5), 0.55, 0);
        add_medium(*s, &fog, nullptr, 0.6, v3(1, 1, 1));
        std::vector<rt_quad_desc> block;
        box_faces(v3(-2.4, -0.6, -0.4), v3(-1.7, 0.6, 0.4), block, 0, placement{}.rotated_y(20));
        add_medium(*s, nullptr, &block, 0.8, v3(1, 1, 1));
        camera_settings c;
        c.aspect_ratio = 16.0 / 9.0;
        c.image_width = 480;
        c.samples_per_pixel = 64;
        c.max_depth = 50;
        c.sampling = RT_SAMPLING_MATERIAL;
        c.vfov = 30;
        c.lookfrom = v3(0, 0, 6);
        c.lookat = v3(0, 0, 0);
        c.sky_bottom = v3(1, 1, 1);
        c.sky_top = v3(1, 1, 1);
        set_camera(*s, c, p, false);
    }
    else if (name == "furnace")
    {
        // gpu_scenes.ixx:33-55: a white sphere under a white sky, every pixel exactly 1 under -p material
        s->spheres.push_back(make_sphere(v3(0, 0, 0), 1.0, s->lambertian(v3(1, 1, 1))));
        camera_settings c;
        c.aspect_ratio = 16.0 / 9.0;
        c.image_width = 480;
        c.samples_per_pixel = 64;
        c.max_depth = 10;
        c.sampling = RT_SAMPLING_MATERIAL;
        c.vfov = 30;
        c.lookfrom = v3(0, 0, 6);
        c.lookat = v3(0, 0, 0);
        c.sky_bottom = v3(1, 1, 1);
        c.sky_top = v3(1, 1, 1);
        set_camera(*s, c, p, false);
    }
    else if (name == "env-furnace" || name == "ggx-furnace")
    {
        // gpu_scenes_environments.ixx:96-110 env-furnace: the white furnace's sphere and camera under a constant map
        // of radiance 1, every pixel exactly 1 under the material's own sampling. ggx-furnace (gpu_scenes.ixx:66-67,
        // one sphere): a white GGX conductor (F0 = 1, roughness sqrt(0.3), alpha 0.3) whose centre keeps, with
        // Turquin's compensation, all of the light (docs/quality.md:136-144)
        int material;
        if (name == "env-furnace")
        {
            material = s->lambertian(v3(1, 1, 1));
        }
        else
        {
            material = s->metal(v3(1, 1, 1), 0.0);
        }
        s->spheres.push_back(make_sphere(v3(0, 0, 0), 1.0, material));
        if (name == "ggx-furnace")
        {
            s->microfacets.assign(s->materials.size(), rt_microfacet_desc{});
            s->microfacets[static_cast<size_t>(material)] = {RT_MICROFACET_CONDUCTOR, 0, std::sqrt(0.3)};
        }
        const int w = p.env_width > 0 ? p.env_width : 64;
        s->has_environment = true;
        s->environment_pixels.assign(static_cast<size_t>(w) * (w / 2) * 3, 1.0f);
        s->environment.image.width = w;
        s->environment.image.height = w / 2;
        s->environment.scale = 1;
        s->quality = 1;
        s->combination = RT_COMBINE_BSDF_ONLY;
        camera_settings c;
        c.aspect_ratio = 16.0 / 9.0;
        c.image_width = 480;
        c.samples_per_pixel = 64;
        c.max_depth = 10;
        c.sampling = RT_SAMPLING_MATERIAL;
        c.vfov = 30;
        c.lookfrom = v3(0, 0, 6);
        c.lookat = v3(0, 0, 0);
        rt_builtin_params q = p;
        q.sampling = RT_SAMPLING_MATERIAL;
        set_camera(*s, c, q, false);
    }
    else if (name == "mesh-ggx")
    {
        // A triangle mesh under an HDR sky: an icosphere of level 8 (1,310,720 triangles) displaced along its normal by
        // 0.15 x 4-octave Perlin turbulence, a rough GGX metal (r = 0.3, F0 (0.95, 0.64, 0.54)), standing on a plane
        // under a glossy coat (rho 0.73, r = 0.2); lit by a 1024 x 512 sky gradient with a 0.5-degree sun of radiance
        // 5e4, 48 degrees high, sampled by its brightness. The NEE/MIS integrator, power heuristic.
        const int level = p.mesh_level > 0 ? std::min(p.mesh_level, 9) : 8;
        std::vector<rt_vec3> points;
        std::vector<std::array<uint32_t, 3>> faces;
        icosphere(level, points, faces);
        const perlin_noise noise(rng);
        const rt_vec3 center{0, 1.3, 0};
        mesh_store mesh;
        mesh.positions.reserve(points.size() * 3);
        for (const rt_vec3& v : points)
        {
            const double r = 1 + 0.15 * noise.turbulence(mul(2.0, v), 4);
            mesh.positions.push_back(static_cast<float>(center.x + r * v.x));
            mesh.positions.push_back(static_cast<float>(center.y + r * v.y));
            mesh.positions.push_back(static_cast<float>(center.z + r * v.z));
        }
        mesh.indices.reserve(faces.size() * 3);
        for (const auto& f : faces)
        {
            mesh.indices.insert(mesh.indices.end(), {f[0], f[1], f[2]});
        }
        const int metal = s->metal(v3(0.95, 0.64, 0.54), 0.0);
        const int plane = s->lambertian(v3(0.73, 0.73, 0.73));
        mesh.material = metal;
        s->meshes.push_back(std::move(mesh));
        s->quads.push_back(make_quad(v3(-100, 0, -100), v3(0, 0, 200), v3(200, 0, 0), plane));
        s->microfacets.resize(s->materials.size());
        for (rt_microfacet_desc& f : s->microfacets)
        {
            f = rt_microfacet_desc{};
        }
        s->microfacets[static_cast<size_t>(metal)] = {RT_MICROFACET_CONDUCTOR, 0, 0.3};
        s->microfacets[static_cast<size_t>(plane)] = {RT_MICROFACET_GLOSS, 0, 0.2};
        const int env_width = p.env_width > 0 ? p.env_width : 1024;
        const double elevation = degrees_to_radians(48);
        const double azimuth = degrees_to_radians(35);
        const rt_vec3 sun{std::cos(elevation) * std::sin(azimuth), std::sin(elevation),
                          std::cos(elevation) * std::cos(azimuth)};
        s->has_environment = true;
        sky_with_sun(env_width, env_width / 2, sun, 0.5, 5e4, s->environment_pixels);
        s->environment.image.width = env_width;
        s->environment.image.height = env_width / 2;
        s->environment.yaw_degrees = 0;
        s->environment.scale = 1;
        s->quality = 1;
        s->combination = RT_COMBINE_POWER_HEURISTIC;
        camera_settings c;
        c.aspect_ratio = 16.0 / 9.0;
        c.image_width = 1920;
        c.samples_per_pixel = 256;
        c.max_depth = 16;
        c.sampling = RT_SAMPLING_MATERIAL;
        c.vfov = 30;
        c.lookfrom = v3(0, 2, 9);
        c.lookat = v3(0, 1.1, 0);
        rt_builtin_params q = p;
        q.sampling = RT_SAMPLING_MATERIAL;
        set_camera(*s, c, q, false);
    }
    else
    {
        error = "unknown built-in scene '" + name + "'";
        return RT_ERR_INVALID;
    }
    if (p.combination >= 0)
    {
        // A combination asks for the NEE/MIS integrator (the reference's quality kernel, -p material/nee/mis), which
        // samples bounces as the material scatters
        s->combination = p.combination;
        s->quality = 1;
        s->camera.sampling = RT_SAMPLING_MATERIAL;
    }
    s->finish();
    out = std::move(s);
    return RT_OK;
}

// ---- serialization: a little-endian binary file of the tables ---------------------------------------------------

namespace
{
constexpr char magic[8] = {'R', 'T', 'B', '2', 'S', 'C', 'N', '1'};

struct writer
{
    FILE* f;
    bool ok = true;
    void bytes(const void* p, size_t n)
    {
        if (n > 0 && std::fwrite(p, 1, n, f) != n)
        {
            ok = false;
        }
    }
    template <class T>
    void value(const T& v) { bytes(&v, sizeof(T)); }
    template <class T>
    void array(const T* p, int64_t n)
    {
        value(n);
        bytes(p, sizeof(T) * static_cast<size_t>(n));
    }
};

struct reader
{
    FILE* f;
    bool ok = true;
    void bytes(void* p, size_t n)
    {
        if (n > 0 && std::fread(p, 1, n, f) != n)
        {
            ok = false;
        }
    }
    template <class T>
    void value(T& v) { bytes(&v, sizeof(T)); }
    template <class T>
    void array(std::vector<T>& out)
    {
        int64_t n = 0;
        value(n);
        if (!ok || n < 0 || n > (int64_t{1} << 34))
        {
            ok = false;
            return;
        }
        out.resize(static_cast<size_t>(n));
        bytes(out.data(), sizeof(T) * static_cast<size_t>(n));
    }
};
} // namespace

rt_status save_scene(const rt_scene_desc& d, const std::string& path, std::string& error)
{
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f)
    {
        error = "cannot open '" + path + "' for writing";
        return RT_ERR_RUNTIME;
    }
    writer w{f};
    w.bytes(magic, sizeof(magic));
    w.array(d.spheres, d.sphere_count);
    w.array(d.materials, d.material_count);
    w.value(d.camera);
    w.array(d.textures, d.texture_count);
    w.value(d.image_count);
    for (int64_t i = 0; i < d.image_count; ++i)
    {
        w.value(d.images[i].width);
        w.value(d.images[i].height);
        w.array(d.images[i].rgb, int64_t{d.images[i].width} * d.images[i].height * 3);
    }
    w.array(d.perlins, d.perlin_count);
    w.array(d.quads, d.quad_count);
    w.value(d.medium_count);
    for (int64_t i = 0; i < d.medium_count; ++i)
    {
        w.value(d.media[i]);
        w.array(d.media[i].quads, d.media[i].quad_count);
    }
    w.array(d.lights, d.light_count);
    w.value(d.combination);
    w.value(d.quality);
    w.array(d.microfacets, d.microfacet_count);
    const int32_t has_env = d.environment ? 1 : 0;
    w.value(has_env);
    if (d.environment)
    {
        w.value(d.environment->yaw_degrees);
        w.value(d.environment->scale);
        w.value(d.environment->image.width);
        w.value(d.environment->image.height);
        w.array(d.environment->image.rgb,
                int64_t{d.environment->image.width} * d.environment->image.height * 3);
    }
    w.value(d.mesh_count);
    for (int64_t i = 0; i < d.mesh_count; ++i)
    {
        w.value(d.meshes[i].material);
        w.array(d.meshes[i].positions, d.meshes[i].vertex_count * 3);
        w.array(d.meshes[i].indices, d.meshes[i].triangle_count * 3);
    }
    const bool ok = w.ok && std::fclose(f) == 0;
    if (!ok)
    {
        error = "writing '" + path + "' failed";
        return RT_ERR_RUNTIME;
    }
    return RT_OK;
}

rt_status load_scene(const std::string& path, std::unique_ptr<scene_store>& out, std::string& error)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f)
    {
        error = "cannot open '" + path + "'";
        return RT_ERR_RUNTIME;
    }
    auto s = std::make_unique<scene_store>();
    reader r{f};
    char head[8] = {};
    r.bytes(head, sizeof(head));
    if (!r.ok || std::memcmp(head, magic, sizeof(magic)) != 0)
    {
        std::fclose(f);
        error = "'" + path + "' is not a scene file";
        return RT_ERR_RUNTIME;
    }
    r.array(s->spheres);
    r.array(s->materials);
    r.value(s->camera);
    r.array(s->textures);
    int64_t images = 0;
    r.value(images);
    for (int64_t i = 0; r.ok && i < images && i < 65536; ++i)
    {
        rt_image_desc im{};
        r.value(im.width);
        r.value(im.height);
        s->image_pixels.emplace_back();
        r.array(s->image_pixels.back());
        s->images.push_back(im);
    }
    r.array(s->perlins);
    r.array(s->quads);
    int64_t media = 0;
    r.value(media);
    for (int64_t i = 0; r.ok && i < media && i < 65536; ++i)
    {
        medium_store m;
        r.value(m.desc);
        r.array(m.quads);
        s->media.push_back(std::move(m));
    }
    r.array(s->lights);
    r.value(s->combination);
    r.value(s->quality);
    r.array(s->microfacets);
    int32_t has_env = 0;
    r.value(has_env);
    if (r.ok && has_env)
    {
        s->has_environment = true;
        r.value(s->environment.yaw_degrees);
        r.value(s->environment.scale);
        r.value(s->environment.image.width);
        r.value(s->environment.image.height);
        r.array(s->environment_pixels);
    }
    int64_t meshes = 0;
    r.value(meshes);
    for (int64_t i = 0; r.ok && i < meshes && i < 65536; ++i)
    {
        mesh_store m;
        r.value(m.material);
        r.array(m.positions);
        r.array(m.indices);
        s->meshes.push_back(std::move(m));
    }
    std::fclose(f);
    if (!r.ok)
    {
        error = "'" + path + "' is truncated or damaged";
        return RT_ERR_RUNTIME;
    }
    s->finish();
    out = std::move(s);
    return RT_OK;
}
} // namespace rtb
