// TEST INFRASTRUCTURE — the CPU oracle of the NEE/MIS integrator (the reference's "quality kernel"), in double.
//
// The reference has this estimator on the GPU only (src/gpu/quality_path.cuh:83-188 trace_quality_ray, with
// light_sampler.cuh:40-103, lamps.cuh:81-146, mis.cuh:30-62, bsdf.cuh:58-201). This is its restatement on the CPU
// renderer of cpu_renderer.h: the same light set (quads and still spheres that glow one solid color, picked uniformly),
// the same densities, the same depth rule and weights, traced in double with the CPU's closest hit and an any-hit
// shadow query, and the CPU's random numbers.
#pragma once

#include "cpu_renderer.h"
#include "ggx_env_cpu.h"

namespace oracle
{
struct lamp
{
    int kind;      // RT_LIGHT_*
    point3 corner; // quad: q; sphere: center
    vec3 u, v, normal;
    double size;   // quad: area; sphere: radius
    color radiance;
    int primitive; // source id
};

struct lamp_sample
{
    vec3 wi;
    double distance = 0;
    double pdf = 0;
};

// lamp_table.cu / lamps.cuh:1-25: every quad and every sphere that stands still whose material is a diffuse_light,
// spheres first, in the scene's order
inline std::vector<lamp> build_lamps(const scene& s)
{
    std::vector<lamp> lamps;
    for (const sphere& sp : s.geometry.spheres)
    {
        const material& m = s.materials[static_cast<size_t>(sp.material)];
        if (m.kind == RT_DIFFUSE_LIGHT && m.texture < 0 && sp.center.direction.length_squared() == 0)
        {
            lamps.push_back({RT_LIGHT_SPHERE, sp.center.origin, {}, {}, {}, sp.radius, m.albedo, sp.id});
        }
    }
    for (const quad& q : s.geometry.quads)
    {
        const material& m = s.materials[static_cast<size_t>(q.material)];
        if (m.kind == RT_DIFFUSE_LIGHT && m.texture < 0)
        {
            lamps.push_back({RT_LIGHT_QUAD, q.q, q.u, q.v, q.normal, q.area, m.albedo, q.id});
        }
    }
    return lamps;
}

// lamps.cuh:81-131 sample_lamp: 2 numbers always; false for the back of a quad or a point inside a sphere
inline bool sample_lamp(const lamp& e, const point3& x, rng& g, lamp_sample& out)
{
    const double a = g.next();
    const double b = g.next();
    if (e.kind == RT_LIGHT_QUAD)
    {
        const vec3 to = (e.corner - x) + a * e.u + b * e.v;
        const double d2 = to.length_squared();
        const double d = std::sqrt(d2);
        out.wi = to / d;
        out.distance = d;
        const double cos_light = -dot(out.wi, e.normal);
        if (!(cos_light > 0))
        {
            return false;
        }
        out.pdf = d2 / (cos_light * e.size);
        return true;
    }
    const vec3 to_center = e.corner - x;
    const double d2 = to_center.length_squared();
    const double r2 = e.size * e.size;
    if (!(d2 > r2))
    {
        return false;
    }
    const double sin_sq_max = r2 / d2;
    const double one_minus_cos_max = sin_sq_max / (1 + std::sqrt(1 - sin_sq_max));
    const double phi = 2 * std::numbers::pi * a;
    const double one_minus_z = b * one_minus_cos_max;
    const double sin_sq = one_minus_z * (2 - one_minus_z);
    const double sin_theta = std::sqrt(sin_sq);
    const double cos_theta = 1 - one_minus_z;
    const onb uvw{unit_vector(to_center)};
    out.wi = uvw.transform({std::cos(phi) * sin_theta, std::sin(phi) * sin_theta, cos_theta});
    const double d = std::sqrt(d2);
    out.distance = d * cos_theta - std::sqrt(std::fmax(0.0, r2 - d2 * sin_sq));
    out.pdf = 1 / (2 * std::numbers::pi * one_minus_cos_max);
    return true;
}

// lamps.cuh:136-146 lamp_pdf: the density of a ray from x that hit lamp e at `distance`
inline double lamp_pdf(const lamp& e, const point3& x, const vec3& unit_dir, double distance)
{
    if (e.kind == RT_LIGHT_QUAD)
    {
        const double cos_light = -dot(unit_dir, e.normal);
        return cos_light > 0 ? distance * distance / (cos_light * e.size) : 0.0;
    }
    const double d2 = (e.corner - x).length_squared();
    const double r2 = e.size * e.size;
    if (!(d2 > r2))
    {
        return 0.0;
    }
    const double sin_sq_max = r2 / d2;
    return 1 / (2 * std::numbers::pi * (sin_sq_max / (1 + std::sqrt(1 - sin_sq_max))));
}

// mis.cuh:30-62: the power heuristic as 1/(1 + r^2), and the two weights
inline double power_weight(double self, double other)
{
    if (!(self > 0))
    {
        return 0;
    }
    const double r = other / self;
    const double w = 1 / (r * r + 1);
    return w == w ? w : 0;
}
inline double light_weight(int c, double p_light, double p_bsdf)
{
    return c == RT_COMBINE_POWER_HEURISTIC ? power_weight(p_light, p_bsdf) : 1.0;
}
inline double bsdf_weight(int c, double p_bsdf, double p_light)
{
    if (c == RT_COMBINE_BSDF_ONLY || !(p_bsdf > 0) || !(p_light > 0))
    {
        return 1.0;
    }
    return c == RT_COMBINE_POWER_HEURISTIC ? power_weight(p_bsdf, p_light) : 0.0;
}

inline double largest_channel(const color& c) { return std::fmax(std::fmax(c.x, c.y), c.z); }

struct quality_scene
{
    const scene& base;
    std::vector<lamp> lamps;
    std::vector<int> lamp_of; // by source id, -1 for none
    int combination;
    double light_pmf;
    bool has_environment = false;
    environment env;
    std::vector<double> energy; // Turquin's table, when a GGX conductor is in the scene

    int light_count() const { return static_cast<int>(lamps.size()) + (has_environment && env.sampled() ? 1 : 0); }
};

// Anything in (0.001, t_max) along r, the lamp `skip` aside (shadow.cuh:26-109 occluded)? The CPU's BVH search with
// that one primitive left out.
inline bool occluded(const scene& s, const ray& r, double t_max, int skip)
{
    return s.geometry.hit_except(r, interval{0.001, t_max}, skip).has_value();
}

// The lobes of bsdf.cuh:30-99 on the CPU
enum class lobe_kind
{
    lambertian,
    isotropic,
    conductor,
    gloss,
    smooth_conductor,
    books_delta,
};

inline lobe_kind lobe_of(const material& m)
{
    if (m.lobe == RT_MICROFACET_CONDUCTOR)
    {
        return m.alpha >= min_ggx_alpha ? lobe_kind::conductor : lobe_kind::smooth_conductor;
    }
    if (m.lobe == RT_MICROFACET_GLOSS)
    {
        return lobe_kind::gloss;
    }
    if (m.kind == RT_LAMBERTIAN)
    {
        return lobe_kind::lambertian;
    }
    if (m.kind == RT_ISOTROPIC)
    {
        return lobe_kind::isotropic;
    }
    return lobe_kind::books_delta;
}

// eval_bsdf (bsdf.cuh:178-201): f * |cos| for a light sample's unit direction wi, and the lobe's density of it
inline color eval_lobe(const quality_scene& q, lobe_kind k, const material& m, const vec3& n, const vec3& wo,
                       const vec3& wi, double& pdf)
{
    switch (k)
    {
    case lobe_kind::lambertian:
        pdf = cosine_density(n, wi);
        return pdf * m.albedo;
    case lobe_kind::isotropic:
        pdf = uniform_sphere_density;
        return uniform_sphere_density * m.albedo;
    case lobe_kind::conductor:
    {
        const color single = ggx_eval(n, wo, wi, m.alpha, m.albedo, pdf);
        return ggx_compensation(q.energy, m.albedo, dot(n, wo), m.roughness) * single;
    }
    case lobe_kind::gloss:
        return gloss_eval(n, wo, wi, m.alpha, m.albedo, pdf);
    default:
        pdf = 0;
        return {0, 0, 0};
    }
}

// quality_path.cuh:83-188 trace_quality_ray, one whole sample
inline color quality_sample(const quality_scene& q, ray r, rng& g, counters& n)
{
    const scene& s = q.base;
    color radiance{0, 0, 0};
    color throughput{1, 1, 1};
    double bsdf_pdf = 0;
    bool specular = true;
    int rays_left = s.camera.max_depth;
    const int lights = q.light_count();
    while (true)
    {
        const auto rec = s.closest_event(r, g);
        ++n.rays;
        if (!rec)
        {
            // background.cuh:44-61: the environment (filtered after the camera and delta vertices; the nearest texel
            // and its density otherwise), or the camera's sky
            if (!q.has_environment)
            {
                return radiance + throughput * s.sky(r.direction);
            }
            if (specular)
            {
                return radiance + throughput * q.env.radiance_filtered(r.direction);
            }
            double density;
            const color le = q.env.radiance(r.direction, density);
            const double p_light = q.env.sampled() ? q.light_pmf * density : 0.0;
            const double w = bsdf_pdf > 0 ? bsdf_weight(q.combination, bsdf_pdf, p_light) : 1.0;
            return radiance + w * (throughput * le);
        }
        // The material with its color at the hit (its texture there; a metal's albedo)
        material m = s.materials[static_cast<size_t>(rec->material)];
        m.albedo = rec->color_at;
        if (m.kind == RT_DIFFUSE_LIGHT)
        {
            double w = 1;
            if (bsdf_pdf > 0)
            {
                const double distance = rec->t * r.direction.length();
                const int k = q.lamp_of[static_cast<size_t>(rec->id)];
                const double p_light =
                    k >= 0 ? q.light_pmf * lamp_pdf(q.lamps[static_cast<size_t>(k)], r.origin,
                                                    unit_vector(r.direction), distance)
                           : 0.0;
                w = bsdf_weight(q.combination, bsdf_pdf, p_light);
            }
            const color c = rec->front_face ? m.albedo : color{0, 0, 0};
            return radiance + w * (throughput * c);
        }
        const lobe_kind lobe = lobe_of(m);
        const bool delta = lobe == lobe_kind::books_delta || lobe == lobe_kind::smooth_conductor;
        const vec3 wo = -unit_vector(r.direction);
        const bool nee = q.combination != RT_COMBINE_BSDF_ONLY && rays_left > 1 && !delta && lights > 0 &&
                         largest_channel(throughput) > 0;
        bool lit = false;
        color contribution{0, 0, 0};
        vec3 light_dir;
        double light_distance = infinity;
        int skip = -1;
        if (nee)
        {
            // light_sampler.cuh:40-75 sample_light: one number picks a light, the lamps first, the map last
            const double xi = g.next();
            int k = static_cast<int>(xi * lights);
            k = std::min(k, lights - 1);
            bool drawn = false;
            color le;
            double p_light = 0;
            if (k < static_cast<int>(q.lamps.size()))
            {
                const lamp& e = q.lamps[static_cast<size_t>(k)];
                lamp_sample ls;
                if (sample_lamp(e, rec->p, g, ls))
                {
                    drawn = true;
                    light_dir = ls.wi;
                    light_distance = ls.distance;
                    le = e.radiance;
                    p_light = q.light_pmf * ls.pdf;
                    skip = e.primitive;
                }
            }
            else
            {
                double density;
                if (q.env.sample(g, light_dir, le, density))
                {
                    drawn = true;
                    p_light = q.light_pmf * density;
                }
            }
            if (drawn)
            {
                double p_bsdf;
                const color f = eval_lobe(q, lobe, m, rec->normal, wo, light_dir, p_bsdf);
                if (p_light > 0 && largest_channel(f) > 0)
                {
                    contribution = (light_weight(q.combination, p_light, p_bsdf) / p_light) * (throughput * (f * le));
                    const double sum = contribution.x + contribution.y + contribution.z;
                    lit = sum > 0 && sum < infinity;
                }
            }
        }
        // the material's sample: bsdf.cuh:108-174
        vec3 wi;
        color weight{1, 1, 1};
        double pdf = 0;
        bool scattered = true;
        switch (lobe)
        {
        case lobe_kind::lambertian:
        {
            const onb uvw{rec->normal};
            wi = uvw.transform(random_cosine_direction(g));
            scattered = dot(rec->normal, wi) > 0;
            weight = m.albedo;
            pdf = cosine_density(rec->normal, wi);
            break;
        }
        case lobe_kind::isotropic:
            wi = random_unit_vector(g);
            weight = m.albedo;
            pdf = uniform_sphere_density;
            break;
        case lobe_kind::conductor:
        {
            const double u1 = g.next();
            const double u2 = g.next();
            scattered = ggx_sample(rec->normal, wo, m.alpha, m.albedo, u1, u2, wi, weight, pdf);
            if (scattered)
            {
                weight = weight * ggx_compensation(q.energy, m.albedo, dot(rec->normal, wo), m.roughness);
            }
            break;
        }
        case lobe_kind::smooth_conductor:
            scattered = dot(rec->normal, wo) > 0;
            wi = unit_vector(reflect(-wo, rec->normal));
            weight = schlick(m.albedo, dot(rec->normal, wo));
            break;
        case lobe_kind::gloss:
        {
            // ggx.cuh:300-324: the coat or the base, half the time each, then the mixture's weight and density
            if (g.next() < 0.5)
            {
                const double u1 = g.next();
                const double u2 = g.next();
                color coat_weight;
                double coat_pdf;
                scattered = ggx_sample(rec->normal, wo, m.alpha, color{gloss_coat_f0, gloss_coat_f0, gloss_coat_f0},
                                       u1, u2, wi, coat_weight, coat_pdf);
            }
            else
            {
                const onb uvw{rec->normal};
                wi = uvw.transform(random_cosine_direction(g));
                scattered = dot(rec->normal, wi) > 0;
            }
            if (scattered)
            {
                const color f = gloss_eval(rec->normal, wo, wi, m.alpha, m.albedo, pdf);
                scattered = pdf > 0;
                if (scattered)
                {
                    weight = (1 / pdf) * f;
                }
            }
            break;
        }
        default: // the books' metal and glass
            if (m.kind == RT_METAL)
            {
                wi = unit_vector(reflect(r.direction, rec->normal)) + m.fuzz * random_unit_vector(g);
                scattered = dot(wi, rec->normal) > 0;
                weight = m.albedo;
            }
            else
            {
                const double ri = rec->front_face ? (1.0 / m.refraction_index) : m.refraction_index;
                const vec3 ud = unit_vector(r.direction);
                const double cos_theta = std::fmin(dot(-ud, rec->normal), 1.0);
                const double sin_theta = std::sqrt(1.0 - cos_theta * cos_theta);
                wi = ri * sin_theta > 1.0 || reflectance(cos_theta, ri) > g.next() ? reflect(ud, rec->normal)
                                                                                    : refract(ud, rec->normal, ri);
            }
            break;
        }
        if (lit)
        {
            ++n.shadow_rays;
            const ray shadow{rec->p, light_dir, r.time};
            if (!occluded(s, shadow, light_distance, skip))
            {
                // through smoke, with the chance of crossing it (shadow.cuh:129-165)
                radiance += s.transmittance(shadow, light_distance) * contribution;
            }
        }
        if (!scattered)
        {
            return radiance;
        }
        throughput = throughput * weight;
        bsdf_pdf = nee ? pdf : 0;
        specular = delta;
        if (q.combination != RT_COMBINE_BSDF_ONLY && throughput.x == 0 && throughput.y == 0 && throughput.z == 0)
        {
            return radiance;
        }
        if (--rays_left == 0)
        {
            return radiance;
        }
        r = ray{rec->p, wi, r.time};
    }
}

inline quality_scene make_quality(const scene& s, const rt_scene_desc& d)
{
    quality_scene q{s, build_lamps(s), {}, d.combination, 0, false, environment{}, {}};
    const size_t ids = s.geometry.spheres.size() + s.geometry.quads.size() + s.geometry.triangles.size();
    q.lamp_of.assign(ids, -1);
    for (size_t k = 0; k < q.lamps.size(); ++k)
    {
        q.lamp_of[static_cast<size_t>(q.lamps[k].primitive)] = static_cast<int>(k);
    }
    if (d.environment)
    {
        q.has_environment = true;
        q.env = make_environment(*d.environment);
    }
    const int n = q.light_count();
    q.light_pmf = n == 0 ? 0.0 : 1.0 / n;
    for (const material& m : s.materials)
    {
        if (m.lobe == RT_MICROFACET_CONDUCTOR && q.energy.empty())
        {
            q.energy = ggx_energy_table();
        }
    }
    return q;
}
} // namespace oracle
