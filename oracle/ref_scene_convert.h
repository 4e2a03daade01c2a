// Test infrastructure, not product: this library's scene tables (rt_scene_desc) converted into the reference's own
// gpu::scene_desc (src/gpu/renderer.h:381-395, member types 43-377), field by field, for the entry points into the
// reference's renderer under oracle/ (ref_gpu_shim.cpp, ref_closest_hit.cu).
#pragma once

#include "renderer.h" // the reference's header, from its source tree

#include <cstdint>

#include "rt_b200.h"

namespace ref_convert
{
inline gpu::vec3d to_ref(const rt_vec3& v) { return {v.x, v.y, v.z}; }

inline gpu::quad_desc to_ref(const rt_quad_desc& q)
{
    gpu::quad_desc r;
    r.q = to_ref(q.q);
    r.u = to_ref(q.u);
    r.v = to_ref(q.v);
    r.material = q.material;
    return r;
}

inline gpu::sphere_desc to_ref(const rt_sphere_desc& s)
{
    gpu::sphere_desc r;
    r.center = to_ref(s.center);
    r.radius = s.radius;
    r.material = s.material;
    r.displacement = to_ref(s.displacement);
    r.uv_cos = s.uv_cos;
    r.uv_sin = s.uv_sin;
    return r;
}

inline gpu::image_desc to_ref(const rt_image_desc& im)
{
    gpu::image_desc r;
    r.width = im.width;
    r.height = im.height;
    const size_t n = static_cast<size_t>(im.width) * static_cast<size_t>(im.height) * 3;
    r.rgb.assign(im.rgb, im.rgb + n);
    return r;
}

inline gpu::camera_desc to_ref(const rt_camera_desc& c)
{
    gpu::camera_desc r;
    r.image_width = c.image_width;
    r.image_height = c.image_height;
    r.sqrt_spp = c.sqrt_spp;
    r.max_depth = c.max_depth;
    r.center = to_ref(c.center);
    r.pixel00_loc = to_ref(c.pixel00_loc);
    r.pixel_delta_u = to_ref(c.pixel_delta_u);
    r.pixel_delta_v = to_ref(c.pixel_delta_v);
    r.defocus = c.defocus != 0;
    r.defocus_disk_u = to_ref(c.defocus_disk_u);
    r.defocus_disk_v = to_ref(c.defocus_disk_v);
    r.sky_bottom = to_ref(c.sky_bottom);
    r.sky_top = to_ref(c.sky_top);
    r.sampling = static_cast<gpu::sampling_strategy>(c.sampling);
    return r;
}

inline gpu::scene_desc to_ref(const rt_scene_desc& d)
{
    gpu::scene_desc s;
    for (int64_t i = 0; i < d.sphere_count; ++i)
    {
        s.spheres.push_back(to_ref(d.spheres[i]));
    }
    for (int64_t i = 0; i < d.material_count; ++i)
    {
        const rt_material_desc& m = d.materials[i];
        gpu::material_desc r;
        r.kind = static_cast<gpu::material_kind>(m.kind);
        r.albedo = to_ref(m.albedo);
        r.fuzz = m.fuzz;
        r.refraction_index = m.refraction_index;
        r.texture = m.texture;
        s.materials.push_back(r);
    }
    s.camera = to_ref(d.camera);
    for (int64_t i = 0; i < d.texture_count; ++i)
    {
        const rt_texture_desc& t = d.textures[i];
        gpu::texture_desc r;
        r.kind = static_cast<gpu::texture_kind>(t.kind);
        r.rgb = to_ref(t.rgb);
        r.inv_scale = t.inv_scale;
        r.even = t.even;
        r.odd = t.odd;
        r.image = t.image;
        r.scale = t.scale;
        r.perlin = t.perlin;
        s.textures.push_back(r);
    }
    for (int64_t i = 0; i < d.image_count; ++i)
    {
        s.images.push_back(to_ref(d.images[i]));
    }
    for (int64_t i = 0; i < d.perlin_count; ++i)
    {
        gpu::perlin_desc p;
        for (int k = 0; k < gpu::perlin_point_count; ++k)
        {
            p.random_vectors[k] = to_ref(d.perlins[i].random_vectors[k]);
            p.perm_x[k] = d.perlins[i].perm_x[k];
            p.perm_y[k] = d.perlins[i].perm_y[k];
            p.perm_z[k] = d.perlins[i].perm_z[k];
        }
        s.perlins.push_back(p);
    }
    for (int64_t i = 0; i < d.quad_count; ++i)
    {
        s.quads.push_back(to_ref(d.quads[i]));
    }
    for (int64_t i = 0; i < d.medium_count; ++i)
    {
        const rt_medium_desc& m = d.media[i];
        gpu::medium_desc r;
        r.boundary = static_cast<gpu::boundary_shape>(m.boundary);
        r.sphere = to_ref(m.sphere);
        for (int64_t k = 0; k < m.quad_count; ++k)
        {
            r.quads.push_back(to_ref(m.quads[k]));
        }
        r.neg_inv_density = m.neg_inv_density;
        r.material = m.material;
        s.media.push_back(r);
    }
    for (int64_t i = 0; i < d.light_count; ++i)
    {
        const rt_light_desc& l = d.lights[i];
        gpu::light_desc r;
        r.kind = static_cast<gpu::light_shape>(l.kind);
        r.quad = to_ref(l.quad);
        r.center = to_ref(l.center);
        r.radius = l.radius;
        r.weight = l.weight;
        s.lights.push_back(r);
    }
    s.quality.combination = static_cast<gpu::light_combination>(d.combination);
    for (int64_t i = 0; i < d.microfacet_count; ++i)
    {
        gpu::microfacet_desc r;
        r.kind = static_cast<gpu::microfacet_kind>(d.microfacets[i].kind);
        r.roughness = d.microfacets[i].roughness;
        s.quality.microfacets.push_back(r);
    }
    if (d.environment)
    {
        gpu::environment_desc e;
        e.image = to_ref(d.environment->image);
        e.yaw_degrees = d.environment->yaw_degrees;
        e.scale = d.environment->scale;
        s.quality.environment = e;
    }
    return s;
}
} // namespace ref_convert
