// An owned scene: std::vector tables behind an rt_scene_desc that points into them. Built-in scenes, loaded files and
// the serving layer's requests all hold their scene this way; the renderer itself only ever reads the plain desc.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "rt_b200.h"

namespace rtb
{
struct mesh_store
{
    std::vector<float> positions;
    std::vector<uint32_t> indices;
    int32_t material = 0;
};

struct medium_store
{
    rt_medium_desc desc{};
    std::vector<rt_quad_desc> quads;
};

struct scene_store
{
    std::vector<rt_sphere_desc> spheres;
    std::vector<rt_material_desc> materials;
    rt_camera_desc camera{};
    std::vector<rt_texture_desc> textures;
    std::vector<rt_image_desc> images;
    std::vector<std::vector<float>> image_pixels;
    std::vector<rt_perlin_desc> perlins;
    std::vector<rt_quad_desc> quads;
    std::vector<medium_store> media;
    std::vector<rt_medium_desc> media_desc;
    std::vector<rt_light_desc> lights;
    int32_t combination = RT_COMBINE_BSDF_ONLY;
    int32_t quality = 0;
    std::vector<rt_microfacet_desc> microfacets;
    bool has_environment = false;
    rt_environment_desc environment{};
    std::vector<float> environment_pixels;
    std::vector<mesh_store> meshes;
    std::vector<rt_mesh_desc> mesh_desc;

    rt_scene_desc desc{};

    // Points desc at the tables; call after the last change to any of them
    const rt_scene_desc& finish();

    int add_material(const rt_material_desc& m)
    {
        materials.push_back(m);
        return static_cast<int>(materials.size()) - 1;
    }
    int add_solid_texture(rt_vec3 rgb);
    int lambertian(rt_vec3 albedo);
    int metal(rt_vec3 albedo, double fuzz);
    int dielectric(double refraction_index);
    int diffuse_light(rt_vec3 emit);

    // A deep copy of any desc (the caller's arrays may die after this returns)
    static std::unique_ptr<scene_store> copy_of(const rt_scene_desc& d);
};

// camera_settings of camera.ixx:86-115 and the frame its constructor computes (camera.ixx:138-182)
struct camera_settings
{
    double aspect_ratio = 1.0;
    int image_width = 100;
    int samples_per_pixel = 10;
    int max_depth = 10;
    int sampling = RT_SAMPLING_MIXTURE;
    double vfov = 90;
    rt_vec3 lookfrom{0, 0, 0};
    rt_vec3 lookat{0, 0, -1};
    rt_vec3 vup{0, 1, 0};
    double defocus_angle = 0;
    double focus_dist = 10;
    rt_vec3 sky_bottom{0, 0, 0};
    rt_vec3 sky_top{0, 0, 0};
};

rt_camera_desc camera_frame(const camera_settings& s, int height_override);

rt_status build_builtin(const std::string& name, const rt_builtin_params& params, std::unique_ptr<scene_store>& out,
                        std::string& error);

rt_status save_scene(const rt_scene_desc& d, const std::string& path, std::string& error);
rt_status load_scene(const std::string& path, std::unique_ptr<scene_store>& out, std::string& error);
}

// The owned scene handle of the C-ABI
struct rt_owned_scene
{
    std::unique_ptr<rtb::scene_store> store;
};
