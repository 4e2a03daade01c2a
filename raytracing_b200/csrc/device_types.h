// Plain data shared by the host code that builds a resident scene and the kernels that render it. Everything the
// kernels read per ray is 16-byte aligned and fetched with 128-bit loads; a BVH node is 64 bytes (4 loads) and holds
// the boxes of BOTH of its children, so one node fetch decides the whole step of the traversal (Aila and Laine,
// "Understanding the Efficiency of Ray Traversal on GPUs", HPG 2009) where the reference's 32-byte node holds its own
// box and a step reads two nodes (src/gpu/bvh.cuh:29-38, 680-693).
#pragma once

#include <cstdint>

#include <vector_types.h>

#ifdef __CUDACC__
#define RTB_HD __host__ __device__
#else
#define RTB_HD
#endif

namespace rtb
{
struct f3
{
    float x, y, z;
};

// A node: the boxes of its two children, laid out per axis so that the slab test of both children reads each axis
// once: x = (lo0, hi0, lo1, hi1), likewise y and z. link[c] >= 0 is an inner node's index; link[c] < 0 is a leaf,
// encoded in the link itself (see leaf_link), so a leaf needs no fetch of its own.
struct alignas(64) bvh_node
{
    float x[4];
    float y[4];
    float z[4];
    int32_t link[2];
    int32_t pad[2];
};
static_assert(sizeof(bvh_node) == 64, "a node is four 16-byte loads");

// The same tree collapsed four wide, for the wavefront's walk: the boxes of up to four children per axis and bound
// (lo_x = the four children's x minima, ...), then their links (a leaf as in bvh_node, traversal_done for an unused
// slot). A walk step reads 128 bytes and decides four children, and a walk takes about half the dependent steps.
struct alignas(64) bvh4_node
{
    float lo_x[4];
    float hi_x[4];
    float lo_y[4];
    float hi_y[4];
    float lo_z[4];
    float hi_z[4];
    int32_t link[4];
    int32_t pad[4];
};
static_assert(sizeof(bvh4_node) == 128, "a wide node is eight 16-byte loads");
// No more nodes to visit, and a wide node's unused slot (a leaf link never takes this value: its kind field would be 3)
constexpr int32_t traversal_done_link = static_cast<int32_t>(0x80000000u);
constexpr int wide_stack = 96;   // the wide walk's stack: up to three entries a level, 32 levels
constexpr int max_wide_depth = wide_stack / 3;

// Primitive kinds; a leaf holds primitives of one kind, contiguous in that kind's array
enum prim_kind : int32_t
{
    kind_sphere = 0,
    kind_quad = 1,
    kind_triangle = 2,
};

constexpr int leaf_count_bits = 4; // at most 15 primitives in a leaf; 0 is the empty leaf
constexpr int max_leaf_size = 15;
constexpr int leaf_start_shift = 6;
constexpr int max_bvh_depth = 64; // the traversal stack's size

// ~link = start << 6 | count << 2 | kind
RTB_HD inline int32_t leaf_link(int32_t start, int32_t count, int32_t kind)
{
    return ~((start << leaf_start_shift) | (count << 2) | kind);
}
RTB_HD inline int32_t leaf_kind(int32_t link) { return (~link) & 3; }
RTB_HD inline int32_t leaf_count(int32_t link) { return ((~link) >> 2) & 15; }
RTB_HD inline int32_t leaf_start(int32_t link) { return (~link) >> leaf_start_shift; }

// A sphere: center and radius, one 16-byte load. A negative radius marks a sphere whose quadratic is solved in FP64
// (its radius is large next to the distances rays travel to it, so FP32 cancels: the radius-1000 ground).
struct alignas(16) sphere4
{
    float cx, cy, cz, r;
};

// A quad as hit_quad reads it (src/gpu/quad.cuh:19-46): a corner, the unit normal u x v, and the dual basis of (u, v)
// in its plane, alpha_axis = v x w and beta_axis = w x u with w = n / |n|^2, 48 bytes: three 16-byte loads.
struct alignas(16) quad12
{
    float qx, qy, qz, nx;
    float ny, nz, ax, ay;
    float az, bx, by, bz;
};

// A triangle: its three vertices as the mesh gives them (a vertex shared by two triangles is the same floats in both,
// which the watertight test needs), 48 bytes (the last three floats unused), three 16-byte loads
struct alignas(16) triangle12
{
    float ax, ay, az, bx;
    float by, bz, cx, cy;
    float cz, pad0, pad1, pad2;
};

// A material as the shading reads it (src/gpu/material.cuh:18-26), with the NEE/MIS integrator's GGX side entry
// (renderer.h:249-261): 48 bytes, three 16-byte loads
struct alignas(16) material12
{
    float r, g, b;   // albedo, emission, or a metal's albedo (F0 for a GGX conductor)
    int32_t kind;    // RT_LAMBERTIAN ...
    float fuzz;
    float ior;
    int32_t lobe;    // RT_MICROFACET_NONE, _CONDUCTOR (the material is a metal of fuzz 0), _GLOSS (a lambertian)
    float alpha;     // the GGX width r^2
    float roughness; // r: the energy table's axis
    int32_t texture; // -1: the color is (r, g, b); otherwise its texture (a checker, an image or a noise)
    int32_t texture_needs; // texture_needs_uv | texture_needs_point: what reading the texture needs of the hit
    float pad2;
};

constexpr int32_t texture_needs_uv = 1;    // an image in the texture: the hit's (u, v)
constexpr int32_t texture_needs_point = 2; // a checker: the hit point, moved exactly onto a sphere

// The environment map (src/gpu/environment_data.h): texels with their sampling density, the alias table's bins, the
// rows' cosines, and the yaw
struct alignas(16) env_texel
{
    float r, g, b, pdf; // radiance; the density Y/S per steradian of the cell's directions
};

struct alignas(8) alias_bin
{
    float q;       // the chance of the bin's own cell, on the 2^-24 grid
    int32_t alias; // the cell that takes the rest
};

struct environment_view
{
    const env_texel* texels;
    const alias_bin* bins;
    const float* row_cos;    // height + 1
    int32_t width, height;
    int32_t log2_bins;
    int32_t sampled;         // the map has light (S > 0) and an alias table: it is a light of the NEE set
    float cos_yaw, sin_yaw;
    float scale;
};

// A shape of the books' lights list (src/gpu/lights.cuh:18-45): what lights_pdf_value and lights_random read
struct alignas(16) light24
{
    quad12 quad;     // RT_LIGHT_QUAD: the hit test of the density
    float ux, uy, uz, area;
    float vx, vy, vz, cdf;
    float cx, cy, cz, radius; // RT_LIGHT_SPHERE
    float weight;
    int32_t kind;
    int32_t twin;    // the global id of the world's primitive with exactly these numbers, or -1
    int32_t pad;
};

// A lamp of the NEE/MIS integrator's light set (src/gpu/lamps.cuh:34-47)
struct alignas(16) emitter20
{
    float cx, cy, cz, size; // quad: corner, area; sphere: center, radius
    float ux, uy, uz;
    int32_t kind;
    float vx, vy, vz;
    int32_t primitive; // its global id
    float nx, ny, nz, pad0;
    float er, eg, eb, pad1;
};

// A divisor d (1 <= d < 2^32) with its multiplier, for division by multiplication (Granlund and Montgomery, "Division by
// Invariant Integers using Multiplication", PLDI 1994): for every n < 2^32, n / d is the high 64 bits of the 128-bit
// product n * magic with magic = floor((2^64 - 1) / d) + 1. The product overshoots n / d by n (magic - 2^64 / d) / 2^64
// < 2^-32, less than the 1/d that n / d's fraction stays below the next integer, so the quotient is exact; d = 1 keeps
// n (magic 0). The kernels turn sample and work-item numbers into passes and pixels this way, where a division would
// be a long software sequence.
struct fast_divisor
{
    uint64_t magic;
    uint32_t d;
    uint32_t pad;
};

inline fast_divisor make_fast_divisor(uint32_t d)
{
    return {d > 1 ? ~uint64_t{0} / d + 1 : 0, d, 0};
}

// The camera (src/gpu/camera.cuh:33-50), pixel grid relative to the center computed in double on the host
struct camera_params
{
    int32_t width, height, sqrt_spp, max_depth;
    float recip_sqrt_spp;
    f3 center;
    f3 center_to_pixel00;
    f3 delta_u, delta_v;
    int32_t defocus;
    f3 disk_u, disk_v;
    f3 sky_bottom, sky_top;
    int32_t sampling;
    // The view's divisors: a round's strata a side (sqrt_spp), a round's passes (sqrt_spp^2), the 8x4 tiles a row
    // ((width + 7) / 8) and the padded pixels (tiles * 32) a pass of samples or work items spans
    fast_divisor div_sqrt_spp;
    fast_divisor div_round_passes;
    fast_divisor div_tiles_x;
    fast_divisor div_padded;
};

// A texture (src/gpu/texture.cuh:10-19): 32 bytes, two 16-byte loads. checker: `even`, `odd` are texture indices
// smaller than its own and inv_scale the cubes' 1 / side; image: `table` indexes the images; noise: the noise tables
struct alignas(16) texture8
{
    int32_t kind; // RT_TEXTURE_*
    int32_t even, odd;
    int32_t table;
    float r, g, b;
    float inv_scale;
};

// Where an image's texels are: texels[offset + j * width + i] is pixel (i, j), rows from the top
struct alignas(16) image_info
{
    int32_t offset, width, height, pad;
};

// A marble texture (the CPU's noise_texture with its own perlin tables, perlin.ixx): 256 gradients (16 bytes each),
// the three permutations of 0..255, and the stripes' frequency
struct alignas(16) noise_table
{
    float4 gradients[256];
    uint8_t perm_x[256];
    uint8_t perm_y[256];
    uint8_t perm_z[256];
    float scale;
    float pad[3];
};

// A sphere's texture frame (sphere.cuh:119-168): the turn of the rotate_y instances around it (u of its texture
// coordinates is read in its own coordinates), and |c|^2 - r^2 and the bound below which a checker's point is moved
// onto the sphere exactly (one Newton step; 0: never)
struct alignas(16) sphere_frame
{
    float cos_theta, sin_theta;
    float k, limit;
};

// At most this many volumes of smoke in a scene: a vertex draws one number per volume, from its dimension blocks 4-15
constexpr int max_media = 48;

// A volume of smoke (src/gpu/constant_medium.cuh:9-27): a box around it over the whole shutter, -1/density, its
// isotropic material, and its boundary: a sphere (center at time 0, radius, motion) when quad_count is 0, otherwise
// boundary quads [first_quad, first_quad + quad_count). 64 bytes.
struct alignas(16) medium16
{
    float lo_x, lo_y, lo_z, neg_inv_density;
    float hi_x, hi_y, hi_z;
    int32_t material;
    float cx, cy, cz, radius;
    float dx, dy, dz;
    int32_t first_quad;
    int32_t quad_count;
    int32_t pad[3];
};

// The resident scene as the kernels see it
struct scene_view
{
    const bvh_node* nodes;
    const bvh4_node* wide_nodes; // the tree four wide (null when it would be deeper than max_wide_depth)
    const sphere4* spheres;     // global ids [0, quad_base)
    const quad12* quads;        // [quad_base, triangle_base)
    const triangle12* triangles;// [triangle_base, ...)
    int32_t quad_base;
    int32_t triangle_base;
    int32_t node_count;
    int32_t prim_count;
    const int32_t* prim_material; // by global id
    const material12* materials;
    const light24* lights;
    int32_t light_count;
    int32_t lamp_count;
    const emitter20* lamps;
    const int32_t* lamp_of;     // by global id, -1: no lamp
    float light_pmf;         // 1 / (lamps + the map if it is sampled)
    int32_t combination;
    int32_t has_environment; // misses see the map (the NEE/MIS integrator only), not the camera's sky
    int32_t flat;            // a small scene of spheres and quads: closest hits test every primitive, no tree walk
    environment_view env;
    // Textures, motion and smoke (the second book); all empty in a scene without them
    const texture8* textures;
    const image_info* images;
    const float4* texels;
    const noise_table* noises;
    const float4* sphere_motion;      // per sphere (leaf order): the center's displacement over the shutter
    const sphere_frame* sphere_frames; // per sphere (leaf order), for textured spheres
    const medium16* media;
    const quad12* boundary_quads;
    int32_t has_motion;      // some sphere moves: rays carry a time, spheres are where they are at it
    int32_t medium_count;
    int32_t medium_base;     // the global id of a particle of media[0]: right after the surface primitives
    int32_t has_textures;    // some material reads a texture (not one solid color)
};

// ---- the same tables in double, for the books' integrator in FP64 (precision::float64, renderer.h:402-409) --------
// They follow the float tables' leaf order and global ids (one tree serves both: its float boxes, widened by
// box_margin, hold every double primitive), so prim_material, the lights' twins and the tree are shared.
struct alignas(16) d4
{
    double x, y, z, w;
};

// A sphere (center, radius), its motion over the shutter (w unused), and its texture frame as sphere_frame
using sphere_d = d4;
using motion_d = d4;
using frame_d = d4; // cos_theta, sin_theta, k, limit

// A quad: corner, unit normal, the dual basis alpha and beta axes (make_quad's numbers, not rounded to float)
struct alignas(16) quad_d
{
    double q[3], n[3], a[3], b[3];
};

struct alignas(16) material_d
{
    double r, g, b;
    double fuzz, ior;
    int32_t kind;
    int32_t texture;
    int32_t texture_needs;
    int32_t pad;
};

struct alignas(16) light_d
{
    quad_d quad;
    double u[3], v[3], c[3];
    double area, cdf, radius, weight;
    int32_t kind;
    int32_t twin;
};

struct alignas(16) texture_d
{
    int32_t kind, even, odd, table;
    double r, g, b, inv_scale;
};

struct alignas(16) noise_d
{
    d4 gradients[256];
    uint8_t perm_x[256];
    uint8_t perm_y[256];
    uint8_t perm_z[256];
    double scale;
};

struct alignas(16) medium_d
{
    double lo[3], hi[3];
    double neg_inv_density;
    double c[3];
    double radius;
    double dm[3];
    int32_t material;
    int32_t first_quad;
    int32_t quad_count;
    int32_t pad;
};

// The camera in double: the pixel grid relative to the center, the lens, the sky
struct camera_d
{
    int32_t width, height, sqrt_spp, max_depth;
    double recip_sqrt_spp;
    double center[3], to_pixel00[3], delta_u[3], delta_v[3], disk_u[3], disk_v[3], sky_bottom[3], sky_top[3];
    int32_t defocus;
    int32_t sampling;
};

struct scene_view_f64
{
    const bvh_node* nodes;      // the float tree (boxes rounded outward), shared with the float tables
    const sphere_d* spheres;    // leaf order, as scene_view's
    const quad_d* quads;
    const int32_t* prim_material;
    const material_d* materials;
    const light_d* lights;
    const texture_d* textures;
    const image_info* images;
    const float4* texels;       // an image's texels are given as floats
    const noise_d* noises;
    const motion_d* sphere_motion;
    const frame_d* sphere_frames;
    const medium_d* media;
    const quad_d* boundary_quads;
    double box_margin;          // how far a double primitive may reach past its float box: node bounds are widened by it
    int32_t node_count;
    int32_t flat;
    int32_t quad_base;
    int32_t prim_count;
    int32_t light_count;
    int32_t has_motion;
    int32_t medium_count;
    int32_t medium_base;
    int32_t has_textures;
    int32_t pad;
};
} // namespace rtb
