/* rt_b200.h — the C-ABI of the B200 path-tracing integrator.
 *
 * A scene goes in as plain tables that refer to each other by index (the reference's gpu::scene_desc,
 * src/gpu/renderer.h:381-395 and its member types at renderer.h:43-377), linear pixels come out. Every entry point
 * returns an rt_status; the reference's C++ API throws instead (renderer.h:518-526, 597-601) and the three exception
 * classes map onto three status codes:
 *   std::runtime_error   -> RT_ERR_RUNTIME  (a CUDA failure, an inconsistent scene)
 *   std::invalid_argument-> RT_ERR_INVALID  (an option out of range)
 *   std::logic_error     -> RT_ERR_LOGIC    (misuse: pixels() before a complete pass, a call on a dead session)
 * rt_last_error_message() returns the message of the calling thread's last failure.
 *
 * All structs are plain data with fixed-width members and explicit padding, so that the layout is the same for C,
 * C++, cgo, ctypes and JNI callers. No CUDA or torch type crosses this boundary.
 */
#ifndef RT_B200_H
#define RT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RT_ABI_VERSION 1

typedef enum rt_status
{
    RT_OK = 0,
    RT_ERR_RUNTIME = 1,     /* std::runtime_error in the reference */
    RT_ERR_INVALID = 2,     /* std::invalid_argument */
    RT_ERR_LOGIC = 3,       /* std::logic_error */
    RT_ERR_NO_DEVICE = 4,   /* no CUDA device: query_device's runtime_error */
    RT_ERR_UNSUPPORTED = 5, /* a scene feature this build does not render (yet): a runtime_error in the reference */
    RT_ERR_CAPACITY = 6,    /* a request beyond a stated limit (the HBM budget, a no-allocation scratch size) */
    RT_ERR_TIMEOUT = 7      /* a bounded wait ran out */
} rt_status;

/* ---- the scene: renderer.h:30-395 as fixed-layout structs ---------------------------------------------------- */

typedef struct rt_vec3
{
    double x, y, z;
} rt_vec3;

/* renderer.h:44-62 texture_kind / texture_desc */
enum { RT_TEXTURE_SOLID = 0, RT_TEXTURE_CHECKER = 1, RT_TEXTURE_IMAGE = 2, RT_TEXTURE_NOISE = 3 };
typedef struct rt_texture_desc
{
    int32_t kind;
    int32_t even, odd;   /* checker: texture indices */
    int32_t image;       /* image: index into images */
    int32_t perlin;      /* noise: index into perlins */
    int32_t pad0;
    rt_vec3 rgb;         /* solid */
    double inv_scale;    /* checker */
    double scale;        /* noise */
} rt_texture_desc;

/* renderer.h:66-71 image_desc: width*height*3 linear floats, rows from the top */
typedef struct rt_image_desc
{
    int32_t width, height;
    const float* rgb;
} rt_image_desc;

/* renderer.h:82-88 perlin_desc */
typedef struct rt_perlin_desc
{
    rt_vec3 random_vectors[256];
    int32_t perm_x[256], perm_y[256], perm_z[256];
} rt_perlin_desc;

/* renderer.h:92-109 material_kind / material_desc */
enum { RT_LAMBERTIAN = 0, RT_METAL = 1, RT_DIELECTRIC = 2, RT_DIFFUSE_LIGHT = 3, RT_ISOTROPIC = 4 };
typedef struct rt_material_desc
{
    int32_t kind;
    int32_t texture;          /* lambertian, diffuse_light, isotropic: index into textures */
    rt_vec3 albedo;           /* metal */
    double fuzz;              /* metal, at most 1 */
    double refraction_index;  /* dielectric */
} rt_material_desc;

/* renderer.h:114-131 sphere_desc (world coordinates, instances baked) */
typedef struct rt_sphere_desc
{
    rt_vec3 center;           /* at time 0 */
    double radius;
    int32_t material;
    int32_t pad0;
    rt_vec3 displacement;     /* motion over the shutter; exactly 0 for a sphere that stands still */
    double uv_cos, uv_sin;    /* the turn of rotate_y instances, for texture coordinates */
} rt_sphere_desc;

/* renderer.h:134-141 quad_desc: points q + a*u + b*v, a, b in [0, 1]; front side u x v */
typedef struct rt_quad_desc
{
    rt_vec3 q, u, v;
    int32_t material;
    int32_t pad0;
} rt_quad_desc;

/* renderer.h:146-162 medium_desc */
enum { RT_BOUNDARY_SPHERE = 0, RT_BOUNDARY_CONVEX_QUADS = 1 };
typedef struct rt_medium_desc
{
    int32_t boundary;
    int32_t material;          /* isotropic */
    rt_sphere_desc sphere;
    const rt_quad_desc* quads;
    int64_t quad_count;
    double neg_inv_density;
} rt_medium_desc;

/* renderer.h:172-193 light_shape / light_desc: the books' lights list, instances baked */
enum { RT_LIGHT_QUAD = 0, RT_LIGHT_SPHERE = 1 };
typedef struct rt_light_desc
{
    int32_t kind;
    int32_t pad0;
    rt_quad_desc quad;
    rt_vec3 center;
    double radius;
    double weight;             /* chance of aiming at it; the weights add up to 1 */
} rt_light_desc;

/* renderer.h:197-203 sampling_strategy */
enum { RT_SAMPLING_UNIFORM = 0, RT_SAMPLING_MATERIAL = 1, RT_SAMPLING_LIGHTS = 2, RT_SAMPLING_MIXTURE = 3 };

/* renderer.h:212-232 camera_desc, as the CPU's camera computed it from its settings (camera.ixx:138-182) */
typedef struct rt_camera_desc
{
    int32_t image_width, image_height;
    int32_t sqrt_spp;          /* a round of strata is sqrt_spp^2 passes */
    int32_t max_depth;         /* rays per path, the camera ray included */
    rt_vec3 center, pixel00_loc, pixel_delta_u, pixel_delta_v;
    int32_t defocus;           /* rays start on the lens disk */
    int32_t sampling;          /* RT_SAMPLING_*: effective_sampling of the requested strategy */
    rt_vec3 defocus_disk_u, defocus_disk_v;
    rt_vec3 sky_bottom, sky_top;
} rt_camera_desc;

/* renderer.h:239-266 light_combination, microfacet_kind / microfacet_desc, environment_desc */
enum { RT_COMBINE_BSDF_ONLY = 0, RT_COMBINE_LIGHTS_ONLY = 1, RT_COMBINE_POWER_HEURISTIC = 2 };
enum { RT_MICROFACET_NONE = 0, RT_MICROFACET_CONDUCTOR = 1, RT_MICROFACET_GLOSS = 2 };
typedef struct rt_microfacet_desc
{
    int32_t kind;
    int32_t pad0;
    double roughness;          /* r in [0, 1]; the GGX width is alpha = r^2 */
} rt_microfacet_desc;

typedef struct rt_environment_desc
{
    rt_image_desc image;       /* equirectangular, +y up, row 0 = +y; finite and >= 0 */
    double yaw_degrees;
    double scale;
} rt_environment_desc;

/* Triangle meshes. The reference traces them only through OptiX (renderer.h:354-377); here they are traced by the
 * same CUDA BVH as the spheres and quads. positions: 3 floats per vertex, world coordinates; indices: 3 per
 * triangle; one scene material for the whole mesh. */
typedef struct rt_mesh_desc
{
    const float* positions;
    int64_t vertex_count;
    const uint32_t* indices;
    int64_t triangle_count;
    int32_t material;
    int32_t pad0;
} rt_mesh_desc;

/* renderer.h:381-395 scene_desc (+ quality_desc renderer.h:268-273, meshes traced by CUDA) */
typedef struct rt_scene_desc
{
    const rt_sphere_desc* spheres;     int64_t sphere_count;
    const rt_material_desc* materials; int64_t material_count;
    rt_camera_desc camera;
    const rt_texture_desc* textures;   int64_t texture_count;
    const rt_image_desc* images;       int64_t image_count;
    const rt_perlin_desc* perlins;     int64_t perlin_count;
    const rt_quad_desc* quads;         int64_t quad_count;
    const rt_medium_desc* media;       int64_t medium_count;
    const rt_light_desc* lights;       int64_t light_count;
    /* quality_desc */
    int32_t combination;               /* RT_COMBINE_*: 0 renders with the books' strategies */
    int32_t quality;                   /* nonzero: render with the NEE/MIS integrator (the reference's quality kernel) */
    const rt_microfacet_desc* microfacets; int64_t microfacet_count; /* 0 or one per material */
    const rt_environment_desc* environment;                          /* NULL: the camera's sky gradient */
    const rt_mesh_desc* meshes;        int64_t mesh_count;
} rt_scene_desc;

/* ---- options and results: renderer.h:404-492, 530-562 -------------------------------------------------------- */

/* renderer.h:402-409 precision: the number type the GPU computes with. RT_FLOAT32 is the hot path. RT_FLOAT64 renders
 * the books' scenes (spheres, moving spheres, quads, smoke, textures; the four books' strategies) with every number of a
 * path in double and 53-bit random numbers, in the persistent form: a mode to compare with, as the reference's. As
 * there, the NEE/MIS integrator (rt_scene_desc.quality) and triangle meshes compute in float only (RT_ERR_INVALID), and
 * a float64 session displays the books' bytes only. */
enum { RT_FLOAT32 = 0, RT_FLOAT64 = 1 };

typedef struct rt_render_options
{
    uint64_t seed;              /* round r draws with seed + r * 2^32 (renderer.h:564-566) */
    int64_t passes;             /* 0: sqrt_spp^2; > 0: exactly that many */
    int32_t arithmetic;         /* RT_FLOAT32 (the hot path) or RT_FLOAT64 (the books' integrator in double) */
    int32_t pad0;
    double launch_seconds;      /* how long one launch is planned to take, (0, 0.5] */
} rt_render_options;

typedef struct rt_kernel_info
{
    char name[32];
    int32_t registers;
    int32_t local_bytes;
    int32_t blocks_per_multiprocessor;
    int32_t threads_per_block;
    int32_t max_threads_per_multiprocessor;
    int32_t multiprocessors;
} rt_kernel_info;

typedef struct rt_render_result
{
    double seconds;             /* render() end to end: validation, BVH, upload, all passes, download */
    double kernel_seconds;      /* the passes alone, timed on the GPU */
    uint64_t rays;              /* path segments: closest-hit queries, camera rays and bounces */
    uint64_t shadow_rays;       /* NEE shadow queries, counted apart */
    int64_t passes;
    int32_t launches;
    int32_t kernel_launches;    /* as rt_render_report's */
    rt_kernel_info kernel;
} rt_render_result;

typedef struct rt_device_info
{
    char name[256];
    int32_t compute_capability_major, compute_capability_minor;
    int32_t multiprocessors;
    int32_t runtime_version, driver_version;
    int32_t pad0;
    double memory_gib;
} rt_device_info;

/* How a session's launches run (no counterpart in the reference, whose renderer has one kernel): the persistent
   kernel, whose lanes each carry a path from its camera ray to its end, or the wavefront, whose paths wait in device
   memory between a shade kernel and a trace kernel that gives each lane a new ray as soon as its own is answered.
   Both make the same image from the same seed. AUTO takes the wavefront for scenes searched through the tree and the
   persistent kernel for the small ones searched flat (and for the counting build). */
enum { RT_FORM_AUTO = 0, RT_FORM_PERSISTENT = 1, RT_FORM_WAVEFRONT = 2 };

typedef struct rt_session_options
{
    uint64_t seed;
    int32_t arithmetic;         /* RT_FLOAT32 or RT_FLOAT64 (a persistent-form session; RT_FORM_WAVEFRONT is refused) */
    int32_t form;               /* RT_FORM_*; 0 (AUTO) where the caller zeroed the struct */
    double launch_seconds;
} rt_session_options;

/* renderer.h:574-579 accumulation */
typedef struct rt_accumulation
{
    int64_t passes;
    int32_t rows;
    int32_t pad0;
} rt_accumulation;

/* renderer.h:583-590 render_report */
typedef struct rt_render_report
{
    rt_accumulation state;
    int32_t launches;
    int32_t kernel_launches;    /* GPU kernels the call launched: a persistent launch's render and reduction, a
                                   wavefront launch's shade and trace per step and its reduction (no counterpart) */
    double gpu_seconds;
    double longest_launch_seconds;
} rt_render_report;

/* ---- entry points ------------------------------------------------------------------------------------------ */

/* The thread's last error message ("" after success). Replaces the what() of the reference's exceptions. */
const char* rt_last_error_message(void);

/* ABI version of the loaded library (RT_ABI_VERSION). */
int32_t rt_abi_version(void);

/* renderer.h:516 query_device(wait_mode): describes the first CUDA device and starts CUDA on it. */
rt_status rt_query_device(rt_device_info* info);

/* Selects the CUDA device this thread's later calls use (the reference renders on the first device only,
 * renderer.h:512-518; one process per GPU calls this with its local rank). */
rt_status rt_set_device(int32_t device);

/* renderer.h:400 count_lamps: the quality integrator's lamps (quads and still spheres glowing one solid color). */
rt_status rt_count_lamps(const rt_scene_desc* scene, int32_t* count);

/* renderer.h:168 is_convex: whether quads bound one convex shape (a medium boundary the GPU can render). */
rt_status rt_is_convex(const rt_quad_desc* quads, int64_t count, int32_t* convex);

/* renderer.h:526 render(scene_desc, render_options) -> render_result. pixels: width*height*3 linear doubles, rows
 * from the top (render_result::pixels, renderer.h:477-478); pixel_count must be width*height*3. */
rt_status rt_render(const rt_scene_desc* scene, const rt_render_options* options, double* pixels,
                    int64_t pixel_count, rt_render_result* result);

/* A scene resident on the device: validated, its BVH built and uploaded once (the first half of the session
 * constructor, renderer.h:596-601). Several sessions and serving requests may share one. */
typedef struct rt_scene rt_scene;
rt_status rt_scene_create(const rt_scene_desc* desc, rt_scene** scene);
rt_status rt_scene_destroy(rt_scene* scene);
/* Primitive and node counts and device bytes of the resident scene, for reports. */
typedef struct rt_scene_stats
{
    int64_t spheres, quads, triangles, nodes, leaves, lamps, lights;
    int64_t device_bytes;
    int32_t depth;
    int32_t max_leaf_size;
    int32_t flat;               /* 1: a small scene of spheres and quads, searched by testing every primitive */
    int32_t pad0;
} rt_scene_stats;
rt_status rt_scene_stats_get(const rt_scene* scene, rt_scene_stats* stats);

/* renderer.h:591-673 session: one view of a resident scene whose image gains passes on demand. */
typedef struct rt_session rt_session;
rt_status rt_session_create(rt_scene* scene, const rt_session_options* options, rt_session** session);
rt_status rt_session_destroy(rt_session* session);
/* set_camera (renderer.h:602): a new view; the image starts over. The strategy must stay the scene's. */
rt_status rt_session_set_camera(rt_session* session, const rt_camera_desc* camera);
rt_status rt_session_state(const rt_session* session, rt_accumulation* state);
/* render_to({passes, 0}) (renderer.h:611): renders until the image has `passes` complete passes. */
rt_status rt_session_render_to(rt_session* session, int64_t passes, rt_render_report* report);
/* render_for(seconds, pass_limit) (renderer.h:618). */
rt_status rt_session_render_for(rt_session* session, double seconds, int64_t pass_limit, rt_render_report* report);
/* pixels() (renderer.h:623): sums / passes as doubles, width*height*3, rows from the top. */
rt_status rt_session_pixels(const rt_session* session, double* pixels, int64_t pixel_count);
/* rays(), shadow_rays(), kernel_seconds() (renderer.h:664-667), since the view was set */
rt_status rt_session_counters(const rt_session* session, uint64_t* rays, uint64_t* shadow_rays,
                              double* kernel_seconds);
rt_status rt_session_kernel(const rt_session* session, rt_kernel_info* info);

/* Renders passes [pass_begin, pass_end) of `camera`'s view of a resident scene and ADDS the samples' sums into
 * device_sums (width*height*3 doubles of device memory the caller owns, rows from the top; zero it to start an
 * image), allocating no device memory at all. This entry point has no counterpart in the reference. It is for
 * callers that cannot call cudaMalloc: a program that owns all of its device memory through its own pool (an engine
 * or a server that reserves its HBM at start-up and hands out pre-sized buffers only), or a thread that must not
 * block on the allocator, which can synchronize the device. The render kernel's scratch (work and ray counters, the
 * per-chunk partial sums) comes from a fixed 64 MiB array in the library's device image instead: an image may have
 * at most 2,796,192 pixels once padded to 8x4 tiles (about 1920x1440), larger ones return RT_ERR_CAPACITY. Every GPU
 * that loads the library holds that array until the process exits. The first call on a device looks up the array's
 * address (cudaGetSymbolAddress) with that device current and creates the device's stream for these calls (a
 * non-blocking stream: a call neither waits for nor delays the caller's streams), so make that first call before any
 * stream capture. Every call shares the array and leaves its contents behind; calls are synchronous (each waits for
 * its own stream), and two calls that overlap on the GPU (from two host threads) race. Passes are rendered in
 * launches of whole 16-pass chunks, aligned to multiples of 16 as a session aligns its launches: when pass_begin and
 * pass_end fall on multiples of 16 (or on the boundaries a session's launches used), the sums equal that session's
 * render of the same seed and passes bit for bit; a range that starts or ends inside a chunk sums that chunk in two
 * parts, equal to the session's to rounding. rays / shadow_rays (may be NULL): this call's counts. */
rt_status rt_render_passes_no_alloc(rt_scene* scene, const rt_camera_desc* camera, uint64_t seed, int64_t pass_begin,
                                    int64_t pass_end, double* device_sums, uint64_t* rays, uint64_t* shadow_rays);

/* ---- the display transform and the image files (renderer.h:278-303, 623-635; image.ixx:93-203) ------------ */

/* renderer.h:286-292 tone_map: how linear light becomes a screen's bytes. BOOKS: the books' bytes (gamma 2 as a
 * square root, clamped to 0.999, times 256 truncated; image::save_png's to_byte). NONE: the light times 2^exposure,
 * clipped to [0, 1], sRGB-encoded. AGX: Troy Sobotka's AgX (16.5 stops on a log2 curve). NEUTRAL: Khronos PBR Neutral,
 * then sRGB. The last three are dithered by interleaved gradient noise of the pixel's position. */
enum { RT_TONE_BOOKS = 0, RT_TONE_NONE = 1, RT_TONE_AGX = 2, RT_TONE_NEUTRAL = 3 };

/* renderer.h:294-303 display_options: a tone map and an exposure in stops, a finite number within +-24
 * (max_exposure); BOOKS takes no exposure (RT_ERR_INVALID otherwise, as check_display, renderer.cu:1204-1220). */
typedef struct rt_display_options
{
    int32_t tone_map;           /* RT_TONE_* */
    int32_t pad0;
    double exposure;
} rt_display_options;

/* session::display(options) (renderer.h:623-635): the image of the complete passes as 4 bytes per pixel (red, green,
 * blue, 255), rows from the top, computed on the GPU from the FP64 sums (the reference's display.cu and tonemap.cu
 * kernels, bit for bit). byte_count must be width*height*4. RT_ERR_LOGIC before the image has a complete pass. */
rt_status rt_session_display(rt_session* session, const rt_display_options* options, uint8_t* rgba,
                             int64_t byte_count);

/* The same transform on an image kept in device memory by the caller (a served frame, the no-allocation entry
 * point's sums): device_sums holds width*height*3 doubles, the sums of `passes` passes; device_rgba receives
 * width*height*4 bytes (4-byte aligned). Queued on `stream` (a cudaStream_t; NULL: the default stream) and not waited
 * for. No counterpart in the reference's API (its session keeps its sums private). */
rt_status rt_display_device(const double* device_sums, int32_t width, int32_t height, int64_t passes,
                            const rt_display_options* options, uint8_t* device_rgba, void* stream);

/* image::save (image.ixx:170-184): writes `pixels` (width*height*3 linear doubles, rows from the top) to `path` in
 * the format its extension names, .pfm or .png in any letter case (RT_ERR_INVALID for another). PFM (save_pfm,
 * image.ixx:157-168): "PF", the size, -1.0, rows from the bottom as little-endian float32, the linear values. PNG
 * (save_png, image.ixx:116-145): 8-bit RGB of the display transform's bytes under `options` (NULL: BOOKS; a tone map
 * other than BOOKS is computed on the GPU, as the reference computes its tone maps' bytes). */
rt_status rt_image_save(const char* path, const double* pixels, int32_t width, int32_t height,
                        const rt_display_options* options);

/* image::mean_radiance (image.ixx:93-103): the average over all pixels of (r + g + b) / 3, summed in pixel order as
 * the reference's average() folds them. */
rt_status rt_image_mean_radiance(const double* pixels, int32_t width, int32_t height, double* mean);

/* The session's image of complete passes saved as rt_image_save saves pixels(), and its mean radiance. */
rt_status rt_session_save(rt_session* session, const char* path, const rt_display_options* options);
rt_status rt_session_mean_radiance(const rt_session* session, double* mean);

/* Device-resident variant for callers that keep the image on the GPU (a served frame, a display transform):
 * the device address of the per-pixel sums (3 doubles per pixel, rows from the top) and of the pass count. */
rt_status rt_session_device_sums(const rt_session* session, const double** sums, int64_t* passes);

/* Per-kernel timing (no counterpart in the reference, whose render_result gives the launches' total only): while on,
 * every kernel a launch runs is bracketed by CUDA events on the session's stream and its time added to its kind's
 * total: [0] the persistent render kernel, [1] the wavefront's shade kernel, [2] its trace kernel, [3] the
 * reductions. Off by default (the events cost a few microseconds a kernel); totals since the view was set. */
enum { RT_KERNEL_RENDER = 0, RT_KERNEL_SHADE = 1, RT_KERNEL_TRACE = 2, RT_KERNEL_REDUCE = 3 };
typedef struct rt_kernel_times
{
    double seconds[4];
    int64_t launches[4];
} rt_kernel_times;
rt_status rt_session_set_timing(rt_session* session, int32_t on);
rt_status rt_session_kernel_times(const rt_session* session, rt_kernel_times* times);

/* The wavefront's autotuner (no counterpart in the reference, whose launch planner sizes launches but never the
 * kernels' shapes, renderer.cu:201-308): short renders of the session's view under candidate launch shapes, one knob
 * after another from the built-in defaults: the trace kernel's register cap (as the minimum blocks per multiprocessor
 * its launch bounds give: 8, or 6 with more registers a thread) and its grid (blocks per multiprocessor); the slot
 * pool, which is the query queue's capacity (two queries a slot); the shade kernel's block size. The best shape stays
 * with the session and is remembered, per device and scene class (flat or tree, integrator, features, triangles,
 * size), for the sessions made after it. The image does not depend on the shape. The view must have no passes yet
 * (RT_ERR_LOGIC otherwise) and starts over afterwards; a persistent-form session has nothing to tune (slots 0). */
typedef struct rt_tuning
{
    int32_t slots;
    int32_t trace_blocks_per_sm;
    int32_t shade_block;
    int32_t trace_min_blocks;
    int32_t trace_registers;    /* the chosen trace kernel's registers a thread */
    int32_t trials;             /* renders measured (0: the shape came from an earlier session's tuning, or defaults) */
    int32_t from_cache;         /* 1: taken from an earlier tuning of the same scene class */
    int32_t pad0;
    double samples_per_second;  /* the chosen shape's measured speed (pixel passes a second) */
    double default_samples_per_second; /* the built-in defaults' */
} rt_tuning;
/* trial_passes: the passes of each measured launch (after a one-chunk launch, as the session's planner probes);
 * 0: enough for about 32 million samples, so that every candidate pool reaches its steady state. */
rt_status rt_session_autotune(rt_session* session, int64_t trial_passes, rt_tuning* result);
rt_status rt_session_tuning(const rt_session* session, rt_tuning* current);
/* Applies a shape an earlier autotune reported (slots, trace_blocks_per_sm, shade_block, trace_min_blocks;
 * the other fields are ignored), so a service can keep its tunings across processes. RT_ERR_INVALID for a value the
 * kernels do not take, RT_ERR_LOGIC for a persistent-form session. */
rt_status rt_session_set_tuning(rt_session* session, const rt_tuning* shape);
/* The autotuner's search on a caller-given measure (its selection logic without a GPU, for tests): the candidates
 * of a GPU whose trace kernels fit max_trace_blocks (default cap) and max_trace_blocks_roomy (roomy cap) blocks a
 * multiprocessor, each measured by measure(shape, user) in samples per second. */
typedef double (*rt_tune_measure_fn)(const rt_tuning* shape, void* user);
rt_status rt_autotune_simulate(int32_t max_trace_blocks, int32_t max_trace_blocks_roomy, rt_tune_measure_fn measure,
                               void* user, rt_tuning* result);

/* The counting build (no counterpart in the reference): while on, launches also count BVH node fetches and sphere,
 * quad and triangle tests (closest-hit and shadow traversals together), the measured work behind the roofline's
 * algorithmic bytes. Slower; off by default. counts: nodes, spheres, quads, triangles since the view was set. */
rt_status rt_session_set_counting(rt_session* session, int32_t on);
rt_status rt_session_fetch_counts(const rt_session* session, uint64_t counts[4]);

/* ---- batched rendering and serving (no counterpart in the reference: one session renders one view, renderer.h:
 * 585-590; here many requests share each refinement step's launches) ------------------------------------------- */

/* One job of a batch: a scene (validated and built for the batch), the seed and passes it renders, and where its
 * image goes (width*height*3 doubles, host memory, rows from the top). */
typedef struct rt_batch_job
{
    const rt_scene_desc* scene;
    uint64_t seed;
    int64_t passes;             /* 0: sqrt_spp^2 */
    double* pixels;
} rt_batch_job;

typedef struct rt_batch_options
{
    int64_t partial_budget_bytes; /* the partials arena a step may use; 0: 1 GiB */
    int32_t use_graph;          /* capture the step into a CUDA graph and replay it */
    int32_t pad0;
} rt_batch_options;

typedef struct rt_batch_report
{
    double seconds;             /* the whole call */
    double setup_seconds;       /* validation, BVH builds and uploads of the jobs' scenes */
    double gpu_seconds;         /* the steps' launches, timed on the GPU */
    uint64_t rays;
    uint64_t shadow_rays;
    int32_t steps;
    int32_t launches;
    int32_t graph;              /* the steps ran as a captured graph */
    int32_t pad0;
} rt_batch_report;

/* Renders every job to its passes in batched steps (many jobs of any size and scene per step; each group of them,
   by search and form, one persistent launch or one wavefront run per step). */
rt_status rt_batch_render(const rt_batch_job* jobs, int32_t count, const rt_batch_options* options,
                          rt_batch_report* report);

typedef struct rt_server rt_server;

typedef struct rt_server_options
{
    int64_t hbm_budget_bytes;   /* what the admitted requests' sums and the step's partials may hold */
    double step_seconds;        /* the GPU time a refinement step aims at */
    int32_t use_graph;
    /* 1: the continuous wavefront. One pool of path slots lives as long as the server, and a request's refinement
     * is published into it while the unclaimed backlog is short, so that no step drains the pool; its first pass is
     * rendered in a batched step of first frames (whose last paths advance through steps of a few slots, not of the
     * whole pool) and handed over. A step runs the pool for about step_seconds of GPU time and returns with work still
     * running. Images equal a session's rendered to one pass, then to the target. 2: the same with the first passes
     * published into the pool too. 0: batched steps (each step a batch of passes, drained before it returns). */
    int32_t continuous;
    /* The continuous wavefront (ignored otherwise): its slot pool (a multiple of 128; 0: 1.5 x 2^20), its steps
     * between two readings of the counts (1-16; 0: 2; a sample published now is claimable from the next group but
     * one), and the unclaimed backlog it keeps published ahead of the slots, in seconds of GPU time at the measured
     * rate, three groups' time if more (0: 0.002). */
    int32_t slots;
    int32_t group_steps;
    double lookahead_seconds;
} rt_server_options;

enum { RT_REQUEST_QUEUED = 0, RT_REQUEST_ACTIVE = 1, RT_REQUEST_DONE = 2, RT_REQUEST_CANCELLED = 3 };

typedef struct rt_request_status
{
    int32_t state;              /* RT_REQUEST_* */
    int32_t pad0;
    int64_t passes;             /* complete passes so far */
    int64_t target;
    double first_frame_seconds; /* from submit to the end of its first pass; < 0 until then */
    double done_seconds;        /* from submit to its target; < 0 until then */
} rt_request_status;

typedef struct rt_server_step_report
{
    double gpu_seconds;
    int32_t admitted;           /* requests admitted this step */
    int32_t first_frames;       /* requests that got their first pass */
    int32_t refined;            /* requests that got more passes */
    int32_t completed;
    int32_t active;
    int32_t queued;
} rt_server_step_report;

typedef struct rt_server_stats
{
    uint64_t rays;
    uint64_t shadow_rays;
    double gpu_seconds;
    int64_t steps;
    int64_t launches;
    int64_t completed;
    int64_t used_bytes;
    /* The continuous wavefront: groups of steps run, and the mean over groups of the pool's slots that queued a ray
     * in the group's last step (1: no slot idle). 0 for batched steps. */
    int64_t groups;
    double busy_slots;
} rt_server_stats;

rt_status rt_server_create(const rt_server_options* options, rt_server** server);
rt_status rt_server_destroy(rt_server* server);
/* Queues a request: a view of a resident scene (the scene must outlive the request), its seed and target passes. */
rt_status rt_server_submit(rt_server* server, rt_scene* scene, const rt_camera_desc* camera, uint64_t seed,
                           int64_t target_passes, int64_t* request_id);
/* One refinement step: admit what the budget allows, first frames first, then refinement; synchronous. */
rt_status rt_server_step(rt_server* server, rt_server_step_report* report);
rt_status rt_server_poll(const rt_server* server, int64_t request_id, rt_request_status* status);
/* The request's image so far (sums / passes); frees a finished request's device memory. */
rt_status rt_server_fetch(rt_server* server, int64_t request_id, double* pixels, int64_t pixel_count);
/* The request's image so far through the display transform (rt_session_display's bytes for its view): the frame a
 * served client is shown. Keeps the request's memory (a later rt_server_fetch frees a finished one). */
rt_status rt_server_display(rt_server* server, int64_t request_id, const rt_display_options* options, uint8_t* rgba,
                            int64_t byte_count);
rt_status rt_server_cancel(rt_server* server, int64_t request_id);
rt_status rt_server_stats_get(const rt_server* server, rt_server_stats* stats);

/* ---- parity hooks (no counterpart in the reference's API: its GpuTests call device functions directly) ------ */

/* Closest-hit queries for given rays on the device: the first hit's primitive in SOURCE index space (spheres
 * 0..S-1, quads S..S+Q-1, triangles S+Q.. in mesh order; -1 for a miss) and its t, for the first-hit parity test
 * (bvh.cuh:576-706 closest_hit; tracer_check_layout.h classes). Host arrays: origins and directions 3 floats each. */
rt_status rt_scene_closest_hits(rt_scene* scene, const float* origins, const float* directions, int64_t count,
                                int32_t* ids, float* ts);

/* The deterministic camera rays of pass `pass` for every pixel of the scene's camera, as the kernel generates them
 * (rows from the top), for the parity test: origins and directions, 3 floats each per pixel. */
rt_status rt_scene_camera_rays(rt_scene* scene, uint64_t seed, int64_t pass, float* origins, float* directions,
                               int64_t pixel_count);

/* ---- built-in scenes (scenes.ixx:79-518, gpu_scenes*.ixx) ---------------------------------------------------- */

/* A scene the library builds from its name, owning its tables. Names: "weekend" (the first book's cover), "cornell",
 * "glass" (the Cornell box with a glass ball), "cornell-mis" (glass under NEE+MIS), "materials", "quads", "furnace"
 * (every pixel exactly 1: a closed white sky), "mesh-ggx" (the displaced 1.3M-triangle icosphere in GGX metal under an
 * HDR sky), "cover-N" (a cover variant of about N random spheres, with its own seed). width, spp, depth override the scene's camera when > 0; scene_seed picks the scene's random
 * content (the CPU's scene generator, mt19937_64 seeded as scenes.ixx's main thread). */
typedef struct rt_builtin_params
{
    int32_t image_width;
    int32_t image_height;       /* 0: from the scene's aspect ratio */
    int32_t samples_per_pixel;  /* rounded to a square as camera.ixx:141 */
    int32_t max_depth;
    int32_t sampling;           /* -1: the scene's own; else RT_SAMPLING_* */
    int32_t combination;        /* -1: the scene's own; else RT_COMBINE_* (nonzero turns on the NEE/MIS integrator) */
    uint64_t scene_seed;
    int32_t sphere_count;       /* cover-N: how many random spheres */
    int32_t mesh_level;         /* mesh-ggx: icosphere subdivision level (8: 1,310,720 triangles) */
    int32_t env_width;          /* mesh-ggx: environment map width (height = width / 2) */
    int32_t pad0;
    double orbit_azimuth;       /* when orbit != 0: the camera orbits the look-at point at its distance (serving */
    double orbit_elevation;     /* requests): azimuth about +y from +z and elevation above the horizon, in degrees */
    int32_t orbit;
    int32_t pad1;
} rt_builtin_params;

typedef struct rt_owned_scene rt_owned_scene;
rt_status rt_builtin_scene(const char* name, const rt_builtin_params* params, rt_owned_scene** scene);
const rt_scene_desc* rt_owned_scene_desc(const rt_owned_scene* scene);
rt_status rt_owned_scene_destroy(rt_owned_scene* scene);
/* The camera of a built-in scene with the given overrides (an orbit, a size), its geometry built at its cheapest. */
rt_status rt_builtin_camera(const char* name, const rt_builtin_params* params, rt_camera_desc* camera);
/* A scene serialized once and fed to every renderer (the oracle, the reference build, this one). */
rt_status rt_scene_save(const rt_scene_desc* scene, const char* path);
rt_status rt_scene_load(const char* path, rt_owned_scene** scene);

#ifdef __cplusplus
}
#endif

#endif /* RT_B200_H */
