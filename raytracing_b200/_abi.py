"""ctypes mirror of include/rt_b200.h: the same structs, field for field, and the entry points' signatures."""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIBRARY = Path(__file__).resolve().parent / "_lib" / "librt_b200.so"

RT_OK, RT_ERR_RUNTIME, RT_ERR_INVALID, RT_ERR_LOGIC, RT_ERR_NO_DEVICE, RT_ERR_UNSUPPORTED, RT_ERR_CAPACITY, \
    RT_ERR_TIMEOUT = range(8)
RT_TEXTURE_SOLID, RT_TEXTURE_CHECKER, RT_TEXTURE_IMAGE, RT_TEXTURE_NOISE = range(4)
RT_LAMBERTIAN, RT_METAL, RT_DIELECTRIC, RT_DIFFUSE_LIGHT, RT_ISOTROPIC = range(5)
RT_LIGHT_QUAD, RT_LIGHT_SPHERE = range(2)
RT_SAMPLING_UNIFORM, RT_SAMPLING_MATERIAL, RT_SAMPLING_LIGHTS, RT_SAMPLING_MIXTURE = range(4)
RT_COMBINE_BSDF_ONLY, RT_COMBINE_LIGHTS_ONLY, RT_COMBINE_POWER_HEURISTIC = range(3)
RT_MICROFACET_NONE, RT_MICROFACET_CONDUCTOR, RT_MICROFACET_GLOSS = range(3)
RT_FLOAT32, RT_FLOAT64 = range(2)
RT_FORM_AUTO, RT_FORM_PERSISTENT, RT_FORM_WAVEFRONT = range(3)
RT_TONE_BOOKS, RT_TONE_NONE, RT_TONE_AGX, RT_TONE_NEUTRAL = range(4)


class Vec3(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


class TextureDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("even", C.c_int32), ("odd", C.c_int32), ("image", C.c_int32),
                ("perlin", C.c_int32), ("pad0", C.c_int32), ("rgb", Vec3), ("inv_scale", C.c_double),
                ("scale", C.c_double)]


class ImageDesc(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("rgb", C.POINTER(C.c_float))]


class PerlinDesc(C.Structure):
    _fields_ = [("random_vectors", Vec3 * 256), ("perm_x", C.c_int32 * 256), ("perm_y", C.c_int32 * 256),
                ("perm_z", C.c_int32 * 256)]


class MaterialDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("texture", C.c_int32), ("albedo", Vec3), ("fuzz", C.c_double),
                ("refraction_index", C.c_double)]


class SphereDesc(C.Structure):
    _fields_ = [("center", Vec3), ("radius", C.c_double), ("material", C.c_int32), ("pad0", C.c_int32),
                ("displacement", Vec3), ("uv_cos", C.c_double), ("uv_sin", C.c_double)]


class QuadDesc(C.Structure):
    _fields_ = [("q", Vec3), ("u", Vec3), ("v", Vec3), ("material", C.c_int32), ("pad0", C.c_int32)]


class MediumDesc(C.Structure):
    _fields_ = [("boundary", C.c_int32), ("material", C.c_int32), ("sphere", SphereDesc),
                ("quads", C.POINTER(QuadDesc)), ("quad_count", C.c_int64), ("neg_inv_density", C.c_double)]


class LightDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("pad0", C.c_int32), ("quad", QuadDesc), ("center", Vec3),
                ("radius", C.c_double), ("weight", C.c_double)]


class CameraDesc(C.Structure):
    _fields_ = [("image_width", C.c_int32), ("image_height", C.c_int32), ("sqrt_spp", C.c_int32),
                ("max_depth", C.c_int32), ("center", Vec3), ("pixel00_loc", Vec3), ("pixel_delta_u", Vec3),
                ("pixel_delta_v", Vec3), ("defocus", C.c_int32), ("sampling", C.c_int32),
                ("defocus_disk_u", Vec3), ("defocus_disk_v", Vec3), ("sky_bottom", Vec3), ("sky_top", Vec3)]


class MicrofacetDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("pad0", C.c_int32), ("roughness", C.c_double)]


class EnvironmentDesc(C.Structure):
    _fields_ = [("image", ImageDesc), ("yaw_degrees", C.c_double), ("scale", C.c_double)]


class DisplayOptions(C.Structure):
    _fields_ = [("tone_map", C.c_int32), ("pad0", C.c_int32), ("exposure", C.c_double)]


class KernelTimes(C.Structure):
    _fields_ = [("seconds", C.c_double * 4), ("launches", C.c_int64 * 4)]


class Tuning(C.Structure):
    _fields_ = [("slots", C.c_int32), ("trace_blocks_per_sm", C.c_int32), ("shade_block", C.c_int32),
                ("trace_min_blocks", C.c_int32), ("trace_registers", C.c_int32), ("trials", C.c_int32),
                ("from_cache", C.c_int32), ("pad0", C.c_int32), ("samples_per_second", C.c_double),
                ("default_samples_per_second", C.c_double)]


TUNE_MEASURE = C.CFUNCTYPE(C.c_double, C.POINTER(Tuning), C.c_void_p)


class MeshDesc(C.Structure):
    _fields_ = [("positions", C.POINTER(C.c_float)), ("vertex_count", C.c_int64),
                ("indices", C.POINTER(C.c_uint32)), ("triangle_count", C.c_int64), ("material", C.c_int32),
                ("pad0", C.c_int32)]


class SceneDesc(C.Structure):
    _fields_ = [("spheres", C.POINTER(SphereDesc)), ("sphere_count", C.c_int64),
                ("materials", C.POINTER(MaterialDesc)), ("material_count", C.c_int64),
                ("camera", CameraDesc),
                ("textures", C.POINTER(TextureDesc)), ("texture_count", C.c_int64),
                ("images", C.POINTER(ImageDesc)), ("image_count", C.c_int64),
                ("perlins", C.POINTER(PerlinDesc)), ("perlin_count", C.c_int64),
                ("quads", C.POINTER(QuadDesc)), ("quad_count", C.c_int64),
                ("media", C.POINTER(MediumDesc)), ("medium_count", C.c_int64),
                ("lights", C.POINTER(LightDesc)), ("light_count", C.c_int64),
                ("combination", C.c_int32), ("quality", C.c_int32),
                ("microfacets", C.POINTER(MicrofacetDesc)), ("microfacet_count", C.c_int64),
                ("environment", C.POINTER(EnvironmentDesc)),
                ("meshes", C.POINTER(MeshDesc)), ("mesh_count", C.c_int64)]


class RenderOptions(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("passes", C.c_int64), ("arithmetic", C.c_int32), ("pad0", C.c_int32),
                ("launch_seconds", C.c_double)]


class KernelInfo(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("registers", C.c_int32), ("local_bytes", C.c_int32),
                ("blocks_per_multiprocessor", C.c_int32), ("threads_per_block", C.c_int32),
                ("max_threads_per_multiprocessor", C.c_int32), ("multiprocessors", C.c_int32)]


class RenderResult(C.Structure):
    _fields_ = [("seconds", C.c_double), ("kernel_seconds", C.c_double), ("rays", C.c_uint64),
                ("shadow_rays", C.c_uint64), ("passes", C.c_int64), ("launches", C.c_int32),
                ("kernel_launches", C.c_int32), ("kernel", KernelInfo)]


class DeviceInfo(C.Structure):
    _fields_ = [("name", C.c_char * 256), ("compute_capability_major", C.c_int32),
                ("compute_capability_minor", C.c_int32), ("multiprocessors", C.c_int32),
                ("runtime_version", C.c_int32), ("driver_version", C.c_int32), ("pad0", C.c_int32),
                ("memory_gib", C.c_double)]


class SessionOptions(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("arithmetic", C.c_int32), ("form", C.c_int32),
                ("launch_seconds", C.c_double)]


class Accumulation(C.Structure):
    _fields_ = [("passes", C.c_int64), ("rows", C.c_int32), ("pad0", C.c_int32)]


class RenderReport(C.Structure):
    _fields_ = [("state", Accumulation), ("launches", C.c_int32), ("kernel_launches", C.c_int32),
                ("gpu_seconds", C.c_double), ("longest_launch_seconds", C.c_double)]


class SceneStats(C.Structure):
    _fields_ = [("spheres", C.c_int64), ("quads", C.c_int64), ("triangles", C.c_int64), ("nodes", C.c_int64),
                ("leaves", C.c_int64), ("lamps", C.c_int64), ("lights", C.c_int64), ("device_bytes", C.c_int64),
                ("depth", C.c_int32), ("max_leaf_size", C.c_int32), ("flat", C.c_int32), ("pad0", C.c_int32)]


class BuiltinParams(C.Structure):
    _fields_ = [("image_width", C.c_int32), ("image_height", C.c_int32), ("samples_per_pixel", C.c_int32),
                ("max_depth", C.c_int32), ("sampling", C.c_int32), ("combination", C.c_int32),
                ("scene_seed", C.c_uint64), ("sphere_count", C.c_int32), ("mesh_level", C.c_int32),
                ("env_width", C.c_int32), ("pad0", C.c_int32), ("orbit_azimuth", C.c_double),
                ("orbit_elevation", C.c_double), ("orbit", C.c_int32), ("pad1", C.c_int32)]


class BatchJob(C.Structure):
    _fields_ = [("scene", C.POINTER(SceneDesc)), ("seed", C.c_uint64), ("passes", C.c_int64),
                ("pixels", C.POINTER(C.c_double))]


class BatchOptions(C.Structure):
    _fields_ = [("partial_budget_bytes", C.c_int64), ("use_graph", C.c_int32), ("pad0", C.c_int32)]


class BatchReport(C.Structure):
    _fields_ = [("seconds", C.c_double), ("setup_seconds", C.c_double), ("gpu_seconds", C.c_double),
                ("rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("steps", C.c_int32), ("launches", C.c_int32),
                ("graph", C.c_int32), ("pad0", C.c_int32)]


class ServerOptions(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_int64), ("step_seconds", C.c_double), ("use_graph", C.c_int32),
                ("continuous", C.c_int32), ("slots", C.c_int32), ("group_steps", C.c_int32),
                ("lookahead_seconds", C.c_double)]


class RequestStatus(C.Structure):
    _fields_ = [("state", C.c_int32), ("pad0", C.c_int32), ("passes", C.c_int64), ("target", C.c_int64),
                ("first_frame_seconds", C.c_double), ("done_seconds", C.c_double)]


class ServerStepReport(C.Structure):
    _fields_ = [("gpu_seconds", C.c_double), ("admitted", C.c_int32), ("first_frames", C.c_int32),
                ("refined", C.c_int32), ("completed", C.c_int32), ("active", C.c_int32), ("queued", C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("gpu_seconds", C.c_double),
                ("steps", C.c_int64), ("launches", C.c_int64), ("completed", C.c_int64), ("used_bytes", C.c_int64),
                ("groups", C.c_int64), ("busy_slots", C.c_double)]


# (name, restype, argtypes) of every entry point declared in include/rt_b200.h
ENTRY_POINTS = [
    ("rt_last_error_message", C.c_char_p, []),
    ("rt_abi_version", C.c_int32, []),
    ("rt_query_device", C.c_int, [C.POINTER(DeviceInfo)]),
    ("rt_set_device", C.c_int, [C.c_int32]),
    ("rt_count_lamps", C.c_int, [C.POINTER(SceneDesc), C.POINTER(C.c_int32)]),
    ("rt_is_convex", C.c_int, [C.POINTER(QuadDesc), C.c_int64, C.POINTER(C.c_int32)]),
    ("rt_render", C.c_int, [C.POINTER(SceneDesc), C.POINTER(RenderOptions), C.POINTER(C.c_double), C.c_int64,
                            C.POINTER(RenderResult)]),
    ("rt_scene_create", C.c_int, [C.POINTER(SceneDesc), C.POINTER(C.c_void_p)]),
    ("rt_scene_destroy", C.c_int, [C.c_void_p]),
    ("rt_scene_stats_get", C.c_int, [C.c_void_p, C.POINTER(SceneStats)]),
    ("rt_session_create", C.c_int, [C.c_void_p, C.POINTER(SessionOptions), C.POINTER(C.c_void_p)]),
    ("rt_session_destroy", C.c_int, [C.c_void_p]),
    ("rt_session_set_camera", C.c_int, [C.c_void_p, C.POINTER(CameraDesc)]),
    ("rt_session_state", C.c_int, [C.c_void_p, C.POINTER(Accumulation)]),
    ("rt_session_render_to", C.c_int, [C.c_void_p, C.c_int64, C.POINTER(RenderReport)]),
    ("rt_session_render_for", C.c_int, [C.c_void_p, C.c_double, C.c_int64, C.POINTER(RenderReport)]),
    ("rt_session_pixels", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_int64]),
    ("rt_session_counters", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                      C.POINTER(C.c_double)]),
    ("rt_session_kernel", C.c_int, [C.c_void_p, C.POINTER(KernelInfo)]),
    ("rt_session_device_sums", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int64)]),
    ("rt_render_passes_no_alloc", C.c_int, [C.c_void_p, C.POINTER(CameraDesc), C.c_uint64, C.c_int64, C.c_int64,
                                            C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("rt_session_display", C.c_int, [C.c_void_p, C.POINTER(DisplayOptions), C.POINTER(C.c_uint8), C.c_int64]),
    ("rt_display_device", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int64, C.POINTER(DisplayOptions),
                                    C.c_void_p, C.c_void_p]),
    ("rt_image_save", C.c_int, [C.c_char_p, C.POINTER(C.c_double), C.c_int32, C.c_int32,
                                C.POINTER(DisplayOptions)]),
    ("rt_image_mean_radiance", C.c_int, [C.POINTER(C.c_double), C.c_int32, C.c_int32, C.POINTER(C.c_double)]),
    ("rt_session_save", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(DisplayOptions)]),
    ("rt_session_mean_radiance", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    ("rt_session_set_timing", C.c_int, [C.c_void_p, C.c_int32]),
    ("rt_session_kernel_times", C.c_int, [C.c_void_p, C.POINTER(KernelTimes)]),
    ("rt_session_autotune", C.c_int, [C.c_void_p, C.c_int64, C.POINTER(Tuning)]),
    ("rt_session_tuning", C.c_int, [C.c_void_p, C.POINTER(Tuning)]),
    ("rt_session_set_tuning", C.c_int, [C.c_void_p, C.POINTER(Tuning)]),
    ("rt_autotune_simulate", C.c_int, [C.c_int32, C.c_int32, TUNE_MEASURE, C.c_void_p, C.POINTER(Tuning)]),
    ("rt_session_set_counting", C.c_int, [C.c_void_p, C.c_int32]),
    ("rt_session_fetch_counts", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64 * 4)]),
    ("rt_scene_closest_hits", C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int64,
                                        C.POINTER(C.c_int32), C.POINTER(C.c_float)]),
    ("rt_scene_camera_rays", C.c_int, [C.c_void_p, C.c_uint64, C.c_int64, C.POINTER(C.c_float),
                                       C.POINTER(C.c_float), C.c_int64]),
    ("rt_builtin_scene", C.c_int, [C.c_char_p, C.POINTER(BuiltinParams), C.POINTER(C.c_void_p)]),
    ("rt_owned_scene_desc", C.POINTER(SceneDesc), [C.c_void_p]),
    ("rt_owned_scene_destroy", C.c_int, [C.c_void_p]),
    ("rt_scene_save", C.c_int, [C.POINTER(SceneDesc), C.c_char_p]),
    ("rt_scene_load", C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    ("rt_builtin_camera", C.c_int, [C.c_char_p, C.POINTER(BuiltinParams), C.POINTER(CameraDesc)]),
    ("rt_batch_render", C.c_int, [C.POINTER(BatchJob), C.c_int32, C.POINTER(BatchOptions), C.POINTER(BatchReport)]),
    ("rt_server_create", C.c_int, [C.POINTER(ServerOptions), C.POINTER(C.c_void_p)]),
    ("rt_server_destroy", C.c_int, [C.c_void_p]),
    ("rt_server_submit", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(CameraDesc), C.c_uint64, C.c_int64,
                                   C.POINTER(C.c_int64)]),
    ("rt_server_step", C.c_int, [C.c_void_p, C.POINTER(ServerStepReport)]),
    ("rt_server_poll", C.c_int, [C.c_void_p, C.c_int64, C.POINTER(RequestStatus)]),
    ("rt_server_fetch", C.c_int, [C.c_void_p, C.c_int64, C.POINTER(C.c_double), C.c_int64]),
    ("rt_server_display", C.c_int, [C.c_void_p, C.c_int64, C.POINTER(DisplayOptions), C.POINTER(C.c_uint8),
                                    C.c_int64]),
    ("rt_server_cancel", C.c_int, [C.c_void_p, C.c_int64]),
    ("rt_server_stats_get", C.c_int, [C.c_void_p, C.POINTER(ServerStats)]),
]

_lib = None


def load() -> C.CDLL:
    """Loads the in-tree library; raises if it was not built (there is no fallback path)."""
    global _lib
    if _lib is None:
        path = Path(os.environ.get("RT_B200_LIBRARY", LIBRARY))
        if not path.exists():
            raise RuntimeError(f"{path} is missing: build it with `python -m raytracing_b200.build`")
        lib = C.CDLL(str(path))
        for name, restype, argtypes in ENTRY_POINTS:
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
    return _lib
