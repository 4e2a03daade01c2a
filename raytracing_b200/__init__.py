"""raytracing_b200: a B200-native path-tracing integrator behind the reference's scene API.

The product is the C-ABI library `_lib/librt_b200.so` (include/rt_b200.h): a scene description in, linear pixels
out, rendered by hand-written sm_100a kernels. This module is the thin Python face of that library, shaped like the
reference's C++ interface (src/gpu/renderer.h): `render(scene, options)` and `Session` for a render that goes on,
with the reference's exception classes mapped onto Python's (runtime_error -> RenderError, invalid_argument ->
ValueError, logic_error -> LogicError). There is no CPU path: if the library is missing, importing works but every
call raises.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _abi
from ._abi import (RT_COMBINE_BSDF_ONLY, RT_COMBINE_LIGHTS_ONLY, RT_COMBINE_POWER_HEURISTIC, RT_SAMPLING_LIGHTS,
                   RT_SAMPLING_MATERIAL, RT_SAMPLING_MIXTURE, RT_SAMPLING_UNIFORM)

__all__ = ["RenderError", "LogicError", "NoDeviceError", "UnsupportedError", "CapacityError", "OwnedScene",
           "builtin_scene", "builtin_camera", "load_scene", "query_device", "render", "Scene", "Session",
           "RenderResult", "batch_render", "BatchResult", "Server", "SAMPLING", "COMBINATION", "library_path"]

SAMPLING = {"uniform": RT_SAMPLING_UNIFORM, "material": RT_SAMPLING_MATERIAL, "lights": RT_SAMPLING_LIGHTS,
            "mixture": RT_SAMPLING_MIXTURE}
FORMS = {"auto": _abi.RT_FORM_AUTO, "persistent": _abi.RT_FORM_PERSISTENT, "wavefront": _abi.RT_FORM_WAVEFRONT}
COMBINATION = {"material": RT_COMBINE_BSDF_ONLY, "nee": RT_COMBINE_LIGHTS_ONLY, "mis": RT_COMBINE_POWER_HEURISTIC}


class RenderError(RuntimeError):
    """std::runtime_error in the reference: a CUDA failure or an inconsistent scene."""


class LogicError(RuntimeError):
    """std::logic_error in the reference: a call in the wrong state."""


class NoDeviceError(RenderError):
    """No CUDA device (query_device's runtime_error)."""


class UnsupportedError(RenderError):
    """A scene feature this build does not render."""


class CapacityError(RenderError):
    """A request beyond a stated limit."""


def library_path() -> str:
    return str(_abi.LIBRARY)


def _lib():
    return _abi.load()


def _check(status: int) -> None:
    if status == _abi.RT_OK:
        return
    message = _lib().rt_last_error_message().decode("utf-8", "replace")
    if status == _abi.RT_ERR_INVALID:
        raise ValueError(message)
    if status == _abi.RT_ERR_LOGIC:
        raise LogicError(message)
    if status == _abi.RT_ERR_NO_DEVICE:
        raise NoDeviceError(message)
    if status == _abi.RT_ERR_UNSUPPORTED:
        raise UnsupportedError(message)
    if status == _abi.RT_ERR_CAPACITY:
        raise CapacityError(message)
    raise RenderError(message)


class OwnedScene:
    """A scene description owned by the library (built in, or loaded from a file)."""

    def __init__(self, handle: C.c_void_p):
        self._handle = handle

    @property
    def desc(self) -> "C._Pointer[_abi.SceneDesc]":
        return _lib().rt_owned_scene_desc(self._handle)

    @property
    def camera(self) -> _abi.CameraDesc:
        return self.desc.contents.camera

    @property
    def width(self) -> int:
        return int(self.camera.image_width)

    @property
    def height(self) -> int:
        return int(self.camera.image_height)

    @property
    def round_passes(self) -> int:
        return int(self.camera.sqrt_spp) ** 2

    def save(self, path: str) -> None:
        _check(_lib().rt_scene_save(self.desc, str(path).encode()))

    def count_lamps(self) -> int:
        n = C.c_int32()
        _check(_lib().rt_count_lamps(self.desc, C.byref(n)))
        return int(n.value)

    def close(self) -> None:
        if self._handle:
            _lib().rt_owned_scene_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _builtin_params(width: int = 0, height: int = 0, spp: int = 0, depth: int = 0,
                    sampling: Optional[str] = None, combination: Optional[str] = None, scene_seed: int = 0,
                    sphere_count: int = 0, mesh_level: int = 0, env_width: int = 0,
                    orbit: Optional[tuple[float, float]] = None) -> _abi.BuiltinParams:
    p = _abi.BuiltinParams()
    p.image_width = width
    p.image_height = height
    p.samples_per_pixel = spp
    p.max_depth = depth
    p.sampling = SAMPLING[sampling] if sampling else -1
    p.combination = COMBINATION[combination] if combination else -1
    p.scene_seed = scene_seed
    p.sphere_count = sphere_count
    p.mesh_level = mesh_level
    p.env_width = env_width
    if orbit is not None:
        p.orbit = 1
        p.orbit_azimuth, p.orbit_elevation = orbit
    return p


def builtin_scene(name: str, **overrides) -> OwnedScene:
    """A scene the library builds by name (the reference's "materials", "weekend", "bouncing", "checker", "earth",
    "perlin", "quads", "light", "cornell", "smoke", "final", "aluminum", "glass"; "cornell-mis", "furnace",
    "feature-furnace", "env-furnace", "ggx-furnace", "mesh-ggx", "cover-N"): the reference's scene code, flattened as its GPU
    translator flattens it. Overrides: width, height, spp, depth, sampling, combination, scene_seed, sphere_count,
    mesh_level, env_width, orbit=(azimuth, elevation) in degrees."""
    p = _builtin_params(**overrides)
    handle = C.c_void_p()
    _check(_lib().rt_builtin_scene(name.encode(), C.byref(p), C.byref(handle)))
    return OwnedScene(handle)


def builtin_camera(name: str, **overrides) -> _abi.CameraDesc:
    """The camera builtin_scene(name, **overrides) would have, without building the scene's geometry."""
    p = _builtin_params(**overrides)
    cam = _abi.CameraDesc()
    _check(_lib().rt_builtin_camera(name.encode(), C.byref(p), C.byref(cam)))
    return cam


def load_scene(path: str) -> OwnedScene:
    handle = C.c_void_p()
    _check(_lib().rt_scene_load(str(path).encode(), C.byref(handle)))
    return OwnedScene(handle)


def set_device(device: int) -> None:
    """The CUDA device this thread's later calls use (one process per GPU passes its local rank)."""
    _check(_lib().rt_set_device(device))


def query_device() -> dict:
    info = _abi.DeviceInfo()
    _check(_lib().rt_query_device(C.byref(info)))
    return {"name": info.name.decode(), "compute_capability": (info.compute_capability_major,
                                                                  info.compute_capability_minor),
            "multiprocessors": info.multiprocessors, "memory_gib": info.memory_gib,
            "runtime_version": info.runtime_version, "driver_version": info.driver_version}


def _kernel_dict(k: _abi.KernelInfo) -> dict:
    return {"name": k.name.decode(), "registers": k.registers, "local_bytes": k.local_bytes,
            "blocks_per_multiprocessor": k.blocks_per_multiprocessor, "threads_per_block": k.threads_per_block,
            "max_threads_per_multiprocessor": k.max_threads_per_multiprocessor,
            "multiprocessors": k.multiprocessors}


@dataclass
class RenderResult:
    """render_result of renderer.h:475-492: pixels are height x width x 3 linear doubles, rows from the top."""
    pixels: np.ndarray
    seconds: float
    kernel_seconds: float
    rays: int
    shadow_rays: int
    passes: int
    launches: int
    kernel: dict


def _desc_of(scene) -> "C._Pointer[_abi.SceneDesc]":
    return scene.desc if isinstance(scene, OwnedScene) else scene


ARITHMETIC = {"float32": _abi.RT_FLOAT32, "float64": _abi.RT_FLOAT64}


def render(scene, seed: int = 0, passes: int = 0, launch_seconds: float = 0.05,
           out: Optional[np.ndarray] = None, arithmetic: str = "float32") -> RenderResult:
    """renderer.h:526 render(): the whole job through the C-ABI, host tables in, host pixels out. arithmetic:
    "float32" (the hot path) or "float64" (the books' integrator in double, renderer.h:402-409)."""
    desc = _desc_of(scene)
    cam = desc.contents.camera
    h, w = int(cam.image_height), int(cam.image_width)
    pixels = out if out is not None else np.empty((h, w, 3), dtype=np.float64)
    if pixels.shape != (h, w, 3) or pixels.dtype != np.float64 or not pixels.flags.c_contiguous:
        raise ValueError("out must be a C-contiguous float64 array of shape (height, width, 3)")
    o = _abi.RenderOptions(seed=seed, passes=passes, arithmetic=ARITHMETIC[arithmetic], launch_seconds=launch_seconds)
    r = _abi.RenderResult()
    _check(_lib().rt_render(desc, C.byref(o), pixels.ctypes.data_as(C.POINTER(C.c_double)), pixels.size,
                            C.byref(r)))
    return RenderResult(pixels, r.seconds, r.kernel_seconds, r.rays, r.shadow_rays, r.passes, r.launches,
                        _kernel_dict(r.kernel))


class Scene:
    """A scene resident on the device: validated, its BVH built and uploaded once."""

    def __init__(self, scene):
        self._owner = scene  # keeps an OwnedScene's tables alive while this lives
        handle = C.c_void_p()
        _check(_lib().rt_scene_create(_desc_of(scene), C.byref(handle)))
        self._handle = handle
        desc = _desc_of(scene).contents
        self.width = int(desc.camera.image_width)
        self.height = int(desc.camera.image_height)

    def stats(self) -> dict:
        s = _abi.SceneStats()
        _check(_lib().rt_scene_stats_get(self._handle, C.byref(s)))
        return {name: getattr(s, name) for name, _ in _abi.SceneStats._fields_}

    def closest_hits(self, origins: np.ndarray, directions: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        o = np.ascontiguousarray(origins, dtype=np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(directions, dtype=np.float32).reshape(-1, 3)
        n = o.shape[0]
        ids = np.empty(n, dtype=np.int32)
        ts = np.empty(n, dtype=np.float32)
        _check(_lib().rt_scene_closest_hits(self._handle, o.ctypes.data_as(C.POINTER(C.c_float)),
                                            d.ctypes.data_as(C.POINTER(C.c_float)), n,
                                            ids.ctypes.data_as(C.POINTER(C.c_int32)),
                                            ts.ctypes.data_as(C.POINTER(C.c_float))))
        return ids, ts

    def camera_rays(self, seed: int, pass_index: int) -> tuple[np.ndarray, np.ndarray]:
        n = self.width * self.height
        o = np.empty((n, 3), dtype=np.float32)
        d = np.empty((n, 3), dtype=np.float32)
        _check(_lib().rt_scene_camera_rays(self._handle, seed, pass_index, o.ctypes.data_as(C.POINTER(C.c_float)),
                                           d.ctypes.data_as(C.POINTER(C.c_float)), n))
        return o, d

    def close(self) -> None:
        if self._handle:
            _lib().rt_scene_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


TONE_MAPS = {"books": _abi.RT_TONE_BOOKS, "none": _abi.RT_TONE_NONE, "agx": _abi.RT_TONE_AGX,
             "neutral": _abi.RT_TONE_NEUTRAL}


def _display_options(tone: str = "books", exposure: float = 0.0) -> _abi.DisplayOptions:
    """renderer.h:294-303 display_options: a tone map (TONE_MAPS) and an exposure in stops."""
    return _abi.DisplayOptions(tone_map=TONE_MAPS[tone], exposure=exposure)


def save_image(path: str, pixels: np.ndarray, tone: str = "books", exposure: float = 0.0) -> None:
    """image::save (image.ixx:170-184): .pfm keeps the linear values, .png the display transform's bytes."""
    px = np.ascontiguousarray(pixels, dtype=np.float64)
    h, w, _ = px.shape
    o = _display_options(tone, exposure)
    _check(_lib().rt_image_save(str(path).encode(), px.ctypes.data_as(C.POINTER(C.c_double)), w, h, C.byref(o)))


def mean_radiance(pixels: np.ndarray) -> float:
    """image::mean_radiance (image.ixx:93-103): the average of (r + g + b) / 3 over the pixels."""
    px = np.ascontiguousarray(pixels, dtype=np.float64)
    h, w, _ = px.shape
    out = C.c_double()
    _check(_lib().rt_image_mean_radiance(px.ctypes.data_as(C.POINTER(C.c_double)), w, h, C.byref(out)))
    return out.value


def display_device(sums_ptr: int, width: int, height: int, passes: int, rgba_ptr: int, tone: str = "books",
                   exposure: float = 0.0, stream: int = 0) -> None:
    """The display transform of device sums into device bytes (rt_display_device), queued on `stream`."""
    o = _display_options(tone, exposure)
    _check(_lib().rt_display_device(C.c_void_p(sums_ptr), width, height, passes, C.byref(o), C.c_void_p(rgba_ptr),
                                    C.c_void_p(stream or None)))


def _tuning_dict(t: _abi.Tuning) -> dict:
    return {name: getattr(t, name) for name, _ in _abi.Tuning._fields_ if name != "pad0"}


def autotune_simulate(measure, max_trace_blocks: int = 8, max_trace_blocks_roomy: int = 6) -> dict:
    """The autotuner's search (the library's own code) on a Python measure(shape dict) -> samples per second."""
    def call(shape, _user):
        return float(measure(_tuning_dict(shape.contents)))

    cb = _abi.TUNE_MEASURE(call)
    t = _abi.Tuning()
    _check(_lib().rt_autotune_simulate(max_trace_blocks, max_trace_blocks_roomy, cb, None, C.byref(t)))
    return _tuning_dict(t)


class Session:
    """renderer.h:591-673 session: one view whose image gains passes on demand; its sums stay on the device."""

    def __init__(self, scene: Scene, seed: int = 0, launch_seconds: float = 0.05, form: str = "auto",
                 arithmetic: str = "float32"):
        """form: "auto", "persistent" or "wavefront" (FORMS): how the launches run; the image is the same.
        arithmetic: "float32" or "float64" (ARITHMETIC; float64 renders the books' scenes in the persistent form)."""
        self._scene = scene
        o = _abi.SessionOptions(seed=seed, arithmetic=ARITHMETIC[arithmetic], form=FORMS[form],
                                launch_seconds=launch_seconds)
        handle = C.c_void_p()
        _check(_lib().rt_session_create(scene._handle, C.byref(o), C.byref(handle)))
        self._handle = handle
        self.width = scene.width
        self.height = scene.height

    def set_camera(self, camera: _abi.CameraDesc) -> None:
        _check(_lib().rt_session_set_camera(self._handle, C.byref(camera)))
        self.width = int(camera.image_width)
        self.height = int(camera.image_height)

    def state(self) -> int:
        a = _abi.Accumulation()
        _check(_lib().rt_session_state(self._handle, C.byref(a)))
        return int(a.passes)

    def render_to(self, passes: int) -> dict:
        r = _abi.RenderReport()
        _check(_lib().rt_session_render_to(self._handle, passes, C.byref(r)))
        return {"passes": r.state.passes, "launches": r.launches, "kernel_launches": r.kernel_launches,
                "gpu_seconds": r.gpu_seconds, "longest_launch_seconds": r.longest_launch_seconds}

    def render_for(self, seconds: float, pass_limit: int) -> dict:
        r = _abi.RenderReport()
        _check(_lib().rt_session_render_for(self._handle, seconds, pass_limit, C.byref(r)))
        return {"passes": r.state.passes, "launches": r.launches, "kernel_launches": r.kernel_launches,
                "gpu_seconds": r.gpu_seconds, "longest_launch_seconds": r.longest_launch_seconds}

    def pixels(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        px = out if out is not None else np.empty((self.height, self.width, 3), dtype=np.float64)
        _check(_lib().rt_session_pixels(self._handle, px.ctypes.data_as(C.POINTER(C.c_double)), px.size))
        return px

    def display(self, tone: str = "books", exposure: float = 0.0) -> np.ndarray:
        """session::display(options) (renderer.h:623-635): height x width x 4 bytes (RGB and 255)."""
        out = np.empty((self.height, self.width, 4), dtype=np.uint8)
        o = _display_options(tone, exposure)
        _check(_lib().rt_session_display(self._handle, C.byref(o), out.ctypes.data_as(C.POINTER(C.c_uint8)),
                                         out.size))
        return out

    def save(self, path: str, tone: str = "books", exposure: float = 0.0) -> None:
        o = _display_options(tone, exposure)
        _check(_lib().rt_session_save(self._handle, str(path).encode(), C.byref(o)))

    def mean_radiance(self) -> float:
        out = C.c_double()
        _check(_lib().rt_session_mean_radiance(self._handle, C.byref(out)))
        return out.value

    def counters(self) -> dict:
        rays = C.c_uint64()
        shadow = C.c_uint64()
        seconds = C.c_double()
        _check(_lib().rt_session_counters(self._handle, C.byref(rays), C.byref(shadow), C.byref(seconds)))
        return {"rays": rays.value, "shadow_rays": shadow.value, "kernel_seconds": seconds.value}

    def kernel(self) -> dict:
        k = _abi.KernelInfo()
        _check(_lib().rt_session_kernel(self._handle, C.byref(k)))
        return _kernel_dict(k)

    def set_tuning(self, shape: dict) -> None:
        """Applies a launch shape (a dict as autotune() and tuning() return)."""
        t = _abi.Tuning(**{k: int(shape[k]) for k in ("slots", "trace_blocks_per_sm", "shade_block",
                                                        "trace_min_blocks")})
        _check(_lib().rt_session_set_tuning(self._handle, C.byref(t)))

    def autotune(self, trial_passes: int = 0) -> dict:
        """The wavefront's autotuner on this view (which must have no passes yet; it starts over afterwards): the
        chosen launch shape and its measured speed against the built-in defaults'."""
        t = _abi.Tuning()
        _check(_lib().rt_session_autotune(self._handle, trial_passes, C.byref(t)))
        return _tuning_dict(t)

    def tuning(self) -> dict:
        t = _abi.Tuning()
        _check(_lib().rt_session_tuning(self._handle, C.byref(t)))
        return _tuning_dict(t)

    def set_timing(self, on: bool) -> None:
        """Per-kernel timing: CUDA events around every kernel of every launch (slows launches a little)."""
        _check(_lib().rt_session_set_timing(self._handle, 1 if on else 0))

    def kernel_times(self) -> dict:
        """{kind: (seconds, launches)} for the persistent render, shade, trace and reduction kernels since the view
        was set (with timing on)."""
        t = _abi.KernelTimes()
        _check(_lib().rt_session_kernel_times(self._handle, C.byref(t)))
        return {name: (t.seconds[k], int(t.launches[k])) for k, name in enumerate(("render", "shade", "trace",
                                                                                      "reduce"))}

    def set_counting(self, on: bool) -> None:
        _check(_lib().rt_session_set_counting(self._handle, 1 if on else 0))

    def fetch_counts(self) -> dict:
        v = (C.c_uint64 * 4)()
        _check(_lib().rt_session_fetch_counts(self._handle, C.byref(v)))
        return {"nodes": v[0], "spheres": v[1], "quads": v[2], "triangles": v[3]}

    def device_sums(self) -> tuple[int, int]:
        ptr = C.c_void_p()
        passes = C.c_int64()
        _check(_lib().rt_session_device_sums(self._handle, C.byref(ptr), C.byref(passes)))
        return int(ptr.value or 0), int(passes.value)

    def close(self) -> None:
        if self._handle:
            _lib().rt_session_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class BatchResult:
    """What one batched render of many jobs returns: each job's image (height x width x 3, rows from the top)."""
    images: list
    seconds: float
    setup_seconds: float
    gpu_seconds: float
    rays: int
    shadow_rays: int
    steps: int
    launches: int
    graph: bool


def batch_render(jobs: list, partial_budget_bytes: int = 0, use_graph: bool = True) -> BatchResult:
    """Renders many jobs together: per step, one launch (persistent kernel) or one run (wavefront) per group of jobs
    over all their work items. jobs: a list of
    (scene, seed, passes) with scene an OwnedScene or a SceneDesc pointer and passes 0 for the camera's sqrt_spp^2."""
    n = len(jobs)
    table = (_abi.BatchJob * max(n, 1))()
    images = []
    for i, (scene, seed, passes) in enumerate(jobs):
        desc = _desc_of(scene)
        cam = desc.contents.camera
        img = np.zeros((int(cam.image_height), int(cam.image_width), 3), dtype=np.float64)
        images.append(img)
        table[i] = _abi.BatchJob(desc, seed, passes, img.ctypes.data_as(C.POINTER(C.c_double)))
    o = _abi.BatchOptions(partial_budget_bytes=partial_budget_bytes, use_graph=1 if use_graph else 0)
    r = _abi.BatchReport()
    _check(_lib().rt_batch_render(table, n, C.byref(o), C.byref(r)))
    return BatchResult(images, r.seconds, r.setup_seconds, r.gpu_seconds, r.rays, r.shadow_rays, r.steps,
                       r.launches, bool(r.graph))


REQUEST_STATES = {0: "queued", 1: "active", 2: "done", 3: "cancelled"}


class Server:
    """A stream of render requests served in batched steps: admission under an HBM budget, a first frame (one pass)
    for every newly admitted request before refinement, each request done at its target passes. `continuous` 1: the
    refinement runs in one pool of path slots kept running across steps, first frames in batched steps of their own;
    2: first frames in the pool too (rt_server_options.continuous)."""

    def __init__(self, hbm_budget_bytes: int = 8 << 30, step_seconds: float = 0.02, use_graph: bool = True,
                 continuous: int = 0, slots: int = 0, group_steps: int = 0, lookahead_seconds: float = 0.0):
        o = _abi.ServerOptions(hbm_budget_bytes=hbm_budget_bytes, step_seconds=step_seconds,
                               use_graph=1 if use_graph else 0, continuous=int(continuous), slots=slots,
                               group_steps=group_steps, lookahead_seconds=lookahead_seconds)
        handle = C.c_void_p()
        _check(_lib().rt_server_create(C.byref(o), C.byref(handle)))
        self._handle = handle
        self._scenes = {}  # request id -> (Scene, camera), kept alive while the request is

    def submit(self, scene: Scene, camera: _abi.CameraDesc, seed: int, target_passes: int) -> int:
        rid = C.c_int64()
        _check(_lib().rt_server_submit(self._handle, scene._handle, C.byref(camera), seed, target_passes,
                                       C.byref(rid)))
        self._scenes[rid.value] = (scene, camera)
        return rid.value

    def step(self) -> dict:
        r = _abi.ServerStepReport()
        _check(_lib().rt_server_step(self._handle, C.byref(r)))
        return {name: getattr(r, name) for name, _ in _abi.ServerStepReport._fields_}

    def poll(self, request_id: int) -> dict:
        s = _abi.RequestStatus()
        _check(_lib().rt_server_poll(self._handle, request_id, C.byref(s)))
        return {"state": REQUEST_STATES[s.state], "passes": s.passes, "target": s.target,
                "first_frame_seconds": s.first_frame_seconds, "done_seconds": s.done_seconds}

    def fetch(self, request_id: int) -> np.ndarray:
        cam = self._scenes[request_id][1]
        px = np.empty((int(cam.image_height), int(cam.image_width), 3), dtype=np.float64)
        _check(_lib().rt_server_fetch(self._handle, request_id, px.ctypes.data_as(C.POINTER(C.c_double)), px.size))
        if self.poll(request_id)["state"] == "done":
            self._scenes.pop(request_id, None)
        return px

    def display(self, request_id: int, tone: str = "books", exposure: float = 0.0) -> np.ndarray:
        """The request's frame so far through the display transform: height x width x 4 bytes."""
        cam = self._scenes[request_id][1]
        out = np.empty((int(cam.image_height), int(cam.image_width), 4), dtype=np.uint8)
        o = _display_options(tone, exposure)
        _check(_lib().rt_server_display(self._handle, request_id, C.byref(o),
                                        out.ctypes.data_as(C.POINTER(C.c_uint8)), out.size))
        return out

    def cancel(self, request_id: int) -> None:
        _check(_lib().rt_server_cancel(self._handle, request_id))
        self._scenes.pop(request_id, None)

    def stats(self) -> dict:
        s = _abi.ServerStats()
        _check(_lib().rt_server_stats_get(self._handle, C.byref(s)))
        return {name: getattr(s, name) for name, _ in _abi.ServerStats._fields_}

    def close(self) -> None:
        if self._handle:
            _lib().rt_server_destroy(self._handle)
            self._handle = None
        self._scenes.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
