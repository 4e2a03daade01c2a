"""The C-ABI boundary without a GPU: the library loads, exports every entry point include/rt_b200.h declares, its
structs have the layout the header gives them, scenes build and serialize deterministically, inconsistent scenes are
refused with the reference's error classes, and a valid scene on a machine without a GPU fails loudly instead of
falling back to a CPU path."""
import ctypes as C
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from raytracing_b200 import _abi

REPO = Path(__file__).resolve().parent.parent
HEADER = REPO / "include" / "rt_b200.h"


def declared_entry_points():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rt_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    names = declared_entry_points()
    assert len(names) >= 25
    for name in names:
        assert hasattr(lib, name), name
    mirrored = {n for n, _, _ in _abi.ENTRY_POINTS}
    assert set(names) == mirrored


def test_abi_version():
    assert _abi.load().rt_abi_version() == 1


STRUCTS = {
    "rt_vec3": _abi.Vec3, "rt_texture_desc": _abi.TextureDesc, "rt_image_desc": _abi.ImageDesc,
    "rt_perlin_desc": _abi.PerlinDesc, "rt_material_desc": _abi.MaterialDesc, "rt_sphere_desc": _abi.SphereDesc,
    "rt_quad_desc": _abi.QuadDesc, "rt_medium_desc": _abi.MediumDesc, "rt_light_desc": _abi.LightDesc,
    "rt_camera_desc": _abi.CameraDesc, "rt_microfacet_desc": _abi.MicrofacetDesc,
    "rt_environment_desc": _abi.EnvironmentDesc, "rt_mesh_desc": _abi.MeshDesc, "rt_scene_desc": _abi.SceneDesc,
    "rt_render_options": _abi.RenderOptions, "rt_kernel_info": _abi.KernelInfo,
    "rt_render_result": _abi.RenderResult, "rt_device_info": _abi.DeviceInfo,
    "rt_session_options": _abi.SessionOptions, "rt_accumulation": _abi.Accumulation,
    "rt_render_report": _abi.RenderReport, "rt_scene_stats": _abi.SceneStats,
    "rt_builtin_params": _abi.BuiltinParams, "rt_batch_job": _abi.BatchJob, "rt_batch_options": _abi.BatchOptions,
    "rt_batch_report": _abi.BatchReport, "rt_server_options": _abi.ServerOptions,
    "rt_request_status": _abi.RequestStatus, "rt_server_step_report": _abi.ServerStepReport,
    "rt_server_stats": _abi.ServerStats, "rt_display_options": _abi.DisplayOptions,
    "rt_kernel_times": _abi.KernelTimes, "rt_tuning": _abi.Tuning,
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc to read the C layout")
def test_struct_layout_matches_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "rt_b200.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'printf("{cname}.{field} %zu\\n", offsetof({cname}, {field}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(REPO / "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                                check=True).stdout.splitlines())
    for cname, py in STRUCTS.items():
        assert int(out[cname]) == C.sizeof(py), cname
        for field, _ in py._fields_:
            assert int(out[f"{cname}.{field}"]) == getattr(py, field).offset, f"{cname}.{field}"


def test_builtin_scenes_build_and_are_deterministic(rt):
    a = rt.builtin_scene("weekend")
    b = rt.builtin_scene("weekend")
    da, db = a.desc.contents, b.desc.contents
    assert da.sphere_count == db.sphere_count
    assert 470 <= da.sphere_count <= 488  # 1 ground + up to 484 small + 3 big (scenes.ixx:79-127)
    for i in range(da.sphere_count):
        assert da.spheres[i].center.x == db.spheres[i].center.x
        assert da.spheres[i].radius == db.spheres[i].radius
    cam = da.camera
    assert (cam.image_width, cam.image_height, cam.sqrt_spp, cam.max_depth) == (1920, 1080, 22, 50)
    assert cam.defocus == 1
    c = rt.builtin_scene("weekend", scene_seed=17)
    assert c.desc.contents.spheres[1].center.x != da.spheres[1].center.x


def test_glass_scene_matches_reference_tables(rt):
    s = rt.builtin_scene("glass", width=600, spp=1024)
    d = s.desc.contents
    assert (d.sphere_count, d.quad_count, d.light_count) == (1, 12, 2)  # 5 walls + lamp + 6 box faces
    assert (d.camera.image_width, d.camera.image_height, d.camera.sqrt_spp) == (600, 600, 32)
    assert d.camera.sampling == rt.SAMPLING["mixture"]
    lamp = d.quads[5]
    assert (lamp.q.x, lamp.q.y, lamp.q.z, lamp.u.x, lamp.v.z) == (343, 554, 332, -130, -105)
    assert d.lights[0].weight == 0.5 and d.lights[1].weight == 0.5
    assert d.lights[1].kind == _abi.RT_LIGHT_SPHERE and d.lights[1].radius == 90
    # the tall block: rotate_y(15) then translate(265, 0, 295) (scenes.ixx:310-315), baked
    corner = d.quads[6].q
    assert corner.x == pytest.approx(265 + 165 * np.sin(np.radians(15)), abs=1e-9)
    assert s.count_lamps() == 1


def test_scene_save_load_round_trip(rt, tmp_path):
    s = rt.builtin_scene("glass", width=32)
    path = tmp_path / "glass.rtscene"
    s.save(str(path))
    t = rt.load_scene(str(path))
    a, b = s.desc.contents, t.desc.contents
    assert bytes(a.camera) == bytes(b.camera)
    assert a.quad_count == b.quad_count and a.light_count == b.light_count
    assert all(bytes(a.quads[i]) == bytes(b.quads[i]) for i in range(a.quad_count))
    bad = tmp_path / "bad.rtscene"
    bad.write_bytes(b"not a scene")
    with pytest.raises(rt.RenderError):
        rt.load_scene(str(bad))


def _scene_with(rt, mutate):
    s = rt.builtin_scene("cornell", width=16)
    mutate(s.desc.contents)
    return s


def test_inconsistent_scenes_are_refused_before_any_gpu_work(rt):
    s = _scene_with(rt, lambda d: setattr(d.quads[0], "material", 999))
    with pytest.raises(rt.RenderError, match="out of range"):
        rt.Scene(s)
    s = _scene_with(rt, lambda d: setattr(d.camera, "sqrt_spp", 0))
    with pytest.raises(rt.RenderError, match="sqrt_spp"):
        rt.Scene(s)
    s = _scene_with(rt, lambda d: setattr(d, "light_count", 0))
    with pytest.raises(rt.RenderError, match="lights list"):
        rt.Scene(s)


def test_second_book_tables_are_validated(rt):
    """Textures, media and their references are checked before anything is built (renderer.cu:688-810)."""
    s = rt.builtin_scene("smoke", width=16)
    d = s.desc.contents
    count = d.medium_count
    d.medium_count = 49  # checked before any entry is read
    with pytest.raises(rt.UnsupportedError, match="volumes of smoke"):
        rt.Scene(s)
    d.medium_count = count
    isotropic = d.media[0].material
    d.media[0].material = d.spheres[0].material if d.sphere_count else 0
    with pytest.raises(rt.RenderError, match="isotropic"):
        rt.Scene(s)
    d.media[0].material = isotropic
    d.media[0].neg_inv_density = 1.0
    with pytest.raises(rt.RenderError, match="density"):
        rt.Scene(s)
    c = rt.builtin_scene("checker", width=16)
    cd = c.desc.contents
    checker = next(i for i in range(cd.texture_count) if cd.textures[i].kind == 1)
    cd.textures[checker].even = checker  # a checker must refer to textures before it
    with pytest.raises(rt.RenderError, match="come before it"):
        rt.Scene(c)
    p = rt.builtin_scene("perlin", width=16)
    p.desc.contents.perlins[0].perm_y[7] = 256
    with pytest.raises(rt.RenderError, match="Perlin"):
        rt.Scene(p)


@pytest.mark.parametrize("name", ["bouncing", "checker", "earth", "perlin", "light", "smoke", "final", "aluminum"])
def test_second_book_scenes_build_and_round_trip(rt, name, tmp_path):
    """The reference's scene list (scenes.ixx:504-518) beyond the first book's: built, saved and loaded unchanged."""
    s = rt.builtin_scene(name, width=32, spp=4)
    d = s.desc.contents
    assert d.camera.image_width == 32
    path = tmp_path / f"{name}.rtscene"
    s.save(str(path))
    t = rt.load_scene(str(path))
    e = t.desc.contents
    for field in ("sphere_count", "quad_count", "texture_count", "image_count", "perlin_count", "medium_count",
                  "light_count", "material_count"):
        assert getattr(d, field) == getattr(e, field), field
    assert bytes(d.camera) == bytes(e.camera)
    if name == "final":
        assert d.sphere_count == 1006 and d.quad_count == 2401 and d.medium_count == 2
        assert d.image_count == 1 and d.perlin_count == 1
    if name == "bouncing":
        assert any(d.spheres[i].displacement.y != 0 for i in range(d.sphere_count))


def test_no_cpu_fallback_without_gpu(rt):
    """A valid scene on a machine without a CUDA device fails loudly: the product has no CPU path."""
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    s = rt.builtin_scene("furnace", width=16)
    with pytest.raises(rt.RenderError):
        rt.render(s, seed=1)
    with pytest.raises(rt.RenderError):
        rt.batch_render([(s, 1, 4)])
    with pytest.raises(rt.RenderError):
        rt.Server()


def test_builtin_camera_matches_the_scene(rt):
    """The camera alone (the geometry built at its cheapest) is the full scene's camera, bit for bit."""
    for name, kw in (("glass", dict(width=96, orbit=(30.0, 10.0))), ("mesh-ggx", dict(width=128, spp=4)),
                     ("cover-30", dict(width=64, scene_seed=4))):
        cam = rt.builtin_camera(name, **kw)
        scene = rt.builtin_scene(name, **kw, **({"mesh_level": 2} if name == "mesh-ggx" else {}))
        assert bytes(cam) == bytes(scene.camera), name


def test_render_options_are_checked(rt):
    s = rt.builtin_scene("furnace", width=16)
    with pytest.raises((ValueError, rt.RenderError)):
        rt.render(s, passes=-1)


def test_integration_shim_compiles_against_the_reference_header(tmp_path):
    """INTEGRATION.md's C++ shim (the reference's gpu:: API on this C-ABI) compiles as written against the
    reference's own src/gpu/renderer.h, warnings as errors (where the reference's sources are present)."""
    from oracle import build_ref

    header = build_ref.reference_root() / "src" / "gpu" / "renderer.h"
    if not header.exists() or shutil.which("g++") is None:
        pytest.skip("the reference's sources (or g++) are not here")
    blocks = re.findall(r"```cpp\n(.*?)```", (REPO / "INTEGRATION.md").read_text(), re.S)
    assert blocks, "INTEGRATION.md has no C++ block"
    source = tmp_path / "renderer_b200.cpp"
    source.write_text(blocks[0])
    r = subprocess.run(["g++", "-std=c++20", "-fsyntax-only", "-Wall", "-Wextra", "-Werror", "-I", str(header.parent),
                        "-I", str(REPO / "include"), str(source)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
