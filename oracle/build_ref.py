"""Builds the reference's own CUDA renderer into oracle/_ref/libref_gpu.so (test infrastructure, not product).

The reference's `gpu_renderer` library is eight CUDA sources under src/gpu (renderer.cu, display.cu, quality.cu,
tonemap.cu, lamp_table.cu, environment_table.cu, CMakeLists.txt:155-165; guides.cu and denoise.cu, added to it by
cmake/optix.cmake:203 with or without OptiX), plain nvcc translation units with no generated code and no external
library. They are compiled here where they lie, unmodified, for sm_100a, with the
flags its build gives them (-fmad=false for display.cu and tonemap.cu), and linked with oracle/ref_gpu_shim.cpp (C
entry points that convert this library's scene tables into the reference's and call its render and display
transforms) and oracle/ref_closest_hit.cu (the reference's device closest_hit on given rays). The output goes only to
oracle/_ref/ (git-ignored; it travels with the checkout to a GPU machine).

Usage: python oracle/build_ref.py [reference root]. The root is the argument, else the environment variable
RT_REFERENCE_ROOT, else a folder named `reference` beside this repository's checkout.
"""
from __future__ import annotations

import concurrent.futures as futures
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
OUT = HERE / "_ref"
LIBRARY = OUT / "libref_gpu.so"
SOURCES = ["renderer.cu", "display.cu", "quality.cu", "tonemap.cu", "lamp_table.cu", "environment_table.cu", "guides.cu",
           "denoise.cu"]
NO_FMAD = {"display.cu", "tonemap.cu"}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{' '.join(cmd)} failed:\n{r.stdout}\n{r.stderr}")


SHIMS = ["ref_gpu_shim.cpp", "ref_closest_hit.cu"]


def reference_root(reference: Path | str | None = None) -> Path:
    """Where the reference's checkout is: the argument, else $RT_REFERENCE_ROOT, else `reference` beside the repo."""
    if reference:
        return Path(reference)
    if os.environ.get("RT_REFERENCE_ROOT"):
        return Path(os.environ["RT_REFERENCE_ROOT"])
    return REPO.parent / "reference"


def build(reference: Path | None = None) -> Path | None:
    """Returns the library's path, or None when the reference's sources are absent (e.g. on a GPU machine, which
    uses the library built beside the checkout)."""
    gpu = reference_root(reference) / "src" / "gpu"
    if not (gpu / "renderer.cu").exists():
        return LIBRARY if LIBRARY.exists() else None
    OUT.mkdir(exist_ok=True)
    inputs = ([gpu / s for s in SOURCES] + [HERE / s for s in SHIMS] +
              [HERE / "ref_scene_convert.h", gpu / "renderer.h", Path(__file__)])
    if LIBRARY.exists() and LIBRARY.stat().st_mtime > max(p.stat().st_mtime for p in inputs):
        return LIBRARY

    def compile_one(source: Path) -> Path:
        obj = OUT / (source.name + ".o")
        flags = ["nvcc", "-std=c++20", "-O3", *ARCH, "-Xcompiler", "-fPIC", "-I", str(gpu), "-I",
                 str(REPO / "include"), "-I", str(HERE)]
        if source.name in NO_FMAD:
            flags.append("-fmad=false")
        _run(flags + ["-c", str(source), "-o", str(obj)])
        return obj

    with futures.ThreadPoolExecutor(max_workers=9) as pool:
        objects = list(pool.map(compile_one, [gpu / s for s in SOURCES] + [HERE / s for s in SHIMS]))
    _run(["nvcc", "-shared", *ARCH, "-cudart", "static", "-o", str(LIBRARY), *map(str, objects)])
    for obj in objects:
        obj.unlink()
    return LIBRARY


SHIM = OUT / "librenderer_b200.so"


def build_shim(reference: Path | None = None) -> Path | None:
    """The reference's gpu:: API served by this library: the shim INTEGRATION.md documents (its first C++ block,
    extracted as written) compiled against the reference's renderer.h, with oracle/shim_driver.cpp, linked to the
    product library. Returns its path, or None without the reference's sources or the product library."""
    import re

    gpu = reference_root(reference) / "src" / "gpu"
    product = REPO / "raytracing_b200" / "_lib" / "librt_b200.so"
    doc = REPO / "INTEGRATION.md"
    if not (gpu / "renderer.h").exists() or not product.exists():
        return SHIM if SHIM.exists() else None
    OUT.mkdir(exist_ok=True)
    inputs = [doc, HERE / "shim_driver.cpp", HERE / "ref_scene_convert.h", gpu / "renderer.h", product, Path(__file__)]
    if SHIM.exists() and SHIM.stat().st_mtime > max(p.stat().st_mtime for p in inputs):
        return SHIM
    blocks = re.findall(r"```cpp\n(.*?)```", doc.read_text(), re.S)
    if not blocks:
        raise RuntimeError("INTEGRATION.md has no C++ block: the shim is missing")
    source = OUT / "renderer_b200.cpp"
    source.write_text(blocks[0])
    _run(["g++", "-std=c++20", "-O2", "-fPIC", "-shared", "-Wall", "-Wextra", "-Werror", "-I", str(gpu), "-I",
          str(REPO / "include"), "-I", str(HERE), str(source), str(HERE / "shim_driver.cpp"), "-o", str(SHIM),
          "-L", str(product.parent), "-lrt_b200", "-Wl,--no-undefined",
          "-Wl,-rpath,$ORIGIN/../../raytracing_b200/_lib"])
    return SHIM


if __name__ == "__main__":
    path = build(Path(sys.argv[1]) if len(sys.argv) > 1 else None)
    print(path if path else "reference sources absent: nothing built")
    shim = build_shim(Path(sys.argv[1]) if len(sys.argv) > 1 else None)
    print(shim if shim else "no shim built (the reference's header or the product library is absent)")
