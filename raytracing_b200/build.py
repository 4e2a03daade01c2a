"""Builds the C-ABI library raytracing_b200/_lib/librt_b200.so for sm_100a, in-tree.

Every source under raytracing_b200/csrc is compiled by nvcc (the .cu for the device with
-gencode arch=compute_100a,code=sm_100a, the .cpp as host code) in parallel, and linked with the CUDA runtime
linked statically, so that the library needs nothing but the driver at run time. Run as
`python -m raytracing_b200.build` or through __graft_entry__.build().
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
REPO = PACKAGE.parent
CSRC = PACKAGE / "csrc"
OUT = PACKAGE / "_lib"
BUILD = PACKAGE / "_build"
LIBRARY = OUT / "librt_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Compiled with -fmad=false: the display transform's bytes follow the order its products and sums are written in,
# as the reference compiles its display units (its CMakeLists.txt:159-165)
NO_FMAD = {"display.cu"}


def nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return found


def _common_flags() -> list[str]:
    return ["-std=c++20", "-O3", "-Xcompiler", "-fPIC", "-I", str(REPO / "include"), "-I", str(CSRC), "-I",
            str(BUILD)]


def _compile(source: Path) -> Path:
    obj = BUILD / (source.name + ".o")
    deps = [source] + sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [REPO / "include" / "rt_b200.h",
                                                                               BUILD / "ggx_energy_table.h"]
    if obj.exists() and obj.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return obj
    cmd = [nvcc()] + _common_flags()
    if source.suffix == ".cu":
        cmd += ARCH + ["-lineinfo", "-Xptxas", "-warn-spills"]
        if source.name in NO_FMAD:
            cmd.append("-fmad=false")
    else:
        cmd += ["-x", "c++"]
    cmd += ["-c", str(source), "-o", str(obj)]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"compiling {source.name} failed:\n{result.stdout}\n{result.stderr}")
    return obj


def _generate_tables() -> None:
    """Runs the build-time generators (csrc/gen): the GGX energy table, compiled into the library as constant data."""
    source = CSRC / "gen" / "ggx_energy_gen.cpp"
    header = BUILD / "ggx_energy_table.h"
    if header.exists() and header.stat().st_mtime >= source.stat().st_mtime:
        return
    exe = BUILD / "ggx_energy_gen"
    compiler = shutil.which("g++") or "c++"
    result = subprocess.run([compiler, "-O2", "-std=c++20", "-pthread", str(source), "-o", str(exe)],
                            capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"compiling {source.name} failed:\n{result.stderr}")
    subprocess.run([str(exe), str(header)], check=True)


def build(verbose: bool = False) -> Path:
    """Compiles and links the library if any source is newer than it; returns its path."""
    BUILD.mkdir(exist_ok=True)
    OUT.mkdir(exist_ok=True)
    _generate_tables()
    sources = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        objects = list(pool.map(_compile, sources))
    if LIBRARY.exists() and LIBRARY.stat().st_mtime >= max(o.stat().st_mtime for o in objects):
        return LIBRARY
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", str(LIBRARY)] + [str(o) for o in objects]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"linking {LIBRARY.name} failed:\n{result.stdout}\n{result.stderr}")
    if verbose:
        print(f"built {LIBRARY}")
    return LIBRARY


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
