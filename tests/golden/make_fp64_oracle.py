"""Makes the FP64 high-spp oracle renders that each workload's error is measured against (test infrastructure).

* glass (the Cornell box with a glass ball) 600 x 600 and the first book's cover scene 400 x 225: the reference's own
  CUDA renderer in double (gpu::render with precision::float64, src/gpu/renderer.h:405-409; its all-books kernel
  renderer.cu:445-451, built from the reference's sources into oracle/_ref), 65,536 passes (256 x 256 strata), mixture
  of light and cosine sampling, depth 50. NEE+MIS renders of the glass box share this expectation: every strategy is
  an unbiased estimator of the same image.
* mesh-ggx (the level-8 icosphere, GGX metal, glossy plane, sun-lit environment) at 240 x 135: the CPU oracle in
  double (the reference renders triangles only through OptiX), NEE with MIS, depth 16, --mesh-spp passes.

Each image is stored as float32 (height x width x 3, rows from the top) in tests/golden/fp64_<name>.npz with its
passes, seed and renderer. Needs a CUDA GPU for the reference's renders. Usage:
    python tests/golden/make_fp64_oracle.py [--out DIR] [--only glass,weekend,mesh-ggx] [--passes N] [--mesh-spp N]
"""
from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO))

CASES = {
    "glass": dict(width=600, spp=1024, depth=50),
    "weekend": dict(width=400, spp=16, depth=50),
    "mesh-ggx": dict(width=240, spp=16),
}


def main() -> int:
    p = argparse.ArgumentParser()
    p.add_argument("--out", default=str(Path(__file__).resolve().parent))
    p.add_argument("--only", default="glass,weekend,mesh-ggx")
    p.add_argument("--passes", type=int, default=65536)
    p.add_argument("--mesh-spp", type=int, default=2048)
    args = p.parse_args()
    import raytracing_b200 as rt
    from oracle import binding as oracle
    from oracle import ref_gpu

    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    for name in args.only.split(","):
        s = rt.builtin_scene(name, **CASES[name])
        seed = 424242
        t0 = time.perf_counter()
        if name == "mesh-ggx":
            img, info = oracle.render(s.desc, s.width, s.height, seed=seed, passes=args.mesh_spp)
            passes, renderer = args.mesh_spp, "CPU oracle (double), oracle/cpu_renderer.h + ggx_env_cpu.h"
            rays = info["rays"]
        else:
            img, info = ref_gpu.render(s.desc, s.width, s.height, seed=seed, passes=args.passes, fp64=True)
            passes, renderer = args.passes, f"reference gpu::render float64 ({info['kernel']})"
            rays = info["rays"]
        seconds = time.perf_counter() - t0
        path = out / f"fp64_{name}.npz"
        np.savez_compressed(path, image=img.astype(np.float32), passes=passes, seed=seed, renderer=renderer,
                            width=s.width, height=s.height)
        print(f"{name}: {s.width}x{s.height}, {passes} passes, {rays} segments in {seconds:.1f} s by {renderer}; "
              f"mean {img.mean():.6f} -> {path}", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
