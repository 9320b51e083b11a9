"""A compact OP-OSEM case for profiling the device kernels.

Seeded Poisson prompts, flat randoms and a lognormal normalisation at the
HRRT geometry of the chosen span; uploads, computes the sensitivity images,
runs `--subsets` subsets and prints the per-kernel device times.  It holds
the span-3 inputs (about 5 GB in the quad layout, 3 GB with --storage 16) and
nothing else large, so
it suits a profiler capture of a single kernel launch.

    python hrrt_reconstruction_b200/profile_case.py --span 3 --subsets 2
"""
import argparse
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def show(ctx, kernels):
    for k in kernels:
        n, ms = ctx.kernel_stats(k)
        print(f"{k:16s} launches {n:4d}  total {ms:9.3f} ms  avg {ms / max(n, 1):8.3f} ms")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--span", type=int, default=3, choices=[3, 9])
    ap.add_argument("--subsets", type=int, default=2)
    ap.add_argument("--storage", default="f32", choices=["f32", "16"])
    args = ap.parse_args()

    import hrrt_reconstruction_b200 as H
    ctx = H.Context(H.hrrt_geometry(span=args.span))
    rng = np.random.default_rng(7)
    shape = ctx.sino_shape
    prompts = rng.poisson(0.64, size=shape).astype(np.int16)
    randoms = np.full(shape, 0.1, np.float32)
    norm = np.exp(np.float32(0.1) * rng.standard_normal(shape, dtype=np.float32)).astype(np.float32)
    ctx.set_profiling(True)
    ctx.upload_inputs(prompts, randoms, norm, storage=H.STORE_16 if args.storage == "16" else H.STORE_F32)
    show(ctx, ["prep_kernel"])
    ctx.reset_kernel_stats()
    ctx.sensitivity()
    ctx.init_image()
    ctx.reset_kernel_stats()
    ctx.osem_subsets(0, args.subsets)
    ctx.set_profiling(False)
    show(ctx, ["fp_kernel", "bp_kernel", "rotback_kernel"])
    ctx.close()


if __name__ == "__main__":
    main()
