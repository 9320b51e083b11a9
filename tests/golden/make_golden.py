"""Generate the golden fixtures from the reference's own projector.

Runs oracle/_ref/libhrrt_ref.so -- the reference's unmodified projector
sources compiled by oracle/Makefile (target "ref"), which needs the reference
source tree -- on the deterministic inputs of tests/golden/inputs.py and
writes:

  tests/golden/golden.json  sha256 digests of bit-exact outputs (geometry
                            tables, forward projections, rotations) and
                            scalars
  tests/golden/golden.npz   size-independent summaries (inputs.reduce) of the
                            floating-point outputs compared with a tolerance
                            (back projection, sensitivity, OSEM subsets)

The preparation step (normalisation mask, 1/(N*A), additive term) lives in
the reference's driver, which does not build from its own few files; the
fixtures use the oracle's restatement of it (oracle/hrrt_oracle.c, orc_prep)
for the OSEM inputs, and record the digests of what it produced so a change
there is caught too.

Usage: python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import inputs as I  # noqa: E402
from geoms import ALL  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402
from oracle.ref import RefProjector  # noqa: E402

# projection views per geometry (a few, spread over the half-circle)
FP_VIEWS = {"small3": [0, 5, 25, 47], "small9": [0, 7, 24, 47], "hrrt9": [0, 37, 143], "hrrt3": [0, 101]}
BP_VIEWS = {"small3": [3, 30], "small9": [0, 41]}
OSEM_GEOMS = ["small3", "small9"]


def tables(R):
    st, ct, sp, cp = R.trig()
    t, r = R.tantheta()
    zi, zf = R.flookup()
    zs, ze, yr, f = R.blookup()
    return {
        "cylwiny": I.digest(R.cylwiny().astype(np.int32)), "sin_theta": I.digest(st), "cos_theta": I.digest(ct),
        "sin_psi": I.digest(sp), "cos_psi": I.digest(cp), "tantheta": I.digest(t), "rescale": I.digest(r),
        "fl_zzi": I.digest(zi), "fl_zzz0": I.digest(zf), "bl_zsa": I.digest(zs), "bl_zea": I.digest(ze),
        "bl_yra": I.digest(yr), "bl_yr2a": I.digest(f), "order": [int(v) for v in R.order()],
        "segmentsize": R.P, "zp": R.zp, "nz": R.nz,
    }


def main():
    js, arrays = {}, {}
    for name in ["small3", "small9", "hrrt9", "hrrt3"]:
        d = ALL[name]
        R = RefProjector(**d)
        e = {"tables": tables(R)}
        cyl = R.cylwiny()
        img = I.image(R.nx, R.zp, R.nz, cyl)
        e["fp"] = {str(v): I.digest(R.fp_pair(img, v)) for v in FP_VIEWS[name]}
        if name in BP_VIEWS:
            rows = I.rows(R.P, R.nx)
            e["rotate"] = {}
            for v in BP_VIEWS[name]:
                ib = R.bp_pair(rows, v)
                for k, a in I.reduce(ib).items():
                    arrays[f"{name}/bp/{v}/{k}"] = a
                e["rotate"][str(v)] = I.digest(R.rotate_add(ib, v, np.zeros(R.image_shape, np.float32)))
        if name in OSEM_GEOMS:
            O = Oracle(precision="f32", **d)
            prompts, randoms, norm, atten, scatter = I.sinograms(R.P, R.views, R.nx)
            p, a, m = O.prep(prompts, randoms, norm, atten, scatter)
            mask = O.norm_zero_mask()
            e["prep"] = {"prompts": I.digest(p), "add": I.digest(a), "mult": I.digest(m), "mask": I.digest(mask),
                         "masked_quads": int((mask[:, 1:] == 0).sum())}
            R.set_norm_zero_mask(mask)
            nf = R.sensitivity(m)
            order = [int(v) for v in R.order()]
            for s in order[:2]:
                for k, v in I.reduce(nf[s]).items():
                    arrays[f"{name}/sens/{s}/{k}"] = v
            image = R.init_image()
            for s in order[:2]:
                R.osem_subset(image, nf[s], p, a, s)
            for k, v in I.reduce(image).items():
                arrays[f"{name}/osem2/{k}"] = v
            e["osem2_post_sum"] = R.post_iteration(image.copy())
        js[name] = e
        print(name, "done")
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(js, f, indent=1, sort_keys=True)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **arrays)


if __name__ == "__main__":
    main()
