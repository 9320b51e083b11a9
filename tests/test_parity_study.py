"""Whole-study parity at full size, per iteration: hrrt_reconstruct (the one
call a user makes, from host buffers) against the reference's own projector
compiled from its unmodified sources and against the FP64 restatement, on the
two plain-OSEM workloads of the reference's configurations:

  span 9: seed-0 phantom, 1e8 counts, randoms 20 %, norm 1, water
          attenuation, 16 subsets x 1 iteration;
  span 3: seed-1 phantom, 3e8 counts, lognormal norm sigma 0.1, scatter 15 %
          of trues, randoms 25 %, 16 subsets x 2 iterations.

The host runs follow CalculateNormfac (hrrt_osem3d_span3.cpp:3760-3865) and
CalculateOsem3d (:4098-4341) with the stock -T min(8, nproc) grouping.  The
forward projector is bit-identical to the reference's; the back projector
differs from its incremental sums by rounding only, so the whole study must
stay within REL_L2 per iteration of both host runs.  The 16-bit-stored forms
(additive and sensitivity terms in bf16 or fp16, int16 prompts) are held to
the precision bar against the FP64 run.
"""
import numpy as np
import pytest

from geoms import HRRT3, HRRT9, product_geom

pytestmark = pytest.mark.gpu

REL_L2 = 1e-4        # the FP32 drop-in against the reference / the FP64 oracle, per iteration
REL_L2_16 = 1e-3     # 16-bit-stored terms against the FP64 oracle, per iteration

STUDIES = {
    "span9": (HRRT9, dict(seed=0, total_counts=1e8, randoms_frac=0.20), 1),
    "span3": (HRRT3, dict(seed=1, total_counts=3e8, randoms_frac=0.25, scatter_frac=0.15, norm_sigma=0.1), 2),
}


@pytest.fixture(scope="module", params=sorted(STUDIES))
def study(request, ref_lib):
    import hrrt_reconstruction_b200 as H
    from hrrt_reconstruction_b200 import phantom
    from oracle import study_parity as SP
    geom, kw, iters = STUDIES[request.param]
    with H.Context(product_geom(geom)) as ctx:
        st = phantom.study(ctx, **kw)
        raw = [st[k] for k in ("prompts", "randoms", "norm", "atten", "scatter")]
        dev = {}
        for name, storage in (("f32", H.STORE_F32), ("bf16", H.STORE_16), ("fp16", H.STORE_F16)):
            dev[name] = [ctx.reconstruct(*raw, storage=storage, iterations=k + 1)[0] for k in range(iters)]
    del st
    pre = SP.prep(geom, *raw)
    host = {"reference": SP.reconstruct("reference", geom, pre, iters),
            "fp64": SP.reconstruct("fp64", geom, pre, iters)}
    return request.param, dev, host


def test_f32_matches_reference_every_iteration(study):
    from oracle import study_parity as SP
    name, dev, host = study
    errs = SP.compare(dev["f32"], {"reference": host["reference"]})["reference"]
    assert all(e <= REL_L2 for e in errs), (name, errs)


def test_f32_matches_fp64_oracle_every_iteration(study):
    from oracle import study_parity as SP
    name, dev, host = study
    errs = SP.compare(dev["f32"], {"fp64": host["fp64"]})["fp64"]
    assert all(e <= REL_L2 for e in errs), (name, errs)
    # the reference itself sits as close to the FP64 run
    ref = [SP.rel_l2(r["image"], f["image"]) for r, f in zip(host["reference"], host["fp64"])]
    assert all(e <= REL_L2 for e in ref), (name, ref)


@pytest.mark.parametrize("storage", ["bf16", "fp16"])
def test_16bit_terms_within_precision_bar(study, storage):
    from oracle import study_parity as SP
    name, dev, host = study
    errs = SP.compare(dev[storage], {"fp64": host["fp64"]})["fp64"]
    assert all(e <= REL_L2_16 for e in errs), (name, storage, errs)
