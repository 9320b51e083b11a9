"""The CPU oracle (oracle/hrrt_oracle.c) pinned against the golden fixtures
made from the reference's own projector (tests/golden/make_golden.py), and --
where the reference build is present -- against that build directly.

Bit-exact outputs (geometry tables, forward projection, rotation) are compared
by sha256 of their bytes; floating-point sums whose order differs from the
reference's (back projection, sensitivity, OSEM) by relative L2 of their
summaries, tolerance written in each test."""
import json
import os

import numpy as np
import pytest

from geoms import ALL
from golden import inputs as I

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "golden.json")))
ARR = np.load(os.path.join(HERE, "golden", "golden.npz"))


def oracle(name, precision):
    from oracle.oracle import Oracle
    return Oracle(precision=precision, **ALL[name])


def summary(prefix):
    return {k: ARR[f"{prefix}/{k}"] for k in ("total", "lead", "last", "samples")}


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def assert_summary_close(arr, prefix, rtol):
    got, want = I.reduce(arr), summary(prefix)
    for k in want:
        e = rel(got[k], want[k])
        assert e <= rtol, f"{prefix}/{k}: rel-L2 {e:.3e} > {rtol}"


@pytest.mark.parametrize("name", ["small3", "small9", "hrrt9", "hrrt3"])
def test_tables_match_reference(name):
    O = oracle(name, "f32")
    g = GOLD[name]["tables"]
    st, ct, sp, cp = O.trig()
    t, r = O.tantheta()
    zi, zf = O.flookup()
    zs, ze, yr, f = O.blookup()
    got = {"cylwiny": O.cylwiny(), "sin_theta": st, "cos_theta": ct, "sin_psi": sp, "cos_psi": cp,
           "tantheta": t, "rescale": r, "fl_zzi": zi, "fl_zzz0": zf, "bl_zsa": zs, "bl_zea": ze, "bl_yra": yr,
           "bl_yr2a": f}
    for k, a in got.items():
        assert I.digest(a) == g[k], k
    assert [int(v) for v in O.order()] == g["order"]
    assert (O.P, O.zp, O.nz) == (g["segmentsize"], g["zp"], g["nz"])


@pytest.mark.parametrize("name", ["small3", "small9", "hrrt9", "hrrt3"])
def test_fp_bit_identical_to_reference(name):
    """The f32 build reproduces the reference's forward projection bit for bit."""
    O = oracle(name, "f32")
    img = I.image(O.nx, O.zp, O.nz, O.cylwiny())
    for v, dg in GOLD[name]["fp"].items():
        assert I.digest(O.fp_pair(img, int(v))) == dg, f"view {v}"


@pytest.mark.parametrize("name", ["small3", "small9"])
def test_fp64_close_to_reference(name):
    """The f64 build samples the same positions: within 1e-6 of the float
    reference (rel-L2), and the f32 build exactly."""
    O64, O32 = oracle(name, "f64"), oracle(name, "f32")
    img = I.image(O64.nx, O64.zp, O64.nz, O64.cylwiny())
    for v in GOLD[name]["fp"]:
        a, b = O64.fp_pair(img, int(v)), O32.fp_pair(img, int(v))
        assert rel(a, b) <= 1e-6
        assert np.array_equal(a == 0, b == 0)


@pytest.mark.parametrize("name", ["small3", "small9"])
@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_bp_and_rotate_match_reference(name, precision):
    """Back projection: summaries within 2e-6 rel-L2 of the reference (its
    incremental sums round differently)."""
    O = oracle(name, precision)
    rows = I.rows(O.P, O.nx)
    for v in GOLD[name]["rotate"]:
        assert_summary_close(O.bp_pair(rows, int(v)), f"{name}/bp/{v}", 2e-6)


def test_rotate_bit_identical_when_reference_present(ref_lib):
    """Rotating the reference's back projection: the f32 build reproduces the
    reference's rotate-back bit for bit."""
    from oracle.ref import RefProjector
    for name in ("small3", "small9"):
        d = ALL[name]
        R = RefProjector(**d)
        O = oracle(name, "f32")
        rows = I.rows(O.P, O.nx)
        for v, dg in GOLD[name]["rotate"].items():
            ib = R.bp_pair(rows, int(v))
            co = O.rotate_add(ib, int(v), np.zeros(O.image_shape, np.float32))
            assert I.digest(co) == dg


@pytest.mark.parametrize("name", ["small3", "small9"])
@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_sensitivity_and_osem_match_reference(name, precision):
    """Prep (digests), inverse sensitivity of two subsets and the image after
    two OP-OSEM subsets: summaries within 2e-6 / 2e-6 rel-L2 of the reference;
    post-iteration sum within 1e-7 relative."""
    O = oracle(name, precision)
    g = GOLD[name]
    prompts, randoms, norm, atten, scatter = I.sinograms(O.P, O.views, O.nx)
    p, a, m = O.prep(prompts, randoms, norm, atten, scatter)
    mask = O.norm_zero_mask()
    assert I.digest(p) == g["prep"]["prompts"]
    assert I.digest(a) == g["prep"]["add"]
    assert I.digest(m) == g["prep"]["mult"]
    assert I.digest(mask) == g["prep"]["mask"]
    assert int((mask[:, 1:] == 0).sum()) == g["prep"]["masked_quads"] > 0
    nf = O.sensitivity(m, nthreads=3)
    order = [int(v) for v in O.order()]
    for s in order[:2]:
        assert_summary_close(nf[s], f"{name}/sens/{s}", 2e-6)
    image = O.init_image()
    for s in order[:2]:
        O.osem_subset(image, nf[s], p, a, s, nthreads=3)
    assert_summary_close(image, f"{name}/osem2", 2e-6)
    post = O.post_iteration(image.copy())
    assert abs(post - g["osem2_post_sum"]) <= 1e-7 * abs(g["osem2_post_sum"])


def test_golden_check_catches_planted_mistakes():
    """A mistake planted in the oracle's output is caught by the same checks:
    one flipped low mantissa bit in a forward projection changes the digest,
    and a 1e-3 relative change of one BP plane breaks the summary tolerance."""
    O = oracle("small9", "f32")
    img = I.image(O.nx, O.zp, O.nz, O.cylwiny())
    v = next(iter(GOLD["small9"]["fp"]))
    fp = O.fp_pair(img, int(v))
    i = np.flatnonzero(fp)[len(np.flatnonzero(fp)) // 2]
    fp.reshape(-1).view(np.uint32)[i] ^= 1
    assert I.digest(fp) != GOLD["small9"]["fp"][v]
    vb = next(iter(GOLD["small9"]["rotate"]))
    ib = O.bp_pair(I.rows(O.P, O.nx), int(vb))
    ib[:, :, 10] *= np.float32(1 + 1e-3)
    with pytest.raises(AssertionError):
        assert_summary_close(ib, f"small9/bp/{vb}", 2e-6)
