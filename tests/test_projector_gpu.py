"""CUDA projector entry points (through the C ABI) against the CPU oracle
(oracle/hrrt_oracle.c) and the golden fixtures made from the reference's own
projector.

  forward projection (forward_proj3d_thread1) : bit-identical to the oracle's
      f32 build, and sha256-identical to the reference's golden outputs
  rotate-back        (rotate_image_buf)       : bit-identical
  back projection    (back_proj3d_thread1)    : the reference accumulates its
      voxel-driven interpolation incrementally along y; the device evaluates
      it directly in single precision.  Against the oracle's f64 build:
      rel-L2 <= 2e-6 and max abs error <= 1e-5 of the buffer's max; against
      the golden summaries: rel-L2 <= 2e-6.
"""
import json
import os

import numpy as np
import pytest

from geoms import ALL, fov_mask, product_geom, random_image, random_rows
from golden import inputs as I

pytestmark = pytest.mark.gpu

BP_REL_L2 = 2e-6
BP_MAX_REL = 1e-5
HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "golden.json")))
ARR = np.load(os.path.join(HERE, "golden", "golden.npz"))


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.fixture(scope="module", params=["small3", "small9", "hrrt9", "hrrt3"])
def pair(request):
    import hrrt_reconstruction_b200 as H
    from oracle.oracle import Oracle
    d = ALL[request.param]
    O32 = Oracle(precision="f32", **d)
    O64 = Oracle(precision="f64", **d)
    ctx = H.Context(product_geom(d))
    yield request.param, O32, O64, ctx
    ctx.close()


def test_fp_pair_bit_identical(pair):
    name, O, _, ctx = pair
    cyl = O.cylwiny()
    img = random_image(ctx.image_shape, cyl, seed=3, zvalid=O.nz)
    nv2 = O.views // 2
    for view in sorted({0, 1, nv2 // 3, nv2 // 2, nv2 - 1}):
        sentinel = np.full(ctx.rows_shape, -7.0, np.float32)
        want = O.fp_pair(img, view, prj=sentinel)
        got = ctx.fp_pair(img, view, prj=sentinel)
        diff = np.nonzero(want.view(np.uint32) != got.view(np.uint32))
        assert diff[0].size == 0, (name, view, diff[0][:5], diff[1][:5], want[diff][:5], got[diff][:5])


def test_fp_pair_matches_reference_golden(pair):
    """sha256 of the device's forward projection equals that of the
    reference's own output on the same image (tests/golden)."""
    name, O, _, ctx = pair
    img = I.image(O.nx, O.zp, O.nz, O.cylwiny())
    for v, dg in GOLD[name]["fp"].items():
        assert I.digest(ctx.fp_pair(img, int(v))) == dg, (name, v)


def test_fp_cylinder_centre_chord(pair):
    """Forward projection of the FOV cylinder (the reference's -I 0 -h mode):
    the centre bin of segment 0 is the FOV chord sampled at y_size steps."""
    name, O, _, ctx = pair
    if name != "hrrt9":
        pytest.skip("HRRT value")
    img = O.init_image().astype(np.float32)
    prj = ctx.fp_pair(img, 0)
    assert prj[100, 128] == np.float32(296.15625)


def test_rotate_add_bit_identical(pair):
    name, O, _, ctx = pair
    cyl = O.cylwiny()
    ib = random_image(ctx.image_shape, cyl, seed=5, zvalid=O.nz)
    corr = random_image(ctx.image_shape, cyl, seed=6, zvalid=O.nz)
    for view in (0, O.views // 8, O.views // 2 - 1):
        want = O.rotate_add(ib, view, corr)
        got = ctx.rotate_add(ib, view, corr)
        assert np.array_equal(want.view(np.uint32), got.view(np.uint32)), (name, view)


def test_bp_pair_matches_oracle(pair):
    name, _, O, ctx = pair
    rows = random_rows(ctx.rows_shape, seed=7)
    m = fov_mask(O.nx, O.cylwiny())
    for view in (0, O.views // 6, O.views // 2 - 1):
        want = O.bp_pair(rows, view)
        got = ctx.bp_pair(rows, view)
        assert np.all(got[~m] == 0)
        assert np.all(got[:, :, O.nz:] == 0)
        w, g = want[m][:, :O.nz], got[m][:, :O.nz]
        e = rel_l2(g, w)
        mx = float(np.max(np.abs(g.astype(np.float64) - w)) / np.max(np.abs(w)))
        assert e <= BP_REL_L2 and mx <= BP_MAX_REL, (name, view, e, mx)


def test_bp_and_rotate_match_reference_golden(pair):
    name, O, _, ctx = pair
    if name not in ("small3", "small9"):
        pytest.skip("golden back projections are kept for the small scanners")
    rows = I.rows(O.P, O.nx)
    for v in GOLD[name]["rotate"]:
        got = ctx.bp_pair(rows, int(v))
        red = I.reduce(got)
        for k in red:
            e = rel_l2(red[k], ARR[f"{name}/bp/{v}/{k}"])
            assert e <= BP_REL_L2, (name, v, k, e)


def test_bp_linear(pair):
    """The back projector is linear: BP(a*u + v) = a*BP(u) + BP(v)."""
    name, _, _, ctx = pair
    u = random_rows(ctx.rows_shape, seed=11)
    v = random_rows(ctx.rows_shape, seed=12)
    a = np.float32(0.75)
    lhs = ctx.bp_pair(a * u + v, 3)
    rhs = a * ctx.bp_pair(u, 3) + ctx.bp_pair(v, 3)
    assert rel_l2(lhs, rhs) < 1e-6


def test_masked_quads(pair):
    """Quads switched off by the norm-zero mask: the forward projection leaves
    their bins as they were, the back projection adds nothing from them."""
    name, O, O64, ctx = pair
    if name not in ("small3", "small9"):
        pytest.skip("small scanners")
    mask = np.ones((O.views // 2, O.nx // 2 + 1), np.int16)
    mask[:, 5:9] = 0
    mask[3, :] = 0
    ctx.set_norm_zero_mask(mask)
    O.set_norm_zero_mask(mask)
    O64.set_norm_zero_mask(mask)
    try:
        img = random_image(ctx.image_shape, O.cylwiny(), seed=8, zvalid=O.nz)
        sentinel = np.full(ctx.rows_shape, -3.0, np.float32)
        for view in (3, 4):
            got = ctx.fp_pair(img, view, prj=sentinel)
            want = O.fp_pair(img, view, prj=sentinel)
            # the oracle zeroes a skipped quad's bins (the reference keeps the
            # previous view's there); compare the quads the projector ran
            live = np.ones(ctx.rows_shape, bool)
            for x in np.flatnonzero(mask[view] == 0):
                live[:, [x, (O.nx - x) % O.nx]] = False
            assert np.array_equal(got.view(np.uint32)[live], want.view(np.uint32)[live])
            rows = random_rows(ctx.rows_shape, seed=13)
            e = rel_l2(ctx.bp_pair(rows, view), O64.bp_pair(rows, view))
            assert e <= BP_REL_L2
    finally:
        ones = np.ones_like(mask)
        ctx.set_norm_zero_mask(ones)
        O.set_norm_zero_mask(ones)
        O64.set_norm_zero_mask(ones)
