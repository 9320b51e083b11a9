"""The device exact adjoint (hrrt_bp_pair HRRT_BP_ADJOINT, and the OSEM loop
with hrrt_set_backprojector) against the oracle's orc_fp_adjoint and the
dot-product test through the C ABI.

Tolerances: against the f64 oracle rel-L2 <= 1e-6 (single-precision sums in
another order); <fp(x), y> = <x, bp(y)> to 1e-6 relative; one OSEM subset
with the adjoint back projector within 1e-5 of the oracle composition."""
import numpy as np
import pytest

from geoms import ALL, product_geom, random_image, random_rows

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.fixture(scope="module", params=["small3", "small9", "hrrt9", "hrrt3"])
def pair(request):
    import hrrt_reconstruction_b200 as H
    from oracle.oracle import Oracle
    d = ALL[request.param]
    ctx = H.Context(product_geom(d))
    yield request.param, Oracle(**d), ctx
    ctx.close()


def test_adjoint_matches_oracle(pair):
    import hrrt_reconstruction_b200 as H
    name, O, ctx = pair
    y = random_rows(ctx.rows_shape, seed=21)
    for v in (0, O.views // 5, O.views // 2 - 1):
        got = ctx.bp_pair(y, v, mode=H.BP_ADJOINT)
        want = O.fp_adjoint(y, v)
        assert rel_l2(got, want) <= 1e-6, (name, v)
        assert np.all(got[:, :, O.nz:] == 0)


def test_dot_product_through_the_c_abi(pair):
    import hrrt_reconstruction_b200 as H
    name, O, ctx = pair
    x = random_image(ctx.image_shape, O.cylwiny(), seed=22, zvalid=O.nz)
    y = random_rows(ctx.rows_shape, seed=23)
    for v in (1, O.views // 3):
        lhs = float(np.sum(ctx.fp_pair(x, v).astype(np.float64) * y))
        rhs = float(np.sum(x.astype(np.float64) * ctx.bp_pair(y, v, mode=H.BP_ADJOINT)))
        assert abs(lhs - rhs) <= 1e-6 * abs(lhs), (name, v, lhs, rhs)


def _rows(sino, view):
    P, V, _ = sino.shape
    return np.concatenate([sino[:, view, :], sino[:, view + V // 2, :]], axis=0)


def test_osem_subset_with_adjoint_backprojector():
    """Sensitivity and one subset with HRRT_BP_ADJOINT against the oracle's
    forward projection, OP ratio and exact adjoint composed here."""
    import hrrt_reconstruction_b200 as H
    from oracle.oracle import Oracle
    d = ALL["small3"]
    O = Oracle(**d)
    rng = np.random.default_rng(24)
    shape = O.sino_shape
    prompts = rng.poisson(2.0, size=shape).astype(np.int16)
    randoms = np.full(shape, 0.1, np.float32)
    with H.Context(product_geom(d)) as ctx:
        ctx.set_backprojector(H.BP_ADJOINT)
        ctx.upload_inputs(prompts, randoms)
        ctx.sensitivity()
        ctx.init_image()
        img0 = ctx.get_image_xyz().astype(np.float64)
        ctx.osem_subsets(0, 1)
        got = ctx.get_image_xyz()
        nf_dev = ctx.get_sensitivity(0)
    p, a, m = O.prep(prompts, randoms)
    fov = np.zeros((O.nx, O.nx), bool)
    cyl = O.cylwiny()
    for x in range(O.nx):
        fov[x, cyl[x, 0]:cyl[x, 1]] = True
    views = O.vieworder(0)[: O.sviews // 2]
    sens = sum(O.fp_adjoint(_rows(m, v), v) for v in views)
    nf = np.where((np.abs(sens) > 5e-2) & fov[:, :, None], 1.0 / np.where(sens == 0, 1, sens), 0.0)
    nf[:, :, O.nz:] = 0
    assert rel_l2(nf_dev, nf) <= 1e-5
    corr = np.zeros(O.image_shape)
    for v in views:
        est = O.fp_pair(img0, v)
        pr, ad = _rows(p, v).astype(np.float64), _rows(a, v).astype(np.float64)
        den = est + ad
        ratio = np.where(pr == 0, 0.0, np.where(den > 1e-10, pr / np.where(den > 1e-10, den, 1), 1.0))
        corr += O.fp_adjoint(ratio, v)
    cl = np.minimum(100.0, np.maximum(0.01, corr))
    want = np.where(fov[:, :, None], np.minimum(1e4, img0 * (cl * nf)), img0)
    assert rel_l2(got, want) <= 1e-5
