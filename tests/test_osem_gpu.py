"""The device OP-OSEM path (upload/prep, sensitivity, subsets, post-iteration)
through the C ABI against the CPU oracle's f64 build and the golden fixtures.

Tolerances (rel-L2 over the FOV): inverse sensitivity 2e-6, image after one
or two subsets 1e-5, after a full iteration 5e-5 (single-precision device sums
in a different order from the oracle's double sums; the reference itself is
within 3e-7 of the oracle after two subsets); the norm-zero mask and the
masked prompts are integers and must be identical.
"""
import json
import os

import numpy as np
import pytest

from geoms import ALL, HRRT3, product_geom
from golden import inputs as I

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "golden.json")))
ARR = np.load(os.path.join(HERE, "golden", "golden.npz"))


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def setup(name, storage=0):
    import hrrt_reconstruction_b200 as H
    from oracle.oracle import Oracle
    d = ALL[name]
    O = Oracle(precision="f64", nthreads=os.cpu_count() or 4, **d)
    ctx = H.Context(product_geom(d))
    prompts, randoms, norm, atten, scatter = I.sinograms(O.P, O.views, O.nx)
    ctx.upload_inputs(prompts, randoms, norm, atten, scatter, storage=storage)
    p, a, m = O.prep(prompts, randoms, norm, atten, scatter)
    return ctx, O, (p, a, m)


@pytest.mark.parametrize("name", ["small3", "small9"])
def test_prep_mask_and_sensitivity(name):
    ctx, O, (p, a, m) = setup(name)
    with ctx:
        assert np.array_equal(ctx.norm_zero_mask(), O.norm_zero_mask())
        ctx.sensitivity()
        nf = O.sensitivity(m)
        for s in range(O.subsets):
            e = rel_l2(ctx.get_sensitivity(s), nf[s])
            assert e <= 2e-6, (s, e)
        for s in [int(v) for v in GOLD[name]["tables"]["order"][:2]]:
            red = I.reduce(ctx.get_sensitivity(s))
            for k in red:
                assert rel_l2(red[k], ARR[f"{name}/sens/{s}/{k}"]) <= 2e-6


@pytest.mark.parametrize("name", ["small3", "small9"])
def test_two_subsets_match_oracle_and_reference(name):
    ctx, O, (p, a, m) = setup(name)
    with ctx:
        ctx.sensitivity()
        ctx.init_image()
        img0 = ctx.get_image_xyz()
        want = O.init_image()
        assert np.array_equal(img0, want.astype(np.float32))
        nf = O.sensitivity(m)
        ctx.osem_subsets(0, 2)
        got = ctx.get_image_xyz()
        for s in [int(v) for v in O.order()[:2]]:
            O.osem_subset(want, nf[s], p, a, s)
        assert rel_l2(got, want) <= 1e-5
        red = I.reduce(got)
        for k in red:
            assert rel_l2(red[k], ARR[f"{name}/osem2/{k}"]) <= 1e-5, k


def test_full_iteration_and_post_sum():
    """One full iteration (16 subsets) with the post-iteration threshold and
    FP64 sum, through hrrt_osem."""
    ctx, O, (p, a, m) = setup("small3")
    with ctx:
        ctx.sensitivity()
        ctx.init_image()
        st = ctx.osem(1)
        assert st.subset_iterations == O.subsets
        got = ctx.get_image_xyz()
        want = O.init_image()
        nf = O.sensitivity(m)
        for s in [int(v) for v in O.order()]:
            O.osem_subset(want, nf[s], p, a, s)
        post = O.post_iteration(want)
        assert rel_l2(got, want) <= 5e-5
        assert abs(st.sum_image - post) <= 5e-5 * abs(post)
        # get_image is the [z][y][x] array the reference's SaveImage writes
        zyx = ctx.get_image()
        assert np.array_equal(zyx, np.transpose(got[:, :, :O.nz], (2, 1, 0)))


@pytest.fixture(scope="module")
def hrrt3_inputs():
    """Full-size HRRT span 3 sinograms (seeded): prompts, randoms and a
    normalisation with a dead bin block; the oracle's prep of them."""
    from oracle.oracle import Oracle
    O = Oracle(precision="f64", nthreads=os.cpu_count() or 4, **HRRT3)
    rng = np.random.default_rng(5)
    sh = O.sino_shape
    prompts = rng.poisson(1.5, size=sh).astype(np.int16)
    randoms = (rng.random(sh, dtype=np.float32) * np.float32(0.1)).astype(np.float32)
    norm = (np.float32(0.9) + np.float32(0.2) * rng.random(sh, dtype=np.float32)).astype(np.float32)
    norm[:, :, 100:103] = 0
    p, a, m = O.prep(prompts, randoms, norm)
    return O, (prompts, randoms, norm), (p, a, m)


def test_hrrt3_one_subset(hrrt3_inputs):
    """Full-size HRRT span 3: prep, subset 0's sensitivity and one subset."""
    import hrrt_reconstruction_b200 as H
    O, raw, (p, a, m) = hrrt3_inputs
    with H.Context(product_geom(HRRT3)) as ctx:
        ctx.upload_inputs(*raw)
        assert np.array_equal(ctx.norm_zero_mask(), O.norm_zero_mask())
        ctx.sensitivity()
        nf = O.sensitivity(m)
        assert rel_l2(ctx.get_sensitivity(0), nf[0]) <= 2e-6
        ctx.init_image()
        ctx.osem_subsets(0, 1)
        want = O.init_image()
        O.osem_subset(want, nf[0], p, a, 0)
        assert rel_l2(ctx.get_image_xyz(), want) <= 1e-5


@pytest.mark.parametrize("storage,tol", [(1, 1e-3), (2, 2e-4)])
def test_16bit_storage_close_to_f32(hrrt3_inputs, storage, tol):
    """Additive / multiplicative terms stored in bf16 (HRRT_STORE_16) or fp16
    (HRRT_STORE_F16): after two subsets within `tol` rel-L2 of the
    f32-stored path."""
    import hrrt_reconstruction_b200 as H
    _, raw, _ = hrrt3_inputs
    imgs = []
    for st in (H.STORE_F32, storage):
        with H.Context(product_geom(HRRT3)) as ctx:
            ctx.upload_inputs(*raw, storage=st)
            ctx.sensitivity()
            ctx.init_image()
            ctx.osem_subsets(0, 2)
            imgs.append(ctx.get_image_xyz())
    e = rel_l2(imgs[1], imgs[0])
    assert e <= tol, e


@pytest.mark.parametrize("storage", [1, 2])
def test_16bit_storage_vs_fp64_oracle(hrrt3_inputs, storage):
    """The 16-bit-stored path against the FP64 oracle of the same projector:
    the sensitivity image of subset 0 and one subset within 1e-3 rel-L2."""
    import hrrt_reconstruction_b200 as H
    O, raw, (p, a, m) = hrrt3_inputs
    with H.Context(product_geom(HRRT3)) as ctx:
        ctx.upload_inputs(*raw, storage=storage)
        ctx.sensitivity()
        nf = O.sensitivity(m)
        assert rel_l2(ctx.get_sensitivity(0), nf[0]) <= 1e-3
        ctx.init_image()
        ctx.osem_subsets(0, 1)
        want = O.init_image()
        O.osem_subset(want, nf[0], p, a, 0)
        e = rel_l2(ctx.get_image_xyz(), want)
        assert e <= 1e-3, e


def test_fp16_storage_range_is_reported():
    """A term beyond fp16's range fails the upload instead of storing infinity."""
    import hrrt_reconstruction_b200 as H
    from oracle.oracle import Oracle
    d = ALL["small9"]
    O = Oracle(**d)
    prompts, randoms, norm, atten, scatter = I.sinograms(O.P, O.views, O.nx)
    with H.Context(product_geom(d)) as ctx:
        ctx.upload_inputs(prompts, randoms, norm, atten, scatter, storage=H.STORE_F16)
        big = randoms.copy()
        big[3, 5, 7] = 1e6
        with pytest.raises(H.HrrtError, match="fp16"):
            ctx.upload_inputs(prompts, big, norm, atten, scatter, storage=H.STORE_F16)
        ctx.upload_inputs(prompts, big, norm, atten, scatter, storage=H.STORE_16)


@pytest.mark.parametrize("name", ["small3", "small9"])
def test_reconstruct_matches_separate_calls(name):
    """hrrt_reconstruct (uploads streamed in subset order, first iteration
    over every quad) gives the image of upload + sensitivity + init + osem
    + get_image bit for bit, norm-zero mask included."""
    import hrrt_reconstruction_b200 as H
    from oracle.oracle import Oracle
    d = ALL[name]
    O = Oracle(**d)
    prompts, randoms, norm, atten, scatter = I.sinograms(O.P, O.views, O.nx)
    with H.Context(product_geom(d)) as ctx:
        ctx.upload_inputs(prompts, randoms, norm, atten, scatter)
        ctx.sensitivity()
        ctx.init_image()
        st1 = ctx.osem(2)
        want = ctx.get_image()
        mask = ctx.norm_zero_mask()
        sens3 = ctx.get_sensitivity(3)
    with H.Context(product_geom(d)) as ctx:
        got, st2 = ctx.reconstruct(prompts, randoms, norm, atten, scatter, iterations=2)
        assert np.array_equal(ctx.norm_zero_mask(), mask)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        assert st2.subset_iterations == st1.subset_iterations and st2.sum_image == st1.sum_image
        # the context is left ready for more iterations
        assert np.array_equal(ctx.get_sensitivity(3).view(np.uint32), sens3.view(np.uint32))


def test_reconstruct_full_size(hrrt3_inputs):
    import hrrt_reconstruction_b200 as H
    _, raw, _ = hrrt3_inputs
    with H.Context(product_geom(HRRT3)) as ctx:
        ctx.upload_inputs(*raw)
        ctx.sensitivity()
        ctx.init_image()
        ctx.osem(1)
        want = ctx.get_image()
    with H.Context(product_geom(HRRT3)) as ctx:
        got, st = ctx.reconstruct(*raw, iterations=1)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
