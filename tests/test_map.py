"""MAP reconstruction, technique 1 of je_hrrt_osem3d (-b 1,beta): Green's
one-step-late prior (dpfcalc.c) and the update pt_cal_updateimage_mapem.

CPU: the oracle's prior (oracle/hrrt_oracle.c, single-precision build) is
bit-identical to the reference's own calculate_DPF_image (dpfcalc.c compiled
unmodified into oracle/_ref/libmap_ref.so); the reference's update forms
1/nf_inv with _mm_rcp_ps, within 1.5 * 2^-12 of the exact reciprocal used
here.  GPU: the device prior equals the reference's except where the host's
expf is not correctly rounded (one ulp of a term, ~1e-3 of voxels); subsets
with MAP are within 2e-5 of the FP64 oracle; the command line's -b equals
the library."""
import os
import subprocess

import numpy as np
import pytest

from geoms import ALL, product_geom, random_image
from golden import inputs as I

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HAVE_REF = os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libmap_ref.so"))


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_oracle_prior_known_cases():
    """The prior is an odd function of the local differences: 0 inside a flat
    image, opposite for a bump and a dip, and 0 on the first and last planes
    and the first and last x rows."""
    from oracle.oracle import Oracle
    O = Oracle(precision="f32", **ALL["small9"])
    shape = (O.nx, O.nx, O.zp)
    cyl = np.asarray(O.cylwiny()).reshape(-1, 2)
    flat = np.zeros(shape, np.float32)
    for x in range(O.nx):
        flat[x, cyl[x, 0]:cyl[x, 1], :O.nz] = 3.0
    df = O.map_dpf(flat)
    assert np.all(df[24:40, 24:40, 2:O.nz - 2] == 0) and np.any(df != 0)  # only the FOV's edges show
    bump = flat.copy()
    bump[32, 32, 20] = 6.0
    dip = flat.copy()
    dip[32, 32, 20] = 0.0
    db, dd = O.map_dpf(bump), O.map_dpf(dip)
    assert db[32, 32, 20] > 0 and dd[32, 32, 20] < 0
    assert db[31, 32, 20] < 0  # the neighbour sees a larger centre
    x = random_image(shape, O.cylwiny(), seed=5, zvalid=O.nz)
    d = O.map_dpf(x)
    assert np.all(d[:, :, 0] == 0) and np.all(d[:, :, O.nz - 1:] == 0)
    assert np.all(d[0] == 0) and np.all(d[O.nx - 1] == 0)


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref/libmap_ref.so not built")
@pytest.mark.parametrize("name", ["small9", "hrrt9"])
def test_oracle_prior_matches_reference(name):
    from oracle import ref
    from oracle.oracle import Oracle
    O = Oracle(precision="f32", **ALL[name])
    x = random_image((O.nx, O.nx, O.zp), O.cylwiny(), seed=3, zvalid=O.nz)
    want = ref.map_dpf(x, O.nz, np.asarray(O.cylwiny()).reshape(-1, 2))
    got = O.map_dpf(x)
    assert np.count_nonzero(want) > 1000
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref/libmap_ref.so not built")
def test_reference_update_reciprocal_tolerance():
    """pt_cal_updateimage_mapem with the host's _mm_rcp_ps against the same
    update with the exact reciprocal: each voxel agrees to 1.5 * 2^-12 of
    1/nf_inv relative to the denominator beta * prior + 1/nf_inv (the
    approximation's bound carried through the division; where that
    denominator nears 0 the update is unstable in the reference itself), and
    they differ somewhere."""
    from oracle import ref
    from oracle.oracle import Oracle
    O = Oracle(precision="f32", **ALL["small9"])
    shape = (O.nx, O.nx, O.zp)
    cyl = np.asarray(O.cylwiny()).reshape(-1, 2)
    rng = np.random.default_rng(7)
    img = random_image(shape, O.cylwiny(), seed=8, zvalid=O.nz) + np.float32(0.5)
    corr = rng.uniform(0.5, 2.0, shape).astype(np.float32)
    nf = rng.uniform(0.01, 0.1, shape).astype(np.float32)
    dpf = O.map_dpf(img)
    beta = 0.2
    got = ref.map_update(img, corr, nf, dpf, cyl, beta, 1e10)
    den = np.float32(beta) * dpf + np.float32(1) / nf
    q = corr / den
    exact = np.minimum(np.float32(1e10), img * np.minimum(np.float32(100), np.maximum(np.float32(0.1), q)))
    mask = np.zeros(shape, bool)
    for x in range(O.nx):
        mask[x, cyl[x, 0]:cyl[x, 1], :] = True
    rel = np.abs(got[mask] - exact[mask]) / np.abs(exact[mask])
    bound = 1.5 * 2.0 ** -12 * (1.0 / nf[mask]) / np.abs(den[mask]) + 4e-7
    assert np.all(rel <= bound) and rel.max() > 0
    assert np.array_equal(got[~mask], img[~mask])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small9", "hrrt9"])
def test_device_prior_matches_reference(name):
    import hrrt_reconstruction_b200 as H
    from oracle.oracle import Oracle
    d = ALL[name]
    O = Oracle(precision="f32", **d)
    with H.Context(product_geom(d)) as ctx:
        ctx.set_map(1, 0.5)
        x = random_image(ctx.image_shape, O.cylwiny(), seed=3, zvalid=O.nz)
        got = ctx.map_prior(x)
    want = O.map_dpf(x)
    nz = np.count_nonzero(want)
    assert nz > 1000
    # the device's exponential is the correctly rounded one; the host's expf
    # (glibc, <= 0.502 ulp) misses it for ~7e-4 of arguments, by one ulp
    assert np.count_nonzero(got != want) <= 2e-3 * nz
    assert np.abs(got - want).max() <= 4e-6
    if HAVE_REF:
        from oracle import ref
        r = ref.map_dpf(x, O.nz, np.asarray(O.cylwiny()).reshape(-1, 2))
        assert np.array_equal(want.view(np.uint32), r.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small3", "small9"])
@pytest.mark.parametrize("psf", [False, True])
def test_map_subsets_match_oracle(name, psf):
    """Subset 0 with the OSEM update, subsets 1-3 with MAP (first_subset 1),
    against the FP64 oracle's osem_subset / osem_subset_map."""
    import hrrt_reconstruction_b200 as H
    from oracle.oracle import Oracle
    d = ALL[name]
    O = Oracle(precision="f64", nthreads=os.cpu_count() or 4, **d)
    if psf:
        O.set_psf(True)
    prompts, randoms, norm, atten, scatter = I.sinograms(O.P, O.views, O.nx)
    p, a, m = O.prep(prompts, randoms, norm, atten, scatter)
    nf = O.sensitivity(m)
    # beta well below the sensitivity: where beta * prior nears -1/nf_inv the
    # update divides by ~0 and even the oracle's f32 and f64 builds part
    sens = 1.0 / nf[0][nf[0] > 0]
    beta = float(0.02 * np.median(sens))
    with H.Context(product_geom(d)) as ctx:
        if psf:
            ctx.set_psf(True)
        ctx.upload_inputs(prompts, randoms, norm, atten, scatter)
        ctx.sensitivity()
        ctx.set_map(1, beta, first_subset=1)
        ctx.init_image()
        ctx.osem_subsets(0, 4)
        got = ctx.get_image_xyz()
    want = O.init_image()
    order = O.order()
    O.osem_subset(want, nf[int(order[0])], p, a, int(order[0]))
    for k in range(1, 4):
        O.osem_subset_map(want, nf[int(order[k])], p, a, int(order[k]), beta)
    assert rel_l2(got, want) <= 2e-5
    # the prior changed the result
    plain = O.init_image()
    for k in range(4):
        O.osem_subset(plain, nf[int(order[k])], p, a, int(order[k]))
    assert rel_l2(plain, want) > 1e-3


@pytest.mark.gpu
def test_cli_map(tmp_path):
    import hrrt_reconstruction_b200 as H
    from hrrt_reconstruction_b200 import build
    build.build_cli()
    cli = os.path.join(ROOT, "hrrt_reconstruction_b200", "hrrt_osem3d_gpu")
    with H.Context(H.hrrt_geometry(span=9)) as ctx:
        shape = ctx.sino_shape
        rng = np.random.default_rng(17)
        prompts = rng.poisson(1.0, size=shape).astype(np.int16)
        delayed = np.full(shape, 0.1, np.float32)
        ctx.upload_inputs(prompts, delayed)
        ctx.sensitivity()
        ctx.set_map(1, 0.05, 5)
        ctx.init_image()
        ctx.osem(1)
        want = ctx.get_image()
    prompts.tofile(tmp_path / "p.s")
    delayed.tofile(tmp_path / "d.s")
    out = tmp_path / "img.i"
    r = subprocess.run([cli, "-p", str(tmp_path / "p.s"), "-d", str(tmp_path / "d.s"), "-o", str(out), "-W", "3",
                        "-I", "1", "-m", "9,67", "-b", "1,0.05"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, np.float32).reshape(want.shape)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    r = subprocess.run([cli, "-p", str(tmp_path / "p.s"), "-d", str(tmp_path / "d.s"), "-o", str(out), "-W", "3",
                        "-b", "2,0.05"], capture_output=True, text=True, timeout=600)
    assert r.returncode != 0 and "technique 1" in r.stderr
