"""PSF resolution modelling (-B; psf.cpp).

CPU: the library's make1d_psf_filter taps (host code) are bit-identical to the
restatement in oracle/hrrt_oracle.c and to the reference's own psf.cpp, whose
convolve3d the restatement's single-precision build equals bit for bit.  GPU: convolve3d on the device is
bit-identical to the oracle's single-precision build on every test geometry
(same taps, same sum order, no fused multiply-adds); the sensitivity images and
one subset with PSF are within 2e-6 / 1e-5 of the FP64 oracle (as without PSF);
the command line's -B gives the library's image bit for bit."""
import os
import subprocess

import numpy as np
import pytest

from geoms import ALL, product_geom, random_image
from golden import inputs as I

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PARAMS = [(0.0, 0.0, 0.0), (2.0, 5.0, 0.1), (3.0, 0.0, 0.0)]


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("params", PARAMS)
@pytest.mark.parametrize("pixel", [1.21875, 2.4375])
def test_psf_taps_match_oracle(params, pixel):
    import hrrt_reconstruction_b200 as H
    from oracle.oracle import Oracle
    O = Oracle(**ALL["small9"])
    got = H.psf_kernel(*params, pixel_size=pixel)
    want = O.psf_kernel(*params, pixel_size=pixel)
    assert got.size == want.size and got.size % 2 == 1
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert abs(float(got.sum(dtype=np.float64)) - 1.0) < 1e-6


def test_psf_default_is_the_hrrt_kernel():
    """fwhm1 = 0 selects 0.9 / 2.5 sigma (mm) and ratio 0.05: 13 taps at
    1.21875 mm, peak in the middle."""
    import hrrt_reconstruction_b200 as H
    k = H.psf_kernel()
    assert k.size == 13 and int(np.argmax(k)) == 6 and np.allclose(k, k[::-1])


@pytest.mark.parametrize("params", PARAMS)
@pytest.mark.parametrize("name", ["small3", "hrrt9"])
def test_psf_equals_reference(ref_lib, name, params):
    """The reference's own make1d_psf_filter and convolve3d (psf.cpp compiled
    unmodified into oracle/_ref/libhrrt_ref.so, kernels set up as
    hrrt_osem3d_span3.cpp:4521-4540 does) against the restatement's taps and
    single-precision convolve3d and the library's host taps, bit for bit."""
    import hrrt_reconstruction_b200 as H
    from oracle.oracle import Oracle
    d = ALL[name]
    R = ref_lib.RefProjector(nthreads=4, **d)
    taps = R.set_psf(*params)
    assert np.array_equal(taps.view(np.uint32), H.psf_kernel(*params, pixel_size=d["binsize"]).view(np.uint32))
    O = Oracle(precision="f32", **d)
    assert np.array_equal(taps.view(np.uint32), O.psf_kernel(*params, pixel_size=d["binsize"]).view(np.uint32))
    O.set_psf(True, *params)
    x = random_image(O.image_shape, O.cylwiny(), seed=33, zvalid=O.nz)
    assert np.array_equal(R.psf(x).view(np.uint32), O.psf(x).view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("params", PARAMS[:2])
def test_psf_convolve_equals_reference_on_device(ref_lib, params):
    """hrrt_psf_convolve against the reference's convolve3d, HRRT span 9."""
    import hrrt_reconstruction_b200 as H
    d = ALL["hrrt9"]
    R = ref_lib.RefProjector(nthreads=8, **d)
    R.set_psf(*params)
    with H.Context(product_geom(d)) as ctx:
        ctx.set_psf(True, *params)
        x = random_image(ctx.image_shape, R.cylwiny(), seed=34, zvalid=R.nz)
        got = ctx.psf(x)
    assert np.array_equal(got.view(np.uint32), R.psf(x).view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small3", "small9", "hrrt9"])
@pytest.mark.parametrize("params", PARAMS[:2])
def test_psf_convolve_bit_identical(name, params):
    import hrrt_reconstruction_b200 as H
    from oracle.oracle import Oracle
    d = ALL[name]
    O = Oracle(precision="f32", **d)
    O.set_psf(True, *params)
    with H.Context(product_geom(d)) as ctx:
        ctx.set_psf(True, *params)
        x = random_image(ctx.image_shape, O.cylwiny(), seed=31, zvalid=O.nz)
        got = ctx.psf(x)
    want = O.psf(x)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small3", "small9"])
def test_psf_sensitivity_and_subset(name):
    import hrrt_reconstruction_b200 as H
    from oracle.oracle import Oracle
    d = ALL[name]
    O = Oracle(precision="f64", nthreads=os.cpu_count() or 4, **d)
    O.set_psf(True)
    prompts, randoms, norm, atten, scatter = I.sinograms(O.P, O.views, O.nx)
    p, a, m = O.prep(prompts, randoms, norm, atten, scatter)
    nf = O.sensitivity(m)
    with H.Context(product_geom(d)) as ctx:
        ctx.set_psf(True)
        ctx.upload_inputs(prompts, randoms, norm, atten, scatter)
        ctx.sensitivity()
        for s in range(O.subsets):
            assert rel_l2(ctx.get_sensitivity(s), nf[s]) <= 2e-6, s
        ctx.init_image()
        ctx.osem_subsets(0, 2)
        got = ctx.get_image_xyz()
    want = O.init_image()
    order = O.order()
    for k in range(2):
        O.osem_subset(want, nf[int(order[k])], p, a, int(order[k]))
    assert rel_l2(got, want) <= 1e-5


@pytest.mark.gpu
def test_cli_psf(tmp_path):
    import hrrt_reconstruction_b200 as H
    from hrrt_reconstruction_b200 import build
    build.build_cli()
    cli = os.path.join(ROOT, "hrrt_reconstruction_b200", "hrrt_osem3d_gpu")
    with H.Context(H.hrrt_geometry(span=9)) as ctx:
        shape = ctx.sino_shape
        rng = np.random.default_rng(17)
        prompts = rng.poisson(1.0, size=shape).astype(np.int16)
        delayed = np.full(shape, 0.1, np.float32)
        ctx.set_psf(True, 2.0, 5.0, 0.1)
        ctx.upload_inputs(prompts, delayed)
        ctx.sensitivity()
        ctx.init_image()
        ctx.osem(1)
        want = ctx.get_image()
    prompts.tofile(tmp_path / "p.s")
    delayed.tofile(tmp_path / "d.s")
    out = tmp_path / "img.i"
    r = subprocess.run([cli, "-p", str(tmp_path / "p.s"), "-d", str(tmp_path / "d.s"), "-o", str(out), "-W", "3",
                        "-I", "1", "-m", "9,67", "-B", "2,5,0.1"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, np.float32).reshape(want.shape)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert "OSEM3D-OP-PSF" in (tmp_path / "img.i.hdr").read_text()
