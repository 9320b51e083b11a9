"""Smoothed randoms from a coincidence histogram (gen_delays).

CPU: the crystal-singles estimate of the library (host code, hrrt_lm_crystal_singles)
is bit-identical to the restatement in oracle/lm_oracle.c and to the reference's
own compute_csings_from_drates, and recovers the singles rates that generated the
delayed counts.  GPU: hrrt_lm_smooth_randoms against the
oracle's compute_delays restatement (float sums in another order: rel-L2 <= 1e-6),
and the command line with -d pointing at a .ch file."""
import os
import subprocess

import numpy as np
import pytest

from oracle import lm

NC = lm.NCRYSTALS
TAU = 6.0e-9
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def singles_model(seed, live=1.0):
    """Crystal singles rates (cps) [layer][ring][head][x]: a smooth axial and
    transaxial profile with 10 % crystal-to-crystal variation; a fraction
    `live` of the crystals is non-zero (dead crystals read zero)."""
    rng = np.random.default_rng(seed)
    z = np.exp(-0.5 * ((np.arange(104) - 51.5) / 40.0) ** 2)
    x = 0.7 + 0.3 * np.cos((np.arange(72) - 35.5) / 72 * np.pi)
    s = 4.0e4 * z[None, :, None, None] * x[None, None, None, :] * np.ones((2, 104, 8, 72))
    s *= 1.0 + 0.1 * rng.standard_normal(s.shape)
    s *= rng.random(s.shape) < live
    return s.astype(np.float32).reshape(-1)


def coinc_hist(seed, duration, live=1.0):
    s = singles_model(seed, live)
    d = lm.delayed_counts_from_singles(s, duration, TAU)
    prompts = (3 * d).astype(np.int32)
    return np.concatenate([prompts, d]).astype(np.int32), s


def test_crystal_singles_match_oracle_and_model():
    import hrrt_reconstruction_b200 as H
    h, s = coinc_hist(1, 600.0)
    got, it = H.crystal_singles(h[NC:], 600.0, TAU)
    want, it_o = lm.crystal_singles(h[NC:], 600.0, TAU)
    assert it == it_o
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    live = s > 0
    rel = np.abs(got[live] - s[live]) / s[live]
    assert np.median(rel) < 1e-2, np.median(rel)


@pytest.mark.parametrize("seed,duration,live,noise", [(1, 60.0, 1.0, False), (2, 300.0, 0.97, True)])
def test_crystal_singles_equal_reference(seed, duration, live, noise):
    """The reference's own compute_csings_from_drates (gen_delays_lib.cpp
    compiled unmodified into oracle/_ref/lmhist_ref) against the restatement
    and the library's host estimate, bit for bit, iterations included;
    Poisson-noisy counts make the estimator iterate."""
    import hrrt_reconstruction_b200 as H
    from oracle import lm_ref
    if not lm_ref.available():
        pytest.skip("oracle/_ref/lmhist_ref not built")
    ch, _ = coinc_hist(seed, duration, live)
    d = ch[NC:]
    if noise:
        d = np.random.default_rng(seed).poisson(d).astype(np.int32)
    want, it = lm_ref.crystal_singles(d, duration, TAU)
    got, it_o = lm.crystal_singles(d, duration, TAU)
    assert it_o == it and np.array_equal(np.asarray(got, np.float32).view(np.uint32), want.view(np.uint32))
    lib, it_l = H.crystal_singles(d, duration, TAU)
    assert it_l == it and np.array_equal(np.asarray(lib, np.float32).view(np.uint32), want.view(np.uint32))
    if noise:
        assert it > 1


def test_crystal_singles_dead_crystals_and_defaults():
    import hrrt_reconstruction_b200 as H
    h, s = coinc_hist(2, 1.0, live=0.5)
    got, _ = H.crystal_singles(h[NC:])  # scan duration 1 s, tau 6 ns
    want, _ = lm.crystal_singles(h[NC:], 1.0, TAU)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert np.all(got[h[NC:] == 0] == 0)


@pytest.fixture(scope="module", params=[9, 3])
def span_pair(request):
    import hrrt_reconstruction_b200 as H
    O = lm.LMOracle(request.param)
    D = H.Listmode(request.param)
    yield request.param, O, D
    D.close()


@pytest.mark.gpu
def test_smooth_randoms_match_oracle(span_pair):
    """4 % of the crystals live (the oracle walks every pair of a live A
    crystal on one core)."""
    span, O, D = span_pair
    h, _ = coinc_hist(3 + span, 300.0, live=0.04)
    got, it = D.smooth_randoms(h, 300.0)
    want, it_o = lm.smooth_randoms(O, h, 300.0)
    assert it == it_o
    assert got.shape == want.shape and np.all(got >= 0)
    assert np.count_nonzero(want) > 1000
    w = want.astype(np.float64)
    e = float(np.linalg.norm(got.astype(np.float64) - w) / np.linalg.norm(w))
    assert e <= 1e-6, e
    assert np.array_equal(got == 0, want == 0)


@pytest.mark.gpu
def test_cli_coincidence_histogram_as_randoms(tmp_path):
    """-d file.ch: the command line computes the smoothed randoms over the
    scan duration of the prompt sinogram's header and reconstructs with
    them (rel-L2 <= 1e-5 against the library fed the same randoms: the
    randoms' float sums vary at rounding level between runs)."""
    import hrrt_reconstruction_b200 as H
    from hrrt_reconstruction_b200 import build
    build.build_cli()
    cli = os.path.join(ROOT, "hrrt_reconstruction_b200", "hrrt_osem3d_gpu")
    h, _ = coinc_hist(7, 120.0)
    with H.Listmode(9) as L:
        randoms, _ = L.smooth_randoms(h, 120.0)
    with H.Context(H.hrrt_geometry(span=9)) as ctx:
        shape = ctx.sino_shape
        rng = np.random.default_rng(8)
        prompts = rng.poisson(1.0, size=shape).astype(np.int16)
        ctx.upload_inputs(prompts, randoms.reshape(shape))
        ctx.sensitivity()
        ctx.init_image()
        ctx.osem(1)
        want = ctx.get_image()
    prompts.tofile(tmp_path / "p.s")
    (tmp_path / "p.s.hdr").write_text("!INTERFILE\nimage duration := 120\n")
    h.tofile(tmp_path / "r.ch")
    out = tmp_path / "img.i"
    r = subprocess.run([cli, "-p", str(tmp_path / "p.s"), "-d", str(tmp_path / "r.ch"), "-o", str(out), "-W", "3",
                        "-I", "1", "-m", "9,67"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, np.float32).reshape(want.shape)
    e = float(np.linalg.norm(got.astype(np.float64) - want) / np.linalg.norm(want.astype(np.float64)))
    assert e <= 1e-5, e
    (tmp_path / "p.s.hdr").write_text("!INTERFILE\n")
    r = subprocess.run([cli, "-p", str(tmp_path / "p.s"), "-d", str(tmp_path / "r.ch"), "-o", str(out), "-W", "3",
                        "-I", "1", "-m", "9,67"], capture_output=True, text=True, timeout=600)
    assert r.returncode != 0 and "scan duration" in r.stderr
