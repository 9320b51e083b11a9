"""The hrrt_osem3d_gpu command line: the reference's flags and flat files.

CPU: argument handling (usage, required inputs, refused options) -- all of
which exit before a GPU is touched.  GPU: a span-9 OP-OSEM reconstruction
from flat files gives the same image, bit for bit, as the library called
directly on the same arrays; a span-9 attenuation file drives a span-3
reconstruction exactly like the expanded span-3 attenuation
(Atten3D_Span9, hrrt_osem3d_span3.cpp:1762-1796); a 2D scatter segment with
span-9 scale factors exactly like its 3D expansion (drv:1136-1179, 4407-4421)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "hrrt_reconstruction_b200", "hrrt_osem3d_gpu")


@pytest.fixture(scope="module")
def cli():
    from hrrt_reconstruction_b200 import build
    build.build_cli()
    if not os.path.exists(CLI):
        pytest.skip("hrrt_osem3d_gpu not built")
    return CLI


def run(cli, *args):
    return subprocess.run([cli, *args], capture_output=True, text=True, timeout=600)


def test_usage_and_argument_errors(cli):
    r = run(cli)
    assert r.returncode == 1 and "usage" in r.stdout
    r = run(cli, "-o", "x.i", "-W", "3")
    assert r.returncode == 1 and "-p prompts and -d delayed are required" in r.stderr
    r = run(cli, "-p", "a", "-d", "b", "-o", "x.i", "-W", "2")
    assert r.returncode == 1 and "-W 3" in r.stderr
    for opt, word in (("-A", "MAP"), ("-t", "trues")):
        r = run(cli, opt, "x", "-p", "a", "-d", "b", "-o", "x.i", "-W", "3")
        assert r.returncode == 1 and word in r.stderr
    r = run(cli, "-B", "x", "-p", "a", "-d", "b", "-o", "x.i", "-W", "3")
    assert r.returncode == 1 and "-B" in r.stderr
    r = run(cli, "-X", "128", "-p", "a", "-d", "b", "-o", "x.i", "-W", "3")
    assert r.returncode == 1 and "256" in r.stderr


def span_segments(span, maxdel=67, nrings=104):
    G = (maxdel - (span - 1) // 2) // span
    nz = 2 * nrings - 1
    yb, npl = [0], [nz]
    for g in range(1, G + 1):
        zmin = (span + 1) // 2 + (g - 1) * span
        yb += [zmin, zmin]
        npl += [nz - 2 * zmin] * 2
    off = np.concatenate([[0], np.cumsum(npl)[:-1]])
    return yb, npl, off


def expand_span9(a9, views=288, bins=256):
    """Span-3 attenuation from a span-9 one: the same axial plane of the
    span-9 segment of the same sign whose ring-difference range holds the
    span-3 segment's."""
    yb3, np3, off3 = span_segments(3)
    yb9, np9, off9 = span_segments(9)
    a9 = a9.reshape(-1, views, bins)
    out = np.empty((sum(np3), views, bins), np.float32)
    for s in range(len(yb3)):
        h = (s + 1) // 2
        g = (h + 1) // 3
        src = 0 if g == 0 else (2 * g - 1 if s % 2 == 1 else 2 * g)
        p9 = off9[src] + yb3[s] - yb9[src]
        out[off3[s]:off3[s] + np3[s]] = a9[p9:p9 + np3[s]]
    return out


@pytest.mark.gpu
def test_span9_reconstruction_matches_library(cli, tmp_path):
    import hrrt_reconstruction_b200 as H
    g = H.hrrt_geometry(span=9)
    with H.Context(g) as ctx:
        shape = ctx.sino_shape
        rng = np.random.default_rng(11)
        prompts = rng.poisson(1.2, size=shape).astype(np.int16)
        delayed = np.full(shape, 0.15, np.float32)
        norm = (0.9 + 0.2 * rng.random(shape, dtype=np.float32)).astype(np.float32)
        atten = (1.0 + rng.random(shape, dtype=np.float32)).astype(np.float32)
        for name, a in (("p.s", prompts), ("d.s", delayed), ("n.s", norm), ("a.s", atten)):
            a.tofile(tmp_path / name)
        ctx.upload_inputs(prompts, delayed, norm, atten)
        ctx.sensitivity()
        ctx.init_image()
        ctx.osem(2)
        want = ctx.get_image()
    out = tmp_path / "img.i"
    r = run(cli, "-p", str(tmp_path / "p.s"), "-d", str(tmp_path / "d.s"), "-n", str(tmp_path / "n.s"), "-a",
            str(tmp_path / "a.s"), "-o", str(out), "-W", "3", "-I", "2", "-S", "16", "-m", "9,67", "-N", "-T", "8")
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, np.float32).reshape(want.shape)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    hdr = (tmp_path / "img.i.hdr").read_text()
    assert "!INTERFILE" in hdr and "matrix size [3] := 207" in hdr and "number of iterations := 2" in hdr
    assert "reconstruction method := inki-2006-may-OSEM3D-OP" in hdr


@pytest.mark.gpu
def test_span9_attenuation_for_span3(cli, tmp_path):
    import hrrt_reconstruction_b200 as H
    rng = np.random.default_rng(12)
    with H.Context(H.hrrt_geometry(span=9)) as c9:
        a9 = (1.0 + rng.random(c9.sino_shape, dtype=np.float32)).astype(np.float32)
    g3 = H.hrrt_geometry(span=3)
    with H.Context(g3) as ctx:
        shape = ctx.sino_shape
        prompts = rng.poisson(0.8, size=shape).astype(np.int16)
        delayed = np.full(shape, 0.1, np.float32)
        a3 = expand_span9(a9)
        assert a3.shape == shape
        prompts.tofile(tmp_path / "p.s")
        delayed.tofile(tmp_path / "d.s")
        a9.tofile(tmp_path / "a9.s")
        ctx.upload_inputs(prompts, delayed, None, a3)
        ctx.sensitivity()
        ctx.init_image()
        ctx.osem(1)
        want = ctx.get_image()
    out = tmp_path / "img3.i"
    r = run(cli, "-p", str(tmp_path / "p.s"), "-d", str(tmp_path / "d.s"), "-a", str(tmp_path / "a9.s"), "-o",
            str(out), "-W", "3", "-I", "1", "-m", "3,67")
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, np.float32).reshape(want.shape)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def scatter_2d_to_3d(sc2d, sf9, span):
    """The reference's 2D-scatter input (drv:4407-4421): convert_s9_s3
    (drv:1136-1162) makes span-3 plane factors from the span-9 ones -- a walk
    over the span-3 segments three at a time, each next segment a trimmed
    copy of the previous -- and apply_scale_factors (drv:1169-1179) scales 2D
    plane yr_bottom+yr into plane yr of every segment."""
    yb, npl, off = span_segments(span)
    P = sum(npl)
    if span == 9:
        sf = sf9.astype(np.float32)
    else:
        sf = np.zeros(P, np.float32)
        i = j = 0
        for th in range(0, len(yb), 3):
            n = npl[th]
            sf[i:i + n] = sf9[j:j + n] / np.float32(3.0)
            i += n
            j += n
            for k in (1, 2):
                so = yb[th + k] - yb[th + k - 1]
                m = n - 2 * so
                sf[i:i + m] = sf[i - n + so:i - n + so + m]
                n = m
                i += m
    out = np.empty((P,) + sc2d.shape[1:], np.float32)
    for s in range(len(yb)):
        for yr in range(npl[s]):
            out[off[s] + yr] = sc2d[yb[s] + yr] * sf[off[s] + yr]
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("span", [9, 3])
def test_scatter_2d_with_scale_factors(cli, tmp_path, span):
    """-s with an unscaled 2D scatter segment + 2209 span-9 scale factors
    reconstructs exactly like the expanded 3D scatter."""
    import hrrt_reconstruction_b200 as H
    rng = np.random.default_rng(13 + span)
    with H.Context(H.hrrt_geometry(span=span)) as ctx:
        shape = ctx.sino_shape
        nz = ctx.info.nz
        sc2d = (0.05 * rng.random((nz,) + shape[1:], dtype=np.float32)).astype(np.float32)
        sf9 = (0.5 + rng.random(2209, dtype=np.float32)).astype(np.float32)
        s3 = scatter_2d_to_3d(sc2d, sf9, span)
        assert s3.shape == shape
        prompts = rng.poisson(0.8, size=shape).astype(np.int16)
        delayed = np.full(shape, 0.1, np.float32)
        prompts.tofile(tmp_path / "p.s")
        delayed.tofile(tmp_path / "d.s")
        np.concatenate([sc2d.reshape(-1), sf9]).tofile(tmp_path / "s2d.s")
        ctx.upload_inputs(prompts, delayed, None, None, s3)
        ctx.sensitivity()
        ctx.init_image()
        ctx.osem(1)
        want = ctx.get_image()
    out = tmp_path / "img.i"
    r = run(cli, "-p", str(tmp_path / "p.s"), "-d", str(tmp_path / "d.s"), "-s", str(tmp_path / "s2d.s"), "-o",
            str(out), "-W", "3", "-I", "1", "-m", f"{span},67")
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, np.float32).reshape(want.shape)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
