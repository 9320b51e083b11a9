"""Runs oracle/_ref/lmhist_ref -- the reference's OWN listmode code (LUT
creation, rebin_event, the packet decode and histogram, convert_span9, the
crystal singles of gen_delays),
compiled unmodified from its sources by oracle/Makefile.

TEST INFRASTRUCTURE.  Only tests/ and bench.py's listmode parity check use
this module, as the checker of oracle/lm_oracle.c and of the device
histogrammer.  Every call runs the program in a child process: the
reference's reader ends its process on a read past the end of its input, and
its histogram state is process-global.
"""
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
EXE = os.path.join(HERE, "_ref", "lmhist_ref")

SOL = np.dtype([("nsino", np.int32), ("d", np.float32), ("z", np.float32)])
NXD = 144            # crystals x DOI layers of a head
NYCRYS = 104
PACKET_EVENTS = 1 << 20   # the reader's packet (PACKET_SIZE, LM_Reader_mp.hpp)
PLANES = {3: 6367, 9: 2209}
NBLOCKS = 936


def available():
    return os.path.exists(EXE)


def _run(*args, timeout=600):
    r = subprocess.run([EXE, *map(str, args)], capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"lmhist_ref {args[0]} failed ({r.returncode}): {r.stderr[-400:]}")
    return r


def tables(span=3, maxrd=67):
    """-> dict(sol [21][144][144] SOL, c_zpos [104], c_zpos2 [104],
    segplane [63][207] int16) as the reference's init_sol builds them."""
    with tempfile.TemporaryDirectory() as d:
        fn = os.path.join(d, "t.bin")
        _run("tables", span, maxrd, fn)
        raw = open(fn, "rb").read()
    n_sol = 21 * NXD * NXD
    o = 0
    sol = np.frombuffer(raw, SOL, n_sol, o).reshape(21, NXD, NXD)
    o += n_sol * SOL.itemsize
    zpos = np.frombuffer(raw, np.float32, NYCRYS, o)
    o += NYCRYS * 4
    zpos2 = np.frombuffer(raw, np.float32, NYCRYS, o)
    o += NYCRYS * 4
    segplane = np.frombuffer(raw, np.int16, 63 * (2 * NYCRYS - 1), o).reshape(63, 2 * NYCRYS - 1)
    return dict(sol=sol.copy(), c_zpos=zpos.copy(), c_zpos2=zpos2.copy(), segplane=segplane.copy())


def rebin_events(ev, span=3, maxrd=67):
    """rebin_event for each row (mp, alayer, ax, ay, blayer, bx, by) of
    `ev` (int32 [n][7]) -> int32 [n] sinogram addresses (-1: none).  Rows
    must be valid emission classes (mp 1..20, layers 0/1, crystals in range)."""
    ev = np.ascontiguousarray(ev, np.int32)
    assert ev.ndim == 2 and ev.shape[1] == 7
    with tempfile.TemporaryDirectory() as d:
        fi, fo = os.path.join(d, "ev.bin"), os.path.join(d, "addr.bin")
        ev.tofile(fi)
        _run("rebin", span, maxrd, fi, fo)
        return np.fromfile(fo, np.int32)


def convert_span9(span3, maxrd=67, nrings=104):
    """The reference's in-place fold of a span-3 int16 sinogram; returns the
    whole array after the call (its first 2209 planes hold the span-9 one)."""
    s = np.ascontiguousarray(span3, np.int16).copy()
    with tempfile.TemporaryDirectory() as d:
        fn = os.path.join(d, "s.bin")
        s.tofile(fn)
        _run("span9", maxrd, nrings, fn)
        return np.fromfile(fn, np.int16).reshape(s.shape)


def crystal_singles(delayed_counts, scan_duration=1.0, tau=6.0e-9):
    """The reference's compute_csings_from_drates (gen_delays_lib.cpp:235-255)
    on int32 [119808] delayed crystal counts -> (float32 singles rates,
    iterations)."""
    dc = np.ascontiguousarray(delayed_counts, np.int32).reshape(-1)
    assert dc.size == 2 * 104 * 8 * 72
    with tempfile.TemporaryDirectory() as d:
        fi, fo = os.path.join(d, "dc.bin"), os.path.join(d, "sr.bin")
        dc.tofile(fi)
        _run("singles", repr(float(tau)), repr(float(scan_duration)), fi, fo)
        raw = np.fromfile(fo, np.uint8)
    return raw[:dc.size * 4].view(np.float32).copy(), int(raw[dc.size * 4:].view(np.int32)[0])


def histogram(words, span=3, mode=1, duration=1, flags=0, maxrd=67, coinc=False):
    """One frame of the l64 word stream (uint32 pairs ew1, ew2) through the
    reference's reader, rebinner and histogram (lmhistogram's PRO_RAN,
    prompts-only or trues mode).  The frame must end by `duration` before
    the stream does, and the stream must hold no transmission (DOI 7)
    events: the reference's emission path reaches its transmission table
    for them, which only a transmission run builds.

    -> dict(prompts, delayed: int16 sinograms (delayed zero outside PRO_RAN),
    hc: head-curve text, frame_start, duration, total_prompts,
    total_randoms, singles [936] and, with coinc, the coincidence
    histogram uint32 [2][119808])."""
    w = np.ascontiguousarray(words, np.uint32)
    assert w.size % 2 == 0 and duration > 0
    S = PLANES[span] * 256 * 288
    with tempfile.TemporaryDirectory() as d:
        fw, fs, fh, ft, fc = (os.path.join(d, n) for n in ("w.l64", "s.bin", "hc.txt", "st.txt", "c.bin"))
        w.tofile(fw)
        args = ["histogram", span, maxrd, mode, duration, flags, fw, fs, fh, ft] + ([fc] if coinc else [])
        _run(*args)
        sino = np.fromfile(fs, np.int16).reshape(2, S)
        hc = open(fh).read()
        st = {}
        singles = np.zeros(NBLOCKS, np.int32)
        for line in open(ft):
            k, *v = line.split()
            if k == "singles":
                singles[int(v[0])] = int(v[1])
            else:
                st[k] = int(v[0])
        out = dict(prompts=sino[0], delayed=sino[1], hc=hc, frame_start=st["frame_start"], duration=st["duration"],
                   total_prompts=st["prompts"], total_randoms=st["randoms"], singles=singles)
        if coinc:
            out["coinc"] = np.fromfile(fc, np.uint32).reshape(2, -1)
        return out


def coinc_in_reference_layout(cc):
    """A coincidence histogram [2][doi 2][ring 104][head 8][x 72] (the
    archive program's layout, histogram_mp_fromarchive.cpp:916) summed into
    the indexes the rewrite's rebin_packet forms (doi * 59904 + head * 72 +
    x + ring * 7488, histogram_mp.cpp:1218-1222), for comparison with
    histogram(coinc=True)."""
    c = np.asarray(cc, np.uint64).reshape(2, 2, 104, 8, 72)
    doi, ring, head, x = np.meshgrid(np.arange(2), np.arange(104), np.arange(8), np.arange(72), indexing="ij")
    idx = (doi * 59904 + head * 72 + x + ring * 7488).ravel()
    out = np.zeros((2, 2 * 59904 + 104 * 7488), np.uint64)
    for k in range(2):
        np.add.at(out[k], idx, c[k].ravel())
    return out
