"""The lmhistogram command line (lmhistogram_gpu, lmhistogram_mp.cpp:427-1118).

CPU: header and option errors are reported before any device work.  GPU: a
listmode file with a clock-reset tag, block singles and two 2-s frames in -PR
span-3 mode gives, frame by frame, the oracle's prompts (.s), trues folded
into span 9 (.tr.s), coincidence histogram (.ch), head curve (_lm.hc) and
header values; the default (trues) mode over the whole stream likewise."""
import os
import subprocess

import numpy as np
import pytest

from oracle import lm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HALFLIFE = 6586.2
HEADER = """!INTERFILE
!originating system := HRRT
isotope halflife := {halflife}
lower level := 400
!study date (dd:mm:yryr) := 30:12:2009
!study time (hh:mm:ss) := 15:50:00
dose_assay_date (dd:mm:yryr) := 30:12:2009
dose_assay_time (hh:mm:ss) := 15:40:00
{extra}"""


def cli():
    from hrrt_reconstruction_b200 import build
    build.build_library()
    return build.build_lmhistogram()


def write_scan(tmp_path, words, extra="", halflife=HALFLIFE):
    path = tmp_path / "scan.l64"
    np.asarray(words, np.uint32).tofile(path)
    (tmp_path / "scan.l64.hdr").write_text(HEADER.format(halflife=halflife, extra=extra))
    return path


def run(args, **kw):
    return subprocess.run([cli()] + [str(a) for a in args], capture_output=True, text=True, timeout=900, **kw)


def read_header(path):
    out = {}
    for line in open(path):
        if " := " in line:
            k, v = line.rstrip("\n").split(" := ", 1)
            out[k] = v
    return out


def test_errors_before_device_work(tmp_path):
    w = np.zeros(16, np.uint32)
    r = run([tmp_path / "none.l64"])
    assert r.returncode == 1 and "File not found" in r.stderr
    p = tmp_path / "scan.l64"
    w.tofile(p)
    r = run([p])
    assert r.returncode == 1 and "header" in r.stderr
    write_scan(tmp_path, w, halflife=0)
    r = run([p])
    assert r.returncode == 1 and "No isotope halflife" in r.stderr
    write_scan(tmp_path, w, extra="!PET data type := transmission\n")
    r = run([p])
    assert r.returncode == 1 and "transmission" in r.stderr
    write_scan(tmp_path, w)
    for bad in (["-d", "x"], ["-d", "0*3"], ["--span", "7"], ["--add", "a.s"], ["--scan"], ["--bogus"]):
        r = run([p] + bad)
        assert r.returncode == 1, bad
    r = run(["--help"])
    assert r.returncode == 0 and "usage" in r.stdout


def frame_oracle(O, w, durations):
    """The oracle driven like the command line: seek to the clock reset, then
    each frame at its file offset."""
    O.reset_clock()
    pos = O.seek(w, 0)
    assert pos > 0
    frames = []
    for dur in durations:
        s, d, st, hc, rates, _ = O.histogram_hc(w[pos:], duration=dur, offset=pos)
        frames.append((s, d, st, hc, rates, O.last_crystal_counts.copy()))
        pos += st["words_used"]
    return frames


def check_header(h, st, rates, f, nsinos):
    assert int(h["image duration"]) == st["duration"] > 0
    assert int(h["image relative start time"]) == st["frame_start"]
    assert int(h["frame"]) == f
    assert int(h["Total Prompts"]) == st["prompts"] and int(h["Total Randoms"]) == st["delayed"]
    assert int(h["Total Net Trues"]) == st["prompts"] - st["delayed"]
    for b in (0, 17, 935):
        assert int(h[f"block singles {b}"]) == rates[b]
    av = int(rates.astype(np.int64).sum()) // 936
    assert int(h["average singles per block"]) == av
    dtc = np.exp(8.94e-6 * av)
    assert abs(float(h["Dead time correction factor"]) - dtc) <= 1e-6 * dtc + 1e-6
    dcf1 = 2.0 ** ((st["frame_start"] + 600) / HALFLIFE)
    assert abs(float(h["decay correction factor"]) - dcf1) < 2e-6
    # 1 - 2^(-d/T) is formed from a single-precision power (write_sino,
    # lmhistogram_mp.cpp:590): its cancellation leaves ~3e-4 of the exact value
    d = st["duration"]
    dcf2 = np.log(2.0) * d / (HALFLIFE * (1.0 - 2.0 ** (-d / HALFLIFE)))
    assert abs(float(h["decay correction factor2"]) - dcf2) < 1e-3 * dcf2
    assert int(h["matrix size [3]"]) == nsinos
    assert h["!originating system"] == "HRRT" and h["isotope halflife"] == str(HALFLIFE)


@pytest.mark.gpu
def test_frames_prompts_and_randoms_span3(tmp_path):
    from test_listmode_gpu import singles_stream
    w = singles_stream(13, 500_000, tag_every=100, ms0=0)
    p = write_scan(tmp_path, w, extra="axial compression := 3\n")
    r = run([p, "--PR", "--ra", "-d", "2*2"])
    assert r.returncode == 0, r.stderr
    frames = frame_oracle(lm.LMOracle(3), w, [2, 2])
    hc_text = (tmp_path / "scan_lm.hc").read_text().splitlines()
    hc_blocks = [blk.splitlines() for blk in (tmp_path / "scan_lm.hc").read_text().split(
        "Singles,Randoms,Prompts,Time(ms)\n")[1:]]
    assert len(hc_blocks) == 2 and hc_text[0] == "Singles,Randoms,Prompts,Time(ms)"
    for f, (s, d, st, hc, rates, cc) in enumerate(frames):
        stem = tmp_path / f"scan_frame{f}"
        got = np.fromfile(f"{stem}.s", np.uint16)
        assert np.array_equal(got, s)
        tr = np.fromfile(f"{stem}.tr.s", np.int16)
        assert np.array_equal(tr, lm.convert_span9((s.view(np.int16) - d.view(np.int16)).astype(np.int16)))
        assert np.array_equal(np.fromfile(f"{stem}.ra.s", np.uint16), d)
        assert np.array_equal(np.fromfile(f"{stem}.ch", np.uint32), cc) and cc.sum() > 0
        h = read_header(f"{stem}.s.hdr")
        check_header(h, st, rates, f, 6367)
        assert h["Sinogram data type"] == "prompt" and h["!name of true data file"] == f"{stem}.tr.s"
        assert h["!name of data file"] == f"{stem}.s" and h["axial compression"] == "3"
        ht = read_header(f"{stem}.tr.s.hdr")
        assert ht["axial compression"] == "9" and ht["matrix size [3]"] == "2209"
        assert ht["Sinogram data type"] == "true"
        lines = [tuple(int(x) for x in ln.split(",")) for ln in hc_blocks[f]]
        assert lines == [(int(a[3]), int(a[2]), int(a[1]), int(a[0])) for a in hc]
    assert (tmp_path / "scan.dyn").read_text().split() == ["2", "scan_frame0.s", "scan_frame1.s"]


@pytest.mark.gpu
def test_whole_stream_trues_span9(tmp_path):
    """No frame definition: one frame over the rest of the stream (its
    measured duration in the header), trues in the span-9 sinogram."""
    from test_listmode_gpu import random_stream
    w = random_stream(14, 300_000, tag_every=100, ms0=0)
    p = write_scan(tmp_path, w)
    out = tmp_path / "out" / "trues.s"
    out.parent.mkdir()
    r = run([p, "-o", out])
    assert r.returncode == 0, r.stderr
    (s, d, st, hc, rates, cc), = frame_oracle(lm.LMOracle(9), w, [0])
    assert st["terminated"] == 0
    got = np.fromfile(out, np.uint16)
    O = lm.LMOracle(9)
    O.reset_clock()
    n0 = O.seek(w, 0)
    want, _, _ = O.histogram(w[n0:], mode=lm.TRUES, offset=n0)
    assert np.array_equal(got, want)
    h = read_header(str(out) + ".hdr")
    check_header(h, st, rates, 0, 2209)
    assert h["Sinogram data type"] == "true"
    assert np.array_equal(np.fromfile(tmp_path / "out" / "trues.ch", np.uint32), cc)


@pytest.mark.gpu
def test_missing_clock_reset_and_skip(tmp_path):
    """The first frame needs the 0-ms tag (goto_event(0)); a frame skip
    seeks to its second first."""
    from test_listmode_gpu import random_stream
    w = random_stream(15, 200_000, tag_every=100)  # clock from 5 s, no reset tag
    p = write_scan(tmp_path, w)
    r = run([p])
    assert r.returncode == 1 and "time reset" in r.stderr
    r = run([p, "-d", "1,6"])
    assert r.returncode == 0, r.stderr
    O = lm.LMOracle(9)
    O.reset_clock()
    n = O.seek(w, 6)
    want, _, st = O.histogram(w[n:], mode=lm.TRUES, duration=1, offset=n)
    assert np.array_equal(np.fromfile(tmp_path / "scan.s", np.uint16), want)
    h = read_header(tmp_path / "scan.s.hdr")
    assert h["image relative start time"] == "6" and h["image duration"] == "1"
    r = run([p, "-d", "1,60"])
    assert r.returncode == 1 and "requested time" in r.stderr
