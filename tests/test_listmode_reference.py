"""The listmode path pinned to the reference's OWN code (CPU).

oracle/_ref/lmhist_ref is the reference's histogram_mp.cpp, LM_Reader_mp.cpp,
LM_Rebinner_mp.cpp, convert_span9.cpp, lor_sinogram_map.cpp,
geometry_info.cpp and segment_info_fromarchive.cpp compiled unmodified
(oracle/Makefile).  Against it, bit for bit:

  * the rebinner LUT of init_sol / init_phy_to_pro (lor_sinogram_map.cpp:
    99-221): every SOL entry, the crystal z tables and the segment-plane
    table, for span 3 and span 9, from the restatement (oracle/lm_oracle.c)
    and from the product (hrrt_lm_table);
  * rebin_event (LM_Rebinner_mp.cpp:188-219) for every head pair, DOI layer
    and crystal-x class at seven ring pairs;
  * convert_span9 (convert_span9.cpp:13) over the whole int16 range, against
    the restatement and the product's host fold;
  * whole frames through the reference's reader, rebin_packet and histogram
    (histogram_mp.cpp:1026-1233, :1301-1398) -- prompts and delayed, trues,
    prompts only, border-crystal and no-DOI options, time from the tag count
    -- against the restatement: sinograms, frame start and duration, event
    totals, block singles rates and the head-curve text; the coincidence
    histogram where the reference's reader cuts its packet at the frame end,
    and the reference's count past the frame end where it does not.

The device histogrammer is checked against the restatement in
test_listmode_gpu.py and against this program directly in
test_listmode_reference_gpu.py.
"""
import numpy as np
import pytest

from lm_streams import random_stream, whole_packets
from oracle import lm
from oracle import lm_ref
from oracle.lm import LMOracle

pytestmark = pytest.mark.skipif(not lm_ref.available(), reason="oracle/_ref/lmhist_ref not built "
                                                               "(needs the reference sources)")


def all_classes(seed):
    """Every (mp, alayer, ax, blayer, bx) at ring pairs (0,0), (103,103),
    (0,103), (103,0), (51,52), (20,87) and one random pair each."""
    mp, al, ax, bl, bx = np.meshgrid(np.arange(1, 21), np.arange(2), np.arange(72), np.arange(2), np.arange(72),
                                     indexing="ij")
    base = np.stack([mp.ravel(), al.ravel(), ax.ravel(), bl.ravel(), bx.ravel()], 1)
    n = len(base)
    rows = []
    for ay, by in ((0, 0), (103, 103), (0, 103), (103, 0), (51, 52), (20, 87)):
        rows.append(np.column_stack([base[:, 0], base[:, 1], base[:, 2], np.full(n, ay), base[:, 3], base[:, 4],
                                     np.full(n, by)]))
    r = np.random.default_rng(seed).integers(0, 104, (n, 2))
    rows.append(np.column_stack([base[:, 0], base[:, 1], base[:, 2], r[:, 0], base[:, 3], base[:, 4], r[:, 1]]))
    return np.concatenate(rows).astype(np.int32)


def segplane_of(segs):
    z0, zm, off = segs
    sp = np.full((63, 207), -1, np.int16)
    for i in range(len(z0)):
        pl = np.arange(z0[i], zm[i] + 1)
        sp[i, pl] = pl + off[i]
    return sp


@pytest.mark.parametrize("span", [3, 9])
def test_lut_tables_equal_reference(span):
    import hrrt_reconstruction_b200 as H
    T = lm_ref.tables(span)
    O = LMOracle(span)
    sol = O.sol()
    for k in ("nsino", "d", "z"):
        a, b = T["sol"][k][1:], sol[k][1:]
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), k
    z, z2 = O.zpos()
    assert np.array_equal(T["c_zpos"].view(np.uint32), z.view(np.uint32))
    assert np.array_equal(T["c_zpos2"].view(np.uint32), z2.view(np.uint32))
    assert np.array_equal(T["segplane"], segplane_of(O.segments()))
    # the product's host tables (the device LUT is uploaded from them)
    psol = H.lm_table("sol", span=span)
    for k in ("nsino", "d", "z"):
        assert np.array_equal(psol[k][1:].view(np.uint32), T["sol"][k][1:].view(np.uint32)), k


@pytest.mark.parametrize("span", [3, 9])
def test_rebin_event_every_class_equals_reference(span):
    ev = all_classes(span)
    want = lm_ref.rebin_events(ev, span)
    got = LMOracle(span).rebin_events(ev)
    assert np.array_equal(got, want), np.flatnonzero(got != want)[:10]
    assert (want >= 0).sum() > len(ev) // 3


def test_convert_span9_equals_reference():
    import hrrt_reconstruction_b200 as H
    rng = np.random.default_rng(3)
    s3 = rng.integers(-32768, 32768, 6367 * 288 * 256, dtype=np.int64).astype(np.int16)
    want = lm_ref.convert_span9(s3)[:2209 * 288 * 256]
    assert np.array_equal(lm.convert_span9(s3), want)
    assert np.array_equal(H.convert_span9(s3).reshape(-1), want)


def stream(seed, npackets=3):
    # a tag every 1000 events from 5 s: npackets of 1 Mi events span ~npackets s
    return whole_packets(random_stream(seed, npackets * 1_050_000, doi7=False), npackets)


CASES = [  # span, mode, duration (s), flags
    (9, lm.PROMPTS_AND_DELAYED, 2, 0),
    (9, lm.TRUES, 2, 0),
    (9, lm.PROMPTS_ONLY, 1, 0),
    (9, lm.PROMPTS_AND_DELAYED, 2, lm.IGNORE_BORDER_CRYSTAL | lm.NO_DOI),
    (9, lm.PROMPTS_AND_DELAYED, 1, lm.TIME_FROM_COUNT),
    (3, lm.PROMPTS_AND_DELAYED, 2, 0),
]


@pytest.mark.parametrize("span,mode,duration,flags", CASES)
def test_frame_equals_reference_histogrammer(span, mode, duration, flags):
    w = stream(11 + span + 3 * mode + flags)
    R = lm_ref.histogram(w, span=span, mode=mode, duration=duration, flags=flags)
    O = LMOracle(span)
    O.reset_clock()
    s, d, st, hc, rates, totals = O.histogram_hc(w, mode=mode, duration=duration, flags=flags)
    assert st["terminated"] == 1
    assert np.array_equal(s.view(np.int16), R["prompts"]), np.flatnonzero(s.view(np.int16) != R["prompts"])[:10]
    if mode == lm.PROMPTS_AND_DELAYED:
        assert np.array_equal(d.view(np.int16), R["delayed"])
    assert st["frame_start"] == R["frame_start"] and st["duration"] == R["duration"]
    assert (int(totals[0]), int(totals[1])) == (R["total_prompts"], R["total_randoms"])
    assert np.array_equal(rates, R["singles"])
    # the head curve as the reference prints it: a header, then the lines
    # with no separator between them (histogram_mp.cpp:254, :1306)
    text = "Singles,Randoms,Prompts,Time(ms)\n" + "".join(f"{x[3]},{x[2]},{x[1]},{x[0]}" for x in hc.tolist())
    assert R["hc"] == text


def test_coincidence_histogram_equals_reference():
    """The coincidence histogram of a frame that ends in a later packet on
    the reader's pair grid (a stream without lone words), placed as the
    reference indexes it."""
    w = whole_packets(random_stream(7, 3 * 1_050_000, p_resync=0.0, doi7=False), 3)
    R = lm_ref.histogram(w, span=9, mode=lm.PROMPTS_AND_DELAYED, duration=2, coinc=True)
    O = LMOracle(9)
    O.reset_clock()
    O.histogram_hc(w, mode=lm.PROMPTS_AND_DELAYED, duration=2)
    assert np.array_equal(lm_ref.coinc_in_reference_layout(O.last_crystal_counts), R["coinc"].astype(np.uint64))


def test_reference_counts_coincidences_to_the_packet_cut():
    """Where the reference's coincidence histogram departs from the frame:
    rebin_packet counts every event of the packet the reader loaded, and the
    reader cuts a packet at the frame end only once the frame's start is
    known (check_end_of_frame, histogram_mp.cpp:988-1022).  A frame that ends
    inside the first packet therefore counts that whole packet.  The
    restatement counts the frame's events only; here its histogram of the
    whole first packet equals the reference's."""
    w = whole_packets(random_stream(7, 3 * 1_050_000, p_resync=0.0, doi7=False), 3)
    R = lm_ref.histogram(w, span=9, mode=lm.PROMPTS_AND_DELAYED, duration=1, coinc=True)
    O = LMOracle(9)
    O.reset_clock()
    s, _, st, *_ = O.histogram_hc(w, mode=lm.PROMPTS_AND_DELAYED, duration=1)
    assert np.array_equal(s.view(np.int16), R["prompts"]) and st["words_used"] < w.size // 3
    O.reset_clock()
    O.histogram_hc(w[:w.size // 3], mode=lm.PROMPTS_AND_DELAYED, duration=0)
    assert np.array_equal(lm_ref.coinc_in_reference_layout(O.last_crystal_counts), R["coinc"].astype(np.uint64))
