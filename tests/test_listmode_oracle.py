"""Known-answer tests of the listmode histogrammer restatement
(oracle/lm_oracle.c) and its pins to the reference's own listmode geometry
(gen_delays_lib/geometry_info.cpp, segment_info_fromarchive.cpp, built by
oracle/Makefile target "ref").

Every case follows from the reference's code read directly:
  * EWTYPES classes (histogram_mp.cpp:1056-1062): ew1/ew2 top bits 00/11
    prompt, 00/10 delayed, 01/1x tag, anything else out of sync (advance 1);
  * invalid head pair / crystal indices are dropped (:1124-1145);
  * DOI values other than 0 and 1 are not histogrammed; 7 is transmission;
  * packets of 1 Mi 64-bit events are parsed from their own first word
    (LM_Reader_mp.hpp:39, histogram_mp.cpp:1055);
  * a time tag whose second reaches start + duration ends the frame
    (histogram_mp.cpp:225-260, :334-340);
  * bins are 16-bit and wrap;
  * an LOR through the scanner axis between opposite heads has bin 128.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import lm
from oracle.lm import LMOracle, event_words, interleave, tag_words

SINO_PLANE = 256 * 288


@pytest.fixture(scope="module")
def O3():
    return LMOracle(3)


def words_of(*pairs):
    return np.concatenate([interleave(np.atleast_1d(a), np.atleast_1d(b)) for a, b in pairs]).astype(np.uint32)


def test_sizes():
    assert LMOracle(3).sino_size == 6367 * SINO_PLANE
    assert LMOracle(9).sino_size == 2209 * SINO_PLANE


def test_axis_lor_bin_128_and_segment_0(O3):
    """Heads 0 and 4 face each other (head pair 3); crystal ax on head 0 and
    the same index on head 4 are point-symmetric about the axis, so r = 0
    exactly and the bin is 128; equal ring index gives segment 0 and the
    plane round(z/plane_sep)."""
    sol = O3.sol()
    zpos, zpos2 = O3.zpos()
    for ax in (0, 17, 35, 36, 71):
        for layer in (0, 1):
            s = sol[3, ax + 72 * layer, ax + 72 * layer]
            assert s["nsino"] % 256 == 128
            for ay in (0, 51, 103):
                addr = O3.rebin_event(3, layer, ax, ay, layer, ax, ay)
                plane = int(zpos2[ay])
                assert addr == plane * SINO_PLANE + s["nsino"]
    # planes advance about two per ring (plane_sep is half the ring pitch)
    p = np.floor(zpos2).astype(int)
    assert p[0] == 0 and np.all(np.diff(p) >= 1) and p[-1] in (205, 206)


def test_oblique_lors_land_in_odd_and_even_segments(O3):
    """Ring difference +d and -d go to the two segments 2k-1 and 2k of one
    group (which is which follows the LOR's orientation, through the sign of
    the LUT's 1/d): different plane blocks, same bin.
    Across the axis (d_xy ~ 49.9 cm) a difference of 3 crystals (0.72 cm)
    is 0.93 segment steps of 3*plane_sep/R: group 1; of 6 crystals, group 2."""
    z0, zmax, off = O3.segments()
    seg_of = lambda addr: int(np.searchsorted(off + z0, addr // SINO_PLANE, side="right") - 1)  # noqa: E731
    for d, group in ((3, 1), (6, 2)):
        a = O3.rebin_event(3, 0, 30, 40, 0, 30, 40 + d)
        b = O3.rebin_event(3, 0, 30, 40 + d, 0, 30, 40)
        assert a >= 0 and b >= 0
        assert a % SINO_PLANE == b % SINO_PLANE
        assert {seg_of(a), seg_of(b)} == {2 * group - 1, 2 * group}


def test_event_classes_and_rejections(O3):
    good = event_words(3, 35, 50, 35, 50)
    dly = event_words(3, 35, 50, 35, 50, prompt=False)
    w = words_of(
        good,                                    # prompt
        dly,                                     # delayed
        (np.uint32(0x00000000), np.uint32(0x00000000)),  # 00/00: out of sync -> 1 word, then 00/00 again
        event_words(0, 35, 50, 35, 50),          # head pair 0: invalid
        event_words(21, 35, 50, 35, 50),         # head pair 21: invalid (mpe bits allow up to 63)
        event_words(3, 72, 50, 35, 50),          # ax out of range
        event_words(3, 35, 104, 35, 50),         # ay out of range
        event_words(3, 35, 50, 35, 50, doia=3),  # DOI 3: not histogrammed
        event_words(3, 35, 50, 35, 50, doib=7),  # DOI 7: transmission
        tag_words(0xA0000005),                   # block singles tag
        good,
    )
    sino, dl, st = O3.histogram(w)
    addr = O3.rebin_event(3, 0, 35, 50, 0, 35, 50)
    assert sino[addr] == 2 and dl[addr] == 1
    assert int(sino.sum(dtype=np.int64)) == 2 and int(dl.sum(dtype=np.int64)) == 1
    assert st["prompts"] == 2 and st["delayed"] == 1
    assert st["invalid"] == 4 and st["doi_other"] == 1 and st["doi7"] == 1
    assert st["tags"] == 1 and st["timetags"] == 0
    assert st["resyncs"] == 2  # 00/00 skipped one word at a time: (0,0) then (0, next ew1 00)


def test_prompts_only_and_trues_modes(O3):
    good = event_words(3, 35, 50, 35, 50)
    dly = event_words(3, 35, 50, 35, 50, prompt=False)
    addr = O3.rebin_event(3, 0, 35, 50, 0, 35, 50)
    w = words_of(good, dly, dly)
    s, d, st = O3.histogram(w, mode=lm.PROMPTS_ONLY)
    assert d is None and s[addr] == 1 and int(s.sum(dtype=np.int64)) == 1
    s, d, st = O3.histogram(w, mode=lm.TRUES)
    assert s[addr] == np.uint16(0xFFFF)  # 1 - 2 wraps in the signed 16-bit bin


def test_sixteen_bit_wrap(O3):
    n = 65537
    ew1, ew2 = event_words(np.full(n, 3), np.full(n, 20), np.full(n, 60), np.full(n, 50), np.full(n, 61))
    sino, dl, st = O3.histogram(interleave(ew1, ew2))
    addr = O3.rebin_event(3, 0, 20, 60, 0, 50, 61)
    assert addr >= 0 and sino[addr] == 1 and st["prompts"] == n


def test_untimed_tag_value_is_histogrammed_as_an_event(O3):
    """A tag word whose 32-bit value has bit 31 clear passes through the
    32-bit stream as an event word (histogram_mp.cpp:347-364): bit 30 selects
    prompt, the low 30 bits are the address."""
    sino, dl, st = O3.histogram(words_of(tag_words(0x40000000 | 12345), tag_words(777)))
    assert sino[12345] == 1 and dl[777] == 1 and st["tags"] == 2


def test_packet_boundary_resets_alignment(O3):
    """One lone word shifts packet 0's parse by one; the event straddling the
    packet end is lost and packet 1 parses from its own first word."""
    P = lm.PACKET_WORDS
    ev = interleave(*event_words(3, 35, 50, 35, 50))
    w = np.empty(2 * P, np.uint32)
    w[0] = 0x00000000           # lone word: (0, ew1) is 00/00 -> out of sync
    w[1:P - 1] = np.tile(ev, (P - 2) // 2)
    w[P - 1] = ev[0]            # ew1 of an event whose ew2 opens packet 1
    w[P] = ev[1]
    w[P + 1:] = np.tile(ev, P // 2)[:P - 1]
    sino, dl, st = O3.histogram(w)
    addr = O3.rebin_event(3, 0, 35, 50, 0, 35, 50)
    n0 = (P - 2) // 2           # packet 0: events at odd positions
    n1 = (P - 1) // 2           # packet 1: ew2 at P is out of sync, then aligned
    assert st["prompts"] == n0 + n1
    assert sino[addr] == (n0 + n1) % 65536
    assert st["resyncs"] == 2


def test_time_tags_end_the_frame(O3):
    """Tags every ms from 0 ms, one event after each; duration 2 s: the
    frame starts at the first tag (second 0) and ends at the tag of 2000 ms,
    whose following events belong to the next frame."""
    ms = np.arange(0, 3000)
    ev1, ev2 = event_words(np.full(ms.size, 3), 35, 50, 35, 50)
    t1, t2 = tag_words(0x80000000 | ms.astype(np.uint32))
    w = np.empty(4 * ms.size, np.uint32)
    w[0::4], w[1::4], w[2::4], w[3::4] = t1, t2, ev1, ev2
    O3.reset_clock()
    sino, dl, st = O3.histogram(w, duration=2)
    assert st["terminated"] == 1 and st["frame_start"] == 0 and st["duration"] == 2
    assert st["prompts"] == 2000 and st["timetags"] == 2001
    assert st["words_used"] == 4 * 2000 + 2
    # the next frame continues from there with the carried clock
    sino2, _, st2 = O3.histogram(w[st["words_used"]:], duration=2)
    assert st2["frame_start"] == 2 and st2["prompts"] == 1000 and st2["terminated"] == 0
    O3.reset_clock()


def test_crystals_and_segments_match_reference_build():
    path = os.path.join(os.path.dirname(lm.__file__), "_ref", "liblm_ref.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref/liblm_ref.so not built (needs the reference sources)")
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    for span in (3, 9):
        O = LMOracle(span)
        a = np.zeros((8, 2, 72, 104, 3), np.float32)
        L.lmref_crystals(vp(a.ctypes.data))
        assert np.array_equal(a.view(np.uint32), O.crystals().view(np.uint32))
        z0, zm, off = (np.zeros(63, np.int32) for _ in range(3))
        n, npl, dt = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        L.lmref_segments(span, 67, vp(z0.ctypes.data), vp(zm.ctypes.data), vp(off.ctypes.data), ctypes.byref(n),
                         ctypes.byref(npl), ctypes.byref(dt))
        oz0, ozm, ooff = O.segments()
        k = n.value
        assert np.array_equal(z0[:k], oz0) and np.array_equal(zm[:k], ozm) and np.array_equal(off[:k], ooff)
        assert npl.value == O.nplanes and dt.value == O.L.lm_d_tan_theta(O.t)


def test_device_lut_matches_oracle():
    """The library's host-built LUT (hrrt_lm_table, no GPU needed) equals the
    restatement's bit for bit."""
    import hrrt_reconstruction_b200 as H
    for span in (3, 9):
        O = LMOracle(span)
        sol = H.lm_table("sol", span)
        assert np.array_equal(sol.view(np.uint8), O.sol().view(np.uint8))
        zp, zp2 = O.zpos()
        assert np.array_equal(H.lm_table("zpos", span).view(np.uint32), zp.view(np.uint32))
        assert np.array_equal(H.lm_table("zpos2", span).view(np.uint32), zp2.view(np.uint32))
        z0, zm, off = O.segments()
        assert np.array_equal(H.lm_table("segz0", span), z0)
        assert np.array_equal(H.lm_table("segzmax", span), zm)
        assert np.array_equal(H.lm_table("segzoffset", span), off)


def test_convert_span9_folds_the_span3_histogram_into_span9():
    """convert_span9 (convert_span9.cpp:13) of the span-3 trues equals the
    span-9 rebinning of the same events, bin for bin: the fold's segment
    grouping and plane offsets agree with the span-9 LUT."""
    from test_listmode_gpu import random_stream
    w = random_stream(5, 200_000)
    s3, d3, _ = LMOracle(3).histogram(w)
    s9, d9, _ = LMOracle(9).histogram(w)
    t3 = (s3.view(np.int16) - d3.view(np.int16)).astype(np.int16)
    t9 = (s9.view(np.int16) - d9.view(np.int16)).astype(np.int16)
    got = lm.convert_span9(t3)
    assert got.size == LMOracle(9).sino_size
    assert np.count_nonzero(t9) > 10_000 and np.array_equal(got, t9)


def test_convert_span9_known_planes():
    """Span-9 segment 0 plane q = span-3 segment 0 plane q + segments -1 and
    +1 (203 planes each, after 207) at plane q - 2; segment -1 of span 9
    (197 planes, after 207) starts with span-3 segment -2 (after 207+2*203)."""
    t3 = np.zeros(6367 * SINO_PLANE, np.int16)
    planes = t3.reshape(6367, SINO_PLANE)
    planes[10, 0] = 1
    planes[207 + 8, 0] = 10
    planes[207 + 203 + 8, 0] = 100
    planes[207 + 2 * 203 + 4, 5] = 7
    planes[0, 1] = 32767
    planes[207 + 0, 1] = 1   # segment -1 plane 0 -> span-9 plane 2
    planes[2, 1] = 32767
    got = lm.convert_span9(t3).reshape(2209, SINO_PLANE)
    assert got[10, 0] == 111
    assert got[207 + 4, 5] == 7
    assert got[0, 1] == 32767 and got[2, 1] == -32768  # 16-bit wrap


def test_library_convert_span9_matches_oracle():
    """The library's host fold (hrrt_lm_convert_span9) against the oracle's
    in-place restatement over the full int16 range, with and without the
    delayed subtraction."""
    import hrrt_reconstruction_b200 as H
    rng = np.random.default_rng(3)
    a = rng.integers(-32768, 32768, 6367 * SINO_PLANE, dtype=np.int16)
    d = rng.integers(-32768, 32768, a.size, dtype=np.int16)
    assert np.array_equal(H.convert_span9(a, d), lm.convert_span9((a - d).astype(np.int16)))
    assert np.array_equal(H.convert_span9(a), lm.convert_span9(a))
    with pytest.raises(H.HrrtError):
        H.convert_span9(a, maxrd=66)


def test_frames_at_file_offsets_sum_to_one_pass():
    """Packets count from the file start (LM_Reader_mp.cpp:124): frames
    histogrammed at their file offsets add up, bin for bin and count for
    count, to one pass over the file -- with lone out-of-sync words that put
    the stream at odd word positions across packet boundaries."""
    from test_listmode_gpu import random_stream
    O = LMOracle(9)
    w = random_stream(9, 1_100_000, tag_every=100, p_resync=2e-3)
    assert w.size > lm.PACKET_WORDS
    O.reset_clock()
    s1, d1, st1 = O.histogram(w)
    O.reset_clock()
    s = np.zeros_like(s1)
    d = np.zeros_like(d1)
    pos, frames = 0, []
    while pos < w.size:
        _, _, st = O.histogram(w[pos:], duration=2, sino=s, delayed=d, offset=pos)
        frames.append(st)
        pos += st["words_used"]
        if not st["terminated"]:
            break
    assert len(frames) > 3
    assert np.array_equal(s, s1) and np.array_equal(d, d1)
    for k in ("prompts", "delayed", "resyncs", "invalid", "tags"):
        assert sum(f[k] for f in frames) == st1[k], k


def test_seek_known_answer(O3):
    """goto_event: time tags at 5000, 5001, ... ms with 3 events between;
    a seek to 7 s stops just past the 7000-ms tag and sets the clock's second;
    a seek to 0 needs the 0-ms tag; without one the stream ends first."""
    ev = interleave(*event_words(np.array([1, 1, 1]), np.array([3, 4, 5]), np.array([10, 10, 10]),
                                 np.array([3, 4, 5]), np.array([10, 10, 10])))
    parts = []
    for ms in range(5000, 8000):
        parts.append(interleave(*tag_words(np.uint32(0x80000000 | ms))))
        parts.append(ev)
    w = np.concatenate(parts).astype(np.uint32)
    per = 2 + ev.size
    O3.reset_clock()
    n = O3.seek(w, 7)
    assert n == (7000 - 5000) * per + 2
    assert O3.clock.current_time == 7
    O3.reset_clock()
    assert O3.seek(w, 0) == -1
    w0 = np.concatenate([ev, interleave(*tag_words(np.uint32(0x80000000))), ev]).astype(np.uint32)
    O3.reset_clock()
    assert O3.seek(w0, 0) == ev.size + 2 and O3.clock.current_time == 0
    assert O3.seek(w0, 0, flags=lm.TIME_FROM_COUNT) == 0
