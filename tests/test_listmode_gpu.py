"""Device listmode histogrammer (hrrt_lm_* through the C ABI) against the CPU
restatement oracle/lm_oracle.c: sinograms bit-identical, statistics equal,
on the known-answer streams and on seeded random streams that mix every word
class, several packets, a partial last packet and frame ends."""
import numpy as np
import pytest

from oracle import lm
from lm_streams import random_stream
from oracle.lm import LMOracle, event_words, interleave, tag_words

pytestmark = pytest.mark.gpu

STAT_KEYS = ("words_used", "prompts", "delayed", "timetags", "tags", "invalid", "unmapped", "doi_other", "doi7",
             "resyncs", "frame_start", "duration", "terminated")


FORCE_DIRECT, FORCE_PARTITIONED, FORCE_WIDE = 16, 32, 64  # device path selection (same result)
PATHS = (FORCE_DIRECT, FORCE_PARTITIONED, FORCE_WIDE)


def compare(O, D, words, mode, duration=0, flags=0, path=0):
    O.reset_clock()
    D.reset_clock()
    so, do, sto = O.histogram(words, mode=mode, duration=duration, flags=flags)
    sd, dd, std = D.histogram(words, mode=mode, duration=duration, flags=flags | path)
    assert np.array_equal(so, sd), np.flatnonzero(so != sd)[:10]
    if mode == lm.PROMPTS_AND_DELAYED:
        assert np.array_equal(do, dd), np.flatnonzero(do != dd)[:10]
    for k in STAT_KEYS:
        assert sto[k] == std[k], (k, sto[k], std[k])
    return sto


@pytest.fixture(scope="module", params=[3, 9])
def pair(request):
    import hrrt_reconstruction_b200 as H
    O = LMOracle(request.param)
    D = H.Listmode(request.param)
    yield O, D
    D.close()


def test_known_answer_streams(pair):
    O, D = pair
    good = event_words(3, 35, 50, 35, 50)
    dly = event_words(3, 35, 50, 35, 50, prompt=False)
    w = np.concatenate([interleave(np.atleast_1d(a), np.atleast_1d(b)) for a, b in (
        good, dly, (np.uint32(0), np.uint32(0)), event_words(0, 35, 50, 35, 50), event_words(3, 72, 50, 35, 50),
        event_words(3, 35, 50, 35, 50, doia=3), event_words(3, 35, 50, 35, 50, doib=7), tag_words(0xA0000005),
        tag_words(0x40000000 | 12345), tag_words(777), good)]).astype(np.uint32)
    for mode in (lm.TRUES, lm.PROMPTS_AND_DELAYED, lm.PROMPTS_ONLY):
        for path in PATHS:
            compare(O, D, w, mode, path=path)


def test_wrap_and_trues(pair):
    O, D = pair
    n = 70000
    ew1, ew2 = event_words(np.full(n, 3), np.full(n, 20), np.full(n, 60), np.full(n, 50), np.full(n, 61),
                           prompt=np.arange(n) % 3 != 0)
    w = interleave(ew1, ew2)
    for mode in (lm.TRUES, lm.PROMPTS_AND_DELAYED):
        for path in PATHS:
            compare(O, D, w, mode, path=path)


@pytest.mark.parametrize("seed", [1, 2])
def test_random_stream_packets(pair, seed):
    """About 2.6 packets of mixed words; whole stream and 2-s frames."""
    O, D = pair
    w = random_stream(seed, 2_700_000)
    assert w.size > 2 * lm.PACKET_WORDS
    st = compare(O, D, w, lm.PROMPTS_AND_DELAYED, path=FORCE_DIRECT)
    assert st["prompts"] > 0 and st["resyncs"] > 0 and st["invalid"] > 0 and st["doi7"] > 0
    compare(O, D, w, lm.PROMPTS_AND_DELAYED, path=FORCE_PARTITIONED)
    compare(O, D, w, lm.PROMPTS_AND_DELAYED, path=FORCE_WIDE)
    compare(O, D, w, lm.TRUES, flags=lm.IGNORE_BORDER_CRYSTAL, path=FORCE_PARTITIONED)
    compare(O, D, w, lm.TRUES, flags=lm.IGNORE_BORDER_CRYSTAL, path=FORCE_WIDE)
    compare(O, D, w, lm.PROMPTS_ONLY, flags=lm.NO_DOI, path=FORCE_PARTITIONED)
    compare(O, D, w, lm.PROMPTS_ONLY, flags=lm.NO_DOI, path=FORCE_WIDE)


def test_frames_follow_the_clock(pair):
    """Consecutive 1-s frames (1000 tags each): every frame bit-identical and
    the clock carried from one call to the next."""
    O, D = pair
    w = random_stream(3, 2_500_000, tag_every=800)
    O.reset_clock()
    D.reset_clock()
    pos_o = pos_d = 0
    for k in range(3):
        so, do, sto = O.histogram(w[pos_o:], duration=1)
        sd, dd, std = D.histogram(w[pos_d:], duration=1, flags=PATHS[k % 3])
        assert np.array_equal(so, sd) and np.array_equal(do, dd)
        for key in STAT_KEYS:
            assert sto[key] == std[key], (key, sto[key], std[key])
        assert sto["terminated"] == 1
        pos_o += sto["words_used"]
        pos_d += std["words_used"]


def test_device_entry_adds_into_buffers(pair):
    import torch
    O, D = pair
    w = random_stream(4, 300_000)
    O.reset_clock()
    so, do, _ = O.histogram(w)
    dw = torch.from_numpy(w.view(np.int32)).cuda()
    ds = torch.zeros(D.sino_size, dtype=torch.int16, device="cuda")
    dd = torch.zeros(D.sino_size, dtype=torch.int16, device="cuda")
    for path in (FORCE_DIRECT, FORCE_WIDE):
        D.reset_clock()
        D.histogram_device(dw.data_ptr(), w.size, ds.data_ptr(), dd.data_ptr(), flags=path)
    torch.cuda.synchronize()
    got_s = ds.cpu().numpy().view(np.uint16)
    got_d = dd.cpu().numpy().view(np.uint16)
    assert np.array_equal(got_s, (2 * so.astype(np.uint32)).astype(np.uint16))
    assert np.array_equal(got_d, (2 * do.astype(np.uint32)).astype(np.uint16))


def singles_stream(seed, nevents, tag_every=700, ms0=5000):
    """random_stream's events with block singles tags (random blocks and
    rates) after every time tag, and a clock that skips a millisecond now and
    then."""
    rng = np.random.default_rng(seed)
    base = random_stream(seed, nevents, tag_every=tag_every, p_resync=0.0, ms0=ms0)
    out = []
    i = 0
    while i < base.size:
        if i + 1 < base.size and (base[i] >> 30) == 1 and (base[i + 1] >> 30) == 3:
            out.append(base[i:i + 2])
            tag = (int(base[i]) & 0xffff) | ((int(base[i + 1]) & 0xffff) << 16)
            if (tag & 0xE0000000) == 0x80000000:
                for _ in range(int(rng.integers(0, 4))):
                    blk = int(rng.integers(0, 936))
                    val = int(rng.integers(0, 1 << 19))
                    s1, s2 = tag_words(np.uint32(0xA0000000 | (blk << 19) | val))
                    out.append(np.array([s1, s2], np.uint32))
            i += 2
        else:
            out.append(base[i:i + 1])
            i += 1
    return np.concatenate(out).astype(np.uint32)


@pytest.mark.parametrize("path", PATHS)
def test_head_curve_and_block_singles(pair, path):
    """LM_HEAD_CURVE | LM_CRYSTAL_COUNTS: the per-second lines, the block
    singles averages, the line totals and the coincidence histogram equal the
    oracle's (whole stream, then 1-s frames)."""
    import hrrt_reconstruction_b200 as H
    O, D = pair
    w = singles_stream(11, 2_200_000)
    for duration in (0, 1):
        O.reset_clock()
        D.reset_clock()
        pos = 0
        for k in range(2 if duration else 1):
            so, do, sto, hco, rates_o, tot_o = O.histogram_hc(w[pos:], duration=duration)
            sd, dd, std = D.histogram(w[pos:], duration=duration,
                                      flags=path | H.LM_HEAD_CURVE | H.LM_CRYSTAL_COUNTS)
            assert np.array_equal(so, sd) and np.array_equal(do, dd)
            for key in STAT_KEYS:
                assert sto[key] == std[key], (key, sto[key], std[key])
            hcd = D.head_curve()
            rates_d, tot_d = D.block_singles()
            assert hco.shape[0] > 0
            assert np.array_equal(hcd, hco), (hcd[:3], hco[:3])
            assert np.array_equal(rates_d, rates_o)
            assert tot_d == tot_o
            cc = D.crystal_counts()
            assert cc.sum() > 0 and np.array_equal(cc, O.last_crystal_counts)
            pos += sto["words_used"]


def test_trues_span9_device(pair):
    """hrrt_lm_trues_span9_device: the device histograms' prompts - delayed
    folded into span 9 equal the oracle's convert_span9 of the same trues and
    the library's host fold; full-range random planes wrap like shorts."""
    import torch
    import hrrt_reconstruction_b200 as H
    O, D = pair
    S = D.sino_size
    if O.span != 3:
        buf = torch.zeros(8, dtype=torch.int16, device="cuda")
        with pytest.raises(H.HrrtError):
            D.trues_span9_device(buf.data_ptr(), 0, buf.data_ptr())
        return
    w = random_stream(21, 400_000)
    D.reset_clock()
    dw = torch.from_numpy(w.view(np.int32)).cuda()
    ds = torch.zeros(S, dtype=torch.int16, device="cuda")
    dd = torch.zeros(S, dtype=torch.int16, device="cuda")
    D.histogram_device(dw.data_ptr(), w.size, ds.data_ptr(), dd.data_ptr())
    out = torch.empty(2209 * 288 * 256, dtype=torch.int16, device="cuda")
    D.trues_span9_device(ds.data_ptr(), dd.data_ptr(), out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    p, d = ds.cpu().numpy(), dd.cpu().numpy()
    want = lm.convert_span9((p - d).astype(np.int16))
    assert np.count_nonzero(want) > 10_000 and np.array_equal(got, want)
    assert np.array_equal(got, H.convert_span9(p, d))
    rng = np.random.default_rng(4)
    a = rng.integers(-32768, 32768, S, dtype=np.int16)
    ds.copy_(torch.from_numpy(a))
    D.trues_span9_device(ds.data_ptr(), 0, out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), lm.convert_span9(a))


@pytest.mark.parametrize("path", PATHS)
def test_frames_at_file_offsets(pair, path):
    """hrrt_lm_histogram_at: 2-s frames of a stream with lone out-of-sync
    words, each histogrammed at its file offset (packets counted from the
    file start), equal the oracle's frame for frame; so does a seek
    (goto_event) to 6 s followed by a frame."""
    O, D = pair
    w = random_stream(9, 1_100_000, tag_every=100, p_resync=2e-3)
    O.reset_clock()
    D.reset_clock()
    pos, nframes = 0, 0
    while pos < w.size:
        so, do, sto = O.histogram(w[pos:], duration=2, offset=pos)
        sd, dd, std = D.histogram(w[pos:], duration=2, flags=path, offset=pos)
        assert np.array_equal(so, sd) and np.array_equal(do, dd), (nframes, pos)
        for k in STAT_KEYS:
            assert sto[k] == std[k], (nframes, k, sto[k], std[k])
        pos += sto["words_used"]
        nframes += 1
        if not sto["terminated"]:
            break
    assert nframes > 3
    O.reset_clock()
    D.reset_clock()
    n_o = O.seek(w, 6)
    n_d = D.seek(w, 6)
    assert n_o == n_d > 0
    so, do, sto = O.histogram(w[n_o:], duration=1, offset=n_o)
    sd, dd, std = D.histogram(w[n_d:], duration=1, flags=path, offset=n_d)
    assert np.array_equal(so, sd) and np.array_equal(do, dd)
    assert sto["frame_start"] == std["frame_start"] == 6
    import hrrt_reconstruction_b200 as H
    with pytest.raises(H.HrrtError):
        D.seek(w, 10_000)


@pytest.mark.parametrize("offset", [0, 12345])
def test_streamed_chunks_equal_one_pass(pair, offset):
    """Host streams longer than a chunk (here one packet, 2 Mi words) are
    histogrammed chunk by chunk while the next chunk uploads: the whole
    stream, and 1-s frames that straddle chunk ends, equal the oracle's one
    pass bit for bit, counters included (file offsets with an odd packet
    phase too)."""
    import hrrt_reconstruction_b200 as H
    O, D = pair
    w = random_stream(17, 3_000_000, tag_every=1000, p_resync=1e-3)
    assert w.size > 2 * lm.PACKET_WORDS  # three chunks
    try:
        D.set_chunk(lm.PACKET_WORDS)
        with pytest.raises(H.HrrtError):
            D.set_chunk(lm.PACKET_WORDS + 4)
        for mode in (lm.PROMPTS_AND_DELAYED, lm.TRUES):
            O.reset_clock()
            D.reset_clock()
            so, do, sto = O.histogram(w, mode=mode, offset=offset)
            sd, dd, std = D.histogram(w, mode=mode, offset=offset)
            assert np.array_equal(so, sd)
            if mode == lm.PROMPTS_AND_DELAYED:
                assert np.array_equal(do, dd)
            for k in STAT_KEYS:
                assert sto[k] == std[k], (mode, k, sto[k], std[k])
        O.reset_clock()
        D.reset_clock()
        pos, nframes = 0, 0
        while pos < w.size:
            so, do, sto = O.histogram(w[pos:], duration=1, offset=offset + pos)
            sd, dd, std = D.histogram(w[pos:], duration=1, offset=offset + pos)
            assert np.array_equal(so, sd) and np.array_equal(do, dd), nframes
            for k in STAT_KEYS:
                assert sto[k] == std[k], (nframes, k, sto[k], std[k])
            pos += sto["words_used"]
            nframes += 1
            if not sto["terminated"]:
                break
        assert nframes >= 2
    finally:
        D.set_chunk(0)
