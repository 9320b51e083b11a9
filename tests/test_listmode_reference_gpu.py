"""The device listmode histogrammer against the reference's OWN histogrammer
(oracle/_ref/lmhist_ref: histogram_mp.cpp, LM_Reader_mp.cpp,
LM_Rebinner_mp.cpp and the LUT code compiled unmodified), through the C ABI,
bit for bit: span-3 and span-9 frames of seeded streams that mix every word
class the reference's emission path accepts (lone out-of-sync words, invalid
head pairs and crystals, other DOI values, block-singles tags), in
prompts-and-delayed, trues and prompts-only modes, on each device path; the
head curve, the block singles and -- where the reference's reader cuts its
packet at the frame end -- the coincidence histogram.
"""
import numpy as np
import pytest

from lm_streams import random_stream, whole_packets
from oracle import lm
from oracle import lm_ref

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not lm_ref.available(), reason="oracle/_ref/lmhist_ref not built")]

FORCE_DIRECT, FORCE_PARTITIONED, FORCE_WIDE = 16, 32, 64
HEAD_CURVE, CRYSTAL_COUNTS = 128, 256


def stream(seed, p_resync=1e-4):
    return whole_packets(random_stream(seed, 3 * 1_050_000, p_resync=p_resync, doi7=False), 3)


@pytest.mark.parametrize("span,mode,path", [
    (3, lm.PROMPTS_AND_DELAYED, FORCE_DIRECT),
    (3, lm.PROMPTS_AND_DELAYED, FORCE_WIDE),
    (9, lm.PROMPTS_AND_DELAYED, FORCE_PARTITIONED),
    (9, lm.TRUES, FORCE_DIRECT),
    (9, lm.PROMPTS_ONLY, FORCE_WIDE),
])
def test_device_frame_equals_reference(span, mode, path):
    import hrrt_reconstruction_b200 as H
    w = stream(100 + span + mode)
    R = lm_ref.histogram(w, span=span, mode=mode, duration=2)
    with H.Listmode(span) as D:
        D.reset_clock()
        s, d, st = D.histogram(w, mode=mode, duration=2, flags=path | HEAD_CURVE)
        assert st["frame_start"] == R["frame_start"] and st["duration"] == R["duration"]
        assert np.array_equal(s.view(np.int16), R["prompts"]), np.flatnonzero(s.view(np.int16) != R["prompts"])[:10]
        if mode == lm.PROMPTS_AND_DELAYED:
            assert np.array_equal(d.view(np.int16), R["delayed"])
        hc = D.head_curve()
        text = "Singles,Randoms,Prompts,Time(ms)\n" + "".join(f"{x[3]},{x[2]},{x[1]},{x[0]}" for x in hc.tolist())
        assert R["hc"] == text
        rates, totals = D.block_singles()
        assert np.array_equal(rates, R["singles"])
        assert tuple(int(t) for t in totals) == (R["total_prompts"], R["total_randoms"])


def test_device_coincidence_histogram_equals_reference():
    import hrrt_reconstruction_b200 as H
    w = stream(7, p_resync=0.0)
    R = lm_ref.histogram(w, span=9, mode=lm.PROMPTS_AND_DELAYED, duration=2, coinc=True)
    with H.Listmode(9) as D:
        D.reset_clock()
        D.histogram(w, mode=lm.PROMPTS_AND_DELAYED, duration=2, flags=CRYSTAL_COUNTS)
        cc = D.crystal_counts()
    assert np.array_equal(lm_ref.coinc_in_reference_layout(cc), R["coinc"].astype(np.uint64))
