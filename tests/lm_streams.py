"""Seeded l64 event streams shared by the listmode tests (the word layout of
histogram_mp.cpp:1026-1233, built with oracle/lm.py's word builders)."""
import numpy as np

from oracle.lm import event_words, interleave, tag_words

PACKET_WORDS = 2 << 20  # the reader's packet: 1 Mi 64-bit events (LM_Reader_mp.hpp, PACKET_SIZE)


def random_stream(seed, nevents, tag_every=1000, p_resync=1e-4, p_bad=0.01, p_delayed=0.1, ms0=5000, doi7=True):
    """Seeded l64 words: coincidences (10 % delayed) with random head pairs,
    crystals and DOI (mostly valid), a time tag every `tag_every` events
    counting milliseconds from `ms0` (5 s), block-singles tags, lone
    out-of-sync words.  doi7=False leaves out transmission-flagged (DOI 7)
    events, which the reference's emission path cannot take."""
    rng = np.random.default_rng(seed)
    mp = rng.integers(1, 21, nevents)
    ax, bx = rng.integers(0, 72, nevents), rng.integers(0, 72, nevents)
    ay, by = rng.integers(0, 104, nevents), rng.integers(0, 104, nevents)
    doia = rng.choice([0, 1], nevents)
    doib = rng.choice([0, 1], nevents)
    bad = rng.random(nevents) < p_bad
    kind = rng.integers(0, 5, nevents)
    mp = np.where(bad & (kind == 0), rng.choice([0, 21, 40], nevents), mp)
    ax = np.where(bad & (kind == 1), rng.integers(72, 256, nevents), ax)
    by = np.where(bad & (kind == 2), rng.integers(104, 256, nevents), by)
    doia = np.where(bad & (kind == 3), rng.integers(2, 8 if doi7 else 7, nevents), doia)
    doib = np.where(bad & (kind == 4), 7 if doi7 else 5, doib)
    prompt = rng.random(nevents) >= p_delayed
    ew1, ew2 = event_words(mp, ax, ay, bx, by, doia, doib, prompt)
    ev = interleave(ew1, ew2).reshape(-1, 2)
    # insert tags and lone words
    chunks = []
    ms = ms0
    for i in range(0, nevents, tag_every):
        t1, t2 = tag_words(np.uint32(0x80000000 | ms))
        chunks.append(np.array([[t1, t2]], np.uint32).reshape(-1))
        ms += 1
        if (i // tag_every) % 7 == 3:
            s1, s2 = tag_words(np.uint32(0xA0000000 | (i & 0x7ffff)))
            chunks.append(np.array([s1, s2], np.uint32))
        block = ev[i:i + tag_every].reshape(-1).copy()
        chunks.append(block)
        if rng.random() < p_resync * tag_every:
            chunks.append(np.array([0x00000000], np.uint32))
    return np.concatenate(chunks).astype(np.uint32)


def whole_packets(words, npackets):
    """The first `npackets` whole reader packets of a stream."""
    assert words.size >= npackets * PACKET_WORDS
    return np.ascontiguousarray(words[:npackets * PACKET_WORDS])
