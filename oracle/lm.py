"""ctypes binding of the listmode histogrammer restatement oracle/lm_oracle.c.

TEST INFRASTRUCTURE.  Only tests/ and bench.py's cpu_baseline leg use it, as
the checker.  Built by `make -C oracle oracle` (on demand).
"""
import ctypes
import os

import numpy as np

from oracle.oracle import build as _build

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liblm_oracle.so")

TRUES, PROMPTS_AND_DELAYED, PROMPTS_ONLY = 0, 1, 2
IGNORE_BORDER_CRYSTAL, NO_DOI, TIME_FROM_COUNT = 1, 2, 4
PACKET_WORDS = 2 * 1024 * 1024
NXD = 144

SOL = np.dtype([("nsino", np.int32), ("d", np.float32), ("z", np.float32)])


class Clock(ctypes.Structure):
    _fields_ = [("current_time", ctypes.c_longlong), ("current_time_msec", ctypes.c_longlong),
                ("prev_time", ctypes.c_longlong), ("clock_reset", ctypes.c_int), ("pad", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_longlong) for n in ("words_used", "prompts", "delayed", "timetags", "tags", "invalid",
                                                  "unmapped", "doi_other", "doi7", "resyncs", "frame_start",
                                                  "duration")] + [("terminated", ctypes.c_int), ("pad", ctypes.c_int)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_ if n != "pad"}


_L = None


def lib():
    global _L
    if _L is None:
        if not os.path.exists(LIB):
            _build()
        L = ctypes.CDLL(LIB)
        vp, i = ctypes.c_void_p, ctypes.c_int
        L.lm_create.argtypes = [i, i]
        L.lm_create.restype = vp
        L.lm_destroy.argtypes = [vp]
        L.lm_destroy.restype = None
        L.lm_sino_size.argtypes = [vp]
        L.lm_sino_size.restype = ctypes.c_longlong
        L.lm_nplanes.argtypes = [vp]
        L.lm_d_tan_theta.argtypes = [vp]
        L.lm_d_tan_theta.restype = ctypes.c_double
        for n, a in {"lm_get_sol": [vp, vp], "lm_get_zpos": [vp, vp, vp], "lm_get_seg": [vp, vp, vp, vp, vp],
                     "lm_get_crystals": [vp, vp], "lm_clock_init": [vp]}.items():
            getattr(L, n).argtypes = a
            getattr(L, n).restype = None
        L.lm_rebin_event.argtypes = [vp, i, i, i, i, i, i, i]
        L.lm_rebin_events.argtypes = [vp, ctypes.c_longlong, vp, vp]
        L.lm_rebin_events.restype = None
        L.lm_histogram.argtypes = [vp, vp, ctypes.c_longlong, i, i, i, vp, vp, vp, vp]
        f = ctypes.c_float
        L.lm_histogram_hc.argtypes = [vp, vp, ctypes.c_longlong, ctypes.c_longlong, i, i, i, vp, vp, vp, vp, vp, i,
                                      vp, vp, vp]
        L.lm_seek.argtypes = [vp, ctypes.c_longlong, ctypes.c_longlong, i, i, vp]
        L.lm_histogram_at.argtypes = [vp, vp, ctypes.c_longlong, ctypes.c_longlong, i, i, i, vp, vp, vp, vp]
        L.lm_seek.restype = ctypes.c_longlong
        L.lm_crystal_singles.argtypes = [vp, f, f, vp]
        L.lm_smooth_randoms.argtypes = [vp, vp, f, f, i, vp]
        L.lm_convert_span9.argtypes = [vp, i, i]
        L.lm_convert_span9.restype = None
        _L = L
    return _L


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class LMOracle:
    """LUT + histogrammer for one output span (3 or 9), maxrd 67."""

    def __init__(self, span=3, maxrd=67):
        self.L = lib()
        self.t = self.L.lm_create(span, maxrd)
        if not self.t:
            raise ValueError("unsupported span")
        self.span = span
        self.sino_size = self.L.lm_sino_size(self.t)
        self.nplanes = self.L.lm_nplanes(self.t)
        self.clock = Clock()
        self.L.lm_clock_init(ctypes.byref(self.clock))

    def __del__(self):
        t, self.t = getattr(self, "t", None), None
        if t:
            self.L.lm_destroy(t)

    def reset_clock(self):
        self.L.lm_clock_init(ctypes.byref(self.clock))

    def sol(self):
        a = np.zeros((21, NXD, NXD), SOL)
        self.L.lm_get_sol(self.t, _p(a))
        return a

    def zpos(self):
        a = np.zeros(104, np.float32)
        b = np.zeros(104, np.float32)
        self.L.lm_get_zpos(self.t, _p(a), _p(b))
        return a, b

    def segments(self):
        z0, zm, off = (np.zeros(63, np.int32) for _ in range(3))
        n = ctypes.c_int()
        self.L.lm_get_seg(self.t, _p(z0), _p(zm), _p(off), ctypes.byref(n))
        k = n.value
        return z0[:k], zm[:k], off[:k]

    def crystals(self):
        a = np.zeros((8, 2, 72, 104, 3), np.float32)
        self.L.lm_get_crystals(self.t, _p(a))
        return a

    def rebin_event(self, mp, al, ax, ay, bl, bx, by):
        return self.L.lm_rebin_event(self.t, mp, al, ax, ay, bl, bx, by)

    def rebin_events(self, ev):
        """rebin_event for each row (mp, al, ax, ay, bl, bx, by) of int32 [n][7]"""
        ev = np.ascontiguousarray(ev, np.int32)
        out = np.empty(ev.shape[0], np.int32)
        self.L.lm_rebin_events(self.t, ev.shape[0], _p(ev), _p(out))
        return out

    def histogram(self, words, mode=PROMPTS_AND_DELAYED, duration=0, flags=0, sino=None, delayed=None, offset=0):
        """-> (sino, delayed, stats dict); adds into sino/delayed when given;
        `offset`: the position of words[0] in the file (packets count from
        its start)."""
        w = np.ascontiguousarray(words, np.uint32)
        if sino is None:
            sino = np.zeros(self.sino_size, np.uint16)
        if delayed is None and mode == PROMPTS_AND_DELAYED:
            delayed = np.zeros(self.sino_size, np.uint16)
        st = Stats()
        self.L.lm_histogram_at(self.t, _p(w), w.size, offset, mode, duration, flags, ctypes.byref(self.clock),
                               _p(sino), _p(delayed), ctypes.byref(st))
        return sino, delayed, st.as_dict()

    def histogram_hc(self, words, mode=PROMPTS_AND_DELAYED, duration=0, flags=0, max_lines=1 << 20, offset=0):
        """histogram() that also returns the frame's head curve (int64 [n][4]:
        time ms, prompts, randoms, total singles), the blocks' average singles
        rates [936] and the totals of the lines' prompts and randoms; the
        coincidence histogram is left in self.last_crystal_counts.  `offset`:
        the position of words[0] in the file (packets count from its start)."""
        w = np.ascontiguousarray(words, np.uint32)
        sino = np.zeros(self.sino_size, np.uint16)
        delayed = np.zeros(self.sino_size, np.uint16) if mode == PROMPTS_AND_DELAYED else None
        st = Stats()
        hc = np.zeros((max_lines, 4), np.int64)
        rates = np.zeros(936, np.int32)
        tot = np.zeros(2, np.int64)
        cc = np.zeros(2 * NCRYSTALS, np.uint32)
        n = self.L.lm_histogram_hc(self.t, _p(w), w.size, offset, mode, duration, flags, ctypes.byref(self.clock),
                                   _p(sino), _p(delayed), ctypes.byref(st), _p(hc), max_lines, _p(rates), _p(tot),
                                   _p(cc))
        self.last_crystal_counts = cc
        return sino, delayed, st.as_dict(), hc[:min(n, max_lines)].copy(), rates, (int(tot[0]), int(tot[1]))

    def seek(self, words, target, offset=0, flags=0):
        """goto_event: words consumed up to the time tag reaching `target` s
        (the 0-ms tag for 0), -1 when the stream ends first."""
        w = np.ascontiguousarray(words, np.uint32)
        return self.L.lm_seek(_p(w), w.size, offset, target, flags, ctypes.byref(self.clock))


NCRYSTALS = 2 * 104 * 8 * 72  # [layer][ring][head][x]


def crystal_singles(delayed_counts, scan_duration=1.0, tau=6.0e-9):
    """gen_delays' crystal singles estimate (gen_delays_lib.cpp:163-255):
    -> (singles float32 [119808], iterations)."""
    d = np.ascontiguousarray(delayed_counts, np.int32).reshape(-1)
    assert d.size == NCRYSTALS
    out = np.zeros(NCRYSTALS, np.float32)
    it = lib().lm_crystal_singles(_p(d), tau, scan_duration, _p(out))
    return out, it


def smooth_randoms(oracle, coinc_hist, scan_duration=1.0, tau=6.0e-9, maxrd=67):
    """gen_delays' randoms sinogram (float32, the oracle's span) from a
    coincidence histogram [2][119808] int32 -> (sino, iterations)."""
    h = np.ascontiguousarray(coinc_hist, np.int32).reshape(-1)
    assert h.size == 2 * NCRYSTALS
    out = np.zeros(oracle.sino_size, np.float32)
    it = lib().lm_smooth_randoms(oracle.t, _p(h), scan_duration, tau, maxrd, _p(out))
    return out, it


def convert_span9(span3, maxrd=67, nrings=104):
    """convert_span9: the span-3 int16 sinogram folded into span 9 (returns the
    2209 span-9 planes; 16-bit sums wrap)."""
    w = np.array(span3, np.int16).reshape(-1)
    lib().lm_convert_span9(_p(w), maxrd, nrings)
    return w[:2209 * 288 * 256].copy()


def delayed_counts_from_singles(singles, scan_duration=1.0, tau=6.0e-9):
    """The forward model the estimator inverts (compute_drate,
    gen_delays_lib.cpp:163-193), rounded to counts: a coincidence histogram's
    delayed half for known crystal singles rates."""
    s = np.asarray(singles, np.float64).reshape(2, 104, 8, 72)
    hsum = s.sum(axis=(0, 1, 3))
    facing = np.array([sum(hsum[(h + j + 2) % 8] for j in range(5)) for h in range(8)])
    rate = s * tau * facing[None, None, :, None]
    return np.floor(rate * scan_duration + 0.5).astype(np.int32).reshape(-1)


# ---- word builders (the l64 event layout, histogram_mp.cpp:1026-1233) ----
def event_words(mp, ax, ay, bx, by, doia=0, doib=0, prompt=True):
    """(ew1, ew2) of one coincidence: ew1 top bits 00; ew2 top bits 11
    (prompt) or 10 (delayed); head pair mp in bits 16-18 of ew1 (low 3 bits)
    and of ew2 (high 3 bits); DOI in bits 22-24; crystal x in bits 0-7 and y in
    bits 8-15."""
    mp = np.asarray(mp, np.uint32)
    ew1 = (np.asarray(ax, np.uint32) & 0xff) | ((np.asarray(ay, np.uint32) & 0xff) << 8) | ((mp & 7) << 16) | \
        ((np.asarray(doia, np.uint32) & 7) << 22)
    top = np.where(np.asarray(prompt), np.uint32(0xC0000000), np.uint32(0x80000000)).astype(np.uint32)
    ew2 = (np.asarray(bx, np.uint32) & 0xff) | ((np.asarray(by, np.uint32) & 0xff) << 8) | (((mp >> 3) & 7) << 16) | \
        ((np.asarray(doib, np.uint32) & 7) << 22) | top
    return ew1.astype(np.uint32), ew2.astype(np.uint32)


def tag_words(tag):
    """(ew1, ew2) of a tag word carrying the 32-bit value `tag` (ew1 top
    bits 01, ew2 top bits 11)."""
    tag = np.asarray(tag, np.uint32)
    ew1 = np.uint32(0x40000000) | (tag & 0xffff)
    ew2 = np.uint32(0xC0000000) | ((tag >> 16) & 0xffff)
    return ew1.astype(np.uint32), ew2.astype(np.uint32)


def interleave(ew1, ew2):
    out = np.empty(2 * np.size(ew1), np.uint32)
    out[0::2] = ew1
    out[1::2] = ew2
    return out
