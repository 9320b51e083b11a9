"""ctypes binding of oracle/_ref/libhrrt_ref.so -- the reference's OWN projector.

TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py (its
reference arm and cpu_baseline leg) use this module, as the checker / CPU
baseline.  The library is built by oracle/Makefile from the unmodified
reference sources (hrrt_osem3d/hrrt_osem3dv_sbrt_span3.cpp, nr_utils.cpp,
psf.cpp, scanner_model.cpp) plus oracle/ref_harness.cpp, and travels prebuilt.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libhrrt_ref.so")


def available():
    return os.path.exists(REF_LIB)


_L = None


def lib():
    global _L
    if _L is None:
        if not available():
            raise FileNotFoundError(REF_LIB)
        L = ctypes.CDLL(REF_LIB)
        vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.ref_init.argtypes = [i, i, i, f, f, f, i, i, i, i]
        L.ref_init.restype = i
        for n in ("ref_fp_pair", "ref_bp_pair", "ref_rotate_add"):
            getattr(L, n).argtypes = [vp, i, vp]
            getattr(L, n).restype = i
        L.ref_sensitivity.argtypes = [vp, vp, i]
        L.ref_osem_subset.argtypes = [vp, vp, vp, vp, vp, i, i]
        L.ref_post_iteration.argtypes = [vp, i, i]
        L.ref_post_iteration.restype = ctypes.c_double
        L.ref_init_image.argtypes = [vp, i, i]
        L.ref_sequence.argtypes = [i, vp]
        for n in ("ref_get_segments", "ref_get_trig", "ref_get_tantheta", "ref_get_flookup", "ref_get_blookup"):
            getattr(L, n).restype = None
        L.ref_get_segments.argtypes = [vp, vp, vp]
        L.ref_get_cylwiny.argtypes = [vp]
        L.ref_get_trig.argtypes = [vp, vp, vp, vp]
        L.ref_get_tantheta.argtypes = [vp, vp]
        L.ref_get_flookup.argtypes = [vp, vp]
        L.ref_get_blookup.argtypes = [vp, vp, vp, vp]
        L.ref_psf_setup.argtypes = [f, f, f, vp, i]
        L.ref_psf_setup.restype = i
        L.ref_psf_convolve.argtypes = [vp, vp]
        L.ref_psf_convolve.restype = i
        L.ref_set_norm_zero_mask.argtypes = [vp]
        L.ref_get_norm_zero_mask.argtypes = [vp]
        _L = L
    return _L


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


class RefProjector:
    """The reference projector for one geometry (global state in the .so:
    creating a second RefProjector re-initialises the first)."""

    def __init__(self, nrings=104, nelements=256, nangles=288, ring_radius=234.5, plane_sep=1.21875,
                 binsize=1.21875, span=9, maxdel=67, subsets=16, nthreads=1):
        L = lib()
        rc = L.ref_init(nrings, nelements, nangles, ring_radius, plane_sep, binsize, span, maxdel, subsets,
                        nthreads)
        if rc != 0:
            raise RuntimeError("ref_init failed")
        self.L = L
        self.nthreads = nthreads
        self.P = L.ref_segmentsize()
        self.nseg = L.ref_th_pixels()
        self.groupmax = L.ref_groupmax()
        self.zp = L.ref_zp()
        self.nz = L.ref_z_pixels()
        self.nx = L.ref_x_pixels()
        self.views = L.ref_views()
        self.subsets = subsets
        self.sviews = L.ref_sviews()
        self.span = span
        # plane range after GetScannerParameter's adjustments (drv:3516,
        # :3537-3540) for the default -f ...,6,200 and -k 3
        z_min, z_max, npskip = 6, 200, 3
        if npskip > z_min:
            z_min = npskip
        if z_max > self.nz - npskip:
            z_max = self.nz - npskip
        self.z_min, self.z_max = z_min, z_max

    @property
    def image_shape(self):
        return (self.nx, self.nx, self.zp)

    @property
    def rows_shape(self):
        return (2 * self.P, self.nx)

    def fp_pair(self, img, view, prj=None):
        img = np.ascontiguousarray(img, np.float32)
        out = np.zeros(self.rows_shape, np.float32) if prj is None else np.array(prj, np.float32, copy=True)
        self.L.ref_fp_pair(_p(img), view, _p(out))
        return out

    def bp_pair(self, prj, view):
        prj = np.ascontiguousarray(prj, np.float32)
        out = np.zeros(self.image_shape, np.float32)
        self.L.ref_bp_pair(_p(prj), view, _p(out))
        return out

    def rotate_add(self, imagebuf, view, corr):
        ib = np.ascontiguousarray(imagebuf, np.float32)
        co = np.array(corr, np.float32, copy=True)
        self.L.ref_rotate_add(_p(ib), view, _p(co))
        return co

    def sensitivity(self, mult, nthreads=None):
        m = np.ascontiguousarray(mult, np.float32)
        out = np.zeros((self.subsets,) + self.image_shape, np.float32)
        self.L.ref_sensitivity(_p(m), _p(out), nthreads or self.nthreads)
        return out

    def osem_subset(self, image, nf_inv_subset, prompts, add, isubset, nthreads=None):
        """One OP-OSEM subset in place on `image` ([x][y][zp] float32)."""
        assert image.dtype == np.float32 and image.flags.c_contiguous
        corr = np.zeros(self.image_shape, np.float32)
        nf = np.ascontiguousarray(nf_inv_subset, np.float32)
        p = np.ascontiguousarray(prompts, np.int16)
        a = np.ascontiguousarray(add, np.float32)
        self.L.ref_osem_subset(_p(image), _p(corr), _p(nf), _p(p), _p(a), isubset, nthreads or self.nthreads)
        return image

    def post_iteration(self, image, zmin=None, zmax=None):
        zmin = self.z_min if zmin is None else zmin
        zmax = self.z_max if zmax is None else zmax
        assert 0 <= zmin <= zmax <= self.zp and image.dtype == np.float32 and image.flags.c_contiguous
        return self.L.ref_post_iteration(_p(image), zmin, zmax)

    def init_image(self, zmin=None, zmax=None):
        zmin = self.z_min if zmin is None else zmin
        zmax = self.z_max if zmax is None else zmax
        assert 0 <= zmin <= zmax <= self.zp
        out = np.zeros(self.image_shape, np.float32)
        self.L.ref_init_image(_p(out), zmin, zmax)
        return out

    def order(self):
        o = np.zeros(self.subsets, np.int16)
        self.L.ref_sequence(self.subsets, _p(o))
        return o

    # ---- geometry tables ----
    def segments(self):
        a = np.zeros((3, self.nseg), np.int32)
        self.L.ref_get_segments(_p(a[0]), _p(a[1]), _p(a[2]))
        return a

    def cylwiny(self):
        a = np.zeros((self.nx, 2), np.int16)
        self.L.ref_get_cylwiny(_p(a))
        return a

    def trig(self):
        st = np.zeros(self.nseg, np.float32)
        ct = np.zeros(self.nseg, np.float32)
        sp = np.zeros(self.views, np.float32)
        cp = np.zeros(self.views, np.float32)
        self.L.ref_get_trig(_p(st), _p(ct), _p(sp), _p(cp))
        return st, ct, sp, cp

    def tantheta(self):
        t = np.zeros((self.groupmax, self.nz), np.float32)
        r = np.zeros((self.groupmax, self.nz), np.float32)
        self.L.ref_get_tantheta(_p(t), _p(r))
        return t, r

    def flookup(self):
        n = self.groupmax * 2 * (self.span - 1)
        zi = np.zeros((self.nx, n), np.int32)
        zf = np.zeros((self.nx, n), np.float32)
        self.L.ref_get_flookup(_p(zi), _p(zf))
        return zi, zf

    def blookup(self):
        a = [np.zeros((self.nx, self.groupmax), np.int32) for _ in range(3)]
        f = np.zeros((self.nx, self.groupmax), np.float32)
        self.L.ref_get_blookup(_p(a[0]), _p(a[1]), _p(a[2]), _p(f))
        return a[0], a[1], a[2], f

    def set_psf(self, fwhm1=0.0, fwhm2=0.0, ratio=0.0):
        """-B fwhm1,fwhm2,ratio: the x/y/z kernels of make1d_psf_filter
        (psf.cpp:21-70) for this geometry's voxel sizes; returns the x taps."""
        taps = np.zeros(256, np.float32)
        n = self.L.ref_psf_setup(fwhm1, fwhm2, ratio, _p(taps), taps.size)
        if n < 1:
            raise ValueError("make1d_psf_filter refused these parameters")
        return taps[:n].copy()

    def psf(self, image):
        """convolve3d (psf.cpp:463-540) of an [x][y][zp] image (set_psf first)."""
        im = np.ascontiguousarray(image, np.float32)
        out = np.zeros(self.image_shape, np.float32)
        if self.L.ref_psf_convolve(_p(im), _p(out)) != 0:
            raise RuntimeError("ref_psf_convolve")
        return out

    def set_norm_zero_mask(self, mask):
        m = np.ascontiguousarray(mask, np.int16)
        self.L.ref_set_norm_zero_mask(_p(m))

    def norm_zero_mask(self):
        m = np.zeros((self.views // 2, self.nx // 2 + 1), np.int16)
        self.L.ref_get_norm_zero_mask(_p(m))
        return m


# ---- the MAP prior of je_hrrt_osem3d (oracle/_ref/libmap_ref.so) ----
MAP_LIB = os.path.join(HERE, "_ref", "libmap_ref.so")
_M = None


def map_lib():
    global _M
    if _M is None:
        if not os.path.exists(MAP_LIB):
            raise FileNotFoundError(MAP_LIB)
        M = ctypes.CDLL(MAP_LIB)
        vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        M.ref_map_dpf.argtypes = [vp, i, i, i, vp, vp]
        M.ref_map_dpf.restype = i
        M.ref_map_update.argtypes = [vp, vp, vp, vp, i, i, vp, f, f]
        M.ref_map_update.restype = None
        _M = M
    return _M


def map_dpf(image, nz, cylwiny):
    """calculate_DPF_image(image, NULL, dpf, 1) of the reference (dpfcalc.c)
    on a float32 [nx][nx][zp] image with nz planes."""
    im = np.ascontiguousarray(image, np.float32)
    nx, _, zp = im.shape
    cyl = np.ascontiguousarray(cylwiny, np.int32).reshape(-1)
    out = np.zeros_like(im)
    assert map_lib().ref_map_dpf(_p(im), nx, nz, zp, _p(cyl), _p(out)) == 1
    return out


def map_update(image, corr, nf_inv, dpf, cylwiny, beta, image_max):
    """pt_cal_updateimage_mapem's SSE update (with _mm_rcp_ps of nf_inv) on
    float32 [nx][nx][zp] arrays; returns the new image."""
    im = np.array(image, np.float32, order="C")
    c = np.array(corr, np.float32, order="C")
    nf = np.ascontiguousarray(nf_inv, np.float32)
    d = np.ascontiguousarray(dpf, np.float32)
    nx, _, zp = im.shape
    cyl = np.ascontiguousarray(cylwiny, np.int32).reshape(-1)
    map_lib().ref_map_update(_p(im), _p(c), _p(nf), _p(d), nx, zp, _p(cyl), beta, image_max)
    return im
