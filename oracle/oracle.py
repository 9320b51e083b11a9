"""ctypes binding of the C restatement oracle/hrrt_oracle.c.

TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg use this module, as the checker.  Two builds of one source
(oracle/Makefile, target "oracle"):

  precision="f64"  oracle/_build/liboracle.so      double sums, float positions
  precision="f32"  oracle/_build/liboracle_f32.so  the reference's float order

The libraries are built on demand with `make -C oracle oracle` (gcc only).
"""
import ctypes
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBS = {"f64": os.path.join(HERE, "_build", "liboracle.so"),
        "f32": os.path.join(HERE, "_build", "liboracle_f32.so")}
DTYPES = {"f64": np.float64, "f32": np.float32}

_libs = {}
_lock = threading.Lock()


def build():
    r = subprocess.run(["make", "-s", "-C", HERE, "oracle"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")


def lib(precision="f64"):
    with _lock:
        if precision not in _libs:
            path = LIBS[precision]
            if not os.path.exists(path):
                build()
            L = ctypes.CDLL(path)
            vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
            L.orc_create.argtypes = [i, i, i, f, f, f, i, i, i]
            L.orc_create.restype = vp
            L.orc_destroy.argtypes = [vp]
            L.orc_destroy.restype = None
            for n in ("orc_segmentsize", "orc_zp", "orc_nz", "orc_nx", "orc_nviews", "orc_sviews"):
                getattr(L, n).argtypes = [vp]
                getattr(L, n).restype = i
            L.orc_vieworder.argtypes = [vp, i, i]
            L.orc_set_params.argtypes = [vp, i, f, f, f, f]
            L.orc_set_params.restype = None
            sigs = {
                "orc_order": [vp, vp], "orc_z_range": [vp, i, i, vp], "orc_cylwiny": [vp, vp], "orc_trig": [vp, vp, vp, vp, vp],
                "orc_tantheta": [vp, vp, vp], "orc_flookup": [vp, vp, vp], "orc_blookup": [vp, vp, vp, vp, vp],
                "orc_set_norm_zero_mask": [vp, vp], "orc_get_norm_zero_mask": [vp, vp], "orc_fp_pair": [vp, vp, i, vp], "orc_bp_pair": [vp, vp, i, vp], "orc_fp_adjoint": [vp, vp, i, vp],
                "orc_rotate_add": [vp, vp, i, vp], "orc_prep": [vp, vp, vp, vp, vp, vp, vp, vp, vp],
                "orc_sensitivity": [vp, vp, vp, i], "orc_init_image": [vp, vp, i, i],
                "orc_osem_subset": [vp, vp, vp, vp, vp, i, i],
                "orc_map_dpf": [vp, vp, vp], "orc_osem_subset_map": [vp, vp, vp, vp, vp, i, i, f],
            }
            for n, a in sigs.items():
                getattr(L, n).argtypes = a
                getattr(L, n).restype = None
            L.orc_post_iteration.argtypes = [vp, vp, i, i]
            L.orc_post_iteration.restype = ctypes.c_double
            L.orc_psf_kernel.argtypes = [f, f, f, f, vp, i]
            L.orc_psf_kernel.restype = i
            L.orc_set_psf.argtypes = [vp, i, f, f, f, i, i]
            L.orc_set_psf.restype = i
            L.orc_psf.argtypes = [vp, vp, vp]
            L.orc_psf.restype = None
            assert L.orc_real_bytes() == np.dtype(DTYPES[precision]).itemsize
            _libs[precision] = L
        return _libs[precision]


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class Oracle:
    """The restated OP-OSEM path for one geometry.  Images are [x][y][zp],
    view-pair rows [2*segmentsize][nbins], sinograms in the flat-file layout
    [segmentsize][nviews][nbins]; the real type is float64 or float32."""

    def __init__(self, nrings=104, nelements=256, nangles=288, ring_radius=234.5, plane_sep=1.21875,
                 binsize=1.21875, span=9, maxdel=67, subsets=16, precision="f64", nthreads=1, npskip=3,
                 epsilon1=5e-2, epsilon2=1e-2, epsilon3=1e-10, image_max=1e4, z_min=6, z_max=200):
        self.L = lib(precision)
        self.dtype = DTYPES[precision]
        self.g = self.L.orc_create(nrings, nelements, nangles, ring_radius, plane_sep, binsize, span, maxdel,
                                   subsets)
        if not self.g:
            raise ValueError("unsupported geometry")
        self.L.orc_set_params(self.g, npskip, epsilon1, epsilon2, epsilon3, image_max)
        self.nthreads = nthreads
        self.P = self.L.orc_segmentsize(self.g)
        self.zp = self.L.orc_zp(self.g)
        self.nz = self.L.orc_nz(self.g)
        self.nx = self.L.orc_nx(self.g)
        self.views = self.L.orc_nviews(self.g)
        self.sviews = self.L.orc_sviews(self.g)
        self.subsets = subsets
        self.span = span
        self.groupmax = (maxdel - (span - 1) // 2) // span
        self.nseg = 2 * self.groupmax + 1
        zr = np.zeros(2, np.int32)
        self.L.orc_z_range(self.g, z_min, z_max, _p(zr))
        self.z_min, self.z_max = int(zr[0]), int(zr[1])

    def __del__(self):
        g, self.g = getattr(self, "g", None), None
        if g:
            self.L.orc_destroy(g)

    @property
    def image_shape(self):
        return (self.nx, self.nx, self.zp)

    @property
    def rows_shape(self):
        return (2 * self.P, self.nx)

    @property
    def sino_shape(self):
        return (self.P, self.views, self.nx)

    def _r(self, a):
        return np.ascontiguousarray(a, self.dtype)

    # ---- projector ----
    def fp_pair(self, img, view, prj=None):
        """Rows of one view pair; bins the reference never writes keep the
        values of `prj` (zeros when not given)."""
        img = self._r(img)
        out = np.zeros(self.rows_shape, self.dtype) if prj is None else np.array(prj, self.dtype, copy=True)
        self.L.orc_fp_pair(self.g, _p(img), view, _p(out))
        return out

    def bp_pair(self, rows, view):
        rows = self._r(rows)
        out = np.zeros(self.image_shape, self.dtype)
        self.L.orc_bp_pair(self.g, _p(rows), view, _p(out))
        return out

    def fp_adjoint(self, rows, view, image=None):
        """image + FP^T rows (the exact transpose of fp_pair), image frame."""
        rows = self._r(rows)
        out = np.zeros(self.image_shape, self.dtype) if image is None else np.array(image, self.dtype, copy=True)
        self.L.orc_fp_adjoint(self.g, _p(rows), view, _p(out))
        return out

    def rotate_add(self, imagebuf, view, corr):
        ib = self._r(imagebuf)
        co = np.array(corr, self.dtype, copy=True)
        self.L.orc_rotate_add(self.g, _p(ib), view, _p(co))
        return co

    # ---- driver pieces ----
    def prep(self, prompts, randoms, norm=None, atten=None, scatter=None):
        """-> (prompts masked, additive term, 1/(N*A)); updates the norm-zero mask"""
        f = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)  # noqa: E731
        p = np.ascontiguousarray(prompts, np.int16)
        r, n, a, s = f(randoms), f(norm), f(atten), f(scatter)
        po = np.zeros(self.sino_shape, np.int16)
        ao = np.zeros(self.sino_shape, np.float32)
        mo = np.zeros(self.sino_shape, np.float32)
        self.L.orc_prep(self.g, _p(p), _p(r), _p(n), _p(a), _p(s), _p(po), _p(ao), _p(mo))
        return po, ao, mo

    def set_norm_zero_mask(self, mask):
        m = np.ascontiguousarray(mask, np.int16)
        self.L.orc_set_norm_zero_mask(self.g, _p(m))

    def norm_zero_mask(self):
        m = np.zeros((self.views // 2, self.nx // 2 + 1), np.int16)
        self.L.orc_get_norm_zero_mask(self.g, _p(m))
        return m

    def sensitivity(self, mult, nthreads=None):
        m = np.ascontiguousarray(mult, np.float32)
        out = np.zeros((self.subsets,) + self.image_shape, self.dtype)
        self.L.orc_sensitivity(self.g, _p(m), _p(out), nthreads or self.nthreads)
        return out

    def init_image(self, zmin=None, zmax=None):
        zmin = self.z_min if zmin is None else zmin
        zmax = self.z_max if zmax is None else zmax
        assert 0 <= zmin <= zmax <= self.zp
        out = np.zeros(self.image_shape, self.dtype)
        self.L.orc_init_image(self.g, _p(out), zmin, zmax)
        return out

    def osem_subset(self, image, nf_inv_subset, prompts, add, isubset, nthreads=None):
        """One OP-OSEM subset in place on `image` (C-contiguous, oracle dtype)."""
        assert image.dtype == self.dtype and image.flags.c_contiguous
        nf = self._r(nf_inv_subset)
        p = np.ascontiguousarray(prompts, np.int16)
        a = np.ascontiguousarray(add, np.float32)
        self.L.orc_osem_subset(self.g, _p(image), _p(nf), _p(p), _p(a), isubset, nthreads or self.nthreads)
        return image

    def map_dpf(self, image):
        """calculate_DPF_image technique 1 (dpfcalc.c) of an [x][y][zp] image."""
        im = self._r(image)
        out = np.zeros_like(im)
        self.L.orc_map_dpf(self.g, _p(im), _p(out))
        return out

    def osem_subset_map(self, image, nf_inv_subset, prompts, add, isubset, beta, nthreads=None):
        """One OP-OSEM subset with the MAP (technique 1) update, in place."""
        assert image.dtype == self.dtype and image.flags.c_contiguous
        nf = self._r(nf_inv_subset)
        p = np.ascontiguousarray(prompts, np.int16)
        a = np.ascontiguousarray(add, np.float32)
        self.L.orc_osem_subset_map(self.g, _p(image), _p(nf), _p(p), _p(a), isubset, nthreads or self.nthreads,
                                   beta)
        return image

    def psf_kernel(self, fwhm1=0.0, fwhm2=0.0, ratio=0.0, pixel_size=1.21875):
        """make1d_psf_filter's taps (psf.cpp:21-70); fwhm1 0: the HRRT defaults."""
        k = np.zeros(256, np.float32)
        n = self.L.orc_psf_kernel(fwhm1, fwhm2, ratio, pixel_size, _p(k), 256)
        if n < 1:
            raise ValueError("no PSF kernel for these parameters")
        return k[:n].copy()

    def set_psf(self, on=True, fwhm1=0.0, fwhm2=0.0, ratio=0.0):
        """-B fwhm1,fwhm2,ratio: the PSF in sensitivity and subsets from now on."""
        if self.L.orc_set_psf(self.g, 1 if on else 0, fwhm1, fwhm2, ratio, self.z_min, self.z_max) != 0:
            raise ValueError("no PSF kernel for these parameters")

    def psf(self, image):
        """convolve3d (psf.cpp:463-540) of an [x][y][zp] image on FOV columns."""
        img = self._r(image)
        out = np.zeros(self.image_shape, self.dtype)
        self.L.orc_psf(self.g, _p(img), _p(out))
        return out

    def post_iteration(self, image, zmin=None, zmax=None):
        zmin = self.z_min if zmin is None else zmin
        zmax = self.z_max if zmax is None else zmax
        assert 0 <= zmin <= zmax <= self.zp
        assert image.dtype == self.dtype and image.flags.c_contiguous
        return self.L.orc_post_iteration(self.g, _p(image), zmin, zmax)

    def order(self):
        o = np.zeros(self.subsets, np.int16)
        self.L.orc_order(self.g, _p(o))
        return o

    def vieworder(self, isubset):
        return [self.L.orc_vieworder(self.g, isubset, k) for k in range(self.sviews)]

    # ---- geometry tables ----
    def cylwiny(self):
        a = np.zeros((self.nx, 2), np.int32)
        self.L.orc_cylwiny(self.g, _p(a))
        return a

    def trig(self):
        st = np.zeros(self.nseg, np.float32)
        ct = np.zeros(self.nseg, np.float32)
        sp = np.zeros(self.views, np.float32)
        cp = np.zeros(self.views, np.float32)
        self.L.orc_trig(self.g, _p(st), _p(ct), _p(sp), _p(cp))
        return st, ct, sp, cp

    def tantheta(self):
        t = np.zeros((self.groupmax, self.nz), np.float32)
        r = np.zeros((self.groupmax, self.nz), np.float32)
        self.L.orc_tantheta(self.g, _p(t), _p(r))
        return t, r

    def flookup(self):
        n = self.groupmax * 2 * (self.span - 1)
        zi = np.zeros((self.nx, n), np.int32)
        zf = np.zeros((self.nx, n), np.float32)
        self.L.orc_flookup(self.g, _p(zi), _p(zf))
        return zi, zf

    def blookup(self):
        a = [np.zeros((self.nx, self.groupmax), np.int32) for _ in range(3)]
        f = np.zeros((self.nx, self.groupmax), np.float32)
        self.L.orc_blookup(self.g, _p(a[0]), _p(a[1]), _p(a[2]), _p(f))
        return a[0], a[1], a[2], f
