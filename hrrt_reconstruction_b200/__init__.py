"""hrrt_reconstruction_b200 -- B200 (sm_100a) OSEM hot path of hrrt_osem3d.

Python binding of libhrrt_gpu.so (C ABI in include/hrrt_gpu.h).  It mirrors
the reference's function-level projector interface
(hrrt_osem3d/hrrt_osem3d.h:197-216: forward_proj3d_thread1,
back_proj3d_thread1, rotate_image_buf) and its reconstruction steps
(PrepareNormfac/PrepareOsem3dFiles, CalculateNormfac, Init_Image,
CalculateOsem3d, SaveImage in hrrt_osem3d/hrrt_osem3d_span3.cpp).

The library must be built (``python hrrt_reconstruction_b200/build.py`` or
``__graft_entry__.build()``); importing the package without it raises.  There
is no CPU fallback.
"""
import ctypes
import os

import numpy as np

__all__ = ["Geometry", "HrrtError", "Context", "Batch", "Tuning", "Listmode", "lib", "LIB_PATH", "STORE_F32", "STORE_16", "STORE_F16", "BP_REF", "BP_ADJOINT",
           "geometry_table", "hrrt_geometry"]

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libhrrt_gpu.so")
STORE_F32 = 0
STORE_16 = 1   # bf16 additive and multiplicative terms
STORE_F16 = 2  # fp16 additive and multiplicative terms
BP_REF = 0
BP_ADJOINT = 1


class HrrtError(RuntimeError):
    pass


class Geometry(ctypes.Structure):
    """hrrt_geom: scanner / sinogram / reconstruction parameters."""

    _fields_ = [("nrings", ctypes.c_int), ("nelements", ctypes.c_int), ("nangles", ctypes.c_int),
                ("ring_radius", ctypes.c_float), ("plane_sep", ctypes.c_float), ("binsize", ctypes.c_float),
                ("span", ctypes.c_int), ("maxdel", ctypes.c_int), ("subsets", ctypes.c_int),
                ("rel_fov", ctypes.c_float), ("z_min", ctypes.c_int), ("z_max", ctypes.c_int),
                ("npskip", ctypes.c_int), ("epsilon1", ctypes.c_float), ("epsilon2", ctypes.c_float),
                ("epsilon3", ctypes.c_float), ("image_max", ctypes.c_float)]


class Info(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("zp", ctypes.c_int),
                ("nbins", ctypes.c_int), ("nviews", ctypes.c_int), ("nseg", ctypes.c_int),
                ("groupmax", ctypes.c_int), ("segmentsize", ctypes.c_int), ("subsets", ctypes.c_int),
                ("sviews", ctypes.c_int), ("fov_columns", ctypes.c_int), ("sino_elems", ctypes.c_longlong),
                ("image_elems", ctypes.c_longlong)]


class Stats(ctypes.Structure):
    _fields_ = [("sum_image", ctypes.c_double), ("subset_iterations", ctypes.c_int),
                ("ms_total", ctypes.c_float)]


class LmStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_longlong) for n in ("words_used", "prompts", "delayed", "timetags", "tags", "invalid",
                                                  "unmapped", "doi_other", "doi7", "resyncs", "frame_start",
                                                  "duration")] + [("terminated", ctypes.c_int), ("ms", ctypes.c_float)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class Tuning(ctypes.Structure):
    """hrrt_tuning: launch shape of the projectors (results do not depend on it)."""
    _fields_ = [("fp_planes", ctypes.c_int), ("fp_producer_warps", ctypes.c_int), ("bp_planes", ctypes.c_int),
                ("bp_threads", ctypes.c_int), ("bp_tile", ctypes.c_int), ("fp_ms", ctypes.c_double),
                ("bp_ms", ctypes.c_double)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class BatchStats(ctypes.Structure):
    _fields_ = [("ms_total", ctypes.c_double), ("subset_iterations", ctypes.c_int), ("groups", ctypes.c_int),
                ("graphs", ctypes.c_int), ("graph_launches", ctypes.c_int), ("kernel_launches", ctypes.c_longlong)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


LM_TRUES, LM_PROMPTS_AND_DELAYED, LM_PROMPTS_ONLY = 0, 1, 2
LM_IGNORE_BORDER_CRYSTAL, LM_NO_DOI, LM_TIME_FROM_COUNT = 1, 2, 4
LM_FORCE_DIRECT, LM_FORCE_PARTITIONED, LM_FORCE_WIDE, LM_HEAD_CURVE, LM_CRYSTAL_COUNTS = 16, 32, 64, 128, 256


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run hrrt_reconstruction_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    vp, i, f, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double
    G = ctypes.POINTER(Geometry)
    sig = {
        "hrrt_geom_default": (None, [G]),
        "hrrt_ctx_create": (i, [G, i, ctypes.POINTER(vp)]),
        "hrrt_ctx_destroy": (None, [vp]),
        "hrrt_last_error": (ctypes.c_char_p, [vp]),
        "hrrt_get_info": (i, [vp, ctypes.POINTER(Info)]),
        "hrrt_get_stream": (vp, [vp]),
        "hrrt_upload_inputs": (i, [vp, vp, vp, vp, vp, vp, i]),
        "hrrt_sensitivity": (i, [vp]),
        "hrrt_reconstruct": (i, [vp, vp, vp, vp, vp, vp, i, vp, i, vp, ctypes.POINTER(Stats)]),
        "hrrt_init_image": (i, [vp, vp]),
        "hrrt_osem": (i, [vp, i, ctypes.POINTER(Stats)]),
        "hrrt_osem_subsets": (i, [vp, i, i]),
        "hrrt_get_image": (i, [vp, vp]),
        "hrrt_get_image_xyz": (i, [vp, vp]),
        "hrrt_set_image_xyz": (i, [vp, vp]),
        "hrrt_get_sensitivity": (i, [vp, i, vp]),
        "hrrt_get_norm_zero_mask": (i, [vp, vp]),
        "hrrt_set_norm_zero_mask": (i, [vp, vp]),
        "hrrt_fp_pair": (i, [vp, vp, i, vp]),
        "hrrt_bp_pair": (i, [vp, vp, i, vp, i]),
        "hrrt_forward_project": (i, [vp, vp, vp]),
        "hrrt_bp_pair_noalloc": (i, [vp, vp, i, vp, vp]),
        "hrrt_set_backprojector": (i, [vp, i]),
        "hrrt_rotate_add": (i, [vp, vp, i, vp]),
        "hrrt_geometry_table": (ctypes.c_longlong, [G, ctypes.c_char_p, vp, ctypes.c_size_t]),
        "hrrt_set_profiling": (i, [vp, i]),
        "hrrt_kernel_stats": (i, [vp, ctypes.c_char_p, ctypes.POINTER(i), ctypes.POINTER(d)]),
        "hrrt_reset_kernel_stats": (i, [vp]),
        "hrrt_set_psf": (i, [vp, i, f, f, f]),
        "hrrt_psf_convolve": (i, [vp, vp, vp]),
        "hrrt_set_map": (i, [vp, i, f, i]),
        "hrrt_map_prior": (i, [vp, vp, vp]),
        "hrrt_psf_kernel": (ctypes.c_longlong, [f, f, f, f, vp, i]),
        "hrrt_set_tuning": (i, [vp, ctypes.POINTER(Tuning)]),
        "hrrt_get_tuning": (i, [vp, ctypes.POINTER(Tuning)]),
        "hrrt_autotune": (i, [vp, i, ctypes.POINTER(Tuning)]),
        "hrrt_batch_create": (i, [vp, i, i, vp, vp, ctypes.POINTER(vp)]),
        "hrrt_batch_destroy": (None, [vp]),
        "hrrt_batch_set_frame": (i, [vp, i, vp, vp, vp, i]),
        "hrrt_batch_autotune": (i, [vp, i, ctypes.POINTER(Tuning)]),
        "hrrt_batch_run": (i, [vp, ctypes.POINTER(BatchStats)]),
        "hrrt_batch_get_image": (i, [vp, i, vp, ctypes.POINTER(d)]),
        "hrrt_lm_create": (i, [i, i, i, ctypes.POINTER(vp)]),
        "hrrt_lm_destroy": (None, [vp]),
        "hrrt_lm_last_error": (ctypes.c_char_p, [vp]),
        "hrrt_lm_sino_size": (ctypes.c_longlong, [vp]),
        "hrrt_lm_reset_clock": (i, [vp]),
        "hrrt_lm_get_stream": (vp, [vp]),
        "hrrt_lm_table": (ctypes.c_longlong, [i, i, ctypes.c_char_p, vp, ctypes.c_size_t]),
        "hrrt_lm_histogram": (i, [vp, vp, ctypes.c_longlong, i, i, i, vp, vp, ctypes.POINTER(LmStats)]),
        "hrrt_lm_histogram_device": (i, [vp, vp, ctypes.c_longlong, i, i, i, vp, vp, ctypes.POINTER(LmStats), vp]),
        "hrrt_lm_smooth_randoms": (i, [vp, vp, f, f, vp, ctypes.POINTER(i)]),
        "hrrt_lm_head_curve": (i, [vp, vp, i]),
        "hrrt_lm_crystal_counts": (i, [vp, vp]),
        "hrrt_lm_histogram_at": (i, [vp, vp, ctypes.c_longlong, ctypes.c_longlong, i, i, i, vp, vp, vp]),
        "hrrt_lm_seek": (i, [vp, vp, ctypes.c_longlong, ctypes.c_longlong, i, i, vp]),
        "hrrt_lm_set_chunk": (i, [vp, ctypes.c_longlong]),
        "hrrt_lm_convert_span9": (ctypes.c_longlong, [vp, vp, vp, i]),
        "hrrt_lm_trues_span9_device": (i, [vp, vp, vp, vp, vp]),
        "hrrt_lm_block_singles": (i, [vp, vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
        "hrrt_lm_crystal_singles": (i, [vp, f, f, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


lib = _load()


def hrrt_geometry(span=9, **kw):
    """HRRT model 999 defaults (scanner_model.cpp:124) with overrides."""
    g = Geometry()
    lib.hrrt_geom_default(ctypes.byref(g))
    g.span = span
    for k, v in kw.items():
        setattr(g, k, v)
    return g


_TABLE_DTYPES = {"cylwiny": np.int16, "segments": np.int32, "flookup_zzi": np.int32, "blookup": np.int32,
                 "order": np.int16}


def geometry_table(geom, name):
    """One geometry table (host-only, no GPU needed) as a numpy array."""
    n = lib.hrrt_geometry_table(ctypes.byref(geom), name.encode(), None, 0)
    if n < 0:
        raise HrrtError(f"geometry table {name!r}: status {n}")
    dt = _TABLE_DTYPES.get(name, np.float32)
    out = np.empty(n // np.dtype(dt).itemsize, dt)
    lib.hrrt_geometry_table(ctypes.byref(geom), name.encode(), out.ctypes.data, n)
    return out


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _c(a, dtype):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=dtype)
    return a


class Context:
    """One reconstruction context on one GPU (hrrt_ctx)."""

    def __init__(self, geom=None, device=0):
        self.geom = geom if geom is not None else hrrt_geometry()
        h = ctypes.c_void_p()
        rc = lib.hrrt_ctx_create(ctypes.byref(self.geom), device, ctypes.byref(h))
        self._h = h
        if rc != 0:
            msg = lib.hrrt_last_error(h).decode() if h.value else "no context"
            if h.value:
                lib.hrrt_ctx_destroy(h)
            self._h = ctypes.c_void_p()
            raise HrrtError(f"hrrt_ctx_create: {rc}: {msg}")
        info = Info()
        lib.hrrt_get_info(self._h, ctypes.byref(info))
        self.info = info

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.hrrt_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, what):
        if rc != 0:
            raise HrrtError(f"{what}: {rc}: {lib.hrrt_last_error(self._h).decode()}")

    # ---- shapes ----
    @property
    def image_shape(self):
        i = self.info
        return (i.nx, i.ny, i.zp)

    @property
    def sino_shape(self):
        i = self.info
        return (i.segmentsize, i.nviews, i.nbins)

    @property
    def rows_shape(self):
        i = self.info
        return (2 * i.segmentsize, i.nbins)

    @property
    def stream(self):
        return lib.hrrt_get_stream(self._h)

    # ---- reconstruction ----
    def upload_inputs(self, prompts, randoms, norm=None, atten=None, scatter=None, storage=STORE_F32):
        p = _c(prompts, np.int16)
        r = _c(randoms, np.float32)
        n = _c(norm, np.float32)
        a = _c(atten, np.float32)
        s = _c(scatter, np.float32)
        need = int(np.prod(self.sino_shape))
        for name, arr in (("prompts", p), ("randoms", r), ("norm", n), ("atten", a), ("scatter", s)):
            if arr is not None and arr.size != need:
                raise HrrtError(f"{name}: {arr.size} elements, expected {need}")
        self._check(lib.hrrt_upload_inputs(self._h, _ptr(p), _ptr(r), _ptr(n), _ptr(a), _ptr(s), storage),
                    "upload_inputs")

    def sensitivity(self):
        self._check(lib.hrrt_sensitivity(self._h), "sensitivity")

    def reconstruct(self, prompts, randoms, norm=None, atten=None, scatter=None, storage=STORE_F32, iterations=1,
                    init_image_zyx=None, out=None):
        """upload + sensitivity + init + osem + get_image in one pipelined
        call -> (image [z][y][x], Stats).  Host arrays in pinned memory let
        the uploads overlap the first iteration."""
        p = _c(prompts, np.int16)
        r = _c(randoms, np.float32)
        n = _c(norm, np.float32)
        a = _c(atten, np.float32)
        s = _c(scatter, np.float32)
        need = int(np.prod(self.sino_shape))
        for name, arr in (("prompts", p), ("randoms", r), ("norm", n), ("atten", a), ("scatter", s)):
            if arr is not None and arr.size != need:
                raise HrrtError(f"{name}: {arr.size} elements, expected {need}")
        i = self.info
        if out is None:
            out = np.empty((i.nz, i.ny, i.nx), np.float32)
        elif out.shape != (i.nz, i.ny, i.nx) or out.dtype != np.float32 or not out.flags.c_contiguous:
            raise HrrtError("reconstruct: out must be C-contiguous float32 [nz][ny][nx]")
        im = _c(init_image_zyx, np.float32)
        st = Stats()
        self._check(lib.hrrt_reconstruct(self._h, _ptr(p), _ptr(r), _ptr(n), _ptr(a), _ptr(s), storage, _ptr(im),
                                         iterations, _ptr(out), ctypes.byref(st)), "reconstruct")
        return out, st

    def init_image(self, image_zyx=None):
        im = _c(image_zyx, np.float32)
        self._check(lib.hrrt_init_image(self._h, _ptr(im)), "init_image")

    def osem(self, iterations):
        st = Stats()
        self._check(lib.hrrt_osem(self._h, iterations, ctypes.byref(st)), "osem")
        return st

    def osem_subsets(self, first, count):
        self._check(lib.hrrt_osem_subsets(self._h, first, count), "osem_subsets")

    def get_image(self, out=None):
        """The [z][y][x] image the reference's SaveImage writes; `out`, when
        given, is a C-contiguous float32 array of that shape to fill."""
        i = self.info
        if out is None:
            out = np.empty((i.nz, i.ny, i.nx), np.float32)
        elif out.shape != (i.nz, i.ny, i.nx) or out.dtype != np.float32 or not out.flags.c_contiguous:
            raise HrrtError("get_image: out must be C-contiguous float32 [nz][ny][nx]")
        self._check(lib.hrrt_get_image(self._h, _ptr(out)), "get_image")
        return out

    def get_image_xyz(self):
        out = np.empty(self.image_shape, np.float32)
        self._check(lib.hrrt_get_image_xyz(self._h, _ptr(out)), "get_image_xyz")
        return out

    def set_image_xyz(self, img):
        a = _c(img, np.float32)
        assert a.shape == self.image_shape
        self._check(lib.hrrt_set_image_xyz(self._h, _ptr(a)), "set_image_xyz")

    def get_sensitivity(self, subset):
        out = np.empty(self.image_shape, np.float32)
        self._check(lib.hrrt_get_sensitivity(self._h, subset, _ptr(out)), "get_sensitivity")
        return out

    def norm_zero_mask(self):
        i = self.info
        out = np.empty((i.nviews // 2, i.nbins // 2 + 1), np.int16)
        self._check(lib.hrrt_get_norm_zero_mask(self._h, _ptr(out)), "get_norm_zero_mask")
        return out

    def set_norm_zero_mask(self, mask):
        m = _c(mask, np.int16)
        self._check(lib.hrrt_set_norm_zero_mask(self._h, _ptr(m)), "set_norm_zero_mask")

    # ---- projector entry points (reference function-level interface) ----
    def fp_pair(self, image_xyz, view, prj=None):
        img = _c(image_xyz, np.float32)
        assert img.shape == self.image_shape
        out = np.zeros(self.rows_shape, np.float32) if prj is None else _c(prj, np.float32).copy()
        self._check(lib.hrrt_fp_pair(self._h, _ptr(img), view, _ptr(out)), "fp_pair")
        return out

    def forward_project(self, image_xyz):
        """Full flat-file sinogram [segmentsize][nviews][nbins] of image_xyz."""
        img = _c(image_xyz, np.float32)
        assert img.shape == self.image_shape
        out = np.empty(self.sino_shape, np.float32)
        self._check(lib.hrrt_forward_project(self._h, _ptr(img), _ptr(out)), "forward_project")
        return out

    def bp_pair(self, prj, view, mode=BP_REF):
        p = _c(prj, np.float32)
        assert p.shape == self.rows_shape
        out = np.zeros(self.image_shape, np.float32)
        self._check(lib.hrrt_bp_pair(self._h, _ptr(p), view, _ptr(out), mode), "bp_pair")
        return out

    def set_backprojector(self, mode):
        """BP_REF (the reference's back projector) or BP_ADJOINT (the forward
        projector's exact transpose) for sensitivity() and osem()."""
        self._check(lib.hrrt_set_backprojector(self._h, mode), "set_backprojector")

    def rotate_add(self, imagebuf, view, corr):
        ib = _c(imagebuf, np.float32)
        co = _c(corr, np.float32).copy()
        self._check(lib.hrrt_rotate_add(self._h, _ptr(ib), view, _ptr(co)), "rotate_add")
        return co

    # ---- timing ----
    def set_psf(self, enable=True, fwhm1=0.0, fwhm2=0.0, ratio=0.0):
        """-B fwhm1,fwhm2,ratio: PSF modelling in the sensitivity and the
        subsets from now on (fwhm1 0: the HRRT defaults)."""
        self._check(lib.hrrt_set_psf(self._h, 1 if enable else 0, fwhm1, fwhm2, ratio), "set_psf")

    def psf(self, image_xyz):
        """convolve3d of an [x][y][zp] image on FOV columns (set_psf first)."""
        img = _c(image_xyz, np.float32)
        assert img.shape == self.image_shape
        out = np.empty(self.image_shape, np.float32)
        self._check(lib.hrrt_psf_convolve(self._h, _ptr(img), _ptr(out)), "psf")
        return out

    def set_map(self, technique=1, beta=0.0, first_subset=5):
        """-b technique,beta of je_hrrt_osem3d: MAP (technique 1, Green's
        one-step-late prior) from subset `first_subset` after the image was
        set; technique 0 or beta 0 turns it off."""
        self._check(lib.hrrt_set_map(self._h, technique, beta, first_subset), "set_map")

    def map_prior(self, image_xyz):
        """calculate_DPF_image (technique 1) of an [x][y][zp] image (set_map first)."""
        img = _c(image_xyz, np.float32)
        assert img.shape == self.image_shape
        out = np.empty(self.image_shape, np.float32)
        self._check(lib.hrrt_map_prior(self._h, _ptr(img), _ptr(out)), "map_prior")
        return out

    def set_tuning(self, fp_planes=0, fp_producer_warps=0, bp_planes=0, bp_threads=0, bp_tile=0):
        t = Tuning(fp_planes, fp_producer_warps, bp_planes, bp_threads, bp_tile, 0.0, 0.0)
        self._check(lib.hrrt_set_tuning(self._h, ctypes.byref(t)), "set_tuning")

    def get_tuning(self):
        t = Tuning()
        self._check(lib.hrrt_get_tuning(self._h, ctypes.byref(t)), "get_tuning")
        return t

    def autotune(self, repeats=3):
        """Time every projector launch shape on the current inputs and image;
        keep and return the fastest (Tuning)."""
        t = Tuning()
        self._check(lib.hrrt_autotune(self._h, repeats, ctypes.byref(t)), "autotune")
        return t

    def batch(self, nframes, norm=None, atten=None, storage=STORE_F32):
        """A dynamic study on this context's geometry (Batch)."""
        return Batch(self, nframes, norm=norm, atten=atten, storage=storage)

    def set_profiling(self, on):
        self._check(lib.hrrt_set_profiling(self._h, 1 if on else 0), "set_profiling")

    def kernel_stats(self, name):
        n = ctypes.c_int()
        ms = ctypes.c_double()
        self._check(lib.hrrt_kernel_stats(self._h, name.encode(), ctypes.byref(n), ctypes.byref(ms)),
                    "kernel_stats")
        return n.value, ms.value

    def reset_kernel_stats(self):
        self._check(lib.hrrt_reset_kernel_stats(self._h), "reset_kernel_stats")


LM_SOL = np.dtype([("nsino", np.int32), ("d", np.float32), ("z", np.float32)])


class Batch:
    """hrrt_batch: the frames of a dynamic study, sharing the context's
    geometry and one normalisation / attenuation, each with its own prompts,
    randoms, scatter and iteration count; reconstructed together (the frame
    loop of hrrt_osem3d's main, hrrt_osem3d_span3.cpp:4555-4597)."""

    def __init__(self, ctx, nframes, norm=None, atten=None, storage=STORE_F32):
        self.ctx = ctx
        self.nframes = nframes
        n = _c(norm, np.float32)
        a = _c(atten, np.float32)
        need = int(np.prod(ctx.sino_shape))
        for name, arr in (("norm", n), ("atten", a)):
            if arr is not None and arr.size != need:
                raise HrrtError(f"{name}: {arr.size} elements, expected {need}")
        h = ctypes.c_void_p()
        ctx._check(lib.hrrt_batch_create(ctx._h, nframes, storage, _ptr(n), _ptr(a), ctypes.byref(h)), "batch_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib.hrrt_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_frame(self, frame, prompts, randoms, scatter=None, iterations=1):
        p = _c(prompts, np.int16)
        r = _c(randoms, np.float32)
        s = _c(scatter, np.float32)
        need = int(np.prod(self.ctx.sino_shape))
        for name, arr in (("prompts", p), ("randoms", r), ("scatter", s)):
            if arr is not None and arr.size != need:
                raise HrrtError(f"{name}: {arr.size} elements, expected {need}")
        self.ctx._check(lib.hrrt_batch_set_frame(self._h, frame, _ptr(p), _ptr(r), _ptr(s), iterations),
                        "batch_set_frame")

    def autotune(self, repeats=3):
        t = Tuning()
        self.ctx._check(lib.hrrt_batch_autotune(self._h, repeats, ctypes.byref(t)), "batch_autotune")
        return t

    def run(self):
        st = BatchStats()
        self.ctx._check(lib.hrrt_batch_run(self._h, ctypes.byref(st)), "batch_run")
        return st

    def get_image(self, frame, out=None):
        """-> (image [z][y][x] float32, FP64 image sum of its last iteration)"""
        i = self.ctx.info
        if out is None:
            out = np.empty((i.nz, i.ny, i.nx), np.float32)
        elif out.shape != (i.nz, i.ny, i.nx) or out.dtype != np.float32 or not out.flags.c_contiguous:
            raise HrrtError("get_image: out must be C-contiguous float32 [nz][ny][nx]")
        sm = ctypes.c_double()
        self.ctx._check(lib.hrrt_batch_get_image(self._h, frame, _ptr(out), ctypes.byref(sm)), "batch_get_image")
        return out, sm.value


def psf_kernel(fwhm1=0.0, fwhm2=0.0, ratio=0.0, pixel_size=1.21875):
    """Host-only: make1d_psf_filter's taps (fwhm1 0: the HRRT defaults)."""
    k = np.zeros(256, np.float32)
    n = lib.hrrt_psf_kernel(fwhm1, fwhm2, ratio, pixel_size, _ptr(k), 256)
    if n < 1:
        raise HrrtError("no PSF kernel for these parameters")
    return k[:n].copy()


def crystal_singles(delayed_counts, scan_duration=1.0, tau=6.0e-9):
    """Host-only: gen_delays' crystal singles estimate from the 119808 delayed
    crystal counts of a coincidence histogram -> (singles float32, iterations)."""
    d = np.ascontiguousarray(delayed_counts, np.int32).reshape(-1)
    if d.size != 2 * 104 * 8 * 72:
        raise HrrtError("delayed counts: 119808 crystals expected")
    out = np.zeros(d.size, np.float32)
    it = lib.hrrt_lm_crystal_singles(_ptr(d), scan_duration, tau, _ptr(out))
    return out, it


def convert_span9(span3, delayed=None, maxrd=67):
    """Host-only: convert_span9 of a span-3 int16 sinogram (minus `delayed`
    when given: the -PR trues) -> the 2209-plane span-9 int16 sinogram."""
    a = np.ascontiguousarray(span3).view(np.int16).reshape(-1)
    d = None if delayed is None else np.ascontiguousarray(delayed).view(np.int16).reshape(-1)
    if d is not None and d.size != a.size:
        raise HrrtError("convert_span9: prompts and delayed differ in size")
    out = np.empty(2209 * 288 * 256, np.int16)
    n = lib.hrrt_lm_convert_span9(_ptr(a), _ptr(d) if d is not None else None, _ptr(out), maxrd)
    if n < 0:
        raise HrrtError(f"convert_span9: {n}")
    return out[:n * 288 * 256]


def lm_table(name, span=3, maxrd=67):
    """One listmode rebinning table (host-only): "sol" [21][144][144] LM_SOL,
    "zpos"/"zpos2" float [104], "segz0"/"segzmax"/"segzoffset" int32."""
    n = lib.hrrt_lm_table(span, maxrd, name.encode(), None, 0)
    if n < 0:
        raise HrrtError(f"lm_table({name!r}): {n}")
    if name == "sol":
        out = np.empty((21, 144, 144), LM_SOL)
    elif name.startswith("zpos"):
        out = np.empty(n // 4, np.float32)
    else:
        out = np.empty(n // 4, np.int32)
    lib.hrrt_lm_table(span, maxrd, name.encode(), out.ctypes.data, out.nbytes)
    return out


class Listmode:
    """64-bit HRRT listmode histogrammer on the device (hrrt_lm_* C ABI):
    the rebinner LUT for output span 3 or 9, and the clock carried from one
    frame to the next."""

    def __init__(self, span=3, maxrd=67, device=0):
        h = ctypes.c_void_p()
        rc = lib.hrrt_lm_create(span, maxrd, device, ctypes.byref(h))
        if rc != 0:
            msg = lib.hrrt_lm_last_error(h).decode() if h.value else "hrrt_lm_create failed"
            if h.value:
                lib.hrrt_lm_destroy(h)
            raise HrrtError(f"hrrt_lm_create: {msg} ({rc})")
        self._h = h
        self.span = span
        self.sino_size = lib.hrrt_lm_sino_size(h)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib.hrrt_lm_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, what):
        if rc != 0:
            raise HrrtError(f"{what}: {lib.hrrt_lm_last_error(self._h).decode()} ({rc})")

    def reset_clock(self):
        self._check(lib.hrrt_lm_reset_clock(self._h), "reset_clock")

    @property
    def stream(self):
        """cudaStream_t (int) of the host-buffer entry point."""
        return lib.hrrt_lm_get_stream(self._h)

    def histogram(self, words, mode=LM_PROMPTS_AND_DELAYED, duration=0, flags=0, out=None, offset=0):
        """One frame from host words -> (sino, delayed or None, stats dict);
        `out` = (sino, delayed) uint16 host arrays to fill; `offset` = the
        position of words[0] in the listmode file (packets count from its
        start)."""
        w = _c(words, np.uint32)
        if out is None:
            sino = np.empty(self.sino_size, np.uint16)
            dly = np.empty(self.sino_size, np.uint16) if mode == LM_PROMPTS_AND_DELAYED else None
        else:
            sino, dly = out
        st = LmStats()
        self._check(lib.hrrt_lm_histogram_at(self._h, _ptr(w), w.size, offset, mode, duration, flags, _ptr(sino),
                                             _ptr(dly), ctypes.byref(st)), "lm_histogram")
        return sino, dly, st.as_dict()

    def set_chunk(self, words=0):
        """Host words longer than `words` (a multiple of 2 Mi; 0: 64 Mi) are
        histogrammed in chunks whose upload overlaps the previous chunk's
        histogram; < 0 turns streaming off."""
        self._check(lib.hrrt_lm_set_chunk(self._h, words), "lm_set_chunk")

    def seek(self, words, target, offset=0, flags=0):
        """goto_event: words consumed up to the time tag reaching `target` s
        (the 0-ms tag for 0); raises HrrtError when the stream ends first."""
        w = _c(words, np.uint32)
        n = ctypes.c_longlong()
        self._check(lib.hrrt_lm_seek(self._h, _ptr(w), w.size, offset, target, flags, ctypes.byref(n)), "lm_seek")
        return n.value

    def head_curve(self):
        """The head curve of the last histogram call made with LM_HEAD_CURVE:
        int64 [n][4] (time ms, prompts, randoms, total singles)."""
        n = lib.hrrt_lm_head_curve(self._h, None, 0)
        out = np.zeros((max(n, 0), 4), np.int64)
        if n > 0:
            lib.hrrt_lm_head_curve(self._h, _ptr(out), n)
        return out

    def crystal_counts(self):
        """The coincidence histogram of the last LM_CRYSTAL_COUNTS call:
        uint32 [2][119808] (prompt, delayed)."""
        out = np.zeros(2 * 2 * 104 * 8 * 72, np.uint32)
        self._check(lib.hrrt_lm_crystal_counts(self._h, _ptr(out)), "lm_crystal_counts")
        return out

    def block_singles(self):
        """-> (average singles rate of each of the 936 blocks, (total prompts,
        total randoms) of the head-curve lines) of the last LM_HEAD_CURVE call."""
        rates = np.zeros(936, np.int32)
        tp, tr = ctypes.c_longlong(), ctypes.c_longlong()
        lib.hrrt_lm_block_singles(self._h, _ptr(rates), ctypes.byref(tp), ctypes.byref(tr))
        return rates, (tp.value, tr.value)

    def smooth_randoms(self, coinc_hist, scan_duration=1.0, tau=6.0e-9):
        """gen_delays: the randoms sinogram (float32, this context's span) from
        a coincidence histogram [2][119808] int32 -> (sino, iterations)."""
        h = np.ascontiguousarray(coinc_hist, np.int32).reshape(-1)
        if h.size != 2 * 2 * 104 * 8 * 72:
            raise HrrtError("coincidence histogram: 2 x 119808 counts expected")
        out = np.empty(self.sino_size, np.float32)
        it = ctypes.c_int()
        self._check(lib.hrrt_lm_smooth_randoms(self._h, _ptr(h), scan_duration, tau, _ptr(out), ctypes.byref(it)),
                    "lm_smooth_randoms")
        return out, it.value

    def trues_span9_device(self, d_prompts, d_delayed, d_out, stream=None):
        """Device pointers (ints; d_delayed may be 0): the span-3 prompts minus
        delayed folded into span 9 (2209 planes of int16) on `stream`."""
        self._check(lib.hrrt_lm_trues_span9_device(self._h, ctypes.c_void_p(d_prompts),
                                                   ctypes.c_void_p(d_delayed) if d_delayed else None,
                                                   ctypes.c_void_p(d_out),
                                                   ctypes.c_void_p(stream) if stream else None), "lm_trues_span9")

    def histogram_device(self, d_words, nwords, d_sino, d_delayed=None, mode=LM_PROMPTS_AND_DELAYED, duration=0,
                         flags=0, stream=None):
        """Device pointers (ints); adds into the sinograms; -> stats dict."""
        st = LmStats()
        self._check(lib.hrrt_lm_histogram_device(self._h, ctypes.c_void_p(d_words), nwords, mode, duration, flags,
                                                 ctypes.c_void_p(d_sino),
                                                 ctypes.c_void_p(d_delayed) if d_delayed else None, ctypes.byref(st),
                                                 ctypes.c_void_p(stream) if stream else None), "lm_histogram_device")
        return st.as_dict()
