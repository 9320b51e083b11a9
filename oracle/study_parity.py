"""Per-iteration images of a whole OP-OSEM study on the host checkers.

TEST INFRASTRUCTURE.  Only tests/ and bench.py's parity leg use this module,
as the checker of a device reconstruction.  Two host runs of one study:

  "reference"  the reference's own projector compiled from its unmodified
               sources (oracle/_ref/libhrrt_ref.so): CalculateNormfac's
               sensitivity (hrrt_osem3d_span3.cpp:3760-3865), the subset loop
               of CalculateOsem3d (:4098-4341) with its -T thread grouping,
               the post-iteration pass (:4288-4297);
  "fp64"       the same steps on the C restatement's double-precision build
               (oracle/_build/liboracle.so).

Both start from the prep of the restatement (prepare_norm / norm_ANW
:796-1056 and prepare_osem3dw3 :1649-1818 in single precision: prompts masked
where the norm is zero, the additive term (d*N + s)*A, the sensitivity term
1/(N*A) and the norm-zero quad mask), because the reference's prep lives in its
command-line driver, which is not compiled here; the device's prep is checked
against the same restatement (tests/test_osem_gpu.py).

Images are returned in the layout hrrt_reconstruct writes (SaveImage,
drv:4020-4096): float32 [z][y][x], planes < nz.
"""
import os
import time

import numpy as np


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def stock_threads():
    """-T min(8, nproc): the reference's projector threads are
    threads[Cal1 + thr] of a 16-entry array with Cal1 = 8
    (hrrt_osem3d_span3.cpp:189, :448, :4193)."""
    return max(1, min(8, os.cpu_count() or 1))


def _zyx(img_xyz, nz):
    return np.ascontiguousarray(np.transpose(np.asarray(img_xyz)[:, :, :nz], (2, 1, 0)), np.float32)


def prep(geom, prompts, randoms, norm=None, atten=None, scatter=None):
    """-> (prompts masked, additive term, 1/(N*A), norm-zero mask) of the
    single-precision restatement."""
    from oracle.oracle import Oracle
    O = Oracle(precision="f32", **geom)
    p, a, m = O.prep(prompts, randoms, norm, atten, scatter)
    return p, a, m, O.norm_zero_mask()


def reconstruct(kind, geom, prepped, iterations, nthreads=None):
    """Run `iterations` full iterations (every subset in the reference's
    order, then the post-iteration pass) from the default initial image.

    kind: "reference" or "fp64".  Returns a list with one dict per
    iteration: image ([z][y][x] float32), sum (the post-iteration FP64 sum),
    seconds (host time of that iteration; the sensitivity is in "sens_s" of
    the first)."""
    p, a, m, mask = prepped
    if kind == "reference":
        from oracle.ref import RefProjector
        T = nthreads or stock_threads()
        R = RefProjector(nthreads=T, **geom)
        R.set_norm_zero_mask(mask)
        t0 = time.perf_counter()
        nf = R.sensitivity(m, T)
        sens_s = time.perf_counter() - t0
        img = R.init_image()
        order = R.order()
        nz = R.nz
    elif kind == "fp64":
        from oracle.oracle import Oracle
        T = nthreads or (os.cpu_count() or 4)
        R = Oracle(precision="f64", nthreads=T, **geom)
        R.set_norm_zero_mask(mask)
        t0 = time.perf_counter()
        nf = R.sensitivity(m, T)
        sens_s = time.perf_counter() - t0
        img = R.init_image()
        order = R.order()
        nz = R.nz
    else:
        raise ValueError(kind)
    out = []
    for it in range(iterations):
        t0 = time.perf_counter()
        for s in order:
            R.osem_subset(img, nf[int(s)], p, a, int(s), T)
        total = R.post_iteration(img)
        rec = {"image": _zyx(img, nz), "sum": float(total), "seconds": time.perf_counter() - t0, "threads": T}
        if it == 0:
            rec["sens_s"] = sens_s
        out.append(rec)
    return out


def compare(device_images, host_runs):
    """rel-L2 of each device iteration against each host run, per iteration.
    device_images: list of [z][y][x] images; host_runs: {name: reconstruct()}.
    -> {name: [rel-L2 per iteration]}"""
    res = {}
    for name, run in host_runs.items():
        res[name] = [rel_l2(d, h["image"]) for d, h in zip(device_images, run)]
    return res
