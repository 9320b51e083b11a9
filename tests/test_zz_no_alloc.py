"""hrrt_bp_pair_noalloc: the back projection for callers that may not allocate
device memory while they run (a real-time loop that cannot take cudaMalloc's
device synchronisation, a host that gives the library a fixed memory budget at
start-up).  Its scratch is a
static device array inside the library, so the call allocates nothing; the
caller supplies the device input rows and the device output buffer.

Checked through the C ABI against hrrt_bp_pair on two calls in a row (the
static scratch keeps the previous call's contents, so the second call must not
depend on them; the second runs on a stream of the caller's), and the size
limit is checked.  This file is collected last
so that a run stopping at the first failure has run everything else first.
"""
import ctypes

import numpy as np
import pytest

from geoms import HRRT3, SMALL9, product_geom, random_rows

pytestmark = pytest.mark.gpu

REL_L2 = 1e-6  # the back projector tests' tolerance is 2e-6; the two paths add the same two terms


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def call_noalloc(ctx, rows, view, own_stream=False):
    """One call on the context's stream, or on a stream of the caller's."""
    import torch

    import hrrt_reconstruction_b200 as H
    d_in = torch.from_numpy(np.ascontiguousarray(rows, np.float32)).cuda()
    d_out = torch.empty(ctx.image_shape, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    st = torch.cuda.Stream() if own_stream else None
    rc = H.lib.hrrt_bp_pair_noalloc(ctx._h, ctypes.c_void_p(d_in.data_ptr()), view,
                                    ctypes.c_void_p(d_out.data_ptr()),
                                    ctypes.c_void_p(st.cuda_stream) if st is not None else None)
    torch.cuda.synchronize()
    assert rc == 0, H.lib.hrrt_last_error(ctx._h).decode()
    return d_out.cpu().numpy()


@pytest.mark.parametrize("geom", [SMALL9, HRRT3], ids=["small9", "hrrt3"])
def test_noalloc_matches_bp_pair_twice(geom):
    import hrrt_reconstruction_b200 as H
    with H.Context(product_geom(geom)) as ctx:
        nv2 = ctx.info.nviews // 2
        for k, (view, seed) in enumerate(((3, 21), (nv2 - 1, 22))):
            rows = random_rows(ctx.rows_shape, seed=seed)
            want = ctx.bp_pair(rows, view)
            got = call_noalloc(ctx, rows, view, own_stream=k == 1)
            e = rel_l2(got, want)
            assert e <= REL_L2, (k, view, e)
            assert np.array_equal(got == 0, want == 0)


def test_noalloc_rejects_oversized_geometry():
    """A view pair whose quad layout exceeds the 16 MiB static scratch is refused."""
    import torch

    import hrrt_reconstruction_b200 as H
    geom = product_geom(dict(HRRT3, nelements=384))
    with H.Context(geom) as ctx:
        d_in = torch.zeros(ctx.rows_shape, dtype=torch.float32, device="cuda")
        d_out = torch.empty(ctx.image_shape, dtype=torch.float32, device="cuda")
        rc = H.lib.hrrt_bp_pair_noalloc(ctx._h, ctypes.c_void_p(d_in.data_ptr()), 0,
                                        ctypes.c_void_p(d_out.data_ptr()), None)
        assert rc == -1  # HRRT_ERR_ARG
        msg = H.lib.hrrt_last_error(ctx._h).decode()
        assert "scratch" in msg, msg
