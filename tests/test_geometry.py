"""Geometry tables of the product (csrc/geometry.cpp) against the reference's
own dependencies() (hrrt_osem3dv_sbrt_span3.cpp:199-800), bit for bit.  CPU only."""
import numpy as np
import pytest

from geoms import ALL, product_geom, ref_projector

import hrrt_reconstruction_b200 as H


@pytest.mark.parametrize("name", list(ALL))
def test_tables_bit_identical(name, ref_lib):
    d = ALL[name]
    g = product_geom(d)
    R = ref_projector(d)
    assert np.array_equal(H.geometry_table(g, "segments").reshape(3, -1), R.segments())
    assert np.array_equal(H.geometry_table(g, "cylwiny").reshape(-1, 2), R.cylwiny())
    st, ct, sp, cp = R.trig()
    for n, a in (("sin_theta", st), ("cos_theta", ct), ("sin_psi", sp), ("cos_psi", cp)):
        assert np.array_equal(H.geometry_table(g, n).view(np.uint32), a.view(np.uint32)), n
    t, r = R.tantheta()
    assert np.array_equal(H.geometry_table(g, "tantheta").reshape(t.shape).view(np.uint32), t.view(np.uint32))
    assert np.array_equal(H.geometry_table(g, "rescale").reshape(r.shape).view(np.uint32), r.view(np.uint32))
    zi, zf = R.flookup()
    assert np.array_equal(H.geometry_table(g, "flookup_zzi").reshape(zi.shape), zi)
    assert np.array_equal(H.geometry_table(g, "flookup_zzz0").reshape(zf.shape).view(np.uint32), zf.view(np.uint32))
    a, b, c, f = R.blookup()
    bl = H.geometry_table(g, "blookup").reshape(a.shape + (3,))
    assert np.array_equal(bl[..., 0], a) and np.array_equal(bl[..., 1], b) and np.array_equal(bl[..., 2], c)
    assert np.array_equal(H.geometry_table(g, "blookup_yr2a").reshape(f.shape).view(np.uint32), f.view(np.uint32))
    assert np.array_equal(H.geometry_table(g, "order"), R.order())


def test_hrrt_sizes():
    """Segment and plane counts of lmhistogram_mp.cpp:105-116 (and the segment
    sizes of get_info, hrrt_osem3dv_sbrt_span3.cpp:159-191)."""
    for span, nseg, planes in ((9, 15, 2209), (3, 45, 6367)):
        g = H.hrrt_geometry(span=span)
        seg = H.geometry_table(g, "segments").reshape(3, -1)
        assert seg.shape[1] == nseg
        assert int((seg[1] - seg[0] + 1).sum()) == planes
        # FOV: rel_fov 0.95 of 128 pixels -> 46441 columns
        cyl = H.geometry_table(g, "cylwiny").reshape(-1, 2)
        assert int((cyl[:, 1] - cyl[:, 0]).sum()) == 46441


def test_subset_order_16():
    """sequence() (hrrt_osem3d_span3.cpp:535-580) for 16 subsets."""
    g = H.hrrt_geometry()
    assert H.geometry_table(g, "order").tolist() == [0, 8, 1, 9, 2, 10, 3, 11, 4, 12, 5, 13, 6, 14, 7, 15]


def test_bad_geometry_rejected():
    g = H.hrrt_geometry(span=4)
    with pytest.raises(H.HrrtError):
        H.geometry_table(g, "segments")
