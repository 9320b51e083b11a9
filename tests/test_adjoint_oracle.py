"""The oracle's exact adjoint of the forward projector (orc_fp_adjoint): the
dot-product test <FP x, y> = <x, FP^T y> in both builds.  The reference has no
such operator (its back projector is not the forward projector's transpose);
the test is the definition."""
import numpy as np
import pytest

from geoms import ALL, random_image, random_rows


@pytest.mark.parametrize("name", ["small3", "small9", "hrrt9"])
@pytest.mark.parametrize("precision,tol", [("f64", 1e-13), ("f32", 1e-5)])
def test_dot_product(name, precision, tol):
    from oracle.oracle import Oracle
    O = Oracle(precision=precision, **ALL[name])
    x = random_image(O.image_shape, O.cylwiny(), seed=1, zvalid=O.nz)
    y = random_rows(O.rows_shape, seed=2)
    for v in (0, 5, O.views // 2 - 1):
        lhs = float(np.sum(O.fp_pair(x, v).astype(np.float64) * y))
        rhs = float(np.sum(x.astype(np.float64) * O.fp_adjoint(y, v)))
        assert abs(lhs - rhs) <= tol * abs(lhs), (v, lhs, rhs)


def test_adjoint_is_not_the_reference_back_projector():
    """Sanity: the transpose differs from the reference's back projection
    followed by its rotate-back (different interpolation)."""
    from oracle.oracle import Oracle
    O = Oracle(**ALL["small9"])
    y = random_rows(O.rows_shape, seed=3)
    adj = O.fp_adjoint(y, 4)
    ref = O.rotate_add(O.bp_pair(y, 4), 4, np.zeros(O.image_shape))
    assert np.linalg.norm(adj - ref) > 1e-3 * np.linalg.norm(ref)
