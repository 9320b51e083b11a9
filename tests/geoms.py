"""Geometries used by the tests: HRRT model 999 at span 3 and 9, and two
small scanners (same code paths, seconds on the CPU checker)."""
import numpy as np

HRRT9 = dict(nrings=104, nelements=256, nangles=288, ring_radius=234.5, plane_sep=1.21875, binsize=1.21875,
             span=9, maxdel=67, subsets=16)
HRRT3 = dict(HRRT9, span=3)
SMALL3 = dict(nrings=24, nelements=64, nangles=96, ring_radius=58.625, plane_sep=1.21875, binsize=1.21875,
              span=3, maxdel=13, subsets=16)
SMALL9 = dict(nrings=32, nelements=64, nangles=96, ring_radius=58.625, plane_sep=1.21875, binsize=1.21875,
              span=9, maxdel=22, subsets=16)

ALL = {"hrrt9": HRRT9, "hrrt3": HRRT3, "small3": SMALL3, "small9": SMALL9}


def product_geom(d):
    import hrrt_reconstruction_b200 as H
    return H.hrrt_geometry(**d)


def ref_projector(d, nthreads=1):
    from oracle.ref import RefProjector
    return RefProjector(nthreads=nthreads, **d)


def fov_mask(nx, cyl):
    m = np.zeros((nx, nx), bool)
    for x in range(nx):
        m[x, cyl[x, 0]:cyl[x, 1]] = True
    return m


def random_image(shape, cyl, seed=0, zvalid=None):
    """Smooth positive image on the FOV columns, [x][y][zp]."""
    rng = np.random.default_rng(seed)
    nx, _, zp = shape
    img = rng.random(shape, dtype=np.float32) * 0.5 + 0.5
    # smooth along z a little so interpolation matters
    img = (img + np.roll(img, 1, axis=2) + np.roll(img, -1, axis=2)) / 3.0
    m = fov_mask(nx, cyl)
    img *= m[:, :, None]
    nz = zvalid if zvalid is not None else zp - 1
    img[:, :, nz:] = 0
    return np.ascontiguousarray(img.astype(np.float32))


def random_rows(shape, seed=1):
    rng = np.random.default_rng(seed)
    return (rng.random(shape, dtype=np.float32) * 2.0).astype(np.float32)
