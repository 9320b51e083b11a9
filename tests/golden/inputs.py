"""Deterministic inputs for the golden fixtures.

Every input is an exact function of integer indices evaluated in float32, so
the same arrays are rebuilt bit for bit on any machine (no random generator
state is involved).  Shared by make_golden.py (which ran the reference on
them) and the tests (which run the oracle and the device path on them).
"""
import numpy as np


def fov_mask(cyl, nx):
    m = np.zeros((nx, nx), bool)
    for x in range(nx):
        m[x, cyl[x][0]:cyl[x][1]] = True
    return m


def image(nx, zp, nz, cyl):
    """[x][y][zp] float32: a positive pattern on the FOV columns, planes < nz."""
    x, y, z = np.meshgrid(np.arange(nx), np.arange(nx), np.arange(zp), indexing="ij")
    v = ((x * 7 + y * 13 + z * 29) % 61).astype(np.float32) / np.float32(61.0) + np.float32(0.25)
    v *= fov_mask(cyl, nx)[:, :, None]
    v[:, :, nz:] = 0
    return np.ascontiguousarray(v, np.float32)


def rows(P, nbins):
    """[2*P][nbins] float32 view-pair rows."""
    r, b = np.meshgrid(np.arange(2 * P), np.arange(nbins), indexing="ij")
    return np.ascontiguousarray(((r * 17 + b * 5) % 43).astype(np.float32) / np.float32(43.0), np.float32)


def sinograms(P, nviews, nbins):
    """Flat-file sinograms [P][nviews][nbins]: prompts (int16), randoms,
    normalisation with a dead detector block, attenuation (some < 1)."""
    p, v, b = np.meshgrid(np.arange(P), np.arange(nviews), np.arange(nbins), indexing="ij")
    prompts = ((p * 3 + v * 7 + b * 11) % 9).astype(np.int16)
    randoms = ((p + v * 3 + b * 5) % 13).astype(np.float32) / np.float32(26.0)
    norm = np.float32(0.75) + ((p * 5 + v + b * 3) % 11).astype(np.float32) / np.float32(22.0)
    norm[:, (v[0, :, 0] % 24) < 2, :] = 0  # dead detector views
    norm[:, :, nbins // 2 - 3:nbins // 2 - 1] = 0  # dead bins
    atten = np.float32(0.9) + ((p + v * 2 + b) % 17).astype(np.float32) / np.float32(8.0)
    scatter = ((p * 2 + v + b * 7) % 7).astype(np.float32) / np.float32(35.0)
    return (np.ascontiguousarray(prompts), np.ascontiguousarray(randoms, np.float32),
            np.ascontiguousarray(norm, np.float32), np.ascontiguousarray(atten, np.float32),
            np.ascontiguousarray(scatter, np.float32))


def reduce(a):
    """Size-independent summary of a float array, for tolerance checks:
    total, per-leading-index sums, per-last-index sums, 512 fixed samples."""
    a = np.asarray(a, np.float64)
    flat = a.reshape(-1)
    idx = (np.arange(512, dtype=np.int64) * 2654435761) % flat.size
    return {
        "total": np.array([flat.sum()]),
        "lead": a.reshape(a.shape[0], -1).sum(axis=1),
        "last": a.reshape(-1, a.shape[-1]).sum(axis=0),
        "samples": flat[idx],
    }


def digest(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
