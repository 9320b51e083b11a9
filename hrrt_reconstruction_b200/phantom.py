"""Seeded synthetic HRRT study: phantom, mu-map and the four sinograms the
reference reads (-p prompts int16, -d randoms, -n norm, -a attenuation
correction factors, -s scatter), in its flat-file layout.

No scanner data ships with the reference, so every benchmark and parity run
uses this generator.  The forward model is the one OP-OSEM assumes
(hrrt_osem3d_span3.cpp:1641-1818 with the ratio of :2500-2503):

    E[prompts] = FP(x) / (N*A) + r + s/N

with A = exp(FP(mu)) (the attenuation correction factor, >= 1), N the
normalisation (1 or per-bin lognormal), r a flat randoms level and s a smooth
scatter background stored in the normalised units the reference expects.
Prompts are Poisson draws, saturated to int16.

Phantom: water cylinder r = 100 mm, length 200 mm, activity 1 (mu = 0.0096
/mm), with six hot spheres of radius 5, 7.5, 10, 12.5, 15, 18 mm and activity
4, placed from the seed: each centre is drawn uniformly inside the cylinder
(shrunk by the sphere radius + 2 mm) and redrawn until it is at least 2 mm
from every sphere already placed.
"""
import numpy as np

MU_WATER = 0.0096
SPHERE_RADII = (5.0, 7.5, 10.0, 12.5, 15.0, 18.0)


def _grid(ctx):
    i = ctx.info
    g = ctx.geom
    xs = (np.arange(i.nx) - i.nx // 2) * g.binsize
    zs = (np.arange(i.zp) - (i.nz - 1) / 2.0) * g.plane_sep
    return xs, zs


def sphere_centres(seed, cyl_r=100.0, half_len=100.0):
    rng = np.random.default_rng(seed)
    placed = []
    for r in SPHERE_RADII:
        for _ in range(10000):
            rr = (cyl_r - r - 2.0) * np.sqrt(rng.random())
            th = 2 * np.pi * rng.random()
            c = np.array([rr * np.cos(th), rr * np.sin(th), (2 * rng.random() - 1) * (half_len - r - 2.0)])
            if all(np.linalg.norm(c - p) >= r + q + 2.0 for p, q in placed):
                placed.append((c, r))
                break
        else:
            raise RuntimeError("could not place spheres")
    return placed


def phantom(ctx, seed=0, activity=1.0, sphere_activity=4.0, sphere_scale=None, cyl_r=100.0, half_len=100.0):
    """Activity image [x][y][zp] on the context's grid (zero outside the FOV)."""
    i = ctx.info
    xs, zs = _grid(ctx)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    inside = (X ** 2 + Y ** 2) <= cyl_r ** 2
    zin = (np.abs(zs) <= half_len) & (np.arange(i.zp) < i.nz)
    img = np.zeros((i.nx, i.ny, i.zp), np.float32)
    img[inside[:, :, None] & zin[None, None, :]] = activity
    for k, (c, r) in enumerate(sphere_centres(seed, cyl_r, half_len)):
        a = sphere_activity if sphere_scale is None else sphere_activity * sphere_scale[k]
        d2 = (X - c[0]) ** 2 + (Y - c[1]) ** 2
        for z in np.nonzero(np.abs(zs - c[2]) <= r)[0]:
            if z >= i.nz:
                continue
            m = d2 + (zs[z] - c[2]) ** 2 <= r ** 2
            img[m, z] = a
    return img


def mu_map(ctx, cyl_r=100.0, half_len=100.0):
    img = phantom(ctx, seed=0, activity=MU_WATER, sphere_activity=MU_WATER, cyl_r=cyl_r, half_len=half_len)
    return img


def study(ctx, seed=0, total_counts=1e8, randoms_frac=0.20, scatter_frac=0.0, norm_sigma=0.0, sphere_scale=None,
          mu_line=None):
    """Sinograms of one synthetic study (all in the flat-file layout).

    Returns dict(prompts int16, randoms, norm or None, atten, scatter or None,
    image (the phantom), trues (noise-free)).  `mu_line` may pass a precomputed
    FP(mu) to reuse across frames.
    """
    rng = np.random.default_rng(seed + 1000)
    img = phantom(ctx, seed=seed, sphere_scale=sphere_scale)
    fp = ctx.forward_project(img)
    if mu_line is None:
        mu_line = ctx.forward_project(mu_map(ctx))
    atten = np.exp(mu_line, dtype=np.float32)
    if norm_sigma > 0:
        norm = np.exp(norm_sigma * rng.standard_normal(fp.shape, dtype=np.float32)).astype(np.float32)
    else:
        norm = None
    nn = norm if norm is not None else np.float32(1.0)
    t = fp / (nn * atten)
    nbins = fp.shape[2]
    # bins the projector never writes stay empty
    valid = fp > 0
    t_sum = float(t.sum(dtype=np.float64))
    scatter = None
    s_sum = 0.0
    if scatter_frac > 0:
        u = (np.arange(nbins) - nbins / 2.0) / (nbins / 4.0)
        prof = np.exp(-0.5 * u * u).astype(np.float32)
        s_shape = np.broadcast_to(prof, fp.shape) * valid
        s_over_n = s_shape / nn
        k = scatter_frac * t_sum / float(s_over_n.sum(dtype=np.float64))
        scatter = (k * s_shape).astype(np.float32)
        s_sum = scatter_frac * t_sum
    # randoms: flat over the bins the scanner sees, a fraction of all prompts
    nvalid = int(valid.sum())
    trues_and_scatter = t_sum + s_sum
    r_total = randoms_frac / (1.0 - randoms_frac) * trues_and_scatter
    scale = total_counts / (trues_and_scatter + r_total)
    t *= np.float32(scale)
    if scatter is not None:
        scatter *= np.float32(scale)
    r_level = np.float32(r_total * scale / nvalid)
    randoms = np.where(valid, r_level, np.float32(0)).astype(np.float32)
    mean = t + randoms + (scatter / nn if scatter is not None else 0)
    prompts = np.minimum(rng.poisson(mean), 32767).astype(np.int16)
    return dict(prompts=prompts, randoms=randoms, norm=norm, atten=atten, scatter=scatter, image=img,
                trues=t.astype(np.float32))
