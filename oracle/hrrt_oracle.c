/*
 * hrrt_oracle.c -- CPU restatement of the hrrt_osem3d OP-OSEM hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; see hrrt_oracle.h for the two
 * builds and how the oracle is pinned).  Plain C99, compiled with
 * -ffp-contract=off so that every float expression is the sequence of
 * IEEE single-precision operations the reference's SSE2 build performs.
 *
 * Reference files cited below, within the reference project:
 *   sbrt = hrrt_osem3d/hrrt_osem3dv_sbrt_span3.cpp   (projector, geometry)
 *   drv  = hrrt_osem3d/hrrt_osem3d_span3.cpp         (driver, update)
 *   fio  = hrrt_osem3d/file_io_processor.cpp         (flat-file reader)
 *
 * The back projection is restated as the direct sum the reference's
 * incremental scheme evaluates (sbrt:4162-4660; the direct form is the
 * reference's own y = c-1 start, sbrt:4285-4320): every voxel of the rotated
 * frame receives, for each ray through it, the linear interpolation of the
 * zero-padded sinogram at the row's blookup offset.  The reference's
 * incremental form reaches the same sums with a different rounding, so the
 * back projection is compared with a tolerance in both builds.
 */
#include "hrrt_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef orc_real R;

/* the reference code base's single-precision PI (sbrt uses the PI macro) */
#define ORC_PI 3.14159265358979f

struct orc_geom {
  /* scanner / image */
  int nrings, nbins, nviews, span, maxdel, subsets, groupmax, nseg, zshift;
  int nx, ny, nz, zp, c, segmentsize, sviews;
  float ring_radius, plane_sep, ring_spacing, x_size, y_size, rfov;
  /* driver parameters (drv:232, :289, :371-374) */
  int npskip, z_min, z_max;
  float eps1, eps2, eps3, image_max;
  /* tables */
  int *yb, *yt, *soff;               /* [nseg] */
  float *sin_theta, *cos_theta;      /* [nseg] */
  float *sin_psi, *cos_psi;          /* [nviews] */
  float *vcos, *vsin;                /* [groupmax][zshift] */
  int *cyl;                          /* [ny][2] */
  float *tantheta, *rescale;         /* [groupmax][nz] */
  int *fl_zzi;                       /* [ny][groupmax*2*zshift] */
  float *fl_zzz0;
  int *bl_zsa, *bl_zea, *bl_yra;     /* [ny][groupmax] */
  float *bl_yr2a;
  float *bp_scale;                   /* [nseg] */
  int16_t *nzmask;                   /* [nviews/2][nbins/2+1] */
  int *vieworder;                    /* [subsets][sviews] */
  int16_t *order;                    /* [subsets] */
  /* PSF resolution modelling (psf.cpp), off unless orc_set_psf */
  int psf_on, psf_h;                 /* half width h of the x / y kernels (taps -h..h-1 used) */
  int psf_zmin, psf_zmax;            /* planes of the z convolution */
  float *psf_fx, *psf_fy, *psf_fz;   /* [2h+1] */
  float *psf_normz;                  /* [zp] inverted z tap sums */
};

int orc_real_bytes(void) { return (int)sizeof(R); }
int orc_segmentsize(const orc_geom *g) { return g->segmentsize; }
int orc_zp(const orc_geom *g) { return g->zp; }
int orc_nz(const orc_geom *g) { return g->nz; }
int orc_nx(const orc_geom *g) { return g->nx; }
int orc_nviews(const orc_geom *g) { return g->nviews; }
int orc_sviews(const orc_geom *g) { return g->sviews; }
int orc_vieworder(const orc_geom *g, int s, int k) { return g->vieworder[s * g->sviews + k]; }
void orc_order(const orc_geom *g, int16_t *o) { memcpy(o, g->order, sizeof(int16_t) * g->subsets); }

/* z range of GetScannerParameter (drv:3516, :3537-3540) */
void orc_z_range(const orc_geom *g, int z_min, int z_max, int *out) {
  const int nz = g->nz;
  if (z_max == 0) z_max = nz - z_min;
  if (g->npskip > z_min) z_min = g->npskip;
  if (z_max > nz - g->npskip) z_max = nz - g->npskip;
  out[0] = z_min;
  out[1] = z_max;
}

void orc_set_params(orc_geom *g, int npskip, float eps1, float eps2, float eps3, float image_max) {
  g->npskip = npskip;
  g->eps1 = eps1;
  g->eps2 = eps2;
  g->eps3 = eps3;
  g->image_max = image_max;
}

void orc_destroy(orc_geom *g) {
  if (!g) return;
  void *p[] = {g->yb, g->yt, g->soff, g->sin_theta, g->cos_theta, g->sin_psi, g->cos_psi, g->vcos, g->vsin,
               g->cyl, g->tantheta, g->rescale, g->fl_zzi, g->fl_zzz0, g->bl_zsa, g->bl_zea, g->bl_yra,
               g->bl_yr2a, g->bp_scale, g->nzmask, g->vieworder, g->order,
               g->psf_fx, g->psf_fy, g->psf_fz, g->psf_normz};
  for (size_t i = 0; i < sizeof(p) / sizeof(p[0]); i++) free(p[i]);
  free(g);
}

#define NEW(T, n) ((T *)calloc((size_t)(n) > 0 ? (size_t)(n) : 1, sizeof(T)))

/* get_info (sbrt:159-191): plane range of segment group `group` */
static void group_planes(int nrings, int span, int group, int *zmin, int *zmax) {
  if (group == 0) {
    *zmin = 0;
    *zmax = 2 * nrings - 2;
  } else {
    *zmin = (span + 1) / 2 + (group - 1) * span;
    *zmax = 2 * nrings - 2 - *zmin;
  }
}

orc_geom *orc_create(int nrings, int nelements, int nangles, float ring_radius, float plane_sep, float binsize,
                     int span, int maxdel, int subsets) {
  if (span < 3 || span % 2 == 0 || nelements < 8 || nelements % 4 || nangles % 2 || subsets < 1 ||
      nangles % subsets)
    return NULL;
  orc_geom *g = NEW(orc_geom, 1);
  g->nrings = nrings;
  g->nbins = nelements;
  g->nviews = nangles;
  g->span = span;
  g->subsets = subsets;
  g->ring_radius = ring_radius;
  g->plane_sep = plane_sep;
  g->npskip = 3;
  g->z_min = 6;
  g->z_max = 200;
  g->eps1 = 5.E-2f;
  g->eps2 = 1.E-2f;
  g->eps3 = 1.E-10f;
  g->image_max = 1.E4f;
  /* GetScannerParameter (drv:3452-3551) */
  g->nz = nrings * 2 - 1;
  g->zp = (g->nz % 4 == 0) ? g->nz : (g->nz / 4 + 1) * 4;
  g->ring_spacing = 2.0f * plane_sep;
  g->groupmax = (maxdel - (span - 1) / 2) / span;
  if (g->groupmax < 1) {
    free(g);
    return NULL;
  }
  /* dependencies (sbrt:199-330), zoom = 1 */
  g->maxdel = g->groupmax * span + (span - 1) / 2;
  g->nx = g->ny = nelements;
  g->c = g->nx / 2;
  g->x_size = (binsize * nelements) / (1.0f * g->nx);
  g->y_size = g->x_size;
  g->sviews = nangles / subsets;
  g->nseg = 2 * g->groupmax + 1;
  g->zshift = span - 1;
  g->rfov = 0.95f * g->x_size * g->nx / 2.0f;
  const int nx = g->nx, ny = g->ny, nz = g->nz, G = g->groupmax, ZS = g->zshift, c = g->c;

  /* cylindrical window cylwiny (sbrt:339-356) */
  g->cyl = NEW(int, 2 * ny);
  for (int y = 0; y < ny; y++) {
    int flag = 0;
    for (int x = 0; x < nx; x++) {
      const int dx = x - c, dy = y - c;
      const float r2 = dx * g->x_size * dx * g->x_size + dy * g->y_size * dy * g->y_size;
      if (sqrtf(r2) <= g->rfov) {
        if (flag == 0) g->cyl[2 * y] = x;
        flag = 1;
      } else {
        if (flag == 1) g->cyl[2 * y + 1] = x;
        flag = 0;
      }
    }
  }

  /* segment angles and end-plane angles (sbrt:427-444) */
  g->sin_theta = NEW(float, g->nseg);
  g->cos_theta = NEW(float, g->nseg);
  g->vcos = NEW(float, G * ZS);
  g->vsin = NEW(float, G * ZS);
  g->sin_theta[0] = 0.0f;
  g->cos_theta[0] = 1.0f;
  for (int gr = 1; gr <= G; gr++) {
    float t = gr * span * g->ring_spacing;
    t = sqrtf(t * t + (2 * ring_radius) * (2 * ring_radius));
    g->sin_theta[2 * gr - 1] = gr * span * g->ring_spacing / t;
    g->cos_theta[2 * gr - 1] = (2.0f * ring_radius) / t;
    g->sin_theta[2 * gr] = -g->sin_theta[2 * gr - 1];
    g->cos_theta[2 * gr] = g->cos_theta[2 * gr - 1];
    for (int z = 0; z < ZS; z++) {
      const int zmin = span * gr - (span - 1) / 2;
      const int mean_rd = zmin + (z + 1) / 2;
      float u = mean_rd * g->ring_spacing;
      u = sqrtf(u * u + (2 * ring_radius) * (2 * ring_radius));
      g->vcos[(gr - 1) * ZS + z] = (2.0f * ring_radius) / u;
      g->vsin[(gr - 1) * ZS + z] = mean_rd * g->ring_spacing / u;
    }
  }

  /* plane ranges (sbrt:446-468); internal segment order is the file order */
  g->yb = NEW(int, g->nseg);
  g->yt = NEW(int, g->nseg);
  g->soff = NEW(int, g->nseg);
  g->yt[0] = nz - 1;
  for (int gr = 1; gr <= G; gr++) {
    int zmin, zmax;
    group_planes(nrings, span, gr, &zmin, &zmax);
    if (zmax - zmin + 1 < 2 * ZS + 1) {
      orc_destroy(g);
      return NULL;
    }
    g->yb[2 * gr] = g->yb[2 * gr - 1] = zmin;
    g->yt[2 * gr] = g->yt[2 * gr - 1] = zmax;
  }
  for (int s = 0; s < g->nseg; s++) {
    g->soff[s] = g->segmentsize;
    g->segmentsize += g->yt[s] - g->yb[s] + 1;
  }

  /* view angles (sbrt:476-486): single-precision sin, double sqrt */
  g->sin_psi = NEW(float, nangles);
  g->cos_psi = NEW(float, nangles);
  g->sin_psi[0] = 0.0f;
  g->cos_psi[0] = 1.0f;
  g->sin_psi[nangles / 2] = 1.0f;
  g->cos_psi[nangles / 2] = 0.0f;
  const float dpsi = ORC_PI / nangles;
  for (int v = 1; v < nangles / 2; v++) {
    g->sin_psi[v] = sinf(v * dpsi);
    g->cos_psi[v] = (float)sqrt(1. - (double)(g->sin_psi[v] * g->sin_psi[v]));
    g->sin_psi[nangles - v] = g->sin_psi[v];
    g->cos_psi[nangles - v] = -g->cos_psi[v];
  }

  /* calculatevieworder (sbrt:144-152) and sequence (drv:535-580) */
  g->vieworder = NEW(int, subsets * g->sviews);
  for (int i = 0; i < subsets; i++)
    for (int k = 0; k < g->sviews; k++) g->vieworder[i * g->sviews + k] = i + subsets * k;
  g->order = NEW(int16_t, subsets);
  {
    int *done = NEW(int, subsets);
    done[0] = 1;
    for (int i = 1; i < subsets; ++i) {
      int ibest = 0, dbest = 0, j = 0;
      while (j < subsets) {
        while (j < subsets && done[j] == 1) j += 1;
        if (j < subsets) {
          const int k = g->order[i - 1];
          int d = abs(j - k);
          if (subsets - abs(j - k) < d) d = subsets - abs(j - k);
          if (d > dbest) {
            dbest = d;
            ibest = j;
          }
          j += 1;
        }
      }
      g->order[i] = (int16_t)ibest;
      done[ibest] = 1;
    }
    free(done);
  }

  /* tantheta / rescalearray with end-plane angles (sbrt:529-542) */
  g->tantheta = NEW(float, G * nz);
  g->rescale = NEW(float, G * nz);
  for (int th = 2, gr = 0; th < g->nseg; th += 2, gr++) {
    for (int yr = g->yb[th]; yr <= g->yt[th]; yr++) {
      float t = g->sin_theta[th] / g->cos_theta[th];
      float r = g->y_size / fabsf(g->cos_theta[th]);
      int zs = yr - g->yb[th];
      if (zs >= ZS) zs = g->yt[th] - yr;
      if (zs < ZS) {
        t = g->vsin[gr * ZS + zs] / g->vcos[gr * ZS + zs];
        t = -t;
        r = g->y_size / fabsf(g->vcos[gr * ZS + zs]);
      }
      t = -t / 1.0f;
      g->tantheta[gr * nz + yr] = t;
      g->rescale[gr * nz + yr] = r;
    }
  }

  /* flookup: end-plane positions of the forward projection (sbrt:545-578) */
  const int FS = G * 2 * ZS;
  g->fl_zzi = NEW(int, ny * FS);
  g->fl_zzz0 = NEW(float, ny * FS);
  for (int y = 0; y < ny; y++)
    for (int th = 2, gr = 0; th < g->nseg; th += 2, gr++) {
      int i = y * FS + gr * ZS * 2;
      for (int yr = g->yb[th]; yr < g->yb[th] + ZS; yr++, i++) {
        const float zz = yr + ((y - c) * g->tantheta[gr * nz + yr]);
        const int z = (int)zz;
        g->fl_zzz0[i] = zz - z;
        g->fl_zzi[i] = z;
      }
      for (int yr = g->yt[th] - ZS + 1; yr <= g->yt[th]; yr++, i++) {
        const float zz = yr + ((y - c) * g->tantheta[gr * nz + yr]);
        const int z = (int)zz;
        g->fl_zzz0[i] = zz - z;
        g->fl_zzi[i] = z;
      }
    }

  /* blookup: per-row plane window of the back projection (sbrt:672-700) */
  g->bl_zsa = NEW(int, ny * G);
  g->bl_zea = NEW(int, ny * G);
  g->bl_yra = NEW(int, ny * G);
  g->bl_yr2a = NEW(float, ny * G);
  for (int y = 0; y < ny; y++)
    for (int th = 2, gr = 0; th < g->nseg; th += 2, gr++) {
      const float tb = -g->sin_theta[th] / g->cos_theta[th];
      const float yr0 = -(y - c) * tb;
      float yr2 = fabsf(yr0) - (int)fabsf(yr0);
      int yri2 = (int)yr0;
      if (yr0 < 0) {
        yr2 = 1 - yr2;
        yri2 -= 1;
      }
      int zs = g->yb[th] - 1 - yri2, ze = g->yt[th] - yri2, yr = g->yb[th] - 1;
      if (zs < 0) {
        yr = yr - zs;
        zs = 0;
      }
      if (ze > nz - 1) ze = nz - 1;
      const int i = y * G + gr;
      g->bl_zsa[i] = zs;
      g->bl_zea[i] = ze;
      g->bl_yra[i] = yr;
      g->bl_yr2a[i] = yr2;
    }

  /* per-segment back-projection weight (sbrt:1637-1649) */
  g->bp_scale = NEW(float, g->nseg);
  for (int k = 0; k < g->nseg; k++)
    g->bp_scale[k] = g->cos_theta[k] * g->cos_theta[k] * g->cos_theta[k] * span * g->ring_spacing / (2 * ring_radius);

  /* norm_zero_mask: all quads active until a normalisation is read (sbrt:333) */
  g->nzmask = NEW(int16_t, (nangles / 2) * (nx / 2 + 1));
  for (int i = 0; i < (nangles / 2) * (nx / 2 + 1); i++) g->nzmask[i] = 1;
  return g;
}

void orc_cylwiny(const orc_geom *g, int *cyl) { memcpy(cyl, g->cyl, sizeof(int) * 2 * g->ny); }
void orc_trig(const orc_geom *g, float *st, float *ct, float *sp, float *cp) {
  memcpy(st, g->sin_theta, sizeof(float) * g->nseg);
  memcpy(ct, g->cos_theta, sizeof(float) * g->nseg);
  memcpy(sp, g->sin_psi, sizeof(float) * g->nviews);
  memcpy(cp, g->cos_psi, sizeof(float) * g->nviews);
}
void orc_tantheta(const orc_geom *g, float *t, float *r) {
  memcpy(t, g->tantheta, sizeof(float) * g->groupmax * g->nz);
  memcpy(r, g->rescale, sizeof(float) * g->groupmax * g->nz);
}
void orc_flookup(const orc_geom *g, int *zzi, float *zzz0) {
  const size_t n = (size_t)g->ny * g->groupmax * 2 * g->zshift;
  memcpy(zzi, g->fl_zzi, sizeof(int) * n);
  memcpy(zzz0, g->fl_zzz0, sizeof(float) * n);
}
void orc_blookup(const orc_geom *g, int *zsa, int *zea, int *yra, float *yr2a) {
  const size_t n = (size_t)g->ny * g->groupmax;
  memcpy(zsa, g->bl_zsa, sizeof(int) * n);
  memcpy(zea, g->bl_zea, sizeof(int) * n);
  memcpy(yra, g->bl_yra, sizeof(int) * n);
  memcpy(yr2a, g->bl_yr2a, sizeof(float) * n);
}
void orc_get_norm_zero_mask(const orc_geom *g, int16_t *m) {
  memcpy(m, g->nzmask, sizeof(int16_t) * (g->nviews / 2) * (g->nx / 2 + 1));
}
void orc_set_norm_zero_mask(orc_geom *g, const int16_t *m) {
  memcpy(g->nzmask, m, sizeof(int16_t) * (g->nviews / 2) * (g->nx / 2 + 1));
}

/* ------------------------------------------------------------------------ */
/* Forward projection                                                       */
/* ------------------------------------------------------------------------ */

/* Bilinear sample of the image column at the rotated position of voxel
 * (xx, yy), all zp planes (forward_proj3d_view1_thread, sbrt:1848-1890).
 * The reference tests xx0 twice and never yy0 > nx-2; a sample in the disk
 * never reaches the far edge, and the flat-index guard below keeps the
 * restatement inside the array if one ever did.  Returns 0 when the point
 * is outside (the reference then zeroes the column). */
static int sample(const orc_geom *g, const R *img, int xx, int yy, float cosv, float sinv, R *out) {
  const int nx = g->nx, c = g->c, zp = g->zp;
  const float xx0 = (xx - c) * cosv - (yy - c) * sinv + c;
  const float yy0 = (xx - c) * sinv + (yy - c) * cosv + c;
  if (xx0 < 0 || xx0 > nx - 2 || yy0 < 0 || xx0 > nx - 2) return 0;
  const int ix = (int)xx0, iy = (int)yy0;
  const float x1 = xx0 - ix, y1 = yy0 - iy;
  const size_t b1 = ((size_t)ix * g->ny + iy) * zp, b2 = b1 + (size_t)g->ny * zp, b3 = b1 + zp, b4 = b2 + zp;
  if (b4 + zp > (size_t)nx * g->ny * zp) return 0;
  const float w0 = (1 - x1) * (1 - y1), w1 = x1 * (1 - y1), w2 = y1 * (1 - x1), w3 = y1 * x1;
  const R *r1 = img + b1, *r2 = img + b2, *r3 = img + b3, *r4 = img + b4;
  if (x1 != 0 && y1 != 0) {
    for (int z = 0; z < zp; z++) out[z] = (r1[z] * w0 + r2[z] * w1) + (r3[z] * w2 + r4[z] * w3);
  } else if (x1 == 0 && y1 != 0) {
    for (int z = 0; z < zp; z++) out[z] = r1[z] * w0 + r3[z] * w2;
  } else if (x1 != 0 && y1 == 0) {
    for (int z = 0; z < zp; z++) out[z] = r1[z] * w0 + r2[z] * w1;
  } else {
    for (int z = 0; z < zp; z++) out[z] = r1[z];
  }
  return 1;
}

/* forward_proj3d_view1_thread (sbrt:1728-1978) and the copy into the
 * estimate rows of forward_proj3d_thread1 (sbrt:1373-1449).
 * Per quad x the four lanes are bins (view,x), (view,nx-x), (view+90,x),
 * (view+90,nx-x); `pam` holds the lanes of the rows y < c and `pam2` those
 * of the mirrored rows nx-y. */
void orc_fp_pair(const orc_geom *g, const R *img, int view, R *rows) {
  const int nx = g->nx, c = g->c, nz = g->nz, zp = g->zp, G = g->groupmax, ZS = g->zshift, N = g->nbins;
  const int ss = g->segmentsize, FS = G * 2 * ZS;
  const float cosv = g->cos_psi[view], sinv = g->sin_psi[view];
  /* lanes: [plane][4], with one zero plane beyond nz for z+1 reads */
  R *pam = NEW(R, (zp + 2) * 4), *pam2 = NEW(R, (zp + 2) * 4);
  R *rim[8];
  for (int i = 0; i < 8; i++) rim[i] = NEW(R, zp);
  R *p0 = NEW(R, nz * 4);                       /* theta 0 lanes [plane][4] */
  R *p1 = NEW(R, (size_t)(G + 1) * nz * 4);     /* segment 2k lanes, k = 1..G */
  R *p2 = NEW(R, (size_t)(G + 1) * nz * 4);     /* segment 2k-1 */
#define L(a, k, z, l) a[(((size_t)(k)) * nz + (z)) * 4 + (l)]
  for (int x = 1; x <= c; x++) {
    const int *cy = g->cyl + 2 * x;
    const int masked = g->nzmask[view * (nx / 2 + 1) + x] == 0;
    if (cy[0] == 0 && cy[1] == 0) continue;  /* the copy skips such quads */
    memset(p0, 0, sizeof(R) * nz * 4);
    memset(p1, 0, sizeof(R) * (G + 1) * nz * 4);
    memset(p2, 0, sizeof(R) * (G + 1) * nz * 4);
    if (cy[0] != cy[1] && !masked) {
      /* centre row y = c initialises every plane (sbrt:1818-1846) */
      const int cx[4] = {x, nx - x, c, c}, cyy[4] = {c, c, x, nx - x};
      for (int i = 0; i < 4; i++)
        if (!sample(g, img, cx[i], cyy[i], cosv, sinv, rim[i])) memset(rim[i], 0, sizeof(R) * zp);
      for (int z = 0; z < nz; z++)
        for (int l = 0; l < 4; l++) L(p0, 0, z, l) = rim[l][z];
      for (int k = 1; k <= G; k++)
        for (int z = g->yb[2 * k]; z <= g->yt[2 * k]; z++)
          for (int l = 0; l < 4; l++) L(p1, k, z, l) = L(p2, k, z, l) = rim[l][z];
      for (int y = cy[0]; y < c; y++) {
        const int px[8] = {x, nx - x, nx - y, nx - y, x, nx - x, y, y};
        const int py[8] = {y, y, x, nx - x, nx - y, nx - y, x, nx - x};
        for (int i = 0; i < 8; i++)
          if (!sample(g, img, px[i], py[i], cosv, sinv, rim[i])) memset(rim[i], 0, sizeof(R) * zp);
        for (int z = 0; z < nz; z++)
          for (int l = 0; l < 4; l++) {
            pam[z * 4 + l] = rim[l][z];
            pam2[z * 4 + l] = rim[4 + l][z];
          }
        /* theta 0 */
        for (int z = 0; z < nz; z++)
          for (int l = 0; l < 4; l++) L(p0, 0, z, l) = L(p0, 0, z, l) + (pam[z * 4 + l] + pam2[z * 4 + l]);
        const int *zi1 = g->fl_zzi + y * FS, *zi2 = g->fl_zzi + (nx - y) * FS;
        const float *f1a = g->fl_zzz0 + y * FS, *f2a = g->fl_zzz0 + (nx - y) * FS;
        for (int th = 2, gr = 0; th < g->nseg; th += 2, gr++) {
          const int k = th / 2;
          int yri = gr * ZS * 2;
          if (zi1[yri] < 0) continue;
          if (zi2[yri + ZS * 2 - 1] > nz - 1) continue;
          /* end planes: per-plane positions; the weight of one row's sample
           * is the mirrored row's fraction (sbrt:1914-1921) */
          int yr;
          for (yr = g->yb[th]; yr < g->yb[th] + ZS; yr++, yri++) {
            const int z = zi1[yri], z2 = zi2[yri];
            const float f1 = f1a[yri], f2 = f2a[yri];
            for (int l = 0; l < 4; l++) {
              L(p1, k, yr, l) = L(p1, k, yr, l) + ((pam2[(z2 + 1) * 4 + l] + pam[z * 4 + l]) * f2 +
                                                   (pam[(z + 1) * 4 + l] + pam2[z2 * 4 + l]) * f1);
              L(p2, k, yr, l) = L(p2, k, yr, l) + ((pam[(z2 + 1) * 4 + l] + pam2[z * 4 + l]) * f2 +
                                                   (pam2[(z + 1) * 4 + l] + pam[z2 * 4 + l]) * f1);
            }
          }
          /* middle planes: one position, advancing a plane per plane
           * (sbrt:1922-1938) */
          float zz0 = yr + (y - c) * g->tantheta[gr * nz + yr];
          int z = (int)zz0;
          const float c1 = zz0 - z;
          zz0 = yr + (c - y) * g->tantheta[gr * nz + yr];
          int z2 = (int)zz0;
          const float c2 = zz0 - z2;
          for (; yr <= g->yt[th] - ZS; yr++, z++, z2++)
            for (int l = 0; l < 4; l++) {
              L(p1, k, yr, l) = L(p1, k, yr, l) + (c2 * (pam2[(z2 + 1) * 4 + l] + pam[z * 4 + l]) +
                                                   c1 * (pam[(z + 1) * 4 + l] + pam2[z2 * 4 + l]));
              L(p2, k, yr, l) = L(p2, k, yr, l) + (c2 * (pam[(z2 + 1) * 4 + l] + pam2[z * 4 + l]) +
                                                   c1 * (pam2[(z + 1) * 4 + l] + pam[z2 * 4 + l]));
            }
          for (yr = g->yt[th] - ZS + 1; yr <= g->yt[th]; yr++, yri++) {
            const int ze = zi1[yri], ze2 = zi2[yri];
            const float f1 = f1a[yri], f2 = f2a[yri];
            for (int l = 0; l < 4; l++) {
              L(p1, k, yr, l) = L(p1, k, yr, l) + ((pam2[(ze2 + 1) * 4 + l] + pam[ze * 4 + l]) * f2 +
                                                   (pam[(ze + 1) * 4 + l] + pam2[ze2 * 4 + l]) * f1);
              L(p2, k, yr, l) = L(p2, k, yr, l) + ((pam[(ze2 + 1) * 4 + l] + pam2[ze * 4 + l]) * f2 +
                                                   (pam2[(ze + 1) * 4 + l] + pam[ze2 * 4 + l]) * f1);
            }
          }
        }
      }
      /* scaling (sbrt:1953-1976) */
      for (int z = 0; z < nz; z++)
        for (int l = 0; l < 4; l++) L(p0, 0, z, l) = L(p0, 0, z, l) * g->y_size;
      for (int th = 2, gr = 0; th < g->nseg; th += 2, gr++) {
        const int k = th / 2;
        int yr;
        for (yr = g->yb[th]; yr < g->yb[th] + ZS; yr++)
          for (int l = 0; l < 4; l++) {
            L(p1, k, yr, l) = L(p1, k, yr, l) * g->rescale[gr * nz + yr];
            L(p2, k, yr, l) = L(p2, k, yr, l) * g->rescale[gr * nz + yr];
          }
        const float cm = g->rescale[gr * nz + yr];
        for (; yr <= g->yt[th] - ZS; yr++)
          for (int l = 0; l < 4; l++) {
            L(p1, k, yr, l) = L(p1, k, yr, l) * cm;
            L(p2, k, yr, l) = L(p2, k, yr, l) * cm;
          }
        for (yr = g->yt[th] - ZS + 1; yr <= g->yt[th]; yr++)
          for (int l = 0; l < 4; l++) {
            L(p1, k, yr, l) = L(p1, k, yr, l) * g->rescale[gr * nz + yr];
            L(p2, k, yr, l) = L(p2, k, yr, l) * g->rescale[gr * nz + yr];
          }
      }
    }
    /* A quad the projector skips (norm-zero mask) keeps, in the reference,
     * the previous view's values in its buffer; the OP ratio discards them
     * because the prompts there are masked to zero.  Here it is zero. */
    if (cy[0] == 0) continue;
    const int xri = N - x;
    /* copy-out (sbrt:1395-1434); for x = c lane 1 overwrites lane 0 */
    for (int yr = 0; yr < nz; yr++) {
      rows[(size_t)yr * N + x] = L(p0, 0, yr, 0);
      rows[(size_t)yr * N + xri] = L(p0, 0, yr, 1);
      rows[(size_t)(yr + ss) * N + x] = L(p0, 0, yr, 2);
      rows[(size_t)(yr + ss) * N + xri] = L(p0, 0, yr, 3);
    }
    for (int k = 1; k <= G; k++) {
      const int yb = g->yb[2 * k];
      for (int yr = yb; yr <= g->yt[2 * k]; yr++) {
        const size_t a = (size_t)(g->soff[2 * k] + yr - yb), b = (size_t)(g->soff[2 * k - 1] + yr - yb);
        rows[a * N + x] = L(p1, k, yr, 0);
        rows[a * N + xri] = L(p1, k, yr, 1);
        rows[(a + ss) * N + x] = L(p1, k, yr, 2);
        rows[(a + ss) * N + xri] = L(p1, k, yr, 3);
        rows[b * N + x] = L(p2, k, yr, 0);
        rows[b * N + xri] = L(p2, k, yr, 1);
        rows[(b + ss) * N + x] = L(p2, k, yr, 2);
        rows[(b + ss) * N + xri] = L(p2, k, yr, 3);
      }
    }
  }
#undef L
  free(pam);
  free(pam2);
  for (int i = 0; i < 8; i++) free(rim[i]);
  free(p0);
  free(p1);
  free(p2);
}

/* Sample position of voxel (xx, yy) in the forward projector (as sample()):
 * the four corner offsets into the image and their weights; 0 when outside. */
static int sample_taps(const orc_geom *g, int xx, int yy, float cosv, float sinv, size_t b[4], float w[4]) {
  const int nx = g->nx, c = g->c, zp = g->zp;
  const float xx0 = (xx - c) * cosv - (yy - c) * sinv + c;
  const float yy0 = (xx - c) * sinv + (yy - c) * cosv + c;
  if (xx0 < 0 || xx0 > nx - 2 || yy0 < 0 || xx0 > nx - 2) return 0;
  const int ix = (int)xx0, iy = (int)yy0;
  const float x1 = xx0 - ix, y1 = yy0 - iy;
  b[0] = ((size_t)ix * g->ny + iy) * zp;
  b[1] = b[0] + (size_t)g->ny * zp;
  b[2] = b[0] + zp;
  b[3] = b[1] + zp;
  if (b[3] + zp > (size_t)nx * g->ny * zp) return 0;
  w[0] = (1 - x1) * (1 - y1);
  w[1] = x1 * (1 - y1);
  w[2] = y1 * (1 - x1);
  w[3] = y1 * x1;
  return 1;
}

/* Exact adjoint of orc_fp_pair: image += FP^T rows for one view pair.  Every
 * step of the forward projection is transposed: the copy into the rows (for
 * quad x = c the bins of lanes 1 and 3 are the ones written), the scaling,
 * the z interpolation of each segment (end planes with their own positions,
 * middle planes advancing one plane per plane, the same skipped groups), the
 * centre-row initialisation and the bilinear samples.  No counterpart in the
 * reference, whose back projector is not the transpose of its forward
 * projector; <FP x, y> = <x, FP^T y> holds to rounding. */
void orc_fp_adjoint(const orc_geom *g, const R *rows, int view, R *img) {
  const int nx = g->nx, c = g->c, nz = g->nz, zp = g->zp, G = g->groupmax, ZS = g->zshift, N = g->nbins;
  const int ss = g->segmentsize, FS = G * 2 * ZS;
  const float cosv = g->cos_psi[view], sinv = g->sin_psi[view];
  R *q0 = NEW(R, nz * 4);
  R *q1 = NEW(R, (size_t)(G + 1) * nz * 4);
  R *q2 = NEW(R, (size_t)(G + 1) * nz * 4);
  R *gp = NEW(R, (size_t)(nz + 2) * 4), *gp2 = NEW(R, (size_t)(nz + 2) * 4);
#define L(a, k, z, l) a[(((size_t)(k)) * nz + (z)) * 4 + (l)]
  for (int x = 1; x <= c; x++) {
    const int *cy = g->cyl + 2 * x;
    if (cy[0] == 0) continue;                     /* no rows written */
    if (cy[0] == cy[1]) continue;                 /* never projected */
    if (g->nzmask[view * (nx / 2 + 1) + x] == 0) continue;
    const int xri = N - x;
    /* transpose of the copy-out: lane values from the rows */
    memset(q0, 0, sizeof(R) * nz * 4);
    memset(q1, 0, sizeof(R) * (G + 1) * nz * 4);
    memset(q2, 0, sizeof(R) * (G + 1) * nz * 4);
    const int l0 = (x == c) ? 1 : 0, l2 = (x == c) ? 3 : 2;  /* for x = c the later lane wins */
    for (int yr = 0; yr < nz; yr++) {
      L(q0, 0, yr, l0) += rows[(size_t)yr * N + x];
      if (x != c) L(q0, 0, yr, 1) += rows[(size_t)yr * N + xri];
      L(q0, 0, yr, l2) += rows[(size_t)(yr + ss) * N + x];
      if (x != c) L(q0, 0, yr, 3) += rows[(size_t)(yr + ss) * N + xri];
      for (int l = 0; l < 4; l++) L(q0, 0, yr, l) *= g->y_size;
    }
    for (int k = 1; k <= G; k++) {
      const int th = 2 * k, gr = k - 1, yb = g->yb[th];
      for (int yr = yb; yr <= g->yt[th]; yr++) {
        const size_t a = (size_t)(g->soff[th] + yr - yb), b = (size_t)(g->soff[th - 1] + yr - yb);
        int zs = yr - yb;
        if (zs >= ZS) zs = g->yt[th] - yr;
        const float sc = (zs < ZS) ? g->rescale[gr * nz + yr] : g->rescale[gr * nz + yb + ZS];
        L(q1, k, yr, l0) += rows[a * N + x];
        L(q1, k, yr, l2) += rows[(a + ss) * N + x];
        L(q2, k, yr, l0) += rows[b * N + x];
        L(q2, k, yr, l2) += rows[(b + ss) * N + x];
        if (x != c) {
          L(q1, k, yr, 1) += rows[a * N + xri];
          L(q1, k, yr, 3) += rows[(a + ss) * N + xri];
          L(q2, k, yr, 1) += rows[b * N + xri];
          L(q2, k, yr, 3) += rows[(b + ss) * N + xri];
        }
        for (int l = 0; l < 4; l++) {
          L(q1, k, yr, l) *= sc;
          L(q2, k, yr, l) *= sc;
        }
      }
    }
    size_t tb[4];
    float tw[4];
    /* centre row: every plane of every segment took the four centre samples */
    {
      const int cx[4] = {x, nx - x, c, c}, cyy[4] = {c, c, x, nx - x};
      for (int i = 0; i < 4; i++) {
        if (!sample_taps(g, cx[i], cyy[i], cosv, sinv, tb, tw)) continue;
        for (int z = 0; z < nz; z++) {
          R v = L(q0, 0, z, i);
          for (int k = 1; k <= G; k++)
            if (z >= g->yb[2 * k] && z <= g->yt[2 * k]) v += L(q1, k, z, i) + L(q2, k, z, i);
          for (int t = 0; t < 4; t++) img[tb[t] + z] += tw[t] * v;
        }
      }
    }
    for (int y = cy[0]; y < c; y++) {
      memset(gp, 0, sizeof(R) * (nz + 2) * 4);
      memset(gp2, 0, sizeof(R) * (nz + 2) * 4);
      for (int z = 0; z < nz; z++)
        for (int l = 0; l < 4; l++) {
          gp[z * 4 + l] += L(q0, 0, z, l);
          gp2[z * 4 + l] += L(q0, 0, z, l);
        }
      const int *zi1 = g->fl_zzi + y * FS, *zi2 = g->fl_zzi + (nx - y) * FS;
      const float *f1a = g->fl_zzz0 + y * FS, *f2a = g->fl_zzz0 + (nx - y) * FS;
      for (int th = 2, gr = 0; th < g->nseg; th += 2, gr++) {
        const int k = th / 2;
        int yri = gr * ZS * 2;
        if (zi1[yri] < 0) continue;
        if (zi2[yri + ZS * 2 - 1] > nz - 1) continue;
        int yr;
        for (yr = g->yb[th]; yr < g->yb[th] + ZS; yr++, yri++) {
          const int z = zi1[yri], z2 = zi2[yri];
          const float f1 = f1a[yri], f2 = f2a[yri];
          for (int l = 0; l < 4; l++) {
            const R r1 = L(q1, k, yr, l), r2 = L(q2, k, yr, l);
            gp2[(z2 + 1) * 4 + l] += f2 * r1; gp[z * 4 + l] += f2 * r1;
            gp[(z + 1) * 4 + l] += f1 * r1;   gp2[z2 * 4 + l] += f1 * r1;
            gp[(z2 + 1) * 4 + l] += f2 * r2;  gp2[z * 4 + l] += f2 * r2;
            gp2[(z + 1) * 4 + l] += f1 * r2;  gp[z2 * 4 + l] += f1 * r2;
          }
        }
        float zz0 = yr + (y - c) * g->tantheta[gr * nz + yr];
        int z = (int)zz0;
        const float c1 = zz0 - z;
        zz0 = yr + (c - y) * g->tantheta[gr * nz + yr];
        int z2 = (int)zz0;
        const float c2 = zz0 - z2;
        for (; yr <= g->yt[th] - ZS; yr++, z++, z2++)
          for (int l = 0; l < 4; l++) {
            const R r1 = L(q1, k, yr, l), r2 = L(q2, k, yr, l);
            gp2[(z2 + 1) * 4 + l] += c2 * r1; gp[z * 4 + l] += c2 * r1;
            gp[(z + 1) * 4 + l] += c1 * r1;   gp2[z2 * 4 + l] += c1 * r1;
            gp[(z2 + 1) * 4 + l] += c2 * r2;  gp2[z * 4 + l] += c2 * r2;
            gp2[(z + 1) * 4 + l] += c1 * r2;  gp[z2 * 4 + l] += c1 * r2;
          }
        for (yr = g->yt[th] - ZS + 1; yr <= g->yt[th]; yr++, yri++) {
          const int ze = zi1[yri], ze2 = zi2[yri];
          const float f1 = f1a[yri], f2 = f2a[yri];
          for (int l = 0; l < 4; l++) {
            const R r1 = L(q1, k, yr, l), r2 = L(q2, k, yr, l);
            gp2[(ze2 + 1) * 4 + l] += f2 * r1; gp[ze * 4 + l] += f2 * r1;
            gp[(ze + 1) * 4 + l] += f1 * r1;   gp2[ze2 * 4 + l] += f1 * r1;
            gp[(ze2 + 1) * 4 + l] += f2 * r2;  gp2[ze * 4 + l] += f2 * r2;
            gp2[(ze + 1) * 4 + l] += f1 * r2;  gp[ze2 * 4 + l] += f1 * r2;
          }
        }
      }
      /* the eight samples of this row; planes >= nz of pam/pam2 are zero in
       * the forward projection, so their gradient is dropped */
      const int px[8] = {x, nx - x, nx - y, nx - y, x, nx - x, y, y};
      const int py[8] = {y, y, x, nx - x, nx - y, nx - y, x, nx - x};
      for (int i = 0; i < 8; i++) {
        if (!sample_taps(g, px[i], py[i], cosv, sinv, tb, tw)) continue;
        const R *src = (i < 4) ? gp : gp2;
        const int l = i & 3;
        for (int z = 0; z < nz; z++) {
          const R v = src[z * 4 + l];
          for (int t = 0; t < 4; t++) img[tb[t] + z] += tw[t] * v;
        }
      }
    }
  }
#undef L
  free(q0);
  free(q1);
  free(q2);
  free(gp);
  free(gp2);
}

/* ------------------------------------------------------------------------ */
/* Back projection                                                          */
/* ------------------------------------------------------------------------ */

/* back_proj3d_thread1 + back_proj3d_view_n1thread (sbrt:1622-1699,
 * sbrt:4162-4660) as direct sums.  Rows are first weighted by
 * cos^3(theta)*span*ring_spacing/(2R) (sbrt:1637-1649); the segment planes
 * are zero-padded by one plane at each end (sbrt:1684-1687).  For quad x and
 * row y < c, sumt1 (voxels (x,y), (nx-x,y), (nx-y,x), (nx-y,nx-x)) adds
 * segment 2k at blookup[y] and segment 2k-1 at blookup[nx-y]; sumt2 (voxels
 * (x,nx-y), (nx-x,nx-y), (y,x), (y,nx-x)) the converse.  The reference
 * assigns a voxel's first ray and adds its second (sbrt:4560-4640); the sum
 * over both rays is what is stored.  Planes >= nz stay zero. */
void orc_bp_pair(const orc_geom *g, const R *rows_in, int view, R *ib) {
  const int nx = g->nx, c = g->c, nz = g->nz, zp = g->zp, G = g->groupmax, N = g->nbins, ss = g->segmentsize;
  const size_t vol = (size_t)nx * g->ny * zp;
  memset(ib, 0, sizeof(R) * vol);
  /* weighted rows */
  R *rows = NEW(R, (size_t)2 * ss * N);
  for (int s = 0, r = 0; s < g->nseg; s++)
    for (int yr = g->yb[s]; yr <= g->yt[s]; yr++, r++)
      for (int xr = 0; xr < N; xr++) {
        rows[(size_t)r * N + xr] = rows_in[(size_t)r * N + xr] * g->bp_scale[s];
        rows[(size_t)(r + ss) * N + xr] = rows_in[(size_t)(r + ss) * N + xr] * g->bp_scale[s];
      }
  /* lanes [plane+1][4] with a zero plane at each end of every segment */
  const int PL = nz + 2;
  R *q0 = NEW(R, PL * 4), *q1 = NEW(R, (size_t)(G + 1) * PL * 4), *q2 = NEW(R, (size_t)(G + 1) * PL * 4);
  R *s1 = NEW(R, nz * 4), *s2 = NEW(R, nz * 4);
#define Q(a, k, z, l) a[(((size_t)(k)) * PL + (z) + 1) * 4 + (l)]
  for (int x = 0; x <= c; x++) {
    const int ystart = g->cyl[2 * x], yend = g->cyl[2 * x + 1];
    if (ystart == 0 && yend == 0) continue;
    if (g->nzmask[view * (nx / 2 + 1) + x] == 0) continue;  /* masked: zero contribution */
    const int xri = N - x;
    memset(q0, 0, sizeof(R) * PL * 4);
    memset(q1, 0, sizeof(R) * (G + 1) * PL * 4);
    memset(q2, 0, sizeof(R) * (G + 1) * PL * 4);
    for (int z = 0; z < nz; z++) {
      Q(q0, 0, z, 0) = rows[(size_t)z * N + x];
      Q(q0, 0, z, 1) = rows[(size_t)z * N + xri];
      Q(q0, 0, z, 2) = rows[(size_t)(z + ss) * N + x];
      Q(q0, 0, z, 3) = rows[(size_t)(z + ss) * N + xri];
    }
    for (int k = 1; k <= G; k++) {
      const int yb = g->yb[2 * k];
      for (int yr = yb; yr <= g->yt[2 * k]; yr++) {
        const size_t a = (size_t)(g->soff[2 * k] + yr - yb), b = (size_t)(g->soff[2 * k - 1] + yr - yb);
        Q(q1, k, yr, 0) = rows[a * N + x];
        Q(q1, k, yr, 1) = rows[a * N + xri];
        Q(q1, k, yr, 2) = rows[(a + ss) * N + x];
        Q(q1, k, yr, 3) = rows[(a + ss) * N + xri];
        Q(q2, k, yr, 0) = rows[b * N + x];
        Q(q2, k, yr, 1) = rows[b * N + xri];
        Q(q2, k, yr, 2) = rows[(b + ss) * N + x];
        Q(q2, k, yr, 3) = rows[(b + ss) * N + xri];
      }
    }
    for (int y = ystart; y <= c; y++) {
      for (int z = 0; z < nz; z++)
        for (int l = 0; l < 4; l++) s1[z * 4 + l] = s2[z * 4 + l] = Q(q0, 0, z, l);
      if (y == c) {
        /* centre row: every ray passes plane yr = z (sbrt:4260-4270) */
        for (int k = 1; k <= G; k++)
          for (int z = g->yb[2 * k]; z <= g->yt[2 * k]; z++)
            for (int l = 0; l < 4; l++) s1[z * 4 + l] = s1[z * 4 + l] + (Q(q1, k, z, l) + Q(q2, k, z, l));
      } else {
        for (int gr = 0; gr < G; gr++) {
          const int k = gr + 1;
          const int i1 = y * G + gr, i2 = (nx - y) * G + gr;
          const float f1 = g->bl_yr2a[i1], f2 = g->bl_yr2a[i2];
          for (int z = g->bl_zsa[i1], yr = g->bl_yra[i1]; z <= g->bl_zea[i1]; z++, yr++)
            for (int l = 0; l < 4; l++) {
              s1[z * 4 + l] = s1[z * 4 + l] + (Q(q1, k, yr, l) + f1 * (Q(q1, k, yr + 1, l) - Q(q1, k, yr, l)));
              s2[z * 4 + l] = s2[z * 4 + l] + (Q(q2, k, yr, l) + f1 * (Q(q2, k, yr + 1, l) - Q(q2, k, yr, l)));
            }
          for (int z = g->bl_zsa[i2], yr = g->bl_yra[i2]; z <= g->bl_zea[i2]; z++, yr++)
            for (int l = 0; l < 4; l++) {
              s1[z * 4 + l] = s1[z * 4 + l] + (Q(q2, k, yr, l) + f2 * (Q(q2, k, yr + 1, l) - Q(q2, k, yr, l)));
              s2[z * 4 + l] = s2[z * 4 + l] + (Q(q1, k, yr, l) + f2 * (Q(q1, k, yr + 1, l) - Q(q1, k, yr, l)));
            }
        }
      }
      /* scatter the lanes onto their voxels */
      const int v1[4][2] = {{x, y}, {nx - x, y}, {nx - y, x}, {nx - y, nx - x}};
      const int v2[4][2] = {{x, nx - y}, {nx - x, nx - y}, {y, x}, {y, nx - x}};
      for (int l = 0; l < 4; l++) {
        if (x == c && (l & 1)) continue;  /* bin nx-c is bin c */
        R *o = ib + ((size_t)v1[l][0] * g->ny + v1[l][1]) * zp;
        for (int z = 0; z < nz; z++) o[z] += s1[z * 4 + l];
        if (y == c) continue;  /* the centre row has only the sumt1 voxels */
        o = ib + ((size_t)v2[l][0] * g->ny + v2[l][1]) * zp;
        for (int z = 0; z < nz; z++) o[z] += s2[z * 4 + l];
      }
    }
  }
#undef Q
  free(rows);
  free(q0);
  free(q1);
  free(q2);
  free(s1);
  free(s2);
}

/* ------------------------------------------------------------------------ */
/* Rotation back to the image frame                                         */
/* ------------------------------------------------------------------------ */

/* rotateimage2 (sbrt:1137-1186): positions advance incrementally along y in
 * single precision; (int) truncates toward zero, so a position in (-1, 0)
 * passes the bounds test, as in the reference. */
static void rotate_rows(const orc_geom *g, const R *ib, int view, R *out, int xs, int xe) {
  const int nx = g->nx, ny = g->ny, zp = g->zp;
  const float cosv = g->cos_psi[view] / 1.0f;
  const float sinv = -g->sin_psi[view] / 1.0f;
  const float xxx0 = -nx / 2 * cosv + ny / 2 * sinv + nx / 2;
  const float yyy0 = -nx / 2 * sinv - ny / 2 * cosv + ny / 2;
  for (unsigned x = (unsigned)xs; x < (unsigned)xe; x++) {
    const int ystart = g->cyl[2 * x], yend = g->cyl[2 * x + 1];
    float xx0 = xxx0 - ystart * sinv + x * cosv;
    float yy0 = yyy0 + ystart * cosv + x * sinv;
    for (int y = ystart; y < yend; y++) {
      const int xx = (int)xx0, yy = (int)yy0;
      if (xx < 0 || xx > nx - 2 || yy < 0 || yy > nx - 2) {
        xx0 -= sinv;
        yy0 += cosv;
        continue;
      }
      const float x1 = xx0 - xx, y1 = yy0 - yy;
      const float c1 = (1 - x1) * (1 - y1), c2 = x1 * (1 - y1), c3 = y1 * (1 - x1), c4 = y1 * x1;
      const R *i1 = ib + ((size_t)xx * ny + yy) * zp, *i2 = i1 + (size_t)ny * zp, *i3 = i1 + zp, *i4 = i2 + zp;
      R *o = out + ((size_t)x * ny + y) * zp;
      for (int z = 0; z < zp; z++) o[z] = o[z] + ((i1[z] * c1 + i2[z] * c2) + (i3[z] * c3 + i4[z] * c4));
      xx0 -= sinv;
      yy0 += cosv;
    }
  }
}

void orc_rotate_add(const orc_geom *g, const R *ib, int view, R *out) { rotate_rows(g, ib, view, out, 0, g->nx); }

/* ------------------------------------------------------------------------ */
/* Driver pieces                                                            */
/* ------------------------------------------------------------------------ */

/* PrepareNormfac / PrepareOsem3dFiles for OP weighting (-W 3):
 *  - normalisation planes within npskip of a segment's ends are zeroed as
 *    they are read (fio:133-137);
 *  - norm_zero_mask[v][x] = 0 when the normalisation is zero in every plane
 *    for all four bins of the quad (drv:865-903);
 *  - 1/(N*A) with A clamped to >= 1 (norm_ANW, drv:796-821);
 *  - additive term (randoms*N + scatter)*A with the unclamped A, and
 *    prompts zeroed where N == 0 (prepare_osem3dw3, drv:1649-1760 and
 *    mulprojection / addprojection / the attenuation pass that follows). */
void orc_prep(orc_geom *g, const int16_t *prompts, const float *randoms, const float *norm, const float *atten,
              const float *scatter, int16_t *p_out, float *add_out, float *mult_out) {
  const int V = g->nviews, N = g->nbins, ss = g->segmentsize;
  const size_t plane = (size_t)V * N;
  unsigned char *mask = NEW(unsigned char, plane);
  for (int s = 0; s < g->nseg; s++) {
    const int ns = g->yt[s] - g->yb[s] + 1;
    for (int r = 0; r < ns; r++) {
      const int kill = (r < g->npskip || r + g->npskip >= ns);
      const size_t base = (size_t)(g->soff[s] + r) * plane;
      for (size_t i = 0; i < plane; i++) {
        const size_t j = base + i;
        const float nf = norm ? (kill ? 0.0f : norm[j]) : 1.0f;
        const float araw = atten ? atten[j] : 1.0f;
        const float ac = (araw < 1.0f) ? 1.0f : araw;
        float m;
        if (nf > 0.0f) {
          const float den = nf * ac;
          m = (den > g->eps2) ? 1.0f / den : 0.0f;
        } else {
          m = nf;
        }
        mult_out[j] = m;
        float a = randoms[j] * nf;
        if (scatter) a = a + scatter[j];
        add_out[j] = a * araw;
        p_out[j] = (nf == 0.0f) ? 0 : prompts[j];
        if (nf != 0.0f) mask[i] = 1;
      }
    }
  }
  (void)ss;
  for (int v = 0; v < V / 2; v++)
    for (int x = 1; x <= N / 2; x++) {
      const int z = !mask[(size_t)v * N + x] && !mask[(size_t)(v + V / 2) * N + x] &&
                    !mask[(size_t)v * N + N - x] && !mask[(size_t)(v + V / 2) * N + N - x];
      g->nzmask[v * (g->nx / 2 + 1) + x] = z ? 0 : 1;
    }
  free(mask);
}

/* the rows of one view pair out of a flat-file sinogram (drv:2145-2154) */
static void gather_pair_f(const orc_geom *g, const float *sino, int view, R *rows) {
  const int V = g->nviews, N = g->nbins, ss = g->segmentsize;
  for (int j = 0; j < ss; j++)
    for (int xr = 0; xr < N; xr++) {
      rows[(size_t)j * N + xr] = sino[((size_t)j * V + view) * N + xr];
      rows[(size_t)(j + ss) * N + xr] = sino[((size_t)j * V + view + V / 2) * N + xr];
    }
}

/* OP ratio pt_update_est_w3 (drv:2474-2520) on one pair's estimate */
static void ratio_pair(const orc_geom *g, R *est, const int16_t *prompts, const float *add, int view) {
  const int V = g->nviews, N = g->nbins, ss = g->segmentsize;
  for (int h = 0; h < 2; h++)
    for (int j = 0; j < ss; j++)
      for (int xr = 0; xr < N; xr++) {
        const size_t f = ((size_t)j * V + view + h * (V / 2)) * N + xr;
        R *e = est + ((size_t)(j + h * ss)) * N + xr;
        const R den = *e + (R)add[f];
        if (prompts[f] == 0) *e = 0;
        else if (den > g->eps3) *e = (R)prompts[f] / den;
        else *e = 1;
      }
}

typedef struct {
  const orc_geom *g;
  const R *image;
  const int16_t *prompts;
  const float *add;   /* OSEM: additive term; sensitivity: 1/(N*A) */
  int view;
  R *est, *ib;
  int sens;
} pair_job;

/* pt_osem3d_proj_thread1 (drv:1910-1938) and pt_back_proj3d_thread1
 * (drv:1896-1908): one view pair */
static void *pair_worker(void *arg) {
  pair_job *j = (pair_job *)arg;
  const orc_geom *g = j->g;
  if (j->sens) {
    gather_pair_f(g, j->add, j->view, j->est);
  } else {
    memset(j->est, 0, sizeof(R) * 2 * g->segmentsize * g->nbins);
    orc_fp_pair(g, j->image, j->view, j->est);
    ratio_pair(g, j->est, j->prompts, j->add, j->view);
  }
  orc_bp_pair(g, j->est, j->view, j->ib);
  return NULL;
}

typedef struct {
  const orc_geom *g;
  R *const *ib;
  const int *views;
  int n, xs, xe;
  R *out;
} rot_job;

static void *rot_worker(void *arg) {
  rot_job *r = (rot_job *)arg;
  for (int i = 0; i < r->n; i++) rotate_rows(r->g, r->ib[i], r->views[i], r->out, r->xs, r->xe);
  return NULL;
}

/* the subset's pairs in groups of T (CalculateOsem3d, drv:4161-4260):
 * projections in parallel, then the rotate-backs added in view order
 * (rotate_image_buf, sbrt:1701-1725), threads splitting the columns */
static void run_subset_pairs(const orc_geom *g, int isubset, int T, const R *image, const int16_t *prompts,
                             const float *add, int sens, R *corr) {
  const size_t vol = (size_t)g->nx * g->ny * g->zp, rows = (size_t)2 * g->segmentsize * g->nbins;
  const int npairs = g->sviews / 2;
  if (T < 1) T = 1;
  if (T > npairs) T = npairs;
  R **est = NEW(R *, T), **ib = NEW(R *, T);
  for (int t = 0; t < T; t++) {
    est[t] = NEW(R, rows);
    ib[t] = NEW(R, vol);
  }
  pthread_t *th = NEW(pthread_t, T);
  pair_job *jobs = NEW(pair_job, T);
  rot_job *rj = NEW(rot_job, T);
  int *views = NEW(int, T);
  for (int v0 = 0; v0 < npairs; v0 += T) {
    const int n = (npairs - v0 < T) ? npairs - v0 : T;
    for (int t = 0; t < n; t++) {
      views[t] = g->vieworder[isubset * g->sviews + v0 + t];
      jobs[t] = (pair_job){g, image, prompts, add, views[t], est[t], ib[t], sens};
      pthread_create(&th[t], NULL, pair_worker, &jobs[t]);
    }
    for (int t = 0; t < n; t++) pthread_join(th[t], NULL);
    for (int t = 0; t < T; t++) {
      rj[t] = (rot_job){g, ib, views, n, g->nx * t / T, g->nx * (t + 1) / T, corr};
      pthread_create(&th[t], NULL, rot_worker, &rj[t]);
    }
    for (int t = 0; t < T; t++) pthread_join(th[t], NULL);
  }
  for (int t = 0; t < T; t++) {
    free(est[t]);
    free(ib[t]);
  }
  free(est);
  free(ib);
  free(th);
  free(jobs);
  free(rj);
  free(views);
}

/* ---- PSF resolution modelling (psf.cpp) ---------------------------------- */

/* make1d_psf_filter (psf.cpp:21-70): two Gaussians (fwhm1, fwhm2 in mm, the
 * second scaled by ratio) sampled at the pixel size over 2h+1 taps and
 * normalised; fwhm1 == 0 selects the HRRT defaults.  Returns the tap count
 * written to k (capacity cap), or -1. */
int orc_psf_kernel(float fwhm1, float fwhm2, float ratio, float pixel_size, float *k, int cap) {
  if (fwhm1 == 0.0) {
    fwhm1 = (float)(0.9 * sqrt(8.0 * log(2.0)));
    fwhm2 = (float)(2.5 * sqrt(8.0 * log(2.0)));
    ratio = 0.05f;
  }
  if (!(fwhm1 > 0.0)) return -1;
  int size;
  if (fwhm2 > 0.0 && ratio > 0.0)
    size = 2 * ((int)(1.5 * fwhm2 * sqrt(log(10.0) / log(2.)) / pixel_size / 2.0)) + 1;
  else
    size = 2 * ((int)(1.5 * fwhm1 * sqrt(log(10.0) / log(2.)) / pixel_size / 2.0)) + 1;
  if (size > cap) return -1;
  const float sigma1 = (float)(fwhm1 / (sqrt(8.0 * log(2.0)) * pixel_size));
  const float sigma2 = (float)(fwhm2 / (sqrt(8.0 * log(2.0)) * pixel_size));
  const int bin0 = (size - 1) / 2;
  float norm = 0.0f;
  for (int b = 0; b < size; b++) {
    k[b] = (float)exp(-0.5 * (pow((double)(b - bin0) / sigma1, 2.0)));
    if (fwhm2 > 0.0 && ratio > 0.0) k[b] = (float)(k[b] + ratio * exp(-0.5 * (pow((double)(b - bin0) / sigma2, 2.0))));
    norm += k[b];
  }
  for (int b = 0; b < size; b++) k[b] /= norm;
  return size;
}

int orc_set_psf(orc_geom *g, int on, float fwhm1, float fwhm2, float ratio, int z_min, int z_max) {
  free(g->psf_fx);
  free(g->psf_fy);
  free(g->psf_fz);
  free(g->psf_normz);
  g->psf_fx = g->psf_fy = g->psf_fz = g->psf_normz = NULL;
  g->psf_on = 0;
  if (!on) return 0;
  float kx[256], ky[256], kz[256];
  const int nx = orc_psf_kernel(fwhm1, fwhm2, ratio, g->x_size, kx, 256);
  const int ny = orc_psf_kernel(fwhm1, fwhm2, ratio, g->y_size, ky, 256);
  const int nz = orc_psf_kernel(fwhm1, fwhm2, ratio, g->plane_sep, kz, 256);
  if (nx < 1 || ny < 1 || nz < 1 || nx != ny) return -1;
  g->psf_h = (nx - 1) / 2;
  g->psf_fx = NEW(float, nx);
  g->psf_fy = NEW(float, ny);
  g->psf_fz = NEW(float, nz > ny ? nz : ny);
  memcpy(g->psf_fx, kx, sizeof(float) * nx);
  memcpy(g->psf_fy, ky, sizeof(float) * ny);
  memcpy(g->psf_fz, kz, sizeof(float) * nz);
  /* convolveyz's z tap sums (psf.cpp:397-416): the loop bound and the index
   * both use the y kernel's half width */
  const int h = (ny - 1) / 2;
  g->psf_normz = NEW(float, g->zp);
  for (int z = 0; z < g->zp; z++) g->psf_normz[z] = 0.0f;
  for (int mask = -h; mask < h; mask++)
    for (int z = 0; z < g->zp; z++) {
      const int m2 = z + mask;
      if (m2 < z_min || m2 >= z_max) continue;
      g->psf_normz[z] += g->psf_fz[mask + h];
    }
  for (int z = 0; z < g->zp; z++)
    if (g->psf_normz[z] > 0) g->psf_normz[z] = 1 / g->psf_normz[z];
  g->psf_zmin = z_min;
  g->psf_zmax = z_max;
  g->psf_on = 1;
  return 0;
}

/* convolve3d (psf.cpp:463-540): convolvex (:163-206) into a buffer, then
 * convolveyz (:350-460), on FOV columns; out may be in */
void orc_psf(const orc_geom *g, const R *in, R *out) {
  const int N = g->nx, zp = g->zp, h = g->psf_h;
  const size_t vol = (size_t)N * g->ny * zp;
  R *buf = NEW(R, vol), *col = NEW(R, zp), *acc = NEW(R, zp);
  for (int x = 0; x < N; x++) {
    if (g->cyl[2 * x + 1] == 0) continue;
    for (int y = g->cyl[2 * x]; y < g->cyl[2 * x + 1]; y++) {
      for (int z = 0; z < zp; z++) acc[z] = 0;
      float norm = 0;
      for (int mask = -h; mask < h; mask++) {
        const int m2 = x + mask;
        if (m2 < g->cyl[2 * y] || m2 >= g->cyl[2 * y + 1]) continue;
        const R c = (R)g->psf_fx[mask + h];
        norm += g->psf_fx[mask + h];
        for (int z = 0; z < zp; z++) acc[z] = acc[z] + in[((size_t)m2 * N + y) * zp + z] * c;
      }
      R *o = buf + ((size_t)x * N + y) * zp;
      if (norm != 1 && norm != 0) {
        const R c = (R)(1 / norm);
        for (int z = 0; z < zp; z++) o[z] = acc[z] * c;
      } else {
        for (int z = 0; z < zp; z++) o[z] = acc[z];
      }
    }
  }
  for (int x = 0; x < N; x++) {
    if (g->cyl[2 * x + 1] == 0) continue;
    for (int y = g->cyl[2 * x]; y < g->cyl[2 * x + 1]; y++) {
      for (int z = 0; z < zp; z++) col[z] = 0;
      float norm = 0;
      for (int mask = -h; mask < h; mask++) {
        const int m2 = y + mask;
        if (m2 < g->cyl[2 * x] || m2 >= g->cyl[2 * x + 1]) continue;
        const R c = (R)g->psf_fy[mask + h];
        norm += g->psf_fy[mask + h];
        for (int z = 0; z < zp; z++) col[z] = col[z] + buf[((size_t)x * N + m2) * zp + z] * c;
      }
      R *o = out + ((size_t)x * N + y) * zp;
      for (int z = 0; z < zp; z++) o[z] = 0;
      if (norm != 0) {
        for (int mask = -h; mask < h; mask++) {
          int zs = g->psf_zmin - mask, ze = g->psf_zmax - mask;
          if (zs < 0) zs = 0;
          if (ze > g->nz) ze = g->nz;
          const R f = (R)g->psf_fy[mask + h];
          for (int z = zs; z < ze; z++) o[z] = o[z] + col[z + mask] * f;
        }
        const R c = (R)(1 / norm);
        for (int z = 0; z < zp; z++) o[z] = o[z] * ((R)g->psf_normz[z] * c);
      }
    }
  }
  free(buf);
  free(col);
  free(acc);
}

/* CalculateNormfac (drv:3760-3865): per subset the back projection of
 * 1/(N*A), inverted where |.| > epsilon1 on FOV columns, planes < nz
 * (pt_normfac_calculate, drv:1852-1894) */
void orc_sensitivity(const orc_geom *g, const float *mult, R *nf_inv, int nthreads) {
  const size_t vol = (size_t)g->nx * g->ny * g->zp;
  R *nf = NEW(R, vol);
  for (int s = 0; s < g->subsets; s++) {
    memset(nf, 0, sizeof(R) * vol);
    run_subset_pairs(g, s, nthreads, NULL, NULL, mult, 1, nf);
    if (g->psf_on) orc_psf(g, nf, nf); /* drv:3835-3841 */
    R *out = nf_inv + (size_t)s * vol;
    memset(out, 0, sizeof(R) * vol);
    for (int x = 0; x < g->nx; x++)
      for (int y = g->cyl[2 * x]; y < g->cyl[2 * x + 1]; y++)
        for (int z = 0; z < g->nz; z++) {
          const size_t i = ((size_t)x * g->ny + y) * g->zp + z;
          const R a = nf[i];
          out[i] = (fabs((double)a) > g->eps1) ? (R)1 / a : (R)0;
        }
  }
  free(nf);
}

/* Init_Image default (drv:3996-4004) */
void orc_init_image(const orc_geom *g, R *image, int z_min, int z_max) {
  memset(image, 0, sizeof(R) * (size_t)g->nx * g->ny * g->zp);
  for (int x = 0; x < g->nx; x++) {
    if (g->cyl[2 * x] == g->cyl[2 * x + 1]) continue;
    for (int y = g->cyl[2 * x]; y < g->cyl[2 * x + 1]; y++)
      for (int z = z_min; z < z_max; z++) image[((size_t)x * g->ny + y) * g->zp + z] = 1;
  }
}

/* SSE min/max: _mm_max_ps(a, b) = a > b ? a : b, so a NaN in b passes */
static R sse_max(R a, R b) { return a > b ? a : b; }
static R sse_min(R a, R b) { return a < b ? a : b; }

/* one OP-OSEM subset: the subset's pairs (FP, ratio, BP, rotate-back into
 * the correction image) and the update pt_cal_updateimage (drv:2018-2059):
 * image = min(image_max, image * (min(100, max(0.01, corr)) * nf_inv)) on
 * FOV columns, every plane */
void orc_osem_subset(const orc_geom *g, R *image, const R *nf, const int16_t *prompts, const float *add,
                     int isubset, int nthreads) {
  const size_t vol = (size_t)g->nx * g->ny * g->zp;
  R *corr = NEW(R, vol);
  if (g->psf_on) { /* the projection of the blurred image, the blurred correction (drv:4172, :4229) */
    R *ipsf = NEW(R, vol);
    orc_psf(g, image, ipsf);
    run_subset_pairs(g, isubset, nthreads, ipsf, prompts, add, 0, corr);
    free(ipsf);
    orc_psf(g, corr, corr);
  } else {
    run_subset_pairs(g, isubset, nthreads, image, prompts, add, 0, corr);
  }
  const R amax = (R)100.00f, amin = (R)0.01f, imax = (R)g->image_max;
  for (int x = 0; x < g->nx; x++)
    for (int y = g->cyl[2 * x]; y < g->cyl[2 * x + 1]; y++) {
      const size_t b = ((size_t)x * g->ny + y) * g->zp;
      for (int z = 0; z < g->zp; z++) {
        const R cl = sse_min(amax, sse_max(amin, corr[b + z]));
        image[b + z] = sse_min(imax, image[b + z] * (cl * nf[b + z]));
      }
    }
  free(corr);
}

/* ---- MAP, technique 1 of je_hrrt_osem3d (-b 1,beta): Green's one-step-late
 * prior.  calculate_DPF_image (je_hrrt_osem3d/dpfcalc.c:23-31, :66-85,
 * :266-300): maxPET = 1.2 x the image maximum over the FOV columns (never
 * below 0), delta = maxPET / 20, and for every FOV voxel with 1 <= x < nx-1,
 * 1 <= z < nz-1 the sum of tanh((c - n) / delta) = (e - 1) / (e + 1),
 * e = exp(2 (c - n) / delta), over the 6 face neighbours plus sqrt(0.5)
 * times the sum over the 12 edge neighbours in the source's order; the two
 * sums in the working precision, their combination in double.  Elsewhere 0. */
static R map_tanh(R r, R delta) {
  const R e = sizeof(R) == 4 ? (R)expf((float)(2 * r / delta)) : (R)exp((double)(2 * r / delta));
  return (e - 1) / (e + 1);
}

void orc_map_dpf(const orc_geom *g, const R *image, R *dpf) {
  const int N = g->nx, zp = g->zp, nz = g->nz;
  R mx = 0;
  for (int x = 0; x < N; x++)
    for (int y = g->cyl[2 * x]; y < g->cyl[2 * x + 1]; y++)
      for (int z = 0; z < nz; z++)
        if (image[((size_t)x * N + y) * zp + z] > mx) mx = image[((size_t)x * N + y) * zp + z];
  const R maxpet = (R)(1.2 * (double)mx);
  const R delta = (R)((double)maxpet / 20.0);
  memset(dpf, 0, sizeof(R) * (size_t)N * N * zp);
#define IM(a, b, c) image[((size_t)(a) * N + (b)) * zp + (c)]
  for (int x = 1; x < N - 1; x++)
    for (int y = g->cyl[2 * x]; y < g->cyl[2 * x + 1]; y++)
      for (int z = 1; z < nz - 1; z++) {
        const R c = IM(x, y, z);
        R a = map_tanh(c - IM(x, y, z - 1), delta);
        a = a + map_tanh(c - IM(x, y, z + 1), delta);
        a = a + map_tanh(c - IM(x - 1, y, z), delta);
        a = a + map_tanh(c - IM(x + 1, y, z), delta);
        a = a + map_tanh(c - IM(x, y - 1, z), delta);
        a = a + map_tanh(c - IM(x, y + 1, z), delta);
        R b = map_tanh(c - IM(x - 1, y, z - 1), delta);
        b = b + map_tanh(c - IM(x, y - 1, z - 1), delta);
        b = b + map_tanh(c - IM(x + 1, y, z - 1), delta);
        b = b + map_tanh(c - IM(x, y + 1, z - 1), delta);
        b = b + map_tanh(c - IM(x - 1, y - 1, z), delta);
        b = b + map_tanh(c - IM(x - 1, y + 1, z), delta);
        b = b + map_tanh(c - IM(x + 1, y - 1, z), delta);
        b = b + map_tanh(c - IM(x + 1, y + 1, z), delta);
        b = b + map_tanh(c - IM(x - 1, y, z + 1), delta);
        b = b + map_tanh(c - IM(x, y - 1, z + 1), delta);
        b = b + map_tanh(c - IM(x + 1, y, z + 1), delta);
        b = b + map_tanh(c - IM(x, y + 1, z + 1), delta);
        dpf[((size_t)x * N + y) * zp + z] = (R)((double)a + sqrt(0.5) * (double)b);
      }
#undef IM
}

/* one OP-OSEM subset with the MAP update pt_cal_updateimage_mapem
 * (je_hrrt_osem3d/hrrt_osem3d.cpp:2031-2073, wired at :4439-4463): the prior
 * of the image before the update, then on FOV columns, every plane,
 * image = min(image_max, image * min(100, max(0.1, corr / (beta * dpf + 1 / nf_inv)))).
 * The reference forms 1 / nf_inv with _mm_rcp_ps (relative error up to
 * 1.5 * 2^-12); here it is the exact reciprocal. */
void orc_osem_subset_map(const orc_geom *g, R *image, const R *nf, const int16_t *prompts, const float *add,
                         int isubset, int nthreads, float beta) {
  const size_t vol = (size_t)g->nx * g->ny * g->zp;
  R *corr = NEW(R, vol), *dpf = NEW(R, vol);
  if (g->psf_on) {
    R *ipsf = NEW(R, vol);
    orc_psf(g, image, ipsf);
    run_subset_pairs(g, isubset, nthreads, ipsf, prompts, add, 0, corr);
    free(ipsf);
    orc_psf(g, corr, corr);
  } else {
    run_subset_pairs(g, isubset, nthreads, image, prompts, add, 0, corr);
  }
  orc_map_dpf(g, image, dpf);
  const R amax = (R)100.00f, amin = (R)0.1f, imax = (R)g->image_max, b = (R)beta;
  for (int x = 0; x < g->nx; x++)
    for (int y = g->cyl[2 * x]; y < g->cyl[2 * x + 1]; y++) {
      const size_t o = ((size_t)x * g->ny + y) * g->zp;
      for (int z = 0; z < g->zp; z++) {
        const R q = corr[o + z] / (b * dpf[o + z] + (R)1 / nf[o + z]);
        image[o + z] = sse_min(imax, image[o + z] * sse_min(amax, sse_max(amin, q)));
      }
    }
  free(dpf);
  free(corr);
}

/* end of an iteration (drv:4288-4297): sum over the FOV and planes
 * [z_min, z_max), values below 1e-16 set to 0 */
double orc_post_iteration(const orc_geom *g, R *image, int z_min, int z_max) {
  double sum = 0;
  for (int x = 0; x < g->nx; x++)
    for (int y = g->cyl[2 * x]; y < g->cyl[2 * x + 1]; y++) {
      R *p = image + ((size_t)x * g->ny + y) * g->zp;
      for (int z = z_min; z < z_max; z++) {
        sum += (double)p[z];
        if ((double)p[z] < 1e-16) p[z] = 0;
      }
    }
  return sum;
}
