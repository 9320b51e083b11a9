/*
 * hrrt_oracle.h -- CPU restatement of the hrrt_osem3d OP-OSEM hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  The tests, the smoke check and the benchmark's
 * CPU-baseline leg use it as the checker; the product never calls it.
 *
 * One source, two builds (oracle/Makefile):
 *   liboracle_f32.so  orc_real = float: every operation in the reference's
 *                     single-precision expression order (the reference is an
 *                     SSE2 build without fused multiply-add), so the forward
 *                     projection and the rotation are bit-identical to it;
 *   liboracle.so      orc_real = double: the same sample positions (the
 *                     geometry and interpolation weights stay float, exactly
 *                     as the reference computes them) with all sums, scales,
 *                     ratios and updates carried in double: the FP64 oracle.
 *
 * Parity pins: against the reference's own projector compiled from its
 * unmodified sources (oracle/_ref/libhrrt_ref.so, oracle/Makefile target
 * "ref") and against the golden fixtures in tests/golden/ made from it by
 * tests/golden/make_golden.py.
 *
 * Array conventions (those of the reference's buffers):
 *   image     [x][y][zp]            zp = z planes padded to a multiple of 4
 *   rows      [2*segmentsize][nbins] one view pair: view, then view+nviews/2
 *   sinogram  [segmentsize][nviews][nbins]  flat-file layout
 */
#ifndef HRRT_ORACLE_H
#define HRRT_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifndef ORC_REAL
#define ORC_REAL double
#endif
typedef ORC_REAL orc_real;

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_geom orc_geom;

/* dependencies() + GetScannerParameter(); NULL on an unsupported geometry */
orc_geom *orc_create(int nrings, int nelements, int nangles, float ring_radius, float plane_sep, float binsize,
                     int span, int maxdel, int subsets);
void orc_destroy(orc_geom *g);
/* -k npskip, -e epsilon1,epsilon2,epsilon3, -u image_max (drv:232, :371-374) */
void orc_set_params(orc_geom *g, int npskip, float eps1, float eps2, float eps3, float image_max);
int orc_real_bytes(void);
/* the plane range [z_min, z_max) after the driver's adjustments for npskip */
void orc_z_range(const orc_geom *g, int z_min, int z_max, int *out /* [2] */);
int orc_segmentsize(const orc_geom *g);
int orc_zp(const orc_geom *g);
int orc_nz(const orc_geom *g);
int orc_nx(const orc_geom *g);
int orc_nviews(const orc_geom *g);
int orc_sviews(const orc_geom *g);
int orc_vieworder(const orc_geom *g, int isubset, int k);
void orc_order(const orc_geom *g, int16_t *order);
/* geometry tables, for pinning against the reference's own */
void orc_cylwiny(const orc_geom *g, int *cyl /* [ny][2] */);
void orc_trig(const orc_geom *g, float *sin_theta, float *cos_theta, float *sin_psi, float *cos_psi);
void orc_tantheta(const orc_geom *g, float *tantheta, float *rescale /* [groupmax][nz] */);
void orc_flookup(const orc_geom *g, int *zzi, float *zzz0 /* [ny][groupmax*2*zshift] */);
void orc_blookup(const orc_geom *g, int *zsa, int *zea, int *yra, float *yr2a /* [ny][groupmax] */);
void orc_set_norm_zero_mask(orc_geom *g, const int16_t *mask /* [nviews/2][nbins/2+1] */);
void orc_get_norm_zero_mask(const orc_geom *g, int16_t *mask);

/* forward projection of one view pair; writes the bins the reference writes */
void orc_fp_pair(const orc_geom *g, const orc_real *img, int view, orc_real *rows);
/* back projection of one view pair into the rotated frame (overwritten) */
void orc_bp_pair(const orc_geom *g, const orc_real *rows, int view, orc_real *imagebuf);
/* image += FP^T rows: the exact transpose of orc_fp_pair (image frame) */
void orc_fp_adjoint(const orc_geom *g, const orc_real *rows, int view, orc_real *image);
/* corr += rotate-back(imagebuf) for one view */
void orc_rotate_add(const orc_geom *g, const orc_real *imagebuf, int view, orc_real *corr);

/* PrepareNormfac + PrepareOsem3dFiles for -W 3: inputs in flat-file layout
 * (norm, atten, scatter may be NULL); outputs prompts masked by the
 * normalisation, additive term, 1/(N*A); updates the norm-zero mask */
void orc_prep(orc_geom *g, const int16_t *prompts, const float *randoms, const float *norm, const float *atten,
              const float *scatter, int16_t *prompts_out, float *add_out, float *mult_out);
/* inverse sensitivity images of every subset: nf_inv [subsets][x][y][zp] */
void orc_sensitivity(const orc_geom *g, const float *mult, orc_real *nf_inv, int nthreads);
/* Init_Image default: 1 on FOV columns for planes [z_min, z_max) */
void orc_init_image(const orc_geom *g, orc_real *image, int z_min, int z_max);
/* one OP-OSEM subset; nf_inv_subset [x][y][zp] */
void orc_osem_subset(const orc_geom *g, orc_real *image, const orc_real *nf_inv_subset, const int16_t *prompts,
                     const float *add, int isubset, int nthreads);
/* post-iteration threshold (< 1e-16 -> 0) and sum over FOV x [z_min, z_max) */
double orc_post_iteration(const orc_geom *g, orc_real *image, int z_min, int z_max);
/* MAP technique 1 (je_hrrt_osem3d): the prior image calculate_DPF_image
 * makes from `image` ([x][y][zp]), and one OP-OSEM subset with the MAP update
 * (exact reciprocal of nf_inv where the reference uses _mm_rcp_ps) */
void orc_map_dpf(const orc_geom *g, const orc_real *image, orc_real *dpf);
void orc_osem_subset_map(const orc_geom *g, orc_real *image, const orc_real *nf_inv_subset, const int16_t *prompts,
                         const float *add, int isubset, int nthreads, float beta);

/* PSF resolution modelling (psf.cpp): the 1D kernel of make1d_psf_filter
 * (returns its size or -1), and convolve3d on FOV columns once orc_set_psf
 * has enabled it (it then also applies in orc_sensitivity and
 * orc_osem_subset, as -B does in the reference; z_min / z_max: the planes of
 * the z convolution) */
int orc_psf_kernel(float fwhm1, float fwhm2, float ratio, float pixel_size, float *k, int cap);
int orc_set_psf(orc_geom *g, int on, float fwhm1, float fwhm2, float ratio, int z_min, int z_max);
void orc_psf(const orc_geom *g, const orc_real *in, orc_real *out);

#ifdef __cplusplus
}
#endif
#endif
