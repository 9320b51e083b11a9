/*
 * map_ref_harness.cpp -- drives the reference's MAP prior
 * (je_hrrt_osem3d/dpfcalc.c, compiled unmodified by including it here) for
 * the oracle's tests.  TEST INFRASTRUCTURE ONLY: built into
 * oracle/_ref/libmap_ref.so by oracle/Makefile.
 *
 * dpfcalc.c reads the image size and the FOV window (cylwiny) from the
 * driver's globals; they are defined here.  ref_map_update restates the
 * one-line SSE update of pt_cal_updateimage_mapem
 * (je_hrrt_osem3d/hrrt_osem3d.cpp:2031-2073) with the same intrinsics, so
 * that the reciprocal approximation (_mm_rcp_ps) is the host CPU's.
 */
#include <pmmintrin.h>
#include <stdlib.h>
#include <string.h>

int x_pixels, y_pixels, z_pixels, z_pixels_simd;
short int **cylwiny;

#include "dpfcalc.c"

namespace {
// [x][y][zp] float image as the reference's float*** (rows of zp)
float ***view3(float *base, int nx, int ny, int zp) {
  float ***p = (float ***)malloc(sizeof(float **) * nx);
  for (int x = 0; x < nx; x++) {
    p[x] = (float **)malloc(sizeof(float *) * ny);
    for (int y = 0; y < ny; y++) p[x][y] = base + ((size_t)x * ny + y) * zp;
  }
  return p;
}
void free3(float ***p, int nx) {
  for (int x = 0; x < nx; x++) free(p[x]);
  free(p);
}
short int **window(const int *cyl, int nx) {
  short int **w = (short int **)malloc(sizeof(short int *) * nx);
  for (int x = 0; x < nx; x++) {
    w[x] = (short int *)malloc(sizeof(short int) * 2);
    w[x][0] = (short int)cyl[2 * x];
    w[x][1] = (short int)cyl[2 * x + 1];
  }
  return w;
}
}  // namespace

extern "C" {

/* calculate_DPF_image(image, NULL, dpf, 1) on an [nx][nx][zp] image with nz
 * planes; dpf gets the same layout.  Returns the reference's return value. */
int ref_map_dpf(const float *image, int nx, int nz, int zp, const int *cyl, float *dpf) {
  x_pixels = y_pixels = nx;
  z_pixels = nz;
  z_pixels_simd = zp / 4;
  cylwiny = window(cyl, nx);
  float *img = (float *)malloc(sizeof(float) * (size_t)nx * nx * zp);
  memcpy(img, image, sizeof(float) * (size_t)nx * nx * zp);
  float ***P = view3(img, nx, nx, zp), ***D = view3(dpf, nx, nx, zp);
  const int r = calculate_DPF_image(P, NULL, D, 1);
  free3(P, nx);
  free3(D, nx);
  free(img);
  for (int x = 0; x < nx; x++) free(cylwiny[x]);
  free(cylwiny);
  return r;
}

/* pt_cal_updateimage_mapem's update of the FOV columns:
 * image = min(image_max, image * min(100, max(0.1, corr / (beta * dpf + rcp(normfac))))),
 * corr = 0; zp a multiple of 4. */
void ref_map_update(float *image, float *corr, const float *normfac, const float *dpf, int nx, int zp,
                    const int *cyl, float beta, float image_max) {
  const __m128 eps = _mm_set_ps1(beta), amax = _mm_set_ps1(100.00), amin = _mm_set_ps1(0.1f),
               zero = _mm_set_ps1(0), coef = _mm_set_ps1(image_max);
  for (int x = 0; x < nx; x++)
    for (int y = cyl[2 * x]; y < cyl[2 * x + 1]; y++) {
      const size_t o = ((size_t)x * nx + y) * zp;
      __m128 *m1 = (__m128 *)(image + o), *m2 = (__m128 *)(corr + o);
      const __m128 *m3 = (const __m128 *)(normfac + o), *m4 = (const __m128 *)(dpf + o);
      for (int z = 0; z < zp / 4; z++) {
        m1[z] = _mm_min_ps(coef, _mm_mul_ps(m1[z], _mm_min_ps(amax, _mm_max_ps(amin, _mm_div_ps(
                                                      m2[z], _mm_add_ps(_mm_mul_ps(eps, m4[z]),
                                                                        _mm_rcp_ps(m3[z])))))));
        m2[z] = zero;
      }
    }
}

}  // extern "C"
