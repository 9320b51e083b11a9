/*
 * ref_harness.cpp -- drives the reference's own projector code.
 *
 * TEST INFRASTRUCTURE.  oracle/Makefile compiles this file together with the
 * UNMODIFIED reference sources hrrt_osem3d/hrrt_osem3dv_sbrt_span3.cpp,
 * hrrt_osem3d/nr_utils.cpp, hrrt_osem3d/psf.cpp and hrrt_osem3d/scanner_model.cpp
 * into oracle/_ref/libhrrt_ref.so.  Only tests/,
 * __graft_entry__.smoke() and bench.py (its reference arm and cpu_baseline)
 * load that library, and only as the checker / CPU baseline.
 *
 * The reference projector translation unit expects globals that the driver
 * hrrt_osem3d/hrrt_osem3d_span3.cpp defines, and the driver's per-thread
 * buffer allocators, ratio, update, sensitivity-inverse and subset-order
 * helpers.  The driver itself does not compile unpatched, so this file
 * restates those pieces (allocation shapes, loop structure, thread grouping
 * and arithmetic), citing the driver line it follows, and calls the
 * reference's own forward_proj3d_thread1 / back_proj3d_thread1 /
 * rotate_image_buf / forward_proj3d2 / back_proj3d2 for all projector work.
 */
#include <pthread.h>
#include <string.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <vector>
#include <algorithm>

#include "hrrt_osem3d.h"
#include "nr_utils.h"
#include "scanner_model.h"

/* psf.cpp */
int make1d_psf_filter(Psf1D *psf);
void convolve3d(float ***image, float ***out, float ***buf);

/* ---- globals the driver defines (hrrt_osem3d_span3.cpp:150-260) ---- */
int nthreads = 1;
int rings = 0;
float ring_radius = 0.f, ring_spacing = 0.f, z_size = 0.f, sino_sampling = 0.f;
float fov = 0.f, rfov = 0.f;
int z_pixels = 0, z_pixels_simd = 0;
int z_min = 6, z_max = 200, npskip = 3;
int radial_pixels = 0, views = 0, maxdel = 0, span = 0, groupmin = 0, groupmax = 0;
int defelements = 0, defangles = 0;
float zoom = 1.0f, newzoom = 1.0f;
float rel_fov = 0.95f;
int max_g = -1;
int **vieworder = NULL;
/* PSF kernels of -B (hrrt_osem3d_span3.cpp:454-456) */
Psf1D *psfx = NULL, *psfy = NULL, *psfz = NULL;

/* allocator hooks the reference's local mm_malloc.h declares */
void *_mm_malloc(size_t size, size_t align) {
  void *p = NULL;
  if (align < sizeof(void *)) align = sizeof(void *);
  if (posix_memalign(&p, align, size ? size : 1) != 0) return NULL;
  return p;
}
void _mm_free(void *p) { free(p); }
void nrerror(const char *) { exit(1); }

/* ---- state ---- */
static int g_ready = 0;
static int g_zp = 0;                 /* z_pixels_simd*4 (208 for HRRT) */
static float ***g_imagebuf[16];      /* per-thread rotated-frame BP buffers */
static float ***g_prjbuf[16];        /* per-thread packed sinogram buffers */
static float **g_est[16];            /* per-thread estimate rows [2*segmentsize][xr] */
static std::vector<float> g_imagebuf_mem[16];
static std::vector<float> g_est_mem[16];
static int g_nbuf = 0;
static float epsilon1 = 5.E-2f, epsilon3 = 1.E-10f, image_max = 1.E4f; /* drv:371-374 */

/* NR-style pointer cube over a contiguous [nx][ny][nz] block */
static float ***cube_ptrs(float *base, int nx, int ny, int nz) {
  float ***t = (float ***)malloc(sizeof(float **) * nx);
  float **rows = (float **)malloc(sizeof(float *) * nx * ny);
  for (int x = 0; x < nx; x++) {
    t[x] = rows + (size_t)x * ny;
    for (int y = 0; y < ny; y++) t[x][y] = base + ((size_t)x * ny + y) * nz;
  }
  return t;
}
static void free_cube_ptrs(float ***t) { if (t) { free(t[0]); free(t); } }

static float **row_ptrs(float *base, int nrows, int ncols) {
  float **r = (float **)malloc(sizeof(float *) * nrows);
  for (int i = 0; i < nrows; i++) r[i] = base + (size_t)i * ncols;
  return r;
}

/* restates alloc_prjxyf_thread (drv:2754-2772): zeroed, each oblique row
 * offset so that index yr_bottom-1 is the first element. */
static float ***alloc_prjbuf(void) {
  float ***prj = (float ***)malloc((size_t)(xr_pixels + 1) * sizeof(float **));
  for (int xr = 0; xr < xr_pixels + 1; xr++) {
    prj[xr] = (float **)malloc((size_t)(th_pixels / 2 + 1) * sizeof(float *));
    /* one extra __m128 so the BP's 208-entry memcpy of row 0 stays in bounds */
    prj[xr][0] = (float *)_mm_malloc((size_t)(z_pixels_simd * 4 + 1) * 16, 16);
    memset(prj[xr][0], 0, (size_t)(z_pixels_simd * 4 + 1) * 16);
    for (int th = 1; th < th_pixels / 2 + 1; th++) {
      size_t n = (size_t)(yr_top[th * 2] - yr_bottom[th * 2] + 13);
      float *p = (float *)_mm_malloc(n * 16, 16);
      memset(p, 0, n * 16);
      prj[xr][th] = p - yr_bottom[th * 2] * 4 + 4;
    }
  }
  return prj;
}
static void free_prjbuf(float ***prj) {
  if (!prj) return;
  for (int xr = 0; xr < xr_pixels + 1; xr++) {
    _mm_free(prj[xr][0]);
    for (int th = 1; th < th_pixels / 2 + 1; th++) _mm_free(prj[xr][th] + yr_bottom[th * 2] * 4 - 4);
    free(prj[xr]);
  }
  free(prj);
}

static void free_buffers(void) {
  for (int i = 0; i < g_nbuf; i++) {
    free_cube_ptrs(g_imagebuf[i]); g_imagebuf[i] = NULL;
    free_prjbuf(g_prjbuf[i]); g_prjbuf[i] = NULL;
    free(g_est[i]); g_est[i] = NULL;
    g_imagebuf_mem[i].clear(); g_imagebuf_mem[i].shrink_to_fit();
    g_est_mem[i].clear(); g_est_mem[i].shrink_to_fit();
  }
  g_nbuf = 0;
}

static void alloc_buffers(int n) {
  free_buffers();
  for (int i = 0; i < n; i++) {
    g_imagebuf_mem[i].assign((size_t)x_pixels * y_pixels * g_zp, 0.f);
    g_imagebuf[i] = cube_ptrs(g_imagebuf_mem[i].data(), x_pixels, y_pixels, g_zp);
    g_prjbuf[i] = alloc_prjbuf();
    g_est_mem[i].assign((size_t)2 * segmentsize * xr_pixels, 0.f);
    g_est[i] = row_ptrs(g_est_mem[i].data(), 2 * segmentsize, xr_pixels);
  }
  g_nbuf = n;
}

extern "C" {

/*
 * Scanner + sinogram set-up.  Follows GetScannerParameter (drv:3452-3551) for
 * a model given by its fields (scanner_model.cpp:124 for HRRT: 104 rings, 256
 * elements, 288 angles, R 234.5 mm, plane sep 1.21875 mm, bin 1.21875 mm),
 * then the reference's own dependencies() (sbrt:199-800).
 */
int ref_init(int nrings, int nelements, int nangles, float crystal_radius, float plane_sep,
             float binsize, int span_, int maxdel_, int subsets_, int nthreads_) {
  if (g_ready) { free_buffers(); free_dependencies(); g_ready = 0; }
  nthreads = nthreads_ < 1 ? 1 : (nthreads_ > 16 ? 16 : nthreads_);
  rings = nrings;
  ring_radius = crystal_radius;
  z_size = plane_sep;
  x_pixels = y_pixels = 0;
  sino_sampling = binsize;
  z_pixels = rings * 2 - 1;
  z_pixels_simd = (z_pixels % 4 == 0) ? z_pixels / 4 : z_pixels / 4 + 1;
  ring_spacing = 2.0f * z_size;
  span = span_;
  maxdel = maxdel_;
  groupmax = (maxdel - (span - 1) / 2) / span;
  groupmin = 0;
  radial_pixels = nelements;
  views = nangles;
  fov = sino_sampling * radial_pixels;
  rfov = sino_sampling * radial_pixels / 2.0f;
  subsets = subsets_;
  zoom = newzoom = 1.0f;
  rel_fov = 0.95f;
  max_g = -1;
  z_min = 6; z_max = 200; npskip = 3;
  if (npskip > z_min) z_min = npskip;
  if (z_max > z_pixels - npskip) z_max = z_pixels - npskip;
  if (!dependencies(0, 0, 0)) return -1;
  g_zp = z_pixels_simd * 4;
  alloc_buffers(nthreads);
  g_ready = 1;
  return 0;
}

int ref_segmentsize(void) { return segmentsize; }
int ref_th_pixels(void) { return th_pixels; }
int ref_groupmax(void) { return groupmax; }
int ref_zp(void) { return g_zp; }
int ref_z_pixels(void) { return z_pixels; }
int ref_x_pixels(void) { return x_pixels; }
int ref_views(void) { return views; }
int ref_maxdel(void) { return maxdel; }

/* table dumps for geometry pinning */
void ref_get_segments(int *ybot, int *ytop, int *segoff) {
  for (int i = 0; i < th_pixels; i++) { ybot[i] = yr_bottom[i]; ytop[i] = yr_top[i]; segoff[i] = segment_offset[i]; }
}
void ref_get_cylwiny(short *out /* [y_pixels][2] */) {
  for (int y = 0; y < y_pixels; y++) { out[2 * y] = cylwiny[y][0]; out[2 * y + 1] = cylwiny[y][1]; }
}
void ref_get_trig(float *sinth, float *costh, float *sinpsi, float *cospsi) {
  for (int i = 0; i < th_pixels; i++) { sinth[i] = sin_theta[i]; costh[i] = cos_theta[i]; }
  for (int v = 0; v < views; v++) { sinpsi[v] = sin_psi[v]; cospsi[v] = cos_psi[v]; }
}
void ref_get_tantheta(float *tan_out, float *rescale_out /* [groupmax][z_pixels] */) {
  for (int g = 0; g < groupmax; g++)
    for (int z = 0; z < z_pixels; z++) {
      tan_out[g * z_pixels + z] = tantheta[g][z];
      rescale_out[g * z_pixels + z] = rescalearray[g][z];
    }
}
void ref_get_flookup(int *zzi, float *zzz0 /* [y_pixels][groupmax*2*ZShift] */) {
  int n = groupmax * 2 * ZShift;
  for (int y = 0; y < y_pixels; y++)
    for (int i = 0; i < n; i++) { zzi[y * n + i] = flookup[y][i].zzi; zzz0[y * n + i] = flookup[y][i].zzz0; }
}
void ref_get_blookup(int *zsa, int *zea, int *yra, float *yr2a /* [y_pixels][groupmax] */) {
  for (int y = 0; y < y_pixels; y++)
    for (int g = 0; g < groupmax; g++) {
      zsa[y * groupmax + g] = blookup[y][g].zsa; zea[y * groupmax + g] = blookup[y][g].zea;
      yra[y * groupmax + g] = blookup[y][g].yra; yr2a[y * groupmax + g] = blookup[y][g].yr2a;
    }
}
/* norm_zero_mask[v][x], v < views/2, x <= x_pixels/2 (sbrt:333, drv:899-909) */
void ref_set_norm_zero_mask(const short *mask) {
  for (int v = 0; v < views / 2; v++)
    for (int x = 0; x <= x_pixels / 2; x++) norm_zero_mask[v][x] = mask[v * (x_pixels / 2 + 1) + x];
}
void ref_get_norm_zero_mask(short *mask) {
  for (int v = 0; v < views / 2; v++)
    for (int x = 0; x <= x_pixels / 2; x++) mask[v * (x_pixels / 2 + 1) + x] = norm_zero_mask[v][x];
}

/*
 * Forward-project one view pair (view, view+views/2) with the reference's
 * forward_proj3d_thread1 (sbrt:1373-1446).  img: [x][y][zp] contiguous.
 * est: [2*segmentsize][xr_pixels]; rows the reference leaves unwritten keep
 * the caller's values.
 */
int ref_fp_pair(const float *img, int view, float *est) {
  if (!g_ready) return -1;
  float ***ima = cube_ptrs((float *)img, x_pixels, y_pixels, g_zp);
  float **prj = row_ptrs(est, 2 * segmentsize, xr_pixels);
  forward_proj3d_thread1(ima, prj, view, 1, g_imagebuf[0], g_prjbuf[0]);
  free(prj);
  free_cube_ptrs(ima);
  return 0;
}

/*
 * Back-project one view pair into the rotated-frame buffer with the
 * reference's back_proj3d_thread1 (sbrt:1622-1699 -> back_proj3d_view_n1thread
 * sbrt:4162-4668).  est is copied first (the reference rescales in place).
 * imagebuf_out: [x][y][zp].
 */
int ref_bp_pair(const float *est, int view, float *imagebuf_out) {
  if (!g_ready) return -1;
  std::vector<float> tmp(est, est + (size_t)2 * segmentsize * xr_pixels);
  float **prj = row_ptrs(tmp.data(), 2 * segmentsize, xr_pixels);
  memcpy(g_imagebuf_mem[0].data(), imagebuf_out, sizeof(float) * (size_t)x_pixels * y_pixels * g_zp);
  back_proj3d_thread1(prj, NULL, view, 1, g_imagebuf[0], g_prjbuf[0]);
  memcpy(imagebuf_out, g_imagebuf_mem[0].data(), sizeof(float) * (size_t)x_pixels * y_pixels * g_zp);
  free(prj);
  return 0;
}

/* corr += rotate-back(imagebuf) with the reference's rotate_image_buf (sbrt:1701-1725) */
int ref_rotate_add(const float *imagebuf, int view, float *corr) {
  if (!g_ready) return -1;
  float ***ib = cube_ptrs((float *)imagebuf, x_pixels, y_pixels, g_zp);
  float ***co = cube_ptrs(corr, x_pixels, y_pixels, g_zp);
  float ****ibs = &ib;
  int v = view;
  int save = nthreads;
  rotate_image_buf(ibs, co, 1, &v);
  nthreads = save;
  free_cube_ptrs(ib);
  free_cube_ptrs(co);
  return 0;
}

/* sequence() (drv:535-580): subset order by maximum circular distance */
int ref_sequence(int sets, short *order) {
  std::vector<int> done(sets, 0);
  order[0] = 0;
  done[0] = 1;
  for (int i = 1; i < sets; ++i) {
    int ibest = 0, dbest = 0, j = 0;
    while (j < sets) {
      while ((j < sets) && (done[j] == 1)) j += 1;
      if (j < sets) {
        int k = order[i - 1];
        int d = abs(j - k);
        if ((sets - abs(j - k)) < d) d = sets - abs(j - k);
        if (d > dbest) { dbest = d; ibest = j; }
        j += 1;
      }
    }
    order[i] = ibest;
    done[ibest] = 1;
  }
  return 0;
}

}  /* extern "C" */

/* ---- OSEM pieces built on the reference projector ---- */
struct PairTask {
  int view;
  int buf;
  const int16_t *prompts;  /* file layout [segmentsize][views][xr] */
  const float *add;        /* file layout */
  const float *mult;       /* file layout, sensitivity input (or NULL) */
  float ***image;
};

/* copy one view pair's rows out of a file-layout sinogram (the largeprj view
 * of largeprj3, drv:2145-2154) */
template <typename T>
static void gather_pair(const T *sino, int view, T *rows) {
  for (int j = 0; j < segmentsize; j++) {
    memcpy(rows + (size_t)j * xr_pixels, sino + ((size_t)j * views + view) * xr_pixels, sizeof(T) * xr_pixels);
    memcpy(rows + (size_t)(j + segmentsize) * xr_pixels,
           sino + ((size_t)j * views + view + views / 2) * xr_pixels, sizeof(T) * xr_pixels);
  }
}

/* OP-OSEM ratio, pt_update_est_w3 (drv:2474-2520), floatFlag==0 */
static void ratio_w3(float *est, const float *add, const int16_t *p, size_t n) {
  for (size_t i = 0; i < n; i++) {
    float den = est[i] + add[i];
    if (p[i] == 0) est[i] = 0;
    else if (den > epsilon3) est[i] = p[i] / den;
    else est[i] = 1.0f;
  }
}

/* pt_osem3d_proj_thread1 (drv:1910-1938): FP, ratio, BP for one pair */
static void *osem_pair_thread(void *arg) {
  PairTask *t = (PairTask *)arg;
  size_t n = (size_t)2 * segmentsize * xr_pixels;
  std::vector<float> add(n);
  std::vector<int16_t> p(n);
  gather_pair(t->add, t->view, add.data());
  gather_pair(t->prompts, t->view, p.data());
  forward_proj3d_thread1(t->image, g_est[t->buf], t->view, 1, g_imagebuf[t->buf], g_prjbuf[t->buf]);
  ratio_w3(g_est_mem[t->buf].data(), add.data(), p.data(), n);
  back_proj3d_thread1(g_est[t->buf], t->image, t->view, 1, g_imagebuf[t->buf], g_prjbuf[t->buf]);
  return NULL;
}

/* pt_back_proj3d_thread1 (drv:1896-1908) for the sensitivity */
static void *sens_pair_thread(void *arg) {
  PairTask *t = (PairTask *)arg;
  gather_pair(t->mult, t->view, g_est_mem[t->buf].data());
  back_proj3d_thread1(g_est[t->buf], NULL, t->view, 1, g_imagebuf[t->buf], g_prjbuf[t->buf]);
  return NULL;
}

/* pt_cal_updateimage (drv:2018-2059) on FOV columns, all zp planes */
static void update_image(float ***image, float ***corr, float ***nf) {
  for (int x = 0; x < x_pixels; x++)
    for (int y = cylwiny[x][0]; y < cylwiny[x][1]; y++) {
      float *im = image[x][y], *co = corr[x][y], *n = nf[x][y];
      for (int z = 0; z < g_zp; z++) {
        float c = co[z];
        float lo = 0.01f < c ? c : 0.01f;     /* _mm_max_ps(amin, c): NaN -> c */
        if (c != c) lo = c;
        float cl = 100.0f < lo ? 100.0f : lo; /* _mm_min_ps(amax, lo) */
        if (lo != lo) cl = lo;
        float v = im[z] * (cl * n[z]);
        float r = image_max < v ? image_max : v;
        if (v != v) r = v;
        im[z] = r;
        co[z] = 0.f;
      }
    }
}

extern "C" {

/*
 * Run the subset loop of CalculateNormfac (drv:3760-3865) for every subset:
 * nf_inv[s] = |BP_s(mult)| > eps1 ? 1/BP_s(mult) : 0 on FOV columns.
 * mult: 1/(N*A) in file layout.  nf_inv: [subsets][x][y][zp], zeroed by caller.
 */
int ref_sensitivity(const float *mult, float *nf_inv, int nthr) {
  if (!g_ready) return -1;
  int T = std::max(1, std::min(nthr, g_nbuf));
  size_t vol = (size_t)x_pixels * y_pixels * g_zp;
  std::vector<float> nf(vol);
  float ***nfp = cube_ptrs(nf.data(), x_pixels, y_pixels, g_zp);
  int save = nthreads;
  nthreads = T;
  for (int s = 0; s < subsets; s++) {
    std::fill(nf.begin(), nf.end(), 0.f);
    int v;
    for (v = 0; v < sviews / 2 - T + 1; v += T) {
      pthread_t th[16];
      PairTask tasks[16];
      for (int t = 0; t < T; t++) {
        tasks[t] = PairTask{vieworder[s][v + t], t, NULL, NULL, mult, NULL};
        pthread_create(&th[t], NULL, sens_pair_thread, &tasks[t]);
      }
      for (int t = 0; t < T; t++) pthread_join(th[t], NULL);
      rotate_image_buf(g_imagebuf, nfp, T, &vieworder[s][v]);
    }
    if (((sviews / 2) % T) != 0) {
      for (v = sviews / 2 - (sviews / 2) % T; v < sviews / 2; v++) {
        int view = vieworder[s][v];
        gather_pair(mult, view, g_est_mem[0].data());
        back_proj3d2(g_est[0], nfp, view, T, g_imagebuf[0], g_prjbuf[0]);
      }
    }
    float *out = nf_inv + (size_t)s * vol;
    for (int x = 0; x < x_pixels; x++)
      for (int y = cylwiny[x][0]; y < cylwiny[x][1]; y++)
        for (int z = 0; z < z_pixels; z++) {
          float a = nf[((size_t)x * y_pixels + y) * g_zp + z];
          out[((size_t)x * y_pixels + y) * g_zp + z] = (fabs(a) > epsilon1) ? (1.0f / a) : 0.f;
        }
  }
  nthreads = save;
  free_cube_ptrs(nfp);
  return 0;
}

/*
 * One OSEM subset (CalculateOsem3d subset body, drv:4161-4260) on the
 * reference projector with T threads, OP weighting (-W 3), no PSF.
 * image, corr: [x][y][zp]; corr must be zero on entry and is zero on exit.
 */
int ref_osem_subset(float *image, float *corr, const float *nf_inv_subset, const int16_t *prompts,
                    const float *add, int isubset, int nthr) {
  if (!g_ready) return -1;
  int T = std::max(1, std::min(nthr, g_nbuf));
  float ***im = cube_ptrs(image, x_pixels, y_pixels, g_zp);
  float ***co = cube_ptrs(corr, x_pixels, y_pixels, g_zp);
  float ***nf = cube_ptrs((float *)nf_inv_subset, x_pixels, y_pixels, g_zp);
  int save = nthreads;
  nthreads = T;
  int v;
  for (v = 0; v < sviews / 2 - T + 1; v += T) {
    pthread_t th[16];
    PairTask tasks[16];
    for (int t = 0; t < T; t++) {
      tasks[t] = PairTask{vieworder[isubset][v + t], t, prompts, add, NULL, im};
      pthread_create(&th[t], NULL, osem_pair_thread, &tasks[t]);
    }
    for (int t = 0; t < T; t++) pthread_join(th[t], NULL);
    rotate_image_buf(g_imagebuf, co, T, &vieworder[isubset][v]);
  }
  if (((sviews / 2) % T) != 0) {
    size_t n = (size_t)2 * segmentsize * xr_pixels;
    std::vector<float> a(n);
    std::vector<int16_t> p(n);
    for (v = sviews / 2 - (sviews / 2) % T; v < sviews / 2; v++) {
      int view = vieworder[isubset][v];
      forward_proj3d2(im, g_est[0], view, 0, g_imagebuf[0], g_prjbuf[0]);
      gather_pair(add, view, a.data());
      gather_pair(prompts, view, p.data());
      ratio_w3(g_est_mem[0].data(), a.data(), p.data(), n);
      back_proj3d2(g_est[0], co, view, 0, g_imagebuf[0], g_prjbuf[0]);
    }
  }
  update_image(im, co, nf);
  nthreads = save;
  free_cube_ptrs(im);
  free_cube_ptrs(co);
  free_cube_ptrs(nf);
  return 0;
}

/* post-iteration pass (drv:4288-4297): FOV, z in [z_min,z_max) */
/*
 * -B fwhm1,fwhm2,ratio: the three 1-D kernels as the driver builds them
 * (hrrt_osem3d_span3.cpp:4521-4540: Gaussian shape, the HRRT scanner model
 * for fwhm1 = 0 defaults, pixel sizes x_size, y_size, z_size) with the
 * reference's make1d_psf_filter.  Copies the x kernel's taps into `taps`
 * (up to cap) and returns their number, or -1.  ref_init first.
 */
int ref_psf_setup(float fwhm1, float fwhm2, float ratio, float *taps, int cap) {
  if (!g_ready) return -1;
  Psf1D **k[3] = {&psfx, &psfy, &psfz};
  const float px[3] = {x_size, y_size, z_size};
  for (int i = 0; i < 3; i++) {
    if (*k[i]) {
      free((*k[i])->kernel);
      free(*k[i]);
    }
    Psf1D *p = (Psf1D *)malloc(sizeof(Psf1D));
    p->kernel = NULL;
    p->fwhm1 = fwhm1;
    p->fwhm2 = fwhm2;
    p->ratio = ratio;
    p->model = scanner_model(999);
    p->type = GaussShape;
    p->pixel_size = px[i];
    if (make1d_psf_filter(p) != 0) return -1;
    *k[i] = p;
  }
  const int n = psfx->kernel_size < cap ? psfx->kernel_size : cap;
  memcpy(taps, psfx->kernel, sizeof(float) * n);
  return psfx->kernel_size;
}

/* convolve3d (psf.cpp:463-540) of an [x][y][zp] image with the kernels of
 * ref_psf_setup, on the reference's own threads. */
int ref_psf_convolve(const float *in, float *out) {
  if (!g_ready || !psfx) return -1;
  size_t vol = (size_t)x_pixels * y_pixels * g_zp;
  std::vector<float> src(in, in + vol), buf(vol, 0.f);
  memset(out, 0, sizeof(float) * vol);
  float ***a = cube_ptrs(src.data(), x_pixels, y_pixels, g_zp);
  float ***o = cube_ptrs(out, x_pixels, y_pixels, g_zp);
  float ***b = cube_ptrs(buf.data(), x_pixels, y_pixels, g_zp);
  convolve3d(a, o, b);
  free_cube_ptrs(a);
  free_cube_ptrs(o);
  free_cube_ptrs(b);
  return 0;
}

double ref_post_iteration(float *image, int zmin, int zmax) {
  double sum = 0;  /* the reference accumulates in a float global */
  float sumf = 0.f;
  for (int x = 0; x < x_pixels; x++)
    for (int y = cylwiny[x][0]; y < cylwiny[x][1]; y++) {
      float *p = image + ((size_t)x * y_pixels + y) * g_zp;
      for (int z = zmin; z < zmax; z++) {
        sumf += p[z];
        sum += p[z];
        if (p[z] < 1e-16) p[z] = 0;
      }
    }
  (void)sumf;
  return sum;
}

/* Init_Image default (drv:3996-4004): 1 on FOV columns for z in [z_min,z_max) */
void ref_init_image(float *image, int zmin, int zmax) {
  memset(image, 0, sizeof(float) * (size_t)x_pixels * y_pixels * g_zp);
  for (int x = 0; x < x_pixels; x++) {
    if (cylwiny[x][0] == cylwiny[x][1]) continue;
    for (int y = cylwiny[x][0]; y < cylwiny[x][1]; y++)
      for (int z = zmin; z < zmax; z++) image[((size_t)x * y_pixels + y) * g_zp + z] = 1.0f;
  }
}

int ref_vieworder(int isubset, int k) { return vieworder[isubset][k]; }
int ref_sviews(void) { return sviews; }
int ref_subsets(void) { return subsets; }

}  /* extern "C" */
