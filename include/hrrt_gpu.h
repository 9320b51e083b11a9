/*
 * hrrt_gpu.h -- C ABI of libhrrt_gpu.so, the B200 (sm_100a) implementation of
 * the 3D OSEM hot path of hrrt_osem3d (andrewcrabb/hrrt_reconstruction).
 *
 * Conventions
 *   - Every call returns 0 (HRRT_OK) on success and a negative hrrt_status on
 *     failure; hrrt_last_error() then describes the failure.  Nothing in the
 *     library calls exit().
 *   - Host buffers are owned by the caller and never retained.
 *   - One context serves one host thread at a time.  All device work of a
 *     context runs in order on that context's CUDA stream; calls that return
 *     host data synchronise that stream.
 *   - Sinogram arrays use the reference flat-file layout
 *       [segment in file order][plane][view][radial bin]   (bins fastest),
 *     i.e. what hrrt_osem3d reads with -p/-d/-n/-a/-s
 *     (hrrt_osem3d/file_io_processor.cpp:144-294).
 *   - Image arrays handed to the projector entry points use the reference's
 *     in-memory layout image[x][y][z] with z padded to a multiple of 4
 *     (hrrt_info.zp); hrrt_get_image returns the on-disk [z][y][x] layout of
 *     SaveImage (hrrt_osem3d/hrrt_osem3d_span3.cpp:4020-4043).
 *   - Sinogram rows handed to hrrt_fp_pair / hrrt_bp_pair use the reference's
 *     per-view-pair layout prj[2*segmentsize][nbins]: rows [0,segmentsize) are
 *     view v, rows [segmentsize,2*segmentsize) view v+nviews/2
 *     (hrrt_osem3d_span3.cpp:2062-2095, :2145-2154).
 */
#ifndef HRRT_GPU_H
#define HRRT_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  HRRT_OK = 0,
  HRRT_ERR_ARG = -1,      /* invalid argument or size */
  HRRT_ERR_CUDA = -2,     /* CUDA runtime error */
  HRRT_ERR_STATE = -3,    /* call made in the wrong order */
  HRRT_ERR_NOMEM = -4,    /* device allocation failed */
  HRRT_ERR_DEVICE = -5,   /* a device-side check reported an error */
  HRRT_ERR_NOT_FOUND = -6 /* hrrt_lm_seek: the stream ends before the requested time */
} hrrt_status;

/* storage types of the sinogram-shaped inputs on the device (prompts are
 * always int16, the reference's own type, exact over its whole range) */
enum {
  HRRT_STORE_F32 = 0,     /* 1/(NA) and additive term float32 (the reference) */
  HRRT_STORE_16 = 1,      /* 1/(NA) and additive term bf16 (8-bit significand, float32 range) */
  HRRT_STORE_F16 = 2      /* 1/(NA) and additive term fp16 (11-bit significand; a term above 65504 is
                             reported by the upload as HRRT_ERR_ARG) */
};

/* back projector variants */
enum {
  HRRT_BP_REF = 0,        /* voxel-driven sinogram interpolation of the reference */
  HRRT_BP_ADJOINT = 1     /* the exact transpose of the forward projector (no counterpart in the reference) */
};

/*
 * Scanner, sinogram and reconstruction parameters.  Field meanings follow the
 * reference: ScannerModel (hrrt_osem3d/scanner_model.h:3-16), the -m span,maxdel
 * -S subsets -f rel_fov,..,z_min,z_max -k npskip -e eps1,eps2,eps3 -u image_max
 * flags (hrrt_osem3d_span3.cpp:3154-3355) and their defaults (:371-374).
 */
typedef struct hrrt_geom {
  int nrings;          /* direct planes: 104 */
  int nelements;       /* radial bins: 256 */
  int nangles;         /* views: 288 */
  float ring_radius;   /* mm: 234.5 */
  float plane_sep;     /* mm: 1.21875 */
  float binsize;       /* mm: 1.21875 */
  int span;            /* 3 or 9 */
  int maxdel;          /* 67 */
  int subsets;         /* 16 */
  float rel_fov;       /* 0.95 */
  int z_min, z_max;    /* 6, 200 */
  int npskip;          /* 3 */
  float epsilon1, epsilon2, epsilon3, image_max;  /* 5e-2, 1e-2, 1e-10, 1e4 */
} hrrt_geom;

typedef struct hrrt_info {
  int nx, ny, nz, zp;        /* image grid; zp = padded z */
  int nbins, nviews;
  int nseg, groupmax, segmentsize;
  int subsets, sviews;
  int fov_columns;
  long long sino_elems;      /* segmentsize*nviews*nbins */
  long long image_elems;     /* nx*ny*zp */
} hrrt_info;

typedef struct hrrt_stats {
  double sum_image;          /* post-iteration sum over the FOV, z in [z_min,z_max), FP64 */
  int subset_iterations;     /* completed */
  float ms_total;            /* device time of the OSEM loop (CUDA events) */
} hrrt_stats;

typedef struct hrrt_ctx hrrt_ctx;

/* HRRT model 999 (scanner_model.cpp:124) at span 9, maxdel 67, 16 subsets */
void hrrt_geom_default(hrrt_geom *g);

/* Replaces GetScannerParameter + dependencies (hrrt_osem3d_span3.cpp:3452-3551,
 * hrrt_osem3dv_sbrt_span3.cpp:199-800): builds all tables on `device`. */
int hrrt_ctx_create(const hrrt_geom *g, int device, hrrt_ctx **out);
void hrrt_ctx_destroy(hrrt_ctx *ctx);
const char *hrrt_last_error(const hrrt_ctx *ctx);
int hrrt_get_info(const hrrt_ctx *ctx, hrrt_info *info);
/* the context's CUDA stream (a cudaStream_t) for callers that time or order work */
void *hrrt_get_stream(hrrt_ctx *ctx);

/*
 * Replaces PrepareNormfac + PrepareOsem3dFiles for OP-OSEM (-W 3): prepare_norm
 * + norm_ANW (hrrt_osem3d_span3.cpp:796-1056) and prepare_osem3dw3 (:1649-1818)
 * with 3D attenuation (Atten3D).  Builds on the device
 *   1/(N*max(A,1)) (0 where N*A <= eps2),  (d*N + s)*A,  prompts zeroed where N==0,
 *   and the norm-zero quad mask,
 * with N's first/last npskip planes of each segment set to 0 when a norm is
 * given (file_io_processor.cpp:168-172).  norm/atten/scatter may be NULL
 * (N=1, A=1, s=0).  `storage` is HRRT_STORE_F32 or HRRT_STORE_16.
 */
int hrrt_upload_inputs(hrrt_ctx *ctx, const int16_t *prompts, const float *randoms, const float *norm,
                       const float *atten, const float *scatter, int storage);

/* Replaces CalculateNormfac (hrrt_osem3d_span3.cpp:3760-3865) with -N: the
 * per-subset inverse sensitivity images stay on the device. */
int hrrt_sensitivity(hrrt_ctx *ctx);

/* Replaces Init_Image (hrrt_osem3d_span3.cpp:3958-4006).  image_zyx NULL: 1 in
 * the FOV for z in [z_min,z_max), else 0; otherwise a flat [z][y][x] image
 * (the -i input, read without flip). */
int hrrt_init_image(hrrt_ctx *ctx, const float *image_zyx);

/* Replaces CalculateOsem3d (hrrt_osem3d_span3.cpp:4098-4341) for OP-OSEM:
 * `iterations` full passes over the subsets in sequence() order. */
int hrrt_osem(hrrt_ctx *ctx, int iterations, hrrt_stats *stats);

/* Run `count` subset-iterations starting at position `first` of the subset
 * order (wrapping), without the post-iteration pass; for benchmarking. */
int hrrt_osem_subsets(hrrt_ctx *ctx, int first, int count);

/* Image out in the SaveImage layout [z][y][x] (nz*ny*nx floats). */
int hrrt_get_image(hrrt_ctx *ctx, float *image_zyx);
/* Image in/out in the internal layout [x][y][zp]. */
int hrrt_get_image_xyz(hrrt_ctx *ctx, float *image_xyz);
int hrrt_set_image_xyz(hrrt_ctx *ctx, const float *image_xyz);
/* Inverse sensitivity of one subset, [x][y][zp]. */
int hrrt_get_sensitivity(hrrt_ctx *ctx, int subset, float *nf_inv_xyz);
/* Quad mask [nviews/2][nbins/2+1] (norm_zero_mask, sbrt:333, drv:899-909). */
int hrrt_get_norm_zero_mask(hrrt_ctx *ctx, int16_t *mask);
int hrrt_set_norm_zero_mask(hrrt_ctx *ctx, const int16_t *mask);

/* Replaces forward_proj3d_thread1 (hrrt_osem3dv_sbrt_span3.cpp:1373-1446):
 * forward-projects image_xyz into the two views (view, view+nviews/2).  Rows
 * and bins the reference leaves unwritten (bin 0, columns outside the FOV,
 * masked quads) keep the caller's values. */
int hrrt_fp_pair(hrrt_ctx *ctx, const float *image_xyz, int view, float *prj);

/* The reconstruction of main (drv:4487-4560: PrepareNormfac, CalculateNormfac,
 * PrepareOsem3dFiles, Init_Image, CalculateOsem3d, SaveImage) in one call,
 * pipelined: the inputs stream in subset order (each view pair's rows as 2D
 * copies; pinned host memory lets them overlap) while the first iteration's
 * sensitivity images and subsets run behind them.  Same arguments and result
 * as hrrt_upload_inputs + hrrt_sensitivity + hrrt_init_image + hrrt_osem +
 * hrrt_get_image; image_zyx receives SaveImage's [z][y][x] image. */
int hrrt_reconstruct(hrrt_ctx *ctx, const int16_t *prompts, const float *randoms, const float *norm,
                     const float *atten, const float *scatter, int storage, const float *init_image_zyx,
                     int iterations, float *image_zyx, hrrt_stats *stats);

/* Replaces the forward projection of Output_CorrectedScan
 * (hrrt_osem3d_span3.cpp:3624-3723, the -I 0 -h mode): forward-projects
 * image_xyz for every view pair into a full flat-file sinogram (zeros where the
 * reference writes nothing). */
int hrrt_forward_project(hrrt_ctx *ctx, const float *image_xyz, float *sino);

/* Replaces back_proj3d_thread1 (sbrt:1622-1699): back-projects prj (not
 * modified) for (view, view+nviews/2) into the rotated frame buffer
 * imagebuf_xyz [x][y][zp] (overwritten).
 * mode HRRT_BP_ADJOINT instead writes FP^T prj in the image frame (every
 * column, overwritten): the exact transpose of hrrt_fp_pair, so that
 * <fp(x), y> = <x, bp(y)> to rounding.  No counterpart in the reference. */
int hrrt_bp_pair(hrrt_ctx *ctx, const float *prj, int view, float *imagebuf_xyz, int mode);

/* The back projector of hrrt_sensitivity / hrrt_osem: HRRT_BP_REF (default,
 * the reference's) or HRRT_BP_ADJOINT (the forward projector's transpose; the
 * ratio is then not weighted by the reference's cos^3 segment factor).
 * Clears the sensitivity images.  No counterpart in the reference. */
int hrrt_set_backprojector(hrrt_ctx *ctx, int mode);

/*
 * Back projection of one view pair that allocates no device memory (no
 * counterpart in the reference, whose projector works on host arrays).  For
 * callers that may not allocate while they run -- a real-time loop that cannot
 * take cudaMalloc's device synchronisation, or a host that grants the library
 * a fixed memory budget at start-up and allows no allocation after it.  The
 * result of hrrt_bp_pair(ctx, ..., HRRT_BP_REF) -- the reference back
 * projector, whatever hrrt_set_backprojector selected -- with the caller's
 * device buffers: d_prj rows [2*segmentsize][nbins] in, d_imagebuf [x][y][zp]
 * out (overwritten), on `stream` (a cudaStream_t; NULL = the context's
 * stream), asynchronously; the caller's current device is left as it was.
 * Its scratch is a static 16 MiB device array in the library (held on every
 * GPU that loads it until exit); geometries whose quad-layout view pair
 * exceeds it are rejected with HRRT_ERR_ARG.  The first call on a device
 * resolves that array's address, so make it before any stream capture.  All
 * calls share the array: calls that overlap on the GPU race.
 */
int hrrt_bp_pair_noalloc(hrrt_ctx *ctx, const float *d_prj, int view, float *d_imagebuf, void *stream);

/* PSF resolution modelling, the -B fwhm1,fwhm2,ratio option of hrrt_osem3d
 * (psf.cpp; drv:3328-3330, :4521-4540).  enable = 1 builds the x, y and z
 * kernels of make1d_psf_filter (fwhm1 = 0: the HRRT defaults) for the voxel
 * sizes; hrrt_sensitivity then blurs each subset's back projection before
 * inverting it (drv:3835-3841), and every OSEM subset projects the blurred
 * image and blurs the correction image before the update (drv:4172, :4229).
 * enable = 0 turns it off.  Either clears the sensitivity images.  Not
 * available together with a batch. */
int hrrt_set_psf(hrrt_ctx *ctx, int enable, float fwhm1, float fwhm2, float ratio);
/* convolve3d (psf.cpp:463-540) of image_xyz on FOV columns into out_xyz
 * (other columns zero) with the kernels hrrt_set_psf built. */
int hrrt_psf_convolve(hrrt_ctx *ctx, const float *image_xyz, float *out_xyz);
/* MAP reconstruction, technique 1 of je_hrrt_osem3d's -b technique,beta
 * (je_hrrt_osem3d/hrrt_osem3d.cpp:3360-3369, :4330-4463): Green's
 * one-step-late prior.  From subset `first_subset` on (counted from the last
 * hrrt_init_image / hrrt_set_image_xyz; the reference's i_min_MAP is 5) each
 * OSEM subset replaces the update with pt_cal_updateimage_mapem (:2031-2073),
 * image = min(image_max, image * min(100, max(0.1, corr / (beta * prior + 1 / nf_inv)))),
 * the prior being calculate_DPF_image (dpfcalc.c) of the image before the
 * update.  The reference forms 1 / nf_inv with _mm_rcp_ps (relative error up
 * to 1.5 * 2^-12); here it is exact.  technique 0 or beta 0 turns MAP off;
 * technique 2 (the MR joint-entropy prior) is refused.  Not available
 * together with a batch.  The je_hrrt_osem3d defaults eps1 = eps2 = 1e-4 and
 * image_max = 1e10 go in the hrrt_geom given to hrrt_ctx_create. */
int hrrt_set_map(hrrt_ctx *ctx, int technique, float beta, int first_subset);
/* calculate_DPF_image (technique 1) of image_xyz into prior_xyz on the
 * device, after hrrt_set_map. */
int hrrt_map_prior(hrrt_ctx *ctx, const float *image_xyz, float *prior_xyz);

/* Host-only (no GPU needed): make1d_psf_filter's taps for one pixel size into
 * `taps` (capacity); returns the tap count or a negative status. */
long long hrrt_psf_kernel(float fwhm1, float fwhm2, float ratio, float pixel_size, float *taps, int capacity);

/* Replaces rotate_image_buf (sbrt:1701-1725) for one view: corr_xyz +=
 * rotate-back(imagebuf_xyz). */
int hrrt_rotate_add(hrrt_ctx *ctx, const float *imagebuf_xyz, int view, float *corr_xyz);

/* Host-only (no GPU needed): copy one geometry table built for `g` into `out`
 * (capacity `bytes`); returns the table's size in bytes, or a negative status.
 * Names: "cylwiny" (int16 [ny][2]), "segments" (int32 [3][nseg]: yr_bottom,
 * yr_top, segment_offset), "sin_theta", "cos_theta", "sin_psi", "cos_psi",
 * "tantheta", "rescale" (float [groupmax][nz]), "flookup_zzi" (int32),
 * "flookup_zzz0" (float) [ny][groupmax*2*(span-1)], "blookup" (int32
 * [ny][groupmax][3]: zsa, zea, yra), "blookup_yr2a" (float [ny][groupmax]),
 * "bp_scale" (float [nseg]), "order" (int16 [subsets]).  Used to pin the
 * tables against the reference's dependencies(). */
long long hrrt_geometry_table(const hrrt_geom *g, const char *name, void *out, size_t bytes);

/* Device kernel timing: enable per-kernel CUDA-event timing on the context
 * stream, and read back launches / total milliseconds per kernel name. */
int hrrt_set_profiling(hrrt_ctx *ctx, int enable);
int hrrt_kernel_stats(hrrt_ctx *ctx, const char *kernel, int *launches, double *total_ms);
int hrrt_reset_kernel_stats(hrrt_ctx *ctx);

/* ------------------------------------------------------------------------ */
/* Launch shapes of the projectors (no counterpart in the reference)         */
/* ------------------------------------------------------------------------ */

/* Results are bit-identical for every shape; only the time changes. */
typedef struct hrrt_tuning {
  int fp_planes;          /* planes per forward-projection task: 7, 9 or 11 (0: 9) */
  int fp_producer_warps;  /* sampling warps of the forward projector: 2..6 (0: as many as fit) */
  int bp_planes;          /* planes per back-projection task: 4 or 8 (0: 8) */
  int bp_threads;         /* threads per back-projection CTA: 256 or 384 (0: 384) */
  int bp_tile;            /* back projection: plane runs side by side in a warp, a power of 2 up to 32;
                             the warp's other tasks take consecutive rows (0: 2 above 12 segment
                             groups, else 4) */
  double fp_ms, bp_ms;    /* filled by the tuners: the chosen shapes' device time per launch */
} hrrt_tuning;

int hrrt_set_tuning(hrrt_ctx *ctx, const hrrt_tuning *t);
int hrrt_get_tuning(hrrt_ctx *ctx, hrrt_tuning *t);
/* Time every shape this geometry admits on the context's current inputs and
 * image (the forward projection and back projection of the first subset,
 * `repeats` launches each; the image is not changed) and keep the fastest. */
int hrrt_autotune(hrrt_ctx *ctx, int repeats, hrrt_tuning *chosen);

/* ------------------------------------------------------------------------ */
/* Dynamic studies: frames sharing one normalisation and attenuation         */
/* ------------------------------------------------------------------------ */

/*
 * Replaces the frame loop of main (hrrt_osem3d_span3.cpp:4555-4597: the
 * sensitivity once, then per frame PrepareOsem3dFiles, Init_Image,
 * CalculateOsem3d(frame), SaveImage; frames found by get_num_frames,
 * hrrt_osem_utils.cpp:39-64).  Here every frame has its own iteration count,
 * and the frames are reconstructed together: each projector launch covers a
 * group of frames (as many as device memory allows, frames with more
 * iterations first), and one iteration of a group -- every subset's
 * projection, back projection and update, and the post-iteration pass -- is
 * one CUDA graph, captured once per (group, active frames) and replayed.  Each
 * frame's image equals what hrrt_upload_inputs + hrrt_sensitivity +
 * hrrt_init_image + hrrt_osem(iterations) give for it alone (bit-identical).
 *
 * A batch uses its context's geometry, back projector, launch shape and
 * sensitivity images: creating it replaces the context's inputs (single-frame
 * calls need hrrt_upload_inputs again).  The context must outlive the batch.
 */
typedef struct hrrt_batch hrrt_batch;

typedef struct hrrt_batch_stats {
  double ms_total;        /* device time of hrrt_batch_run */
  int subset_iterations;  /* summed over the frames */
  int groups;             /* frame groups (launches cover one group) */
  int graphs;             /* CUDA graphs captured */
  int graph_launches;     /* graph replays (one per iteration of a group) */
  long long kernel_launches; /* kernels run by those replays */
} hrrt_batch_stats;

/* norm / atten: flat-file arrays shared by every frame (NULL = 1), copied to
 * the device; storage: HRRT_STORE_F32 or HRRT_STORE_16. */
int hrrt_batch_create(hrrt_ctx *ctx, int nframes, int storage, const float *norm, const float *atten,
                      hrrt_batch **out);
void hrrt_batch_destroy(hrrt_batch *b);
/* The inputs of one frame (prepared at once; the host arrays are not kept) and
 * its iteration count (>= 1). */
int hrrt_batch_set_frame(hrrt_batch *b, int frame, const int16_t *prompts, const float *randoms,
                         const float *scatter, int iterations);
/* hrrt_autotune with the batch's launches (a whole group of frames). */
int hrrt_batch_autotune(hrrt_batch *b, int repeats, hrrt_tuning *chosen);
/* Reconstruct every frame (each from the uniform initial image). */
int hrrt_batch_run(hrrt_batch *b, hrrt_batch_stats *stats);
/* Frame image in the SaveImage layout [z][y][x]; sum_image (may be NULL): the
 * FP64 image sum of its last post-iteration pass. */
int hrrt_batch_get_image(hrrt_batch *b, int frame, float *image_zyx, double *sum_image);

/* ------------------------------------------------------------------------ */
/* Listmode (64-bit HRRT events) to span-3 / span-9 sinograms               */
/* ------------------------------------------------------------------------ */

/* Histogram modes of lmhistogram_mp (histogram_mp.cpp:1301-1398): trues =
 * prompts minus delayed in one sinogram; prompts and delayed in two; prompts
 * only. */
#define HRRT_LM_TRUES 0
#define HRRT_LM_PROMPTS_AND_DELAYED 1
#define HRRT_LM_PROMPTS_ONLY 2
/* flags: the rebinner's border-crystal option (histogram_mp.cpp:1190), no DOI
 * decoding (every event layer 1), time from the count of time tags instead
 * of their value (timetag_processing = 0) */
#define HRRT_LM_IGNORE_BORDER_CRYSTAL 1
#define HRRT_LM_NO_DOI 2
#define HRRT_LM_TIME_FROM_COUNT 4
/* implementation choice (same result): by default events are added straight
 * into the 16-bit bins; FORCE_WIDE counts into 32-bit scratch counters
 * (reductions without a round trip) folded into the 16-bit bins at the end,
 * FORCE_PARTITIONED scatters events by 64 MB partition first and adds each
 * partition in L2.  Both measured slower than the default on B200. */
#define HRRT_LM_FORCE_DIRECT 16
#define HRRT_LM_FORCE_PARTITIONED 32
#define HRRT_LM_FORCE_WIDE 64
/* also collect the frame's head curve and block singles (hrrt_lm_head_curve,
 * hrrt_lm_block_singles); costs one more parse of the words */
#define HRRT_LM_HEAD_CURVE 128
/* also count the coincidence histogram (hrrt_lm_crystal_counts) */
#define HRRT_LM_CRYSTAL_COUNTS 256

/* one line of the head curve (.hc, process_tagword histogram_mp.cpp:241-258):
 * at each change of second, the time, the prompt and delayed events since the
 * previous line and the sum over blocks of their latest singles sample */
typedef struct hrrt_lm_second {
  long long time_ms;
  long long prompts;
  long long randoms;
  long long total_singles;
} hrrt_lm_second;

typedef struct hrrt_lm_stats {
  long long words_used;  /* words consumed: through the tag that ended the frame, or all */
  long long prompts;     /* prompt events histogrammed (next_event_32's count) */
  long long delayed;     /* delayed events */
  long long timetags;    /* time tags processed */
  long long tags;        /* tag words of every kind */
  long long invalid;     /* events failing the head-pair / crystal checks */
  long long unmapped;    /* valid events without a sinogram address */
  long long doi_other;   /* events with a DOI value other than 0, 1 and 7 */
  long long doi7;        /* transmission-flagged events in an emission stream (not histogrammed) */
  long long resyncs;     /* out-of-sync words skipped */
  long long frame_start; /* s, from the time tags */
  long long duration;    /* s histogrammed */
  int terminated;        /* 1 when a time tag ended the frame */
  float ms;              /* device time of the call (CUDA events) */
} hrrt_lm_stats;

typedef struct hrrt_lm hrrt_lm;

/* Replaces LM_Rebinner::init_rebinner (LM_Rebinner_mp.cpp:56-146) with the
 * LUT that hrrt_rebinner_lut writes (lor_sinogram_map.cpp:141-221, depth
 * 1.0 cm): output span 3 or 9, maximum ring difference (67). */
int hrrt_lm_create(int span, int maxrd, int device, hrrt_lm **out);
void hrrt_lm_destroy(hrrt_lm *lm);
const char *hrrt_lm_last_error(const hrrt_lm *lm);
/* bins of one sinogram: planes x 288 views x 256 bins */
long long hrrt_lm_sino_size(const hrrt_lm *lm);
/* the stream the host-buffer entry point runs on (cudaStream_t) */
void *hrrt_lm_get_stream(const hrrt_lm *lm);
/* Host-only (no GPU needed): copy one rebinning table for (span, maxrd) into
 * `out` (capacity `bytes`); returns its size in bytes or a negative status.
 * Names: "sol" ({int32 nsino; float d; float z} [21][144][144], the LUT
 * hrrt_rebinner_lut writes), "zpos", "zpos2" (float [104]), "segz0",
 * "segzmax", "segzoffset" (int32 [45]). */
long long hrrt_lm_table(int span, int maxrd, const char *name, void *out, size_t bytes);
/* forget the clock carried from the previous frame (a new stream) */
int hrrt_lm_reset_clock(hrrt_lm *lm);

/* Replaces the reader / rebinner / histogram threads of lmhistogram_mp for
 * one frame (histogram_mp.cpp:1026-1398; rebin_event, LM_Rebinner_mp.cpp:
 * 188-219): `words` is the raw l64 stream as 32-bit words (ew1, ew2 pairs),
 * packets of 1 Mi events parsed from their own first word; `duration` > 0
 * ends the frame on the first time tag that reaches it (seconds), else the
 * whole stream is one frame.  Host buffers; `sino` / `delayed` (16-bit
 * bins, wrapping like the reference's short sinogram) are overwritten.
 * The clock carries into the next call: pass the remaining words
 * (from stats.words_used) for the next frame. */
int hrrt_lm_histogram(hrrt_lm *lm, const uint32_t *words, long long nwords, int mode, int duration, int flags,
                      uint16_t *sino, uint16_t *delayed, hrrt_lm_stats *stats);
/* hrrt_lm_histogram of words that sit `file_offset` words into the listmode
 * file: the reader's packets of 1 Mi 64-bit events count from the file start
 * (LM_Reader_mp.cpp:124), so the frames of one file, histogrammed call by
 * call at their offsets, parse as one pass over the file does. */
int hrrt_lm_histogram_at(hrrt_lm *lm, const uint32_t *words, long long nwords, long long file_offset, int mode,
                         int duration, int flags, uint16_t *sino, uint16_t *delayed, hrrt_lm_stats *stats);
/* hrrt_lm_histogram[_at] streams host words longer than one chunk: chunks of
 * whole packets go up on a copy stream while the previous chunk is
 * histogrammed, with the same results as one pass (calls asking for the head
 * curve, the coincidence histogram or a forced wide / partitioned path take
 * the whole stream at once).  words: the chunk, a multiple of 2 Mi words
 * (0: 64 Mi words, 256 MB; < 0: never stream).  No counterpart in the
 * reference, whose reader thread overlaps its file reads the same way
 * (LM_Reader_mp.cpp:124). */
int hrrt_lm_set_chunk(hrrt_lm *lm, long long words);
/* goto_event (histogram_mp.cpp:384-425, 619-623): advance over the words
 * (at `file_offset` in the file) to just past the time tag that reaches
 * `target_s` seconds -- for 0, the tag that reads 0 ms, the coincidence
 * processor's clock reset -- setting the handle's clock second on the way;
 * nothing is histogrammed.  With HRRT_LM_TIME_FROM_COUNT a seek to 0 does
 * nothing.  *consumed: the words advanced; HRRT_ERR_NOT_FOUND when the
 * stream ends first. */
int hrrt_lm_seek(hrrt_lm *lm, const uint32_t *words, long long nwords, long long file_offset, int target_s, int flags,
                 long long *consumed);
/* The same on device buffers (words 16-byte aligned, sinograms 4-byte
 * aligned), ADDING into sino / delayed, on `stream` (NULL: the library's). */
int hrrt_lm_histogram_device(hrrt_lm *lm, const uint32_t *d_words, long long nwords, int mode, int duration,
                             int flags, uint16_t *d_sino, uint16_t *d_delayed, hrrt_lm_stats *stats, void *stream);

/* After a hrrt_lm_histogram[_device] call with HRRT_LM_HEAD_CURVE: its head
 * curve lines (copies min(n, capacity), returns n), and its block singles
 * (rates: [936] average of each block's samples over the frame, the
 * header's "block singles i"; the totals of the lines' prompts and randoms,
 * histogram_mp.cpp:181-190 -- the header's totals add the events after the
 * last line, :1387-1388, which are the stats' prompts / delayed). */
int hrrt_lm_head_curve(hrrt_lm *lm, hrrt_lm_second *out, int capacity);
int hrrt_lm_block_singles(hrrt_lm *lm, int *rates, long long *total_prompts, long long *total_randoms);
/* After a call with HRRT_LM_CRYSTAL_COUNTS: the frame's coincidence histogram
 * (the .ch file write_coin_map writes, histogram_mp.cpp:646-680): uint32
 * [2][119808], prompt then delayed counts of both crystals of every emission
 * event with DOI 0/1 (rebin_packet :1212-1223), crystal index
 * layer*59904 + head*72 + x + ring*576.  The reference counts whole packets,
 * so its map also holds the events after a frame's end in the same packet;
 * here it holds the frame's events. */
int hrrt_lm_crystal_counts(hrrt_lm *lm, uint32_t *counts);

/* Smoothed randoms from a coincidence histogram (.ch: int32 [2][119808],
 * prompt then delayed counts per crystal [layer 2][ring 104][head 8][x 72]).
 * Replaces gen_delays (gen_delays_lib/gen_delays_lib.cpp:285-548), which
 * hrrt_osem3d runs when -d names a .ch file (hrrt_osem3d_span3.cpp:4424-4471):
 * crystal singles from the delayed counts (compute_csings_from_drates,
 * :163-255, on the host), then for every crystal pair within maxrd + 6 rings
 * singles(A) * singles(B) * 2 tau * T added to the pair's bin of the
 * context's span (compute_delays, :89-153, on the device).  Crystal A's
 * singles are indexed as gen_delays_fromarchive.cpp:191 does (the library
 * copy's index reads past the array).  sino: the flat float sinogram
 * (hrrt_lm_sino_size floats); scan_duration <= 0 means 1 s, tau <= 0 means
 * 6 ns; *iterations (may be NULL): the singles estimate's iterations.  Sums are
 * accumulated in float with device atomics (order varies at rounding level). */
int hrrt_lm_smooth_randoms(hrrt_lm *lm, const int32_t *coinc_hist, float scan_duration, float tau, float *sino,
                           int *iterations);
/* Host-only (no GPU needed): the crystal singles estimate alone, from the
 * 119808 delayed crystal counts; returns the iterations run. */
int hrrt_lm_crystal_singles(const int32_t *delayed_counts, float scan_duration, float tau, float *singles);

/* convert_span9 (lmhistogram_mp/convert_span9.cpp:13, called from
 * write_sino, lmhistogram_mp.cpp:668-677): the span-3 sinogram (minus the
 * delayed sinogram when `delayed` is not NULL: the trues of -PR mode) folded
 * into the 2209-plane span-9 sinogram, 16-bit sums that wrap like the
 * reference's shorts.  Host code, out of place (span9 holds 2209 planes and
 * may not alias the inputs); returns the span-9 plane count or a negative
 * error code. */
long long hrrt_lm_convert_span9(const int16_t *span3, const int16_t *delayed, int16_t *span9, int maxrd);
/* The same fold on the device from a span-3 handle's histograms (d_delayed
 * may be NULL), enqueued on `stream` (NULL: the handle's stream); 16-byte
 * aligned device buffers, output not aliasing the inputs. */
int hrrt_lm_trues_span9_device(hrrt_lm *lm, const uint16_t *d_prompts, const uint16_t *d_delayed, int16_t *d_span9,
                               void *stream);

#ifdef __cplusplus
}
#endif
#endif /* HRRT_GPU_H */
