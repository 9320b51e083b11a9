// kernels.cuh -- device tables and kernel launchers of the OSEM hot path.
//
// Data layouts on the device
//   image, nf_inv, Bc, Br : [x][y][zp] float, z fastest (the reference's
//                           image[x][y][z], z padded to a multiple of 4).
//   "quad layout"         : one view pair p (views p and p+nviews/2) and one
//                           radial "quad" x in [0, nbins/2] hold 4 lanes
//                             lane 0 = (view p,           bin x)
//                             lane 1 = (view p,           bin nbins-x)
//                             lane 2 = (view p+nviews/2,  bin x)
//                             lane 3 = (view p+nviews/2,  bin nbins-x)
//                           stored as [pair][x][padded plane][lane] with every
//                           segment padded by one zero plane on each side.
//                           This is the reference's packed prjbuf[x][k][yr][4]
//                           (hrrt_osem3dv_sbrt_span3.cpp:1397-1436, :1654-1693)
//                           made contiguous per quad, so FP output, ratio and
//                           BP input stream with 16-byte accesses.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <cstdint>

namespace hrrt {

#ifndef HRRT_FP_SLOTS
#define HRRT_FP_SLOTS 3
#endif
#ifndef HRRT_BP_MIN_BLOCKS
#define HRRT_BP_MIN_BLOCKS 3
#endif
constexpr int kFpPlanes = 9;                   // default planes per forward-projection task (odd: bank-conflict free)
constexpr int kFpSlots = HRRT_FP_SLOTS;       // sampled rows in flight between producers and consumers
constexpr int kFpZPad = 16;     // zeroed entries after each sampled row
constexpr int kFpEndPlanes = 4; // planes per end-plane task (they cost ~2x a middle plane)
constexpr int kFpMaxGroups = 32; // segment groups the forward projector stages per row (22 at span 3)
constexpr int kBpZ = 8;         // z per back-projection task
constexpr int kBpMinBlocks = HRRT_BP_MIN_BLOCKS;  // resident back-projection CTAs per SM (register budget)
constexpr int kBpPad = 8;       // zero planes on each side of a segment in the back projector (>= kBpZ)
constexpr int kAdjCover = 8;    // rotated-frame points whose bilinear footprint covers a voxel (at most 5 on HRRT)

struct FpTask {
  int16_t seg;   // segment (internal = file order)
  int16_t p0;    // first plane, relative to the segment's yr_bottom
  int16_t n;     // planes in this task (<= the launch's plane variant)
  int16_t type;  // 0: segment 0, 1: oblique middle planes, 2: oblique end planes
};

struct FpMid {   // middle-plane sampling of group g at rotated row y < c (sbrt:1933-1947)
  int z;         // int(yr_m + (y-c)*tan), yr_m = yr_bottom + zshift; < 0 => group skipped
  float f;       // its fraction (coef1)
  int z2;        // int(yr_m + (c-y)*tan)
  float f2;      // its fraction (coef2)
};

struct BpLut {   // blookup (sbrt:672-700) in direct form: yr = z + d for z in [zs, ze]
  int zs, ze, d;
  float f;
};

struct DevGeom {
  int nx, nz, zp, c, nseg, groupmax, zshift, segmentsize, pplanes, nviews, nquads;
  int fov_columns, z_min, z_max;
  float y_size, eps1, eps3, image_max;
  float unit;                       // 1.0f, a run-time value (see addp in kernels.cu)
  const int16_t *cyl0, *cyl1;       // [ny]
  const int *ybot, *ytop, *poff;    // [nseg]; poff = padded offset of plane yr_bottom
  const float *rescale;             // [groupmax][nz]
  const float *bp_scale;            // [nseg]
  const FpMid *fpmid;               // [c][groupmax]
  const int2 *fl_zf;                // [ny][groupmax*2*zshift]: (zzi, bits of zzz0)
  const FpMid *fpmid_t;             // fpmid transposed: [groupmax][c] (the exact adjoint's rows are threads)
  const int2 *fl_t;                 // fl_zf transposed: [groupmax*2*zshift][ny]
  const int4 *adj_endr;             // exact adjoint, [groupmax][c]: planes the bottom / top end-plane
                                    //   entries of a row touch (x..y bottom, z..w top; empty: lo > hi)
  int2 *adj_ent;                    // exact adjoint's rotate: per (pair slot, column) the covering
  int *adj_cnt;                     //   rotated-frame points (index, weight bits) [.][kAdjCover], their count
  int adj_pairs;                    //   pair slots the two buffers hold (for every image column)
  const BpLut *bplut;               // [groupmax][ny]
  const int16_t *nzmask;            // [nviews/2][nquads]
  const float *sin_psi, *cos_psi;   // [nviews]
  const short2 *fov_xy;             // [fov_columns]
  const float2 *rotpos;             // [nviews/2][fov_columns] rotate-back sample points
  const FpTask *fptasks;
  int nfptasks;
  const int16_t *plane_seg;         // [segmentsize] segment of each global plane
  const int16_t *pplane_seg;        // [pplanes] segment of each padded plane, -1 on pads
  int *err;                         // device status word: non-zero after a bounded wait gave up
  int *range_err;                   // non-zero after an input exceeded the fp16 range (HRRT_STORE_F16)
  const int *bp_soff;               // [nseg] back projector: shared-memory plane of yr_bottom
  const int *bp_src;                // [bp_splanes] quad-layout plane of each shared plane, -1 = zero
  int bp_splanes;
};

struct QuadWork {  // one (view pair slot, quad) work item
  int16_t slot;    // pair slot within the batch
  int16_t x;       // quad
  int16_t view;    // first view of the pair
  int16_t pad;
};

// Frames of a dynamic study batched into one launch.  Frame f of a launch
// reads and writes its own buffers at f times these strides from frame 0's;
// the geometry, the work list and the inverse sensitivity are shared.  The
// projector kernels run the work list once per frame, frame-major (CTA i is
// item i % nwork of frame i / nwork: one frame's image stays in L2 while its
// CTAs run, and the next frame's CTAs fill the last wave of the previous);
// the image-domain kernels take the frame from blockIdx.y.
// Images, inputs and image sums belong to stored frames, launch frame f being
// stored frame map[f] (map null: f); the scratch (ratio, partials, partial
// sums) belongs to the launch frame.
struct FrameStrides {
  int n;              // frames in the launch
  const int *map;     // [n] stored frame of each launch frame (device), or null
  long long image;    // floats between stored images
  long long input;    // elements between stored prompts (and additive-term) arrays
  long long ratio;    // floats between ratio blocks ([pair slot][quad_pair])
  long long bc;       // floats between back-projection partial blocks (Bc and Br alike)
  long long partial;  // doubles between post-iteration partial-sum arrays
};
inline FrameStrides one_frame() { return FrameStrides{1, nullptr, 0, 0, 0, 0, 0}; }

// launch shape of the projectors (results do not depend on it)
struct ProjTune {
  int fp_planes;  // planes per forward-projection task: 7, 9 or 11 (0: kFpPlanes)
  int fp_pwarps;  // producer warps of the forward projector (0: as many as fit, 2..6)
  int bp_planes;  // planes per back-projection task: 4 or 8 (0: kBpZ)
  int bp_threads; // threads per back-projection CTA: 256 or 384 (0: 384)
  int bp_tile;    // back projection: plane runs side by side in a warp's 32 tasks, a power of 2
                  // up to 32 (the rest of the warp takes consecutive rows; 0: 2 above 12
                  // segment groups, else 4)
};
inline ProjTune default_tune() { return ProjTune{0, 0, 0, 0, 0}; }
constexpr int kFpPlaneVariants[3] = {7, 9, 11};
// warps per forward-projection CTA for each plane variant (register budget)
constexpr int kFpVariantWarps[3] = {32, 32, 24};

// ---- launchers (kernels.cu) ----
// forward projection of the pairs listed in `work` (mode 0: write est*scale into
// `out`; mode 1: write ratio*bp_scale using prompts/add at their global pair).
// `g.fptasks` must be the task list built for tune.fp_planes.
cudaError_t launch_fp(const DevGeom &g, const float *image, const QuadWork *work, int nwork, int mode,
                      const void *prompts, const void *add, int storage, float *out, long long out_pair_stride,
                      const ProjTune &tune, const FrameStrides &fr, cudaStream_t st);
// back projection of quad-layout input into the column (Bc) / row (Br) partials
cudaError_t launch_bp(const DevGeom &g, const float *in, long long in_pair_stride, const QuadWork *work, int nwork,
                      float *bc, float *br, long long vol, const ProjTune &tune, const FrameStrides &fr,
                      cudaStream_t st);
// exact adjoint of the forward projector: z-transpose into the column / row
// partials (rows scaled as the forward projector scales them)
cudaError_t launch_adj(const DevGeom &g, const float *in, long long in_pair_stride, const QuadWork *work, int nwork,
                       float *bc, float *br, long long vol, const FrameStrides &fr, cudaStream_t st);
// bilinear-sampling transpose of the partials of every pair; mode 0: OSEM
// update, 1: inverse sensitivity (FOV columns), 2: out += (every column)
cudaError_t launch_adj_rotate(const DevGeom &g, const int *pair_views, int npairs, const float *bc, const float *br,
                              long long vol, float *image, float *nf_inv, float *out, int mode,
                              const FrameStrides &fr, cudaStream_t st);
// back projection of one view pair's quad-layout input (quads x0..x0+nquads-1)
// with both partial sums added atomically into `out` (zeroed by the caller)
cudaError_t launch_bp_sum(const DevGeom &g, const float *quad, int view, int x0, int nquads, float *out,
                          cudaStream_t st);
// corr = sum over pairs of rotate-back(Bc+Br); mode 0: OSEM update of image with
// nf_inv; mode 1: write the inverse sensitivity into nf_inv; mode 2: corr_out += corr;
// mode 3: corr_out = corr (FOV columns)
cudaError_t launch_rotback(const DevGeom &g, const int *pair_views, int npairs, const float *bc, const float *br,
                           long long vol, float *image, float *nf_inv, float *corr_out, int mode,
                           const FrameStrides &fr, cudaStream_t st);
cudaError_t launch_rotpos(const DevGeom &g, float2 *rotpos, const int *row_start, cudaStream_t st);
// PSF (convolve3d, psf.cpp:463-540): out = yz(x(in)) on the FOV columns, tmp
// holds the x pass; filters of 2h+1 taps (taps -h..h-1 used); normz [zp] the
// inverted z tap sums
cudaError_t launch_psf(const DevGeom &g, const float *in, float *tmp, float *out, const float *filt_x, int hx,
                       const float *filt_y, int hy, const float *normz, cudaStream_t st);
// mode 0: OSEM update of image from the correction volume; 1: inverse
// sensitivity into nf_inv; 2: the MAP update with the prior volume dpf
cudaError_t launch_apply_corr(const DevGeom &g, const float *corr, float *image, float *nf_inv, int mode,
                              cudaStream_t st, const float *dpf = nullptr, float beta = 0.f);
// MAP technique 1 prior (calculate_DPF_image, je_hrrt_osem3d/dpfcalc.c) of
// image into dpf on the FOV columns; mx: one device word of scratch
cudaError_t launch_map_prior(const DevGeom &g, const float *image, unsigned int *mx, float *dpf, cudaStream_t st);
cudaError_t launch_prep(const DevGeom &g, int nbins, const int16_t *prompts, const float *randoms, const float *norm,
                        const float *atten, const float *scatter, int npskip, float eps2, int storage, void *q_prompts,
                        void *q_add, void *q_mult, int *quad_mask_accum, int plane0, int nplanes,
                        cudaStream_t st);
// the same from pair-major staging: for each of `npairs` slots, the rows of
// view pair_views[slot] and its partner, [2 views][segmentsize][nbins]
// (flat_prompts: the prompts are instead the whole [plane][view][bin]
// sinogram on the device)
cudaError_t launch_prep_pairs(const DevGeom &g, int nbins, const int16_t *prompts, const float *randoms,
                              const float *norm, const float *atten, const float *scatter, int npskip, float eps2,
                              int storage, void *q_prompts, void *q_add, void *q_mult, int *quad_mask_accum,
                              const int *pair_views, int npairs, cudaStream_t st,
                              bool flat_prompts = false);
cudaError_t launch_finish_mask(const DevGeom &g, const int *accum, int16_t *nzmask, cudaStream_t st);
// [z][y][x] image of SaveImage (FOV columns, planes < nz) from [x][y][zp]
cudaError_t launch_image_zyx(const DevGeom &g, const float *image, float *out, cudaStream_t st);
cudaError_t launch_init_image(const DevGeom &g, float *image, cudaStream_t st);
// per launch frame f: threshold of its image, the FP64 sum into sum[stored frame]
cudaError_t launch_post_iteration(const DevGeom &g, float *image, double *partial, double *sum,
                                  const FrameStrides &fr, cudaStream_t st);
int post_iteration_blocks(const DevGeom &g);
// copy the quad-layout 1/(NA) of `npairs` view pairs into f32 scratch, times
// the back projector's segment weight (sbrt:1637-1649 applied in place there)
cudaError_t launch_scale_pairs(const DevGeom &g, const void *src, int storage, const int *views, int npairs,
                               float *dst, long long dst_pair_stride, cudaStream_t st);
// quad-layout <-> reference rows [2*segmentsize][nbins]
cudaError_t launch_rows_to_quad(const DevGeom &g, int nbins, const float *rows, float *quad, int apply_bp_scale,
                                cudaStream_t st);
cudaError_t launch_quad_to_rows(const DevGeom &g, int nbins, const float *quad, const QuadWork *work, int nwork,
                                float *rows, cudaStream_t st);
// scatter the quad-layout estimates of a batch of pairs into a flat-file sinogram
cudaError_t launch_quad_to_file(const DevGeom &g, int nbins, const float *quad, long long quad_pair_stride,
                                const QuadWork *work, int nwork, float *sino, cudaStream_t st);
cudaError_t launch_add_partials(const DevGeom &g, const float *bc, const float *br, float *out, cudaStream_t st);

}  // namespace hrrt
