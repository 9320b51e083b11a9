// context.h -- the state behind an hrrt_ctx and the host helpers the C-ABI
// translation units share (hrrt_gpu.cu: single-frame entry points; batch.cu:
// dynamic studies and the launch-shape tuner).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "../../include/hrrt_gpu.h"
#include "geometry.h"
#include "kernels.cuh"

struct hrrt_batch;

struct KernelTimer {
  std::string name;
  cudaEvent_t start, stop;
};

struct hrrt_ctx {
  hrrt::Geometry geo;
  hrrt::DevGeom dg{};
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  std::vector<void *> allocs;

  int storage = -1;
  void *q_prompts = nullptr, *q_add = nullptr, *q_mult = nullptr;
  int16_t *d_nzmask = nullptr;
  int *d_mask_accum = nullptr;
  std::vector<int16_t> nzmask;

  float *d_image = nullptr;
  float *d_nfinv = nullptr;
  float *d_ratio = nullptr, *d_bc = nullptr, *d_br = nullptr;
  float *d_tmp_img = nullptr;  // test entry points
  float *d_rows = nullptr;
  double *d_partial = nullptr, *d_sum = nullptr;
  int *d_pair_views = nullptr;  // [subsets][npairs]
  hrrt::QuadWork *d_work = nullptr;   // fp lists then bp lists, per subset
  std::vector<int> fp_off, fp_cnt, bp_off, bp_cnt;
  int *d_rowstart = nullptr;
  int npairs = 0;               // view pairs per subset
  long long vol = 0;            // nx*ny*zp
  long long quad_pair = 0;      // floats per pair in quad layout
  // launch shape of the projectors, and the forward-projection task list of
  // each plane variant (null where the variant does not fit the geometry)
  hrrt::ProjTune tune = hrrt::default_tune();
  hrrt::FpTask *d_fptasks[3] = {nullptr, nullptr, nullptr};
  int nfptasks[3] = {0, 0, 0};
  bool have_inputs = false, have_sens = false, have_image = false;

  // chunked upload: flat-file planes staged through two device buffers, the
  // copy of one chunk overlapping the prep of the previous one
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_copied[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr};
  // hrrt_reconstruct: further streams that share each subset's strided copies
  cudaStream_t copy_side[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t ev_side[3][2] = {};
  char *stage[2] = {nullptr, nullptr};
  size_t stage_bytes = 0;
  // pipelined reconstruction: the view pairs of one subset staged pair-major
  char *pstage[2] = {nullptr, nullptr};
  size_t pstage_bytes = 0;
  int16_t *pflat = nullptr;  // hrrt_reconstruct: the whole prompt sinogram
  size_t pflat_elems = 0;

  // back projector of the OSEM loop, and the device geometry it runs with
  // (for the adjoint: segment weights of 1, the forward projector's scaling)
  int bp_mode = HRRT_BP_REF;
  hrrt::DevGeom dg_adj{};
  int *d_view1 = nullptr;       // one view index, for single-pair entry points

  // a dynamic study using this context's geometry, mult and sensitivity
  struct hrrt_batch *batch = nullptr;
  // bumped whenever what a captured launch sequence depends on changes (back
  // projector, launch shape, work lists, PSF)
  int config_epoch = 0;

  // PSF resolution modelling (-B): the x / y filters (2h+1 taps), the
  // inverted z tap sums, and three volumes: the blurred image, the
  // correction image and the x pass
  bool psf_on = false;
  int psf_h = 0;
  float *d_psf_fx = nullptr, *d_psf_fy = nullptr, *d_psf_normz = nullptr;
  float *d_image_psf = nullptr, *d_corr = nullptr, *d_psf_tmp = nullptr;
  // MAP technique 1 (je_hrrt_osem3d -b 1,beta): the prior replaces the update
  // from subset map_first on (counted from the last image initialisation)
  bool map_on = false;
  float map_beta = 0.f;
  int map_first = 5;
  long long subsets_done = 0;
  float *d_dpf = nullptr;
  unsigned int *d_mapmax = nullptr;

  bool prof = false;
  std::vector<KernelTimer> pending;
  std::map<std::string, std::pair<int, double>> kstats;

  ~hrrt_ctx() {
    for (auto &t : pending) {
      cudaEventDestroy(t.start);
      cudaEventDestroy(t.stop);
    }
    for (void *p : allocs) cudaFree(p);
    for (int b = 0; b < 2; b++) {
      if (ev_copied[b]) cudaEventDestroy(ev_copied[b]);
      if (ev_free[b]) cudaEventDestroy(ev_free[b]);
    }
    if (copy_stream) cudaStreamDestroy(copy_stream);
    for (int i = 0; i < 3; i++) {
      if (copy_side[i]) cudaStreamDestroy(copy_side[i]);
      for (int b = 0; b < 2; b++)
        if (ev_side[i][b]) cudaEventDestroy(ev_side[i][b]);
    }
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace hrrt_host {

using hrrt::DevGeom;
using hrrt::FrameStrides;
using hrrt::ProjTune;
using hrrt::QuadWork;

inline int fail(hrrt_ctx *ctx, int code, const std::string &msg) {
  if (ctx) ctx->err = msg;
  return code;
}
inline int cuda_fail(hrrt_ctx *ctx, cudaError_t e, const char *where) {
  return fail(ctx, HRRT_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
#define CK(call, where)                                   \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, where); \
  } while (0)

template <typename T>
inline T *dalloc(hrrt_ctx *ctx, size_t n, cudaError_t *e) {
  void *p = nullptr;
  *e = cudaMalloc(&p, n * sizeof(T) + 16);
  if (*e != cudaSuccess) return nullptr;
  *e = cudaMemsetAsync(p, 0, n * sizeof(T) + 16, ctx->stream);
  ctx->allocs.push_back(p);
  return (T *)p;
}
template <typename T>
inline T *dupload(hrrt_ctx *ctx, const std::vector<T> &v, cudaError_t *e) {
  T *p = dalloc<T>(ctx, std::max<size_t>(v.size(), 1), e);
  if (!p) return nullptr;
  if (!v.empty()) *e = cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
  return p;
}

struct Launch {
  hrrt_ctx *ctx;
  KernelTimer t{};
  Launch(hrrt_ctx *c, const char *name) : ctx(c) {
    if (ctx->prof) {
      t.name = name;
      cudaEventCreate(&t.start);
      cudaEventCreate(&t.stop);
      cudaEventRecord(t.start, ctx->stream);
    }
  }
  ~Launch() {
    if (ctx->prof) {
      cudaEventRecord(t.stop, ctx->stream);
      ctx->pending.push_back(t);
    }
  }
};

inline void drain_timers(hrrt_ctx *ctx) {
  for (auto &t : ctx->pending) {
    cudaEventSynchronize(t.stop);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t.start, t.stop);
    auto &s = ctx->kstats[t.name];
    s.first += 1;
    s.second += ms;
    cudaEventDestroy(t.start);
    cudaEventDestroy(t.stop);
  }
  ctx->pending.clear();
}


// The buffers one OSEM subset reads and writes: the context's own (one
// frame), or a batch's frames with their strides.
struct SubsetBufs {
  float *image;
  const void *prompts, *add;
  float *ratio, *bc, *br;
  FrameStrides fr;
};

// defined in hrrt_gpu.cu
SubsetBufs ctx_bufs(hrrt_ctx *ctx);
// fp -> bp (or the adjoint) -> rotate-back + update of subset s, on ctx->stream
int run_subset(hrrt_ctx *ctx, int s, const SubsetBufs &b);
int device_status(hrrt_ctx *ctx);
int range_status(hrrt_ctx *ctx);
int ensure_input_buffers(hrrt_ctx *ctx, int storage);
int build_work_lists(hrrt_ctx *ctx);
int sens_subset(hrrt_ctx *ctx, int s);
// Prepare one set of flat-file inputs into quad-layout buffers qp / qadd (and
// the shared qmult and norm-zero mask), kUploadPlanes planes at a time through
// the context's two staging buffers.  norm / atten are host arrays, or device
// arrays in the flat layout when `norm_atten_device` (not staged then).
int upload_flat(hrrt_ctx *ctx, const int16_t *prompts, const float *randoms, const float *norm, const float *atten,
                const float *scatter, int storage, bool norm_atten_device, void *qp, void *qadd, void *qmult);
// the forward-projection task list of tune.fp_planes into ctx->dg / dg_adj
int apply_tune(hrrt_ctx *ctx, const ProjTune &t);
// convolve3d of the PSF: out = psf(in) on FOV columns (in may equal out)
int run_psf(hrrt_ctx *ctx, const float *in, float *out);
// defined in batch.cu: a context being destroyed leaves its batch unusable
void detach_batch(hrrt_batch *b);

}  // namespace hrrt_host
