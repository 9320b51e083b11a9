// batch.cu -- dynamic studies (hrrt_batch_*) and the projector launch-shape
// tuner (hrrt_autotune, hrrt_batch_autotune); declared in include/hrrt_gpu.h.
//
// A batch holds every frame's prepared inputs and image on the device and the
// scratch of one group of frames.  The frame loop of the reference's main
// (hrrt_osem3d_span3.cpp:4555-4597) becomes, per group, one CUDA graph per
// iteration: the 16 subsets' fp -> bp -> rotate-back+update launches and the
// post-iteration pass, each launch covering the group's frames that still
// iterate.  Frames are ordered by iteration count (descending), so the frames
// active at any iteration are a prefix of their group and a graph is keyed by
// (group start, active frames).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <utility>
#include <vector>

#include "context.h"

using namespace hrrt;
using namespace hrrt_host;

struct hrrt_batch {
  hrrt_ctx *ctx = nullptr;
  int nframes = 0, storage = 0;
  float *d_norm = nullptr, *d_atten = nullptr;  // flat-file copies shared by every frame
  char *q_prompts = nullptr, *q_add = nullptr;  // [frame] quad-layout inputs
  size_t in_elems = 0;                          // elements per frame (lanes)
  float *images = nullptr;                      // [frame][vol]
  double *sums = nullptr;                       // [frame]
  int group = 1;                                // frames per launch
  float *ratio = nullptr, *bc = nullptr, *br = nullptr;  // scratch of one group
  double *partial = nullptr;                    // [group][pb]
  int pb = 0;
  int *d_order = nullptr;                       // [nframes] frames by descending iteration count
  std::vector<int> iters;
  std::vector<char> ready;
  bool lists_built = false;
  std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
  int epoch = -1;  // ctx->config_epoch the graphs were captured under
  std::vector<void *> allocs;

  ~hrrt_batch() {
    for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
    for (void *p : allocs) cudaFree(p);
    if (ctx && ctx->batch == this) ctx->batch = nullptr;
  }
  template <typename T>
  T *alloc(size_t n, cudaError_t *e) {
    void *p = nullptr;
    *e = cudaMalloc(&p, n * sizeof(T) + 16);
    if (*e != cudaSuccess) return nullptr;
    allocs.push_back(p);
    return (T *)p;
  }
  FrameStrides strides(int start, int n) const {
    return FrameStrides{n,
                        d_order + start,
                        ctx->vol,
                        (long long)in_elems,
                        (long long)ctx->npairs * ctx->quad_pair,
                        (long long)ctx->npairs * ctx->vol,
                        (long long)pb};
  }
  SubsetBufs bufs(int start, int n) const {
    return SubsetBufs{images, q_prompts, q_add, ratio, bc, br, strides(start, n)};
  }
};

namespace {

int bfail(hrrt_batch *b, int code, const std::string &m) { return fail(b->ctx, code, m); }
#define CHECK_BATCH(b)                         \
  do {                                         \
    if (!(b) || !(b)->ctx) return HRRT_ERR_ARG; \
  } while (0)

size_t add_bytes(int storage) { return storage == HRRT_STORE_F32 ? 4 : 2; }

// ---------------------------------------------------------------- tuner ----

// device milliseconds per launch of `fn` (one untimed launch first)
template <typename F>
int time_launch(hrrt_ctx *ctx, int repeats, F fn, double *ms_out) {
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a), "tune");
  CK(cudaEventCreate(&b), "tune");
  cudaError_t e = fn();
  if (e == cudaSuccess) e = cudaEventRecord(a, ctx->stream);
  for (int i = 0; i < repeats && e == cudaSuccess; i++) e = fn();
  if (e == cudaSuccess) e = cudaEventRecord(b, ctx->stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(b);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tune");
  *ms_out = ms / repeats;
  return HRRT_OK;
}

// Every forward-projection shape (plane variant x producer warps) and
// back-projection shape of the geometry, timed on subset order[0] with the
// buffers of `bb`; the fastest of each is kept.
int autotune(hrrt_ctx *ctx, const SubsetBufs &bb, int repeats, hrrt_tuning *chosen) {
  if (repeats < 1) repeats = 1;
  const int s = ctx->geo.order[0];
  const bool adj = ctx->bp_mode == HRRT_BP_ADJOINT;
  const QuadWork *fw = ctx->d_work + ctx->fp_off[s], *bw = ctx->d_work + ctx->bp_off[s];
  const ProjTune saved = ctx->tune;
  ProjTune best = saved;
  double best_fp = 1e30, best_bp = 1e30;
  for (int vi = 0; vi < 3; vi++) {
    if (!ctx->d_fptasks[vi]) continue;
    const int cwarps = (ctx->nfptasks[vi] + 31) / 32;
    for (int pw : {2, 3, 4, 6}) {
      if (cwarps + pw > kFpVariantWarps[vi]) continue;
      ProjTune t = saved;
      t.fp_planes = kFpPlaneVariants[vi];
      t.fp_pwarps = pw;
      if (int rc = apply_tune(ctx, t)) return rc;
      const DevGeom &g = adj ? ctx->dg_adj : ctx->dg;
      double ms = 0;
      int rc = time_launch(ctx, repeats, [&] {
        return launch_fp(g, bb.image, fw, ctx->fp_cnt[s], 1, bb.prompts, bb.add, ctx->storage, bb.ratio,
                         ctx->quad_pair, t, bb.fr, ctx->stream);
      }, &ms);
      if (rc) {
        apply_tune(ctx, saved);
        return rc;
      }
      if (ms < best_fp) {
        best_fp = ms;
        best.fp_planes = t.fp_planes;
        best.fp_pwarps = t.fp_pwarps;
      }
    }
  }
  if (int rc = apply_tune(ctx, best)) return rc;
  if (!adj) {
    for (int i = 0; i < 12; i++) {
      ProjTune t = best;
      t.bp_planes = (i & 1) ? 4 : 8;
      t.bp_threads = (i & 2) ? 384 : 256;
      t.bp_tile = (i < 4) ? 2 : (i < 8) ? 4 : 8;
      double ms = 0;
      int rc = time_launch(ctx, repeats, [&] {
        return launch_bp(ctx->dg, bb.ratio, ctx->quad_pair, bw, ctx->bp_cnt[s], bb.bc, bb.br, ctx->vol, t, bb.fr,
                         ctx->stream);
      }, &ms);
      if (rc) return rc;
      if (ms < best_bp) {
        best_bp = ms;
        best.bp_planes = t.bp_planes;
        best.bp_threads = t.bp_threads;
        best.bp_tile = t.bp_tile;
      }
    }
  } else {
    best_bp = 0;
  }
  if (int rc = apply_tune(ctx, best)) return rc;
  if (chosen) {
    chosen->fp_planes = best.fp_planes;
    chosen->fp_producer_warps = best.fp_pwarps;
    chosen->bp_planes = best.bp_planes;
    chosen->bp_threads = best.bp_threads;
    chosen->bp_tile = best.bp_tile;
    chosen->fp_ms = best_fp;
    chosen->bp_ms = best_bp;
  }
  return HRRT_OK;
}

// ----------------------------------------------------------------- batch ----

// sensitivity images (once per normalisation / back projector) and the
// uniform initial image of every frame (Init_Image, drv:3958-4006)
int prepare(hrrt_batch *b) {
  hrrt_ctx *ctx = b->ctx;
  for (int f = 0; f < b->nframes; f++)
    if (!b->ready[f]) return bfail(b, HRRT_ERR_STATE, "batch: every frame needs hrrt_batch_set_frame first");
  if (!ctx->have_sens) {
    for (int s = 0; s < ctx->geo.sp.subsets; s++)
      if (int rc = sens_subset(ctx, s)) return rc;
    ctx->have_sens = true;
  }
  for (int f = 0; f < b->nframes; f++)
    CK(launch_init_image(ctx->dg, b->images + (size_t)f * ctx->vol, ctx->stream), "batch init");
  // frames by descending iteration count (ties in frame order)
  std::vector<int> order(b->nframes);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->iters[x] > b->iters[y]; });
  CK(cudaMemcpyAsync(b->d_order, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice, ctx->stream),
     "batch order");
  CK(cudaStreamSynchronize(ctx->stream), "batch prepare");
  return HRRT_OK;
}

std::vector<int> sorted_iters(const hrrt_batch *b) {
  std::vector<int> it(b->iters);
  std::stable_sort(it.begin(), it.end(), [](int x, int y) { return x > y; });
  return it;
}

// one iteration of frames [start, start+n) of the sorted order, captured once
// (*captured: whether this call captured it)
int iteration_graph(hrrt_batch *b, int start, int n, cudaGraphExec_t *out, bool *captured) {
  *captured = false;
  if (b->epoch != b->ctx->config_epoch) {
    for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
    b->epoch = b->ctx->config_epoch;
  }
  auto key = std::make_pair(start, n);
  auto it = b->graphs.find(key);
  if (it != b->graphs.end()) {
    *out = it->second;
    return HRRT_OK;
  }
  hrrt_ctx *ctx = b->ctx;
  const bool prof = ctx->prof;
  ctx->prof = false;  // no timing events inside the graph
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed), "capture");
  int rc = HRRT_OK;
  const SubsetBufs bb = b->bufs(start, n);
  for (int i = 0; i < ctx->geo.sp.subsets && rc == HRRT_OK; i++) rc = run_subset(ctx, ctx->geo.order[i], bb);
  if (rc == HRRT_OK) {
    cudaError_t e = launch_post_iteration(ctx->dg, b->images, b->partial, b->sums, bb.fr, ctx->stream);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "capture post_iteration");
  }
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
  ctx->prof = prof;
  if (rc != HRRT_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(ctx, e, "capture");
  cudaGraphExec_t exec = nullptr;
  e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "graph instantiate");
  b->graphs[key] = exec;
  *out = exec;
  *captured = true;
  return HRRT_OK;
}

}  // namespace

namespace hrrt_host {
void detach_batch(hrrt_batch *b) {
  if (!b) return;
  for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
  for (void *p : b->allocs) cudaFree(p);
  b->allocs.clear();
  b->ctx = nullptr;
}
}  // namespace hrrt_host

extern "C" {

int hrrt_set_tuning(hrrt_ctx *ctx, const hrrt_tuning *t) {
  if (!ctx || !t) return HRRT_ERR_ARG;
  return apply_tune(ctx, ProjTune{t->fp_planes, t->fp_producer_warps, t->bp_planes, t->bp_threads, t->bp_tile});
}

int hrrt_get_tuning(hrrt_ctx *ctx, hrrt_tuning *t) {
  if (!ctx || !t) return HRRT_ERR_ARG;
  std::memset(t, 0, sizeof(*t));
  t->fp_planes = ctx->tune.fp_planes > 0 ? ctx->tune.fp_planes : kFpPlanes;
  t->fp_producer_warps = ctx->tune.fp_pwarps;
  t->bp_planes = ctx->tune.bp_planes > 0 ? ctx->tune.bp_planes : kBpZ;
  t->bp_threads = ctx->tune.bp_threads;
  t->bp_tile = ctx->tune.bp_tile;
  return HRRT_OK;
}

int hrrt_autotune(hrrt_ctx *ctx, int repeats, hrrt_tuning *chosen) {
  if (!ctx) return HRRT_ERR_ARG;
  if (!ctx->have_inputs || !ctx->have_image)
    return fail(ctx, HRRT_ERR_STATE, "autotune: inputs and image must be set first");
  if (int rc = autotune(ctx, ctx_bufs(ctx), repeats, chosen)) return rc;
  return device_status(ctx);
}

int hrrt_batch_create(hrrt_ctx *ctx, int nframes, int storage, const float *norm, const float *atten,
                      hrrt_batch **out) {
  if (!ctx || !out) return HRRT_ERR_ARG;
  *out = nullptr;
  if (nframes < 1) return fail(ctx, HRRT_ERR_ARG, "batch: nframes must be >= 1");
  if (storage < HRRT_STORE_F32 || storage > HRRT_STORE_F16) return fail(ctx, HRRT_ERR_ARG, "unknown storage");
  if (ctx->batch) return fail(ctx, HRRT_ERR_STATE, "batch: the context already serves a batch");
  if (ctx->psf_on) return fail(ctx, HRRT_ERR_STATE, "batch: PSF modelling runs one frame at a time");
  if (ctx->map_on) return fail(ctx, HRRT_ERR_STATE, "batch: MAP runs one frame at a time");
  if (int rc = ensure_input_buffers(ctx, storage)) return rc;
  const Geometry &g = ctx->geo;
  auto *b = new hrrt_batch();
  b->ctx = ctx;
  b->nframes = nframes;
  b->storage = storage;
  b->iters.assign(nframes, 0);
  b->ready.assign(nframes, 0);
  auto bail = [&](int rc) {
    delete b;
    return rc;
  };
  cudaError_t e = cudaSuccess;
  const size_t flat = (size_t)g.segmentsize * g.nviews * g.nbins;
  for (int i = 0; i < 2; i++) {
    const float *src = i ? atten : norm;
    if (!src) continue;
    float *d = b->alloc<float>(flat, &e);
    if (!d) return bail(fail(ctx, HRRT_ERR_NOMEM, "batch: norm / attenuation"));
    e = cudaMemcpy(d, src, flat * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "batch: norm / attenuation"));
    (i ? b->d_atten : b->d_norm) = d;
  }
  b->in_elems = (size_t)(g.nviews / 2) * ctx->quad_pair;
  b->q_prompts = b->alloc<char>(nframes * b->in_elems * 2, &e);
  b->q_add = b->q_prompts ? b->alloc<char>(nframes * b->in_elems * add_bytes(storage), &e) : nullptr;
  b->images = b->q_add ? b->alloc<float>((size_t)nframes * ctx->vol, &e) : nullptr;
  b->sums = b->images ? b->alloc<double>(nframes, &e) : nullptr;
  b->d_order = b->sums ? b->alloc<int>(nframes, &e) : nullptr;
  if (!b->d_order) return bail(fail(ctx, HRRT_ERR_NOMEM, "batch: frame inputs"));
  // frames per launch: as many as the free memory holds (2 GiB kept back)
  b->pb = post_iteration_blocks(ctx->dg);
  const size_t per = sizeof(float) * ((size_t)ctx->npairs * ctx->quad_pair + 2 * (size_t)ctx->npairs * ctx->vol) +
                     sizeof(double) * (size_t)b->pb;
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b), "batch");
  const size_t reserve = (size_t)2 << 30;
  const long long fit = free_b > reserve ? (long long)((free_b - reserve) / per) : 0;
  b->group = (int)std::max<long long>(1, std::min<long long>(nframes, fit));
  b->ratio = b->alloc<float>((size_t)b->group * ctx->npairs * ctx->quad_pair, &e);
  b->bc = b->ratio ? b->alloc<float>((size_t)b->group * ctx->npairs * ctx->vol, &e) : nullptr;
  b->br = b->bc ? b->alloc<float>((size_t)b->group * ctx->npairs * ctx->vol, &e) : nullptr;
  b->partial = b->br ? b->alloc<double>((size_t)b->group * b->pb, &e) : nullptr;
  if (!b->partial) return bail(fail(ctx, HRRT_ERR_NOMEM, "batch: scratch"));
  ctx->batch = b;
  ctx->have_inputs = false;  // the context's single-frame inputs are replaced
  ctx->have_sens = false;
  *out = b;
  return HRRT_OK;
}

void hrrt_batch_destroy(hrrt_batch *b) {
  if (!b) return;
  if (b->ctx) cudaStreamSynchronize(b->ctx->stream);
  delete b;
}

int hrrt_batch_set_frame(hrrt_batch *b, int frame, const int16_t *prompts, const float *randoms,
                         const float *scatter, int iterations) {
  CHECK_BATCH(b);
  if (frame < 0 || frame >= b->nframes) return bfail(b, HRRT_ERR_ARG, "batch: frame out of range");
  if (!prompts || !randoms) return bfail(b, HRRT_ERR_ARG, "batch: prompts and randoms are required");
  if (iterations < 1) return bfail(b, HRRT_ERR_ARG, "batch: iterations must be >= 1");
  hrrt_ctx *ctx = b->ctx;
  void *qp = b->q_prompts + (size_t)frame * b->in_elems * 2;
  void *qa = b->q_add + (size_t)frame * b->in_elems * add_bytes(b->storage);
  // the shared 1/(NA) and norm-zero mask are rewritten with the same values
  if (int rc = upload_flat(ctx, prompts, randoms, b->d_norm, b->d_atten, scatter, b->storage, true, qp, qa,
                           ctx->q_mult))
    return rc;
  if (!b->lists_built) {
    if (int rc = build_work_lists(ctx)) return rc;
    b->lists_built = true;
  }
  b->iters[frame] = iterations;
  b->ready[frame] = 1;
  return HRRT_OK;
}

int hrrt_batch_autotune(hrrt_batch *b, int repeats, hrrt_tuning *chosen) {
  CHECK_BATCH(b);
  if (int rc = prepare(b)) return rc;
  if (int rc = autotune(b->ctx, b->bufs(0, std::min(b->group, b->nframes)), repeats, chosen)) return rc;
  return device_status(b->ctx);
}

int hrrt_batch_run(hrrt_batch *b, hrrt_batch_stats *stats) {
  CHECK_BATCH(b);
  hrrt_ctx *ctx = b->ctx;
  if (int rc = prepare(b)) return rc;
  const std::vector<int> it = sorted_iters(b);
  const int S = ctx->geo.sp.subsets;
  hrrt_batch_stats st{};
  cudaEvent_t ev0, ev1;
  CK(cudaEventCreate(&ev0), "batch");
  CK(cudaEventCreate(&ev1), "batch");
  cudaEventRecord(ev0, ctx->stream);
  int rc = HRRT_OK;
  for (int start = 0; start < b->nframes && rc == HRRT_OK; start += b->group) {
    const int n = std::min(b->group, b->nframes - start);
    st.groups++;
    for (int k = 0; k < it[start] && rc == HRRT_OK; k++) {
      int nact = 0;
      while (nact < n && it[start + nact] > k) nact++;
      cudaGraphExec_t g = nullptr;
      bool captured = false;
      rc = iteration_graph(b, start, nact, &g, &captured);
      if (rc) break;
      if (captured) st.graphs++;
      cudaError_t e = cudaGraphLaunch(g, ctx->stream);
      if (e != cudaSuccess) {
        rc = cuda_fail(ctx, e, "graph launch");
        break;
      }
      st.graph_launches++;
      st.kernel_launches += 3LL * S + 2;
      st.subset_iterations += nact * S;
    }
  }
  cudaEventRecord(ev1, ctx->stream);
  cudaError_t e = cudaEventSynchronize(ev1);
  float ms = 0.f;
  if (e == cudaSuccess) cudaEventElapsedTime(&ms, ev0, ev1);
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch run");
  if (int r = device_status(ctx)) return r;
  st.ms_total = ms;
  if (stats) *stats = st;
  return HRRT_OK;
}

int hrrt_batch_get_image(hrrt_batch *b, int frame, float *image_zyx, double *sum_image) {
  CHECK_BATCH(b);
  if (!image_zyx) return HRRT_ERR_ARG;
  if (frame < 0 || frame >= b->nframes) return bfail(b, HRRT_ERR_ARG, "batch: frame out of range");
  hrrt_ctx *ctx = b->ctx;
  const Geometry &g = ctx->geo;
  cudaError_t e = cudaSuccess;
  if (!ctx->d_tmp_img) ctx->d_tmp_img = dalloc<float>(ctx, ctx->vol, &e);
  if (!ctx->d_tmp_img) return fail(ctx, HRRT_ERR_NOMEM, "scratch");
  CK(launch_image_zyx(ctx->dg, b->images + (size_t)frame * ctx->vol, ctx->d_tmp_img, ctx->stream), "batch image");
  CK(cudaMemcpyAsync(image_zyx, ctx->d_tmp_img, sizeof(float) * (size_t)g.nz * g.ny * g.nx, cudaMemcpyDeviceToHost,
                     ctx->stream),
     "batch image");
  if (sum_image)
    CK(cudaMemcpyAsync(sum_image, b->sums + frame, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream),
       "batch image");
  CK(cudaStreamSynchronize(ctx->stream), "batch image");
  return HRRT_OK;
}

}  // extern "C"
