// hrrt_gpu.cu -- the C ABI of libhrrt_gpu.so (declared in include/hrrt_gpu.h).
//
// A context owns the geometry tables, the device copies of the prepared
// inputs (quad layout, every view pair), the image, the per-subset inverse
// sensitivity images and the per-subset scratch (OP ratio and the two
// back-projection partials of each view pair of a subset).  One OSEM subset
// is three launches on the context stream:
//   fp_kernel (forward projection + ratio) -> bp_kernel -> rotback_kernel
//   (rotate-back of the nine view pairs fused with the multiplicative update).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "context.h"

using namespace hrrt;
using namespace hrrt_host;

namespace {

// flat-file planes per upload chunk (96 planes of 288 x 256 bins: 127 MB of
// staging per buffer with all five inputs)
constexpr int kUploadPlanes = 96;

// make1d_psf_filter (psf.cpp:21-70): two Gaussians of FWHM fwhm1, fwhm2 (mm)
// -- the second scaled by ratio -- sampled at the pixel size over 2h+1 taps
// (h from 1.5 FWHM at the 10 % level) and normalised by their float sum;
// fwhm1 == 0 selects the HRRT's defaults (0.9 and 2.5 sigma in mm, ratio
// 0.05).  Empty when fwhm1 < 0.
std::vector<float> psf_taps(float fwhm1, float fwhm2, float ratio, float pixel_size) {
  if (fwhm1 == 0.0) {
    fwhm1 = (float)(0.9 * std::sqrt(8.0 * std::log(2.0)));
    fwhm2 = (float)(2.5 * std::sqrt(8.0 * std::log(2.0)));
    ratio = 0.05f;
  }
  if (!(fwhm1 > 0.0)) return {};
  const double w = (fwhm2 > 0.0 && ratio > 0.0) ? fwhm2 : fwhm1;
  const int size = 2 * ((int)(1.5 * w * std::sqrt(std::log(10.0) / std::log(2.)) / pixel_size / 2.0)) + 1;
  if (size < 1 || size > 255) return {};
  const float sigma1 = (float)(fwhm1 / (std::sqrt(8.0 * std::log(2.0)) * pixel_size));
  const float sigma2 = (float)(fwhm2 / (std::sqrt(8.0 * std::log(2.0)) * pixel_size));
  const int bin0 = (size - 1) / 2;
  std::vector<float> k(size);
  float norm = 0.0f;
  for (int b = 0; b < size; b++) {
    k[b] = (float)std::exp(-0.5 * (std::pow((double)(b - bin0) / sigma1, 2.0)));
    if (fwhm2 > 0.0 && ratio > 0.0)
      k[b] = (float)(k[b] + ratio * std::exp(-0.5 * (std::pow((double)(b - bin0) / sigma2, 2.0))));
    norm += k[b];
  }
  for (int b = 0; b < size; b++) k[b] /= norm;
  return k;
}

// Forward-projection tasks shared by every quad: (segment, plane run, kind).
std::vector<FpTask> build_fp_tasks(const Geometry &g, int PL) {
  std::vector<FpTask> mid, ends;
  for (int p0 = 0; p0 < g.nz; p0 += PL) mid.push_back(FpTask{0, (int16_t)p0, (int16_t)std::min(PL, g.nz - p0), 0});
  for (int s = 1; s < g.nseg; s++) {
    const int ns = g.yr_top[s] - g.yr_bottom[s] + 1;
    for (int p0 = g.zshift; p0 < ns - g.zshift; p0 += PL)
      mid.push_back(FpTask{(int16_t)s, (int16_t)p0, (int16_t)std::min(PL, ns - g.zshift - p0), 1});
    // an end-plane run stays inside one end region, so its lookup entries are consecutive
    for (int p0 = 0; p0 < g.zshift; p0 += kFpEndPlanes)
      ends.push_back(FpTask{(int16_t)s, (int16_t)p0, (int16_t)std::min(kFpEndPlanes, g.zshift - p0), 2});
    for (int p0 = ns - g.zshift; p0 < ns; p0 += kFpEndPlanes)
      ends.push_back(FpTask{(int16_t)s, (int16_t)p0, (int16_t)std::min(kFpEndPlanes, ns - p0), 2});
  }
  // one task kind per warp (the kinds cost different amounts per row, and a
  // warp mixing them would set the pace of every row barrier): pad each kind
  // to a multiple of 32 with empty tasks
  std::vector<FpTask> t0, t1;
  for (const FpTask &t : mid) (t.type == 0 ? t0 : t1).push_back(t);
  std::vector<FpTask> out;
  for (auto *lst : {&t0, &t1, &ends}) {
    out.insert(out.end(), lst->begin(), lst->end());
    while (out.size() % 32) out.push_back(FpTask{0, 0, 0, -1});
  }
  return out;
}

// Every shared-memory index the forward projector can form for this geometry
// must lie inside the staged column; checked once here so the kernel needs no
// run-time guards.
std::string validate_fp(const Geometry &g, const std::vector<FpMid> &mid, const std::vector<FpTask> &tasks, int PL) {
  const int ZS = g.zp + kFpZPad, FS = g.flookup_stride();
  int ymin = g.c;
  for (int x = 1; x <= g.c; x++)
    if (g.cyl0[x] != g.cyl1[x]) ymin = std::min<int>(ymin, g.cyl0[x]);
  for (int y = ymin; y < g.c; y++) {
    for (const FpTask &t : tasks) {
      if (t.type < 0) continue;
      if (t.type == 0) {
        if (t.p0 + PL >= ZS) return "fp: segment-0 window out of range";
        continue;
      }
      const int gg = (t.seg + 1) / 2 - 1;
      const FpMid m = mid[(size_t)y * g.groupmax + gg];
      if (m.z < 0) continue;
      if (t.type == 1) {
        const int za = m.z + t.p0 - g.zshift, zb = m.z2 + t.p0 - g.zshift;
        if (za < 0 || zb < 0 || za + PL >= ZS || zb + PL >= ZS) return "fp: middle window out of range";
      } else {
        const int ns = g.yr_top[t.seg] - g.yr_bottom[t.seg] + 1;
        for (int j = 0; j < t.n; j++) {
          const int r = t.p0 + j;
          const int yri = (r < g.zshift) ? r : r - ns + 2 * g.zshift;
          const int li = gg * 2 * g.zshift + yri;
          const int z = g.fl_zzi[(size_t)y * FS + li], z2 = g.fl_zzi[(size_t)(g.ny - y) * FS + li];
          if (z < 0 || z2 < 0 || z + 1 >= ZS || z2 + 1 >= ZS) return "fp: end-plane index out of range";
        }
      }
    }
  }
  return std::string();
}

}  // namespace

namespace hrrt_host {

// reads (and clears) the device status word after the stream has drained
int device_status(hrrt_ctx *ctx) {
  int v = 0;
  cudaError_t e = cudaMemcpyAsync(&v, ctx->dg.err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "status");
  if (v != 0) {
    cudaMemsetAsync(ctx->dg.err, 0, sizeof(int), ctx->stream);
    return fail(ctx, HRRT_ERR_DEVICE, "a device-side bounded wait timed out");
  }
  return HRRT_OK;
}

// reads (and clears) the fp16 range flag the input preparation sets
int range_status(hrrt_ctx *ctx) {
  int v = 0;
  cudaError_t e = cudaMemcpyAsync(&v, ctx->dg.range_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "status");
  if (v != 0) {
    cudaMemsetAsync(ctx->dg.range_err, 0, sizeof(int), ctx->stream);
    return fail(ctx, HRRT_ERR_ARG,
                "an additive or multiplicative term exceeds the fp16 range (65504): use HRRT_STORE_16 or _F32");
  }
  return HRRT_OK;
}

int build_work_lists(hrrt_ctx *ctx) {
  const Geometry &g = ctx->geo;
  const int S = g.sp.subsets;
  std::vector<QuadWork> all;
  std::vector<int> views;
  ctx->fp_off.assign(S, 0);
  ctx->fp_cnt.assign(S, 0);
  ctx->bp_off.assign(S, 0);
  ctx->bp_cnt.assign(S, 0);
  // quads ordered by decreasing rotated-column length (longest work first)
  std::vector<int> xs;
  for (int x = 1; x <= g.c; x++)
    if (g.cyl0[x] != g.cyl1[x]) xs.push_back(x);
  std::stable_sort(xs.begin(), xs.end(), [&](int a, int b) { return g.cyl0[a] < g.cyl0[b]; });
  const int nq = g.nx / 2 + 1;
  for (int s = 0; s < S; s++) {
    for (int k = 0; k < ctx->npairs; k++) views.push_back(g.vieworder[(size_t)s * g.sviews + k]);
    for (int pass = 0; pass < 2; pass++) {
      const int off = (int)all.size();
      for (int x : xs)
        for (int k = 0; k < ctx->npairs; k++) {
          const int v = g.vieworder[(size_t)s * g.sviews + k];
          if (pass == 0 && ctx->nzmask[(size_t)v * nq + x] == 0) continue;
          all.push_back(QuadWork{(int16_t)k, (int16_t)x, (int16_t)v, 0});
        }
      if (pass == 0) {
        ctx->fp_off[s] = off;
        ctx->fp_cnt[s] = (int)all.size() - off;
      } else {
        ctx->bp_off[s] = off;
        ctx->bp_cnt[s] = (int)all.size() - off;
      }
    }
  }
  cudaError_t e = cudaSuccess;
  if (ctx->d_work) {
    cudaFree(ctx->d_work);
    ctx->allocs.erase(std::find(ctx->allocs.begin(), ctx->allocs.end(), (void *)ctx->d_work));
  }
  ctx->d_work = dupload(ctx, all, &e);
  if (!ctx->d_work) return cuda_fail(ctx, e, "work list");
  ctx->config_epoch++;
  if (!ctx->d_pair_views) {
    ctx->d_pair_views = dupload(ctx, views, &e);
    if (!ctx->d_pair_views) return cuda_fail(ctx, e, "pair views");
  }
  CK(e, "work list upload");
  return HRRT_OK;
}

SubsetBufs ctx_bufs(hrrt_ctx *ctx) {
  return SubsetBufs{ctx->d_image, ctx->q_prompts, ctx->q_add, ctx->d_ratio, ctx->d_bc, ctx->d_br, one_frame()};
}

int run_subset(hrrt_ctx *ctx, int s, const SubsetBufs &b) {
  const bool adj = ctx->bp_mode == HRRT_BP_ADJOINT;
  const DevGeom &g = adj ? ctx->dg_adj : ctx->dg;
  const QuadWork *fw = ctx->d_work + ctx->fp_off[s], *bw = ctx->d_work + ctx->bp_off[s];
  const int *pv = ctx->d_pair_views + (size_t)s * ctx->npairs;
  float *nf = ctx->d_nfinv + (size_t)s * ctx->vol;
  const bool single = b.fr.n == 1 && !b.fr.map;
  const bool map = single && ctx->map_on && ctx->subsets_done >= ctx->map_first;
  if (single) ctx->subsets_done++;
  if (map) {
    // je_hrrt_osem3d's subset with MAP (hrrt_osem3d.cpp:4439-4463): the
    // correction image (blurred with -B), the prior of the image before the
    // update, then pt_cal_updateimage_mapem
    const float *proj = b.image;
    if (ctx->psf_on) {
      if (int rc = run_psf(ctx, b.image, ctx->d_image_psf)) return rc;
      proj = ctx->d_image_psf;
    }
    {
      Launch L(ctx, "fp_kernel");
      CK(launch_fp(g, proj, fw, ctx->fp_cnt[s], 1, b.prompts, b.add, ctx->storage, b.ratio, ctx->quad_pair,
                   ctx->tune, b.fr, ctx->stream),
         "fp_kernel");
    }
    if (adj) {
      CK(launch_adj(g, b.ratio, ctx->quad_pair, bw, ctx->bp_cnt[s], b.bc, b.br, ctx->vol, b.fr, ctx->stream),
         "adj_kernel");
      CK(cudaMemsetAsync(ctx->d_corr, 0, sizeof(float) * ctx->vol, ctx->stream), "map");
      CK(launch_adj_rotate(g, pv, ctx->npairs, b.bc, b.br, ctx->vol, nullptr, nullptr, ctx->d_corr, 2, b.fr,
                           ctx->stream),
         "adj_rotate_kernel");
    } else {
      {
        Launch L(ctx, "bp_kernel");
        CK(launch_bp(g, b.ratio, ctx->quad_pair, bw, ctx->bp_cnt[s], b.bc, b.br, ctx->vol, ctx->tune, b.fr,
                     ctx->stream),
           "bp_kernel");
      }
      Launch L(ctx, "rotback_kernel");
      CK(launch_rotback(g, pv, ctx->npairs, b.bc, b.br, ctx->vol, nullptr, nullptr, ctx->d_corr, 3, b.fr,
                        ctx->stream),
         "rotback_kernel");
    }
    if (ctx->psf_on)
      if (int rc = run_psf(ctx, ctx->d_corr, ctx->d_corr)) return rc;
    {
      Launch L(ctx, "map_dpf_kernel");
      CK(launch_map_prior(ctx->dg, b.image, ctx->d_mapmax, ctx->d_dpf, ctx->stream), "map prior");
    }
    Launch L(ctx, "apply_corr_kernel");
    CK(launch_apply_corr(ctx->dg, ctx->d_corr, b.image, nf, 2, ctx->stream, ctx->d_dpf, ctx->map_beta), "map update");
    return HRRT_OK;
  }
  if (ctx->psf_on) {
    // -B (drv:4172, :4201-4202, :4229): project the blurred image, blur the
    // correction image, then update
    if (b.fr.n != 1 || b.fr.map) return fail(ctx, HRRT_ERR_STATE, "PSF runs one frame at a time");
    if (int rc = run_psf(ctx, b.image, ctx->d_image_psf)) return rc;
    {
      Launch L(ctx, "fp_kernel");
      CK(launch_fp(g, ctx->d_image_psf, fw, ctx->fp_cnt[s], 1, b.prompts, b.add, ctx->storage, b.ratio,
                   ctx->quad_pair, ctx->tune, b.fr, ctx->stream),
         "fp_kernel");
    }
    if (adj) {
      CK(launch_adj(g, b.ratio, ctx->quad_pair, bw, ctx->bp_cnt[s], b.bc, b.br, ctx->vol, b.fr, ctx->stream),
         "adj_kernel");
      CK(cudaMemsetAsync(ctx->d_corr, 0, sizeof(float) * ctx->vol, ctx->stream), "psf");
      CK(launch_adj_rotate(g, pv, ctx->npairs, b.bc, b.br, ctx->vol, nullptr, nullptr, ctx->d_corr, 2, b.fr,
                           ctx->stream),
         "adj_rotate_kernel");
    } else {
      CK(launch_bp(g, b.ratio, ctx->quad_pair, bw, ctx->bp_cnt[s], b.bc, b.br, ctx->vol, ctx->tune, b.fr,
                   ctx->stream),
         "bp_kernel");
      CK(launch_rotback(g, pv, ctx->npairs, b.bc, b.br, ctx->vol, nullptr, nullptr, ctx->d_corr, 3, b.fr,
                        ctx->stream),
         "rotback_kernel");
    }
    if (int rc = run_psf(ctx, ctx->d_corr, ctx->d_corr)) return rc;
    CK(launch_apply_corr(g, ctx->d_corr, b.image, nf, 0, ctx->stream), "update");
    return HRRT_OK;
  }
  {
    Launch L(ctx, "fp_kernel");
    CK(launch_fp(g, b.image, fw, ctx->fp_cnt[s], 1, b.prompts, b.add, ctx->storage, b.ratio, ctx->quad_pair,
                 ctx->tune, b.fr, ctx->stream),
       "fp_kernel");
  }
  if (adj) {
    {
      Launch L(ctx, "adj_kernel");
      CK(launch_adj(g, b.ratio, ctx->quad_pair, bw, ctx->bp_cnt[s], b.bc, b.br, ctx->vol, b.fr, ctx->stream),
         "adj_kernel");
    }
    Launch L(ctx, "adj_rotate_kernel");
    CK(launch_adj_rotate(g, pv, ctx->npairs, b.bc, b.br, ctx->vol, b.image, nf, nullptr, 0, b.fr, ctx->stream),
       "adj_rotate_kernel");
    return HRRT_OK;
  }
  {
    Launch L(ctx, "bp_kernel");
    CK(launch_bp(g, b.ratio, ctx->quad_pair, bw, ctx->bp_cnt[s], b.bc, b.br, ctx->vol, ctx->tune, b.fr, ctx->stream),
       "bp_kernel");
  }
  Launch L(ctx, "rotback_kernel");
  CK(launch_rotback(g, pv, ctx->npairs, b.bc, b.br, ctx->vol, b.image, nf, nullptr, 0, b.fr, ctx->stream),
     "rotback_kernel");
  return HRRT_OK;
}

// quad-layout input buffers for `storage` (allocated once per storage type)
int ensure_input_buffers(hrrt_ctx *ctx, int storage) {
  const Geometry &g = ctx->geo;
  cudaError_t e = cudaSuccess;
  if (ctx->storage != storage) {
    for (void *p : {ctx->q_prompts, ctx->q_add, ctx->q_mult})
      if (p) {
        cudaFree(p);
        ctx->allocs.erase(std::find(ctx->allocs.begin(), ctx->allocs.end(), p));
      }
    ctx->q_prompts = ctx->q_add = ctx->q_mult = nullptr;
    ctx->storage = -1;
    const size_t nquad = (size_t)(g.nviews / 2) * ctx->quad_pair;
    const size_t ab = storage == HRRT_STORE_F32 ? 4 : 2;
    ctx->q_prompts = dalloc<char>(ctx, nquad * 2, &e);
    ctx->q_add = ctx->q_prompts ? dalloc<char>(ctx, nquad * ab, &e) : nullptr;
    ctx->q_mult = ctx->q_add ? dalloc<char>(ctx, nquad * ab, &e) : nullptr;
    if (!ctx->q_mult) return fail(ctx, HRRT_ERR_NOMEM, "input allocation");
    ctx->storage = storage;
  }
  if (!ctx->d_mask_accum) {
    ctx->d_mask_accum = dalloc<int>(ctx, (size_t)(g.nviews / 2) * ctx->dg.nquads, &e);
    if (!ctx->d_mask_accum) return fail(ctx, HRRT_ERR_NOMEM, "mask");
  }
  return HRRT_OK;
}

// inverse sensitivity of subset s (CalculateNormfac's subset body)
int sens_subset(hrrt_ctx *ctx, int s) {
  const bool adj = ctx->bp_mode == HRRT_BP_ADJOINT;
  if (ctx->psf_on) {
    // the back projection blurred before its inversion (drv:3835-3841)
    const DevGeom &g = adj ? ctx->dg_adj : ctx->dg;
    const int *pv = ctx->d_pair_views + (size_t)s * ctx->npairs;
    CK(launch_scale_pairs(g, ctx->q_mult, ctx->storage, pv, ctx->npairs, ctx->d_ratio, ctx->quad_pair, ctx->stream),
       "scale_pairs");
    if (adj) {
      CK(launch_adj(g, ctx->d_ratio, ctx->quad_pair, ctx->d_work + ctx->bp_off[s], ctx->bp_cnt[s], ctx->d_bc,
                    ctx->d_br, ctx->vol, one_frame(), ctx->stream),
         "adj_kernel");
      CK(cudaMemsetAsync(ctx->d_corr, 0, sizeof(float) * ctx->vol, ctx->stream), "psf");
      CK(launch_adj_rotate(g, pv, ctx->npairs, ctx->d_bc, ctx->d_br, ctx->vol, nullptr, nullptr, ctx->d_corr, 2,
                           one_frame(), ctx->stream),
         "adj_rotate_kernel");
    } else {
      CK(launch_bp(g, ctx->d_ratio, ctx->quad_pair, ctx->d_work + ctx->bp_off[s], ctx->bp_cnt[s], ctx->d_bc,
                   ctx->d_br, ctx->vol, ctx->tune, one_frame(), ctx->stream),
         "bp_kernel");
      CK(launch_rotback(g, pv, ctx->npairs, ctx->d_bc, ctx->d_br, ctx->vol, nullptr, nullptr, ctx->d_corr, 3,
                        one_frame(), ctx->stream),
         "rotback_kernel");
    }
    if (int rc = run_psf(ctx, ctx->d_corr, ctx->d_corr)) return rc;
    CK(launch_apply_corr(g, ctx->d_corr, nullptr, ctx->d_nfinv + (size_t)s * ctx->vol, 1, ctx->stream), "inverse");
    return HRRT_OK;
  }
  {
    Launch L(ctx, "scale_pairs_kernel");
    CK(launch_scale_pairs(adj ? ctx->dg_adj : ctx->dg, ctx->q_mult, ctx->storage,
                          ctx->d_pair_views + (size_t)s * ctx->npairs, ctx->npairs, ctx->d_ratio, ctx->quad_pair,
                          ctx->stream),
       "scale_pairs");
  }
  if (adj) {
    {
      Launch L(ctx, "adj_kernel");
      CK(launch_adj(ctx->dg_adj, ctx->d_ratio, ctx->quad_pair, ctx->d_work + ctx->bp_off[s], ctx->bp_cnt[s],
                    ctx->d_bc, ctx->d_br, ctx->vol, one_frame(), ctx->stream),
         "adj_kernel");
    }
    Launch L(ctx, "adj_rotate_kernel");
    CK(launch_adj_rotate(ctx->dg_adj, ctx->d_pair_views + (size_t)s * ctx->npairs, ctx->npairs, ctx->d_bc, ctx->d_br,
                         ctx->vol, nullptr, ctx->d_nfinv + (size_t)s * ctx->vol, nullptr, 1, one_frame(), ctx->stream),
       "adj_rotate_kernel");
    return HRRT_OK;
  }
  {
    Launch L(ctx, "bp_kernel");
    CK(launch_bp(ctx->dg, ctx->d_ratio, ctx->quad_pair, ctx->d_work + ctx->bp_off[s], ctx->bp_cnt[s], ctx->d_bc,
                 ctx->d_br, ctx->vol, ctx->tune, one_frame(), ctx->stream),
       "bp_kernel");
  }
  Launch L(ctx, "rotback_kernel");
  CK(launch_rotback(ctx->dg, ctx->d_pair_views + (size_t)s * ctx->npairs, ctx->npairs, ctx->d_bc, ctx->d_br, ctx->vol,
                    nullptr, ctx->d_nfinv + (size_t)s * ctx->vol, nullptr, 1, one_frame(), ctx->stream),
     "rotback_kernel");
  return HRRT_OK;
}

int upload_flat(hrrt_ctx *ctx, const int16_t *prompts, const float *randoms, const float *norm, const float *atten,
                const float *scatter, int storage, bool norm_atten_device, void *qp, void *qadd, void *qmult) {
  const Geometry &g = ctx->geo;
  cudaError_t e = cudaSuccess;
  // staging of the raw flat-file arrays, kUploadPlanes planes at a time
  const float *srcs[4] = {randoms, norm, atten, scatter};
  const size_t plane_elems = (size_t)g.nviews * g.nbins;
  const int CP = std::min(g.segmentsize, kUploadPlanes);
  const size_t chunk = (size_t)CP * plane_elems;
  const size_t need = chunk * (sizeof(int16_t) + 4 * sizeof(float));
  if (ctx->stage_bytes < need) {
    for (int b = 0; b < 2; b++)
      if (ctx->stage[b]) {
        cudaFree(ctx->stage[b]);
        ctx->allocs.erase(std::find(ctx->allocs.begin(), ctx->allocs.end(), (void *)ctx->stage[b]));
        ctx->stage[b] = nullptr;
      }
    ctx->stage_bytes = 0;
    for (int b = 0; b < 2; b++) {
      ctx->stage[b] = dalloc<char>(ctx, need, &e);
      if (!ctx->stage[b]) return fail(ctx, HRRT_ERR_NOMEM, "upload staging");
    }
    ctx->stage_bytes = need;
  }
  if (!ctx->copy_stream) {
    CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking), "copy stream");
    for (int b = 0; b < 2; b++) {
      CK(cudaEventCreateWithFlags(&ctx->ev_copied[b], cudaEventDisableTiming), "upload event");
      CK(cudaEventCreateWithFlags(&ctx->ev_free[b], cudaEventDisableTiming), "upload event");
    }
  }
  CK(cudaMemsetAsync(ctx->d_mask_accum, 0, sizeof(int) * (size_t)(g.nviews / 2) * ctx->dg.nquads, ctx->stream),
     "upload_inputs");
  for (int b = 0; b < 2; b++) CK(cudaEventRecord(ctx->ev_free[b], ctx->stream), "upload_inputs");
  for (int p0 = 0, k = 0; p0 < g.segmentsize && e == cudaSuccess; p0 += CP, k++) {
    const int b = k & 1, np = std::min(CP, g.segmentsize - p0);
    const size_t off = (size_t)p0 * plane_elems, cnt = (size_t)np * plane_elems;
    int16_t *sp = reinterpret_cast<int16_t *>(ctx->stage[b]);
    float *stg[4] = {nullptr, nullptr, nullptr, nullptr};
    e = cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_free[b], 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(sp, prompts + off, cnt * sizeof(int16_t), cudaMemcpyHostToDevice, ctx->copy_stream);
    for (int i = 0; i < 4 && e == cudaSuccess; i++) {
      if (!srcs[i]) continue;
      if (norm_atten_device && (i == 1 || i == 2)) {
        stg[i] = const_cast<float *>(srcs[i]) + off;  // already on the device
        continue;
      }
      stg[i] = reinterpret_cast<float *>(ctx->stage[b] + chunk * sizeof(int16_t) + (size_t)i * chunk * sizeof(float));
      e = cudaMemcpyAsync(stg[i], srcs[i] + off, cnt * sizeof(float), cudaMemcpyHostToDevice, ctx->copy_stream);
    }
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_copied[b], ctx->copy_stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream, ctx->ev_copied[b], 0);
    if (e == cudaSuccess) {
      Launch L(ctx, "prep_kernel");
      e = launch_prep(ctx->dg, g.nbins, sp, stg[0], stg[1], stg[2], stg[3], g.sp.npskip, g.sp.epsilon2, storage,
                      qp, qadd, qmult, ctx->d_mask_accum, p0, np, ctx->stream);
    }
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_free[b], ctx->stream);
  }
  if (e == cudaSuccess) e = launch_finish_mask(ctx->dg, ctx->d_mask_accum, ctx->d_nzmask, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ctx->nzmask.data(), ctx->d_nzmask, ctx->nzmask.size() * sizeof(int16_t),
                        cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamSynchronize(ctx->stream);
    return cuda_fail(ctx, e, "upload_inputs");
  }
  if (storage == HRRT_STORE_F16) return range_status(ctx);
  return HRRT_OK;
}


int run_psf(hrrt_ctx *ctx, const float *in, float *out) {
  Launch L(ctx, "psf_kernel");
  CK(launch_psf(ctx->dg, in, ctx->d_psf_tmp, out, ctx->d_psf_fx, ctx->psf_h, ctx->d_psf_fy, ctx->psf_h,
                ctx->d_psf_normz, ctx->stream),
     "psf");
  return HRRT_OK;
}

int apply_tune(hrrt_ctx *ctx, const ProjTune &t) {
  const int pl = t.fp_planes > 0 ? t.fp_planes : kFpPlanes;
  int vi = -1;
  for (int i = 0; i < 3; i++)
    if (kFpPlaneVariants[i] == pl) vi = i;
  if (vi < 0 || !ctx->d_fptasks[vi]) return fail(ctx, HRRT_ERR_ARG, "tuning: plane variant unavailable for this geometry");
  const int cwarps = (ctx->nfptasks[vi] + 31) / 32;
  if (t.fp_pwarps != 0 && (t.fp_pwarps < 2 || t.fp_pwarps > 6 || cwarps + t.fp_pwarps > kFpVariantWarps[vi]))
    return fail(ctx, HRRT_ERR_ARG, "tuning: producer warps out of range");
  if (t.bp_planes != 0 && t.bp_planes != 4 && t.bp_planes != 8)
    return fail(ctx, HRRT_ERR_ARG, "tuning: back-projection planes must be 4 or 8");
  if (t.bp_threads != 0 && t.bp_threads != 256 && t.bp_threads != 384)
    return fail(ctx, HRRT_ERR_ARG, "tuning: back-projection threads must be 256 or 384");
  if (t.bp_tile < 0 || t.bp_tile > 32 || (t.bp_tile & (t.bp_tile - 1)) != 0)
    return fail(ctx, HRRT_ERR_ARG, "tuning: back-projection tile must be a power of 2 up to 32");
  ctx->tune = t;
  ctx->config_epoch++;
  ctx->dg.fptasks = ctx->dg_adj.fptasks = ctx->d_fptasks[vi];
  ctx->dg.nfptasks = ctx->dg_adj.nfptasks = ctx->nfptasks[vi];
  return HRRT_OK;
}

}  // namespace hrrt_host

extern "C" {

void hrrt_geom_default(hrrt_geom *g) {
  ScannerParams p;
  g->nrings = p.nrings;
  g->nelements = p.nelements;
  g->nangles = p.nangles;
  g->ring_radius = p.ring_radius;
  g->plane_sep = p.plane_sep;
  g->binsize = p.binsize;
  g->span = p.span;
  g->maxdel = p.maxdel;
  g->subsets = p.subsets;
  g->rel_fov = p.rel_fov;
  g->z_min = p.z_min;
  g->z_max = p.z_max;
  g->npskip = p.npskip;
  g->epsilon1 = p.epsilon1;
  g->epsilon2 = p.epsilon2;
  g->epsilon3 = p.epsilon3;
  g->image_max = p.image_max;
}

const char *hrrt_last_error(const hrrt_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void *hrrt_get_stream(hrrt_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int hrrt_ctx_create(const hrrt_geom *gp, int device, hrrt_ctx **out) {
  if (!gp || !out) return HRRT_ERR_ARG;
  *out = nullptr;
  hrrt_ctx *ctx = new hrrt_ctx();
  auto bail = [&](int code) {
    // keep the context so the caller can read the message; destroy on request
    *out = ctx;
    return code;
  };
  ScannerParams p;
  p.nrings = gp->nrings;
  p.nelements = gp->nelements;
  p.nangles = gp->nangles;
  p.ring_radius = gp->ring_radius;
  p.plane_sep = gp->plane_sep;
  p.binsize = gp->binsize;
  p.span = gp->span;
  p.maxdel = gp->maxdel;
  p.subsets = gp->subsets;
  p.rel_fov = gp->rel_fov;
  p.z_min = gp->z_min;
  p.z_max = gp->z_max;
  p.npskip = gp->npskip;
  p.epsilon1 = gp->epsilon1;
  p.epsilon2 = gp->epsilon2;
  p.epsilon3 = gp->epsilon3;
  p.image_max = gp->image_max;
  // z range adjustments of GetScannerParameter (drv:3516, :3537-3540)
  if (p.z_max == 0) p.z_max = (2 * p.nrings - 1) - p.z_min;
  if (p.npskip > p.z_min) p.z_min = p.npskip;
  if (p.z_max > (2 * p.nrings - 1) - p.npskip) p.z_max = (2 * p.nrings - 1) - p.npskip;
  std::string m = ctx->geo.build(p);
  if (!m.empty()) return bail(fail(ctx, HRRT_ERR_ARG, "geometry: " + m));
  Geometry &g = ctx->geo;
  if (g.nx > 32767 || g.segmentsize > 32767) return bail(fail(ctx, HRRT_ERR_ARG, "geometry too large"));
  ctx->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "cudaSetDevice"));
  e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "stream"));

  ctx->npairs = g.sviews / 2;
  ctx->vol = (long long)g.nx * g.ny * g.zp;
  const int nq = g.nx / 2 + 1;
  ctx->quad_pair = (long long)nq * g.padded_planes() * 4;

  // derived device tables
  std::vector<int> poff(g.nseg);
  for (int s = 0; s < g.nseg; s++) poff[s] = g.padded_offset(s);
  std::vector<FpMid> mid((size_t)g.c * g.groupmax);
  const int FS = g.flookup_stride();
  for (int y = 0; y < g.c; y++)
    for (int th = 2, gg = 0; th < g.nseg; th += 2, gg++) {
      const int yr = g.yr_bottom[th] + g.zshift;
      const float t = g.tantheta[(size_t)gg * g.nz + yr];
      float zz = yr + (y - g.c) * t;
      const int z = (int)zz;
      const float f = zz - z;
      zz = yr + (g.c - y) * t;
      const int z2 = (int)zz;
      const float f2 = zz - z2;
      // row 0 is never in the FOV (its mirror row ny is outside the tables)
      const bool skip = y == 0 || g.fl_zzi[(size_t)y * FS + gg * g.zshift * 2] < 0 ||
                        g.fl_zzi[(size_t)(g.ny - y) * FS + gg * g.zshift * 2 + g.zshift * 2 - 1] > g.nz - 1;
      mid[(size_t)y * g.groupmax + gg] = FpMid{skip ? -1 : z, f, z2, f2};
    }
  // back-projection lookup, transposed to [group][row]
  std::vector<BpLut> bpl((size_t)g.ny * g.groupmax);
  for (int y = 0; y < g.ny; y++)
    for (int gg = 0; gg < g.groupmax; gg++) {
      const size_t i = (size_t)y * g.groupmax + gg;
      bpl[(size_t)gg * g.ny + y] = BpLut{g.bl_zsa[i], g.bl_zea[i], g.bl_yra[i] - g.bl_zsa[i], g.bl_yr2a[i]};
    }
  std::vector<short2> fovxy;
  std::vector<int> rowstart(g.nx + 1, 0);
  for (int X = 0; X < g.nx; X++) {
    rowstart[X] = (int)fovxy.size();
    for (int Y = g.cyl0[X]; Y < g.cyl1[X]; Y++) fovxy.push_back(make_short2((short)X, (short)Y));
  }
  rowstart[g.nx] = (int)fovxy.size();
  std::vector<int16_t> plane_seg(g.segmentsize);
  for (int s = 0; s < g.nseg; s++)
    for (int r = 0; r <= g.yr_top[s] - g.yr_bottom[s]; r++) plane_seg[g.segment_offset[s] + r] = (int16_t)s;
  // back-projection shared-memory layout: every segment with kBpPad zero
  // planes on each side; bp_src[i] = quad-layout plane of shared plane i or -1
  std::vector<int> bp_soff(g.nseg), bp_src;
  for (int s = 0; s < g.nseg; s++) {
    const int ns = g.yr_top[s] - g.yr_bottom[s] + 1;
    for (int k = 0; k < kBpPad; k++) bp_src.push_back(-1);
    bp_soff[s] = (int)bp_src.size();
    for (int r = 0; r < ns; r++) bp_src.push_back(g.padded_offset(s) + r);
    for (int k = 0; k < kBpPad; k++) bp_src.push_back(-1);
  }
  // whole groups of 8 planes: the back projector swizzles within them
  while (bp_src.size() % 8) bp_src.push_back(-1);
  // no back-projection window may run past its segment's zero planes
  for (int y = 1; y < g.ny; y++)
    for (int gg = 0; gg < g.groupmax; gg++) {
      const size_t i = (size_t)y * g.groupmax + gg;
      const int zs = g.bl_zsa[i], ze = g.bl_zea[i], d = g.bl_yra[i] - g.bl_zsa[i];
      const int yb = g.yr_bottom[2 * gg + 2], yt = g.yr_top[2 * gg + 2];
      if (ze < zs) return bail(fail(ctx, HRRT_ERR_ARG, "bp: empty plane range"));
      const int z_lo = (zs / kBpZ) * kBpZ, z_hi = (ze / kBpZ) * kBpZ + kBpZ - 1;
      if (z_lo + d < yb - kBpPad || z_hi + d + 1 > yt + kBpPad) return bail(fail(ctx, HRRT_ERR_ARG, "bp: padding"));
    }
  // forward-projection task lists of every plane variant (one task per
  // consumer thread, two producer warps at least); the default variant must
  // fit, the others are offered to the tuner where they do
  std::vector<FpTask> vtasks[3];
  for (int i = 0; i < 3; i++) {
    vtasks[i] = build_fp_tasks(g, kFpPlaneVariants[i]);
    std::string vm = validate_fp(g, mid, vtasks[i], kFpPlaneVariants[i]);
    if (vm.empty() && ((int)vtasks[i].size() + 31) / 32 + 2 > kFpVariantWarps[i])
      vm = "fp: too many projection tasks for one CTA";
    if (!vm.empty()) {
      if (kFpPlaneVariants[i] == kFpPlanes) m = vm;
      vtasks[i].clear();
    }
  }
  if (!m.empty()) return bail(fail(ctx, HRRT_ERR_ARG, m));
  if (g.groupmax > kFpMaxGroups)
    return bail(fail(ctx, HRRT_ERR_ARG, "fp: more segment groups than the projector stages per row"));
  if (g.zp % kBpZ != 0) return bail(fail(ctx, HRRT_ERR_ARG, "padded z must be a multiple of 8"));
  for (int x = 1; x <= g.c; x++)
    if (g.cyl0[x] != g.cyl1[x] && g.cyl0[x] < 1) return bail(fail(ctx, HRRT_ERR_ARG, "FOV reaches the grid edge"));
  if ((size_t)bp_src.size() * 16 > 200 * 1024)
    return bail(fail(ctx, HRRT_ERR_ARG, "sinogram quad exceeds shared memory"));

  DevGeom &d = ctx->dg;
  d.nx = g.nx;
  d.nz = g.nz;
  d.zp = g.zp;
  d.c = g.c;
  d.nseg = g.nseg;
  d.groupmax = g.groupmax;
  d.zshift = g.zshift;
  d.segmentsize = g.segmentsize;
  d.pplanes = g.padded_planes();
  d.nviews = g.nviews;
  d.nquads = nq;
  d.fov_columns = (int)fovxy.size();
  d.z_min = g.sp.z_min;
  d.z_max = g.sp.z_max;
  d.y_size = g.y_size;
  d.eps1 = g.sp.epsilon1;
  d.eps3 = g.sp.epsilon3;
  d.image_max = g.sp.image_max;
  d.unit = 1.0f;
  d.cyl0 = dupload(ctx, g.cyl0, &e);
  d.cyl1 = dupload(ctx, g.cyl1, &e);
  d.ybot = dupload(ctx, g.yr_bottom, &e);
  d.ytop = dupload(ctx, g.yr_top, &e);
  d.poff = dupload(ctx, poff, &e);
  d.rescale = dupload(ctx, g.rescale, &e);
  d.bp_scale = dupload(ctx, g.bp_scale, &e);
  d.fpmid = dupload(ctx, mid, &e);
  std::vector<int2> flzf(g.fl_zzi.size());
  for (size_t i = 0; i < flzf.size(); i++) {
    int bits;
    std::memcpy(&bits, &g.fl_zzz0[i], 4);
    flzf[i] = make_int2(g.fl_zzi[i], bits);
  }
  d.fl_zf = dupload(ctx, flzf, &e);
  // the same two tables with the row fastest, for the exact adjoint
  {
    std::vector<FpMid> mt(mid.size());
    for (int y = 0; y < g.c; y++)
      for (int gg = 0; gg < g.groupmax; gg++) mt[(size_t)gg * g.c + y] = mid[(size_t)y * g.groupmax + gg];
    d.fpmid_t = dupload(ctx, mt, &e);
    std::vector<int2> ft(flzf.size());
    for (int y = 0; y < g.ny; y++)
      for (int i = 0; i < FS; i++) ft[(size_t)i * g.ny + y] = flzf[(size_t)y * FS + i];
    d.fl_t = dupload(ctx, ft, &e);
    // per (group, row y < c): the planes the end-plane entries of rows y and
    // N - y touch (each entry z reaches z and z + 1), bottom end and top end
    std::vector<int4> endr((size_t)g.groupmax * g.c, make_int4(1 << 30, -1, 1 << 30, -1));
    for (int y = 1; y < g.c; y++)
      for (int gg = 0; gg < g.groupmax; gg++) {
        int4 &r = endr[(size_t)gg * g.c + y];
        for (int i = 0; i < 2 * g.zshift; i++)
          for (const int row : {y, g.ny - y}) {
            const int z = g.fl_zzi[(size_t)row * FS + gg * 2 * g.zshift + i];
            if (i < g.zshift) {
              r.x = std::min(r.x, z);
              r.y = std::max(r.y, z + 1);
            } else {
              r.z = std::min(r.z, z);
              r.w = std::max(r.w, z + 1);
            }
          }
      }
    d.adj_endr = dupload(ctx, endr, &e);
    // the exact adjoint's rotate tables, rebuilt for each subset's pairs
    d.adj_pairs = ctx->npairs;
    d.adj_ent = dalloc<int2>(ctx, (size_t)ctx->npairs * g.nx * g.nx * kAdjCover, &e);
    d.adj_cnt = d.adj_ent ? dalloc<int>(ctx, (size_t)ctx->npairs * g.nx * g.nx, &e) : nullptr;
  }
  d.bplut = dupload(ctx, bpl, &e);
  d.sin_psi = dupload(ctx, g.sin_psi, &e);
  d.cos_psi = dupload(ctx, g.cos_psi, &e);
  d.fov_xy = dupload(ctx, fovxy, &e);
  for (int i = 0; i < 3; i++) {
    if (vtasks[i].empty()) continue;
    ctx->d_fptasks[i] = dupload(ctx, vtasks[i], &e);
    ctx->nfptasks[i] = (int)vtasks[i].size();
    if (kFpPlaneVariants[i] == kFpPlanes) {
      d.fptasks = ctx->d_fptasks[i];
      d.nfptasks = ctx->nfptasks[i];
    }
  }
  d.plane_seg = dupload(ctx, plane_seg, &e);
  std::vector<int16_t> pplane_seg(g.padded_planes(), -1);
  for (int s = 0; s < g.nseg; s++)
    for (int r = 0; r <= g.yr_top[s] - g.yr_bottom[s]; r++) pplane_seg[g.padded_offset(s) + r] = (int16_t)s;
  d.pplane_seg = dupload(ctx, pplane_seg, &e);
  d.bp_soff = dupload(ctx, bp_soff, &e);
  d.bp_src = dupload(ctx, bp_src, &e);
  d.bp_splanes = (int)bp_src.size();
  ctx->d_rowstart = dupload(ctx, rowstart, &e);
  d.err = dalloc<int>(ctx, 1, &e);
  d.range_err = dalloc<int>(ctx, 1, &e);
  ctx->nzmask = g.norm_zero_mask;
  ctx->d_nzmask = dupload(ctx, ctx->nzmask, &e);
  d.nzmask = ctx->d_nzmask;
  if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "table upload"));
  float2 *rp = dalloc<float2>(ctx, (size_t)(g.nviews / 2) * d.fov_columns, &e);
  if (!rp) return bail(cuda_fail(ctx, e, "rotpos"));
  d.rotpos = rp;
  e = launch_rotpos(d, rp, ctx->d_rowstart, ctx->stream);
  if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "rotpos kernel"));

  // image, sensitivity, scratch
  ctx->d_image = dalloc<float>(ctx, ctx->vol, &e);
  ctx->d_nfinv = ctx->d_image ? dalloc<float>(ctx, (size_t)g.sp.subsets * ctx->vol, &e) : nullptr;
  ctx->d_ratio = ctx->d_nfinv ? dalloc<float>(ctx, (size_t)ctx->npairs * ctx->quad_pair, &e) : nullptr;
  ctx->d_bc = ctx->d_ratio ? dalloc<float>(ctx, (size_t)ctx->npairs * ctx->vol, &e) : nullptr;
  ctx->d_br = ctx->d_bc ? dalloc<float>(ctx, (size_t)ctx->npairs * ctx->vol, &e) : nullptr;
  const int pb = post_iteration_blocks(d);
  ctx->d_partial = ctx->d_br ? dalloc<double>(ctx, pb, &e) : nullptr;
  ctx->d_sum = ctx->d_partial ? dalloc<double>(ctx, 1, &e) : nullptr;
  if (!ctx->d_sum) return bail(fail(ctx, HRRT_ERR_NOMEM, std::string("device allocation: ") + cudaGetErrorString(e)));
  // the adjoint runs with segment weights of 1 (its rows carry the forward
  // projector's own scaling)
  ctx->dg_adj = d;
  ctx->dg_adj.bp_scale = dupload(ctx, std::vector<float>(g.nseg, 1.0f), &e);
  ctx->d_view1 = dalloc<int>(ctx, 1, &e);
  if (!ctx->dg_adj.bp_scale || !ctx->d_view1) return bail(cuda_fail(ctx, e, "adjoint tables"));
  int rc = build_work_lists(ctx);
  if (rc) return bail(rc);
  e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "create"));
  *out = ctx;
  return HRRT_OK;
}

void hrrt_ctx_destroy(hrrt_ctx *ctx) {
  if (!ctx) return;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->batch) detach_batch(ctx->batch);
  delete ctx;
}

int hrrt_get_info(const hrrt_ctx *ctx, hrrt_info *info) {
  if (!ctx || !info) return HRRT_ERR_ARG;
  const Geometry &g = ctx->geo;
  info->nx = g.nx;
  info->ny = g.ny;
  info->nz = g.nz;
  info->zp = g.zp;
  info->nbins = g.nbins;
  info->nviews = g.nviews;
  info->nseg = g.nseg;
  info->groupmax = g.groupmax;
  info->segmentsize = g.segmentsize;
  info->subsets = g.sp.subsets;
  info->sviews = g.sviews;
  info->fov_columns = g.fov_columns;
  info->sino_elems = (long long)g.segmentsize * g.nviews * g.nbins;
  info->image_elems = (long long)g.nx * g.ny * g.zp;
  return HRRT_OK;
}

int hrrt_upload_inputs(hrrt_ctx *ctx, const int16_t *prompts, const float *randoms, const float *norm,
                       const float *atten, const float *scatter, int storage) {
  if (!ctx) return HRRT_ERR_ARG;
  if (!prompts || !randoms) return fail(ctx, HRRT_ERR_ARG, "prompts and randoms are required");
  if (storage < HRRT_STORE_F32 || storage > HRRT_STORE_F16) return fail(ctx, HRRT_ERR_ARG, "unknown storage");
  if (ctx->batch) return fail(ctx, HRRT_ERR_STATE, "the context serves a batch (hrrt_batch_destroy first)");
  if (int rc = ensure_input_buffers(ctx, storage)) return rc;
  if (int rc = upload_flat(ctx, prompts, randoms, norm, atten, scatter, storage, false, ctx->q_prompts, ctx->q_add,
                           ctx->q_mult))
    return rc;
  int rc = build_work_lists(ctx);
  if (rc) return rc;
  ctx->have_inputs = true;
  ctx->have_sens = false;
  return HRRT_OK;
}

int hrrt_sensitivity(hrrt_ctx *ctx) {
  if (!ctx) return HRRT_ERR_ARG;
  if (!ctx->have_inputs) return fail(ctx, HRRT_ERR_STATE, "hrrt_upload_inputs must come first");
  const Geometry &g = ctx->geo;
  for (int s = 0; s < g.sp.subsets; s++)
    if (int rc = sens_subset(ctx, s)) return rc;
  CK(cudaStreamSynchronize(ctx->stream), "sensitivity");
  ctx->have_sens = true;
  return HRRT_OK;
}

int hrrt_init_image(hrrt_ctx *ctx, const float *image_zyx) {
  if (!ctx) return HRRT_ERR_ARG;
  const Geometry &g = ctx->geo;
  if (!image_zyx) {
    CK(launch_init_image(ctx->dg, ctx->d_image, ctx->stream), "init_image");
  } else {
    // Init_Image with -i (drv:3970-3995): image[y][x][z] = file[z][y][x]
    // restricted to FOV columns; the [z][y][x] file is read as tmp[x][y]
    std::vector<float> h((size_t)ctx->vol, 0.f);
    for (int z = 0; z < g.nz; z++)
      for (int x = 0; x < g.nx; x++)
        for (int y = g.cyl0[x]; y < g.cyl1[x]; y++)
          h[((size_t)y * g.ny + x) * g.zp + z] = image_zyx[((size_t)z * g.nx + x) * g.ny + y];
    CK(cudaMemcpyAsync(ctx->d_image, h.data(), h.size() * 4, cudaMemcpyHostToDevice, ctx->stream), "init_image");
  }
  CK(cudaStreamSynchronize(ctx->stream), "init_image");
  ctx->have_image = true;
  ctx->subsets_done = 0;
  return HRRT_OK;
}

int hrrt_osem_subsets(hrrt_ctx *ctx, int first, int count) {
  if (!ctx || count < 0) return HRRT_ERR_ARG;
  if (!ctx->have_inputs || !ctx->have_sens || !ctx->have_image)
    return fail(ctx, HRRT_ERR_STATE, "inputs, sensitivity and image must be set first");
  const int S = ctx->geo.sp.subsets;
  for (int i = 0; i < count; i++) {
    const int s = ctx->geo.order[(size_t)(((first + i) % S) + S) % S];
    int rc = run_subset(ctx, s, ctx_bufs(ctx));
    if (rc) return rc;
  }
  return HRRT_OK;
}

int hrrt_osem(hrrt_ctx *ctx, int iterations, hrrt_stats *stats) {
  if (!ctx || iterations < 0) return HRRT_ERR_ARG;
  if (!ctx->have_inputs || !ctx->have_sens || !ctx->have_image)
    return fail(ctx, HRRT_ERR_STATE, "inputs, sensitivity and image must be set first");
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a), "event");
  CK(cudaEventCreate(&b), "event");
  cudaEventRecord(a, ctx->stream);
  double sum = 0.0;
  int done = 0;
  for (int it = 0; it < iterations; it++) {
    for (int i = 0; i < ctx->geo.sp.subsets; i++) {
      int rc = run_subset(ctx, ctx->geo.order[i], ctx_bufs(ctx));
      if (rc) {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        return rc;
      }
      done++;
    }
    {
      Launch L(ctx, "post_iter_kernel");
      CK(launch_post_iteration(ctx->dg, ctx->d_image, ctx->d_partial, ctx->d_sum, one_frame(), ctx->stream), "post_iteration");
    }
  }
  cudaEventRecord(b, ctx->stream);
  CK(cudaEventSynchronize(b), "osem");
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (iterations > 0) CK(cudaMemcpy(&sum, ctx->d_sum, sizeof(double), cudaMemcpyDeviceToHost), "sum");
  if (int rc = device_status(ctx)) return rc;
  if (stats) {
    stats->sum_image = sum;
    stats->subset_iterations = done;
    stats->ms_total = ms;
  }
  return HRRT_OK;
}

// Each subset's strided copies (1 KB rows) are dealt out over kCopyStreams
// streams: measured on B200 for the span-3 reconstruction with the projectors
// running, 271 ms with one stream, 267 with two, 262 with four.
#ifndef HRRT_COPY_STREAMS
#define HRRT_COPY_STREAMS 4
#endif
constexpr int kCopyStreams = HRRT_COPY_STREAMS;  // 1..4
static_assert(kCopyStreams >= 1 && kCopyStreams <= 4, "copy streams");

int hrrt_reconstruct(hrrt_ctx *ctx, const int16_t *prompts, const float *randoms, const float *norm,
                     const float *atten, const float *scatter, int storage, const float *init_image_zyx,
                     int iterations, float *image_zyx, hrrt_stats *stats) {
  if (!ctx) return HRRT_ERR_ARG;
  if (!prompts || !randoms || !image_zyx || iterations < 1)
    return fail(ctx, HRRT_ERR_ARG, "prompts, randoms, an output image and iterations >= 1 are required");
  if (storage < HRRT_STORE_F32 || storage > HRRT_STORE_F16) return fail(ctx, HRRT_ERR_ARG, "unknown storage");
  if (ctx->batch) return fail(ctx, HRRT_ERR_STATE, "the context serves a batch (hrrt_batch_destroy first)");
  const Geometry &g = ctx->geo;
  if (int rc = ensure_input_buffers(ctx, storage)) return rc;
  // pair-major staging of one subset's view pairs (the four float inputs),
  // two buffers
  const float *srcs[4] = {randoms, norm, atten, scatter};
  const size_t P = g.segmentsize, N = g.nbins, V = g.nviews;
  const size_t pair_elems = 2 * P * N, set_elems = (size_t)ctx->npairs * pair_elems;
  const size_t need = set_elems * 4 * sizeof(float);
  cudaError_t e = cudaSuccess;
  if (ctx->pstage_bytes < need) {
    for (int b = 0; b < 2; b++)
      if (ctx->pstage[b]) {
        cudaFree(ctx->pstage[b]);
        ctx->allocs.erase(std::find(ctx->allocs.begin(), ctx->allocs.end(), (void *)ctx->pstage[b]));
        ctx->pstage[b] = nullptr;
      }
    ctx->pstage_bytes = 0;
    for (int b = 0; b < 2; b++) {
      ctx->pstage[b] = dalloc<char>(ctx, need, &e);
      if (!ctx->pstage[b]) return fail(ctx, HRRT_ERR_NOMEM, "reconstruct staging");
    }
    ctx->pstage_bytes = need;
  }
  // The prompts go up whole, in one contiguous copy at the full link rate,
  // and the prep reads each subset's rows from there: a view's row of int16
  // prompts is only 512 bytes, short enough to slow a strided host copy.
  const size_t pelems = P * V * N;
  if (ctx->pflat_elems < pelems) {
    if (ctx->pflat) {
      cudaFree(ctx->pflat);
      ctx->allocs.erase(std::find(ctx->allocs.begin(), ctx->allocs.end(), (void *)ctx->pflat));
      ctx->pflat = nullptr;
    }
    ctx->pflat_elems = 0;
    ctx->pflat = dalloc<int16_t>(ctx, pelems, &e);
    if (!ctx->pflat) return fail(ctx, HRRT_ERR_NOMEM, "reconstruct prompts");
    ctx->pflat_elems = pelems;
  }
  if (!ctx->copy_stream) {
    CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking), "copy stream");
    for (int b = 0; b < 2; b++) {
      CK(cudaEventCreateWithFlags(&ctx->ev_copied[b], cudaEventDisableTiming), "event");
      CK(cudaEventCreateWithFlags(&ctx->ev_free[b], cudaEventDisableTiming), "event");
    }
  }
  // the norm-zero mask is not known until every pair is prepared: the first
  // iteration projects every FOV quad (a masked quad's prompts are zero, so
  // its ratio is zero, and the back projector skips it by the mask)
  std::fill(ctx->nzmask.begin(), ctx->nzmask.end(), (int16_t)1);
  if (int rc = build_work_lists(ctx)) return rc;
  if (int rc = hrrt_init_image(ctx, init_image_zyx)) return rc;
  CK(cudaMemsetAsync(ctx->d_mask_accum, 0, sizeof(int) * (size_t)(g.nviews / 2) * ctx->dg.nquads, ctx->stream),
     "reconstruct");
  cudaEvent_t ta, tb;
  CK(cudaEventCreate(&ta), "event");
  CK(cudaEventCreate(&tb), "event");
  auto bail = [&](int rc) {
    cudaStreamSynchronize(ctx->copy_stream);
    for (int i = 0; i < 3; i++)
      if (ctx->copy_side[i]) cudaStreamSynchronize(ctx->copy_side[i]);
    cudaStreamSynchronize(ctx->stream);
    cudaEventDestroy(ta);
    cudaEventDestroy(tb);
    return rc;
  };
  cudaEventRecord(ta, ctx->stream);
  for (int b = 0; b < 2; b++) CK(cudaEventRecord(ctx->ev_free[b], ctx->stream), "reconstruct");
  // ahead of every subset's copies on the copy stream, so each subset's
  // ev_copied also covers it
  CK(cudaMemcpyAsync(ctx->pflat, prompts, sizeof(int16_t) * pelems, cudaMemcpyHostToDevice, ctx->copy_stream),
     "reconstruct prompts");
  const int S = g.sp.subsets;
  // a subset's strided copies are dealt out over kCopyStreams streams
  cudaStream_t cst[kCopyStreams];
  cst[0] = ctx->copy_stream;
  for (int i = 1; i < kCopyStreams; i++) {
    if (!ctx->copy_side[i - 1]) {
      CK(cudaStreamCreateWithFlags(&ctx->copy_side[i - 1], cudaStreamNonBlocking), "copy stream");
      for (int b = 0; b < 2; b++)
        CK(cudaEventCreateWithFlags(&ctx->ev_side[i - 1][b], cudaEventDisableTiming), "event");
    }
    cst[i] = ctx->copy_side[i - 1];
  }
  for (int k = 0; k < S; k++) {
    const int s = g.order[k], b = k & 1;
    float *stg[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int c = 0; c < kCopyStreams && e == cudaSuccess; c++) e = cudaStreamWaitEvent(cst[c], ctx->ev_free[b], 0);
    int nc = 0;
    for (int j = 0; j < ctx->npairs && e == cudaSuccess; j++) {
      const int v = g.vieworder[(size_t)s * g.sviews + j];
      for (int h = 0; h < 2 && e == cudaSuccess; h++) {
        const size_t view = v + h * (V / 2), doff = j * pair_elems + h * P * N;
        for (int i = 0; i < 4 && e == cudaSuccess; i++) {
          if (!srcs[i]) continue;
          stg[i] = reinterpret_cast<float *>(ctx->pstage[b] + (size_t)i * set_elems * sizeof(float));
          e = cudaMemcpy2DAsync(stg[i] + doff, N * sizeof(float), srcs[i] + view * N, V * N * sizeof(float),
                                N * sizeof(float), P, cudaMemcpyHostToDevice, cst[nc++ % kCopyStreams]);
        }
      }
    }
    for (int c = 1; c < kCopyStreams && e == cudaSuccess; c++) {
      e = cudaEventRecord(ctx->ev_side[c - 1][b], cst[c]);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_side[c - 1][b], 0);
    }
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_copied[b], ctx->copy_stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream, ctx->ev_copied[b], 0);
    if (e == cudaSuccess) {
      Launch L(ctx, "prep_kernel");
      e = launch_prep_pairs(ctx->dg, g.nbins, ctx->pflat, stg[0], stg[1], stg[2], stg[3], g.sp.npskip,
                            g.sp.epsilon2, storage, ctx->q_prompts, ctx->q_add, ctx->q_mult, ctx->d_mask_accum,
                            ctx->d_pair_views + (size_t)s * ctx->npairs, ctx->npairs, ctx->stream, true);
    }
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_free[b], ctx->stream);
    if (e == cudaSuccess) e = launch_finish_mask(ctx->dg, ctx->d_mask_accum, ctx->d_nzmask, ctx->stream);
    if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "reconstruct upload"));
    if (int rc = sens_subset(ctx, s)) return bail(rc);
    if (int rc = run_subset(ctx, s, ctx_bufs(ctx))) return bail(rc);
  }
  {
    Launch L(ctx, "post_iter_kernel");
    e = launch_post_iteration(ctx->dg, ctx->d_image, ctx->d_partial, ctx->d_sum, one_frame(), ctx->stream);
    if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "post_iteration"));
  }
  // the mask is complete: the remaining iterations skip masked quads
  e = cudaMemcpyAsync(ctx->nzmask.data(), ctx->d_nzmask, ctx->nzmask.size() * sizeof(int16_t),
                      cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "reconstruct"));
  if (storage == HRRT_STORE_F16)
    if (int rc = range_status(ctx)) return bail(rc);
  if (int rc = build_work_lists(ctx)) return bail(rc);
  ctx->have_inputs = ctx->have_sens = ctx->have_image = true;
  int done = S;
  for (int it = 1; it < iterations; it++) {
    for (int i = 0; i < S; i++, done++)
      if (int rc = run_subset(ctx, g.order[i], ctx_bufs(ctx))) return bail(rc);
    Launch L(ctx, "post_iter_kernel");
    e = launch_post_iteration(ctx->dg, ctx->d_image, ctx->d_partial, ctx->d_sum, one_frame(), ctx->stream);
    if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "post_iteration"));
  }
  double sum = 0.0;
  e = launch_image_zyx(ctx->dg, ctx->d_image, ctx->d_tmp_img ? ctx->d_tmp_img : ctx->d_bc, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(image_zyx, ctx->d_tmp_img ? ctx->d_tmp_img : ctx->d_bc,
                        sizeof(float) * (size_t)g.nz * g.ny * g.nx, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&sum, ctx->d_sum, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaEventRecord(tb, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "reconstruct"));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ta, tb);
  cudaEventDestroy(ta);
  cudaEventDestroy(tb);
  if (int rc = device_status(ctx)) return rc;
  if (stats) {
    stats->sum_image = sum;
    stats->subset_iterations = done;
    stats->ms_total = ms;
  }
  return HRRT_OK;
}

int hrrt_get_image(hrrt_ctx *ctx, float *image_zyx) {
  if (!ctx || !image_zyx) return HRRT_ERR_ARG;
  const Geometry &g = ctx->geo;
  // SaveImage (drv:4020-4043): tmpimage[z][y][x] = image[x][y][z] on FOV
  // columns, transposed on the device
  cudaError_t e = cudaSuccess;
  if (!ctx->d_tmp_img) ctx->d_tmp_img = dalloc<float>(ctx, ctx->vol, &e);
  if (!ctx->d_tmp_img) return fail(ctx, HRRT_ERR_NOMEM, "scratch");
  CK(launch_image_zyx(ctx->dg, ctx->d_image, ctx->d_tmp_img, ctx->stream), "get_image");
  CK(cudaMemcpyAsync(image_zyx, ctx->d_tmp_img, sizeof(float) * (size_t)g.nz * g.ny * g.nx, cudaMemcpyDeviceToHost,
                     ctx->stream),
     "get_image");
  CK(cudaStreamSynchronize(ctx->stream), "get_image");
  return HRRT_OK;
}

int hrrt_get_image_xyz(hrrt_ctx *ctx, float *image_xyz) {
  if (!ctx || !image_xyz) return HRRT_ERR_ARG;
  CK(cudaMemcpyAsync(image_xyz, ctx->d_image, ctx->vol * 4, cudaMemcpyDeviceToHost, ctx->stream), "get_image");
  CK(cudaStreamSynchronize(ctx->stream), "get_image");
  return HRRT_OK;
}

int hrrt_set_image_xyz(hrrt_ctx *ctx, const float *image_xyz) {
  if (!ctx || !image_xyz) return HRRT_ERR_ARG;
  CK(cudaMemcpyAsync(ctx->d_image, image_xyz, ctx->vol * 4, cudaMemcpyHostToDevice, ctx->stream), "set_image");
  CK(cudaStreamSynchronize(ctx->stream), "set_image");
  ctx->have_image = true;
  ctx->subsets_done = 0;
  return HRRT_OK;
}

int hrrt_get_sensitivity(hrrt_ctx *ctx, int subset, float *nf_inv_xyz) {
  if (!ctx || !nf_inv_xyz || subset < 0 || subset >= ctx->geo.sp.subsets) return HRRT_ERR_ARG;
  if (!ctx->have_sens) return fail(ctx, HRRT_ERR_STATE, "no sensitivity");
  CK(cudaMemcpyAsync(nf_inv_xyz, ctx->d_nfinv + (size_t)subset * ctx->vol, ctx->vol * 4, cudaMemcpyDeviceToHost,
                     ctx->stream),
     "get_sensitivity");
  CK(cudaStreamSynchronize(ctx->stream), "get_sensitivity");
  return HRRT_OK;
}

int hrrt_get_norm_zero_mask(hrrt_ctx *ctx, int16_t *mask) {
  if (!ctx || !mask) return HRRT_ERR_ARG;
  std::memcpy(mask, ctx->nzmask.data(), ctx->nzmask.size() * sizeof(int16_t));
  return HRRT_OK;
}

int hrrt_set_norm_zero_mask(hrrt_ctx *ctx, const int16_t *mask) {
  if (!ctx || !mask) return HRRT_ERR_ARG;
  std::memcpy(ctx->nzmask.data(), mask, ctx->nzmask.size() * sizeof(int16_t));
  CK(cudaMemcpyAsync(ctx->d_nzmask, ctx->nzmask.data(), ctx->nzmask.size() * 2, cudaMemcpyHostToDevice, ctx->stream),
     "mask");
  CK(cudaStreamSynchronize(ctx->stream), "mask");
  return build_work_lists(ctx);
}

int hrrt_fp_pair(hrrt_ctx *ctx, const float *image_xyz, int view, float *prj) {
  if (!ctx || !image_xyz || !prj) return HRRT_ERR_ARG;
  const Geometry &g = ctx->geo;
  if (view < 0 || view >= g.nviews / 2) return fail(ctx, HRRT_ERR_ARG, "view must be < nviews/2");
  cudaError_t e = cudaSuccess;
  const size_t rows = (size_t)2 * g.segmentsize * g.nbins;
  if (!ctx->d_tmp_img) ctx->d_tmp_img = dalloc<float>(ctx, ctx->vol, &e);
  if (!ctx->d_rows) ctx->d_rows = ctx->d_tmp_img ? dalloc<float>(ctx, rows, &e) : nullptr;
  if (!ctx->d_rows) return fail(ctx, HRRT_ERR_NOMEM, "scratch");
  std::vector<QuadWork> work;
  const int nq = g.nx / 2 + 1;
  for (int x = 1; x <= g.c; x++)
    if (g.cyl0[x] != g.cyl1[x] && ctx->nzmask[(size_t)view * nq + x] != 0)
      work.push_back(QuadWork{0, (int16_t)x, (int16_t)view, 0});
  QuadWork *dw = dupload(ctx, work, &e);
  if (!dw) return cuda_fail(ctx, e, "work");
  CK(cudaMemcpyAsync(ctx->d_tmp_img, image_xyz, ctx->vol * 4, cudaMemcpyHostToDevice, ctx->stream), "fp_pair");
  CK(cudaMemcpyAsync(ctx->d_rows, prj, rows * 4, cudaMemcpyHostToDevice, ctx->stream), "fp_pair");
  {
    Launch L(ctx, "fp_kernel");
    CK(launch_fp(ctx->dg, ctx->d_tmp_img, dw, (int)work.size(), 0, nullptr, nullptr, 0, ctx->d_ratio, ctx->quad_pair, ctx->tune, one_frame(), ctx->stream),
       "fp_kernel");
  }
  CK(launch_quad_to_rows(ctx->dg, g.nbins, ctx->d_ratio, dw, (int)work.size(), ctx->d_rows, ctx->stream), "unpack");
  CK(cudaMemcpyAsync(prj, ctx->d_rows, rows * 4, cudaMemcpyDeviceToHost, ctx->stream), "fp_pair");
  CK(cudaStreamSynchronize(ctx->stream), "fp_pair");
  cudaFree(dw);
  ctx->allocs.erase(std::find(ctx->allocs.begin(), ctx->allocs.end(), (void *)dw));
  return device_status(ctx);
}
int hrrt_forward_project(hrrt_ctx *ctx, const float *image_xyz, float *sino) {
  if (!ctx || !image_xyz || !sino) return HRRT_ERR_ARG;
  const Geometry &g = ctx->geo;
  cudaError_t e = cudaSuccess;
  if (!ctx->d_tmp_img) ctx->d_tmp_img = dalloc<float>(ctx, ctx->vol, &e);
  if (!ctx->d_tmp_img) return fail(ctx, HRRT_ERR_NOMEM, "scratch");
  const size_t n = (size_t)g.segmentsize * g.nviews * g.nbins;
  float *dsino = nullptr;
  e = cudaMalloc(&dsino, n * sizeof(float));
  if (e != cudaSuccess) return fail(ctx, HRRT_ERR_NOMEM, "sinogram");
  QuadWork *dw = nullptr;
  auto done = [&](int rc) {
    cudaStreamSynchronize(ctx->stream);
    cudaFree(dsino);
    if (dw) cudaFree(dw);
    return rc;
  };
  e = cudaMemsetAsync(dsino, 0, n * sizeof(float), ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ctx->d_tmp_img, image_xyz, ctx->vol * 4, cudaMemcpyHostToDevice, ctx->stream);
  // every active quad of every view pair, in batches of npairs pairs
  const int nq = g.nx / 2 + 1, V2 = g.nviews / 2;
  std::vector<QuadWork> work;
  std::vector<int> off;
  for (int b = 0; b < V2; b += ctx->npairs) {
    off.push_back((int)work.size());
    for (int x = 1; x <= g.c; x++)
      for (int k = 0; k < ctx->npairs && b + k < V2; k++)
        if (g.cyl0[x] != g.cyl1[x] && ctx->nzmask[(size_t)(b + k) * nq + x] != 0)
          work.push_back(QuadWork{(int16_t)k, (int16_t)x, (int16_t)(b + k), 0});
  }
  off.push_back((int)work.size());
  if (e == cudaSuccess) e = cudaMalloc(&dw, work.size() * sizeof(QuadWork) + 16);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dw, work.data(), work.size() * sizeof(QuadWork), cudaMemcpyHostToDevice, ctx->stream);
  for (size_t b = 0; b + 1 < off.size() && e == cudaSuccess; b++) {
    const int cnt = off[b + 1] - off[b];
    {
      Launch L(ctx, "fp_kernel");
      e = launch_fp(ctx->dg, ctx->d_tmp_img, dw + off[b], cnt, 0, nullptr, nullptr, 0, ctx->d_ratio, ctx->quad_pair, ctx->tune, one_frame(), ctx->stream);
    }
    if (e == cudaSuccess)
      e = launch_quad_to_file(ctx->dg, g.nbins, ctx->d_ratio, ctx->quad_pair, dw + off[b], cnt, dsino, ctx->stream);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(sino, dsino, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return done(cuda_fail(ctx, e, "forward_project"));
  return done(device_status(ctx));
}

long long hrrt_psf_kernel(float fwhm1, float fwhm2, float ratio, float pixel_size, float *taps, int capacity) {
  const std::vector<float> k = psf_taps(fwhm1, fwhm2, ratio, pixel_size);
  if (k.empty()) return HRRT_ERR_ARG;
  if (taps && capacity >= (int)k.size()) std::memcpy(taps, k.data(), k.size() * sizeof(float));
  return (long long)k.size();
}

int hrrt_set_psf(hrrt_ctx *ctx, int enable, float fwhm1, float fwhm2, float ratio) {
  if (!ctx) return HRRT_ERR_ARG;
  if (ctx->batch && enable) return fail(ctx, HRRT_ERR_STATE, "PSF: not available while the context serves a batch");
  const Geometry &g = ctx->geo;
  if (!enable) {
    if (ctx->psf_on) {
      ctx->psf_on = false;
      ctx->have_sens = false;
      ctx->config_epoch++;
    }
    return HRRT_OK;
  }
  const std::vector<float> kx = psf_taps(fwhm1, fwhm2, ratio, g.x_size), ky = psf_taps(fwhm1, fwhm2, ratio, g.y_size),
                           kz = psf_taps(fwhm1, fwhm2, ratio, g.z_size);
  if (kx.empty() || ky.empty() || kz.empty()) return fail(ctx, HRRT_ERR_ARG, "PSF: fwhm1 must be >= 0");
  if (kx.size() != ky.size()) return fail(ctx, HRRT_ERR_ARG, "PSF: x and y kernels differ in size");
  // convolveyz's z tap sums (psf.cpp:397-416): loop bound and index both use
  // the y kernel's half width; the sums cover planes [z_min, z_max)
  const int h = (int)(ky.size() - 1) / 2;
  std::vector<float> kzp(std::max(kz.size(), ky.size()), 0.f);
  std::copy(kz.begin(), kz.end(), kzp.begin());
  std::vector<float> normz(g.zp, 0.f);
  for (int mask = -h; mask < h; mask++)
    for (int z = 0; z < g.zp; z++) {
      const int m2 = z + mask;
      if (m2 < g.sp.z_min || m2 >= g.sp.z_max) continue;
      normz[z] += kzp[mask + h];
    }
  for (int z = 0; z < g.zp; z++)
    if (normz[z] > 0) normz[z] = 1 / normz[z];
  cudaError_t e = cudaSuccess;
  for (float **p : {&ctx->d_psf_fx, &ctx->d_psf_fy, &ctx->d_psf_normz})
    if (*p) {
      cudaFree(*p);
      ctx->allocs.erase(std::find(ctx->allocs.begin(), ctx->allocs.end(), (void *)*p));
      *p = nullptr;
    }
  ctx->d_psf_fx = dupload(ctx, kx, &e);
  ctx->d_psf_fy = dupload(ctx, ky, &e);
  ctx->d_psf_normz = dupload(ctx, normz, &e);
  if (!ctx->d_image_psf) ctx->d_image_psf = dalloc<float>(ctx, ctx->vol, &e);
  if (!ctx->d_corr) ctx->d_corr = dalloc<float>(ctx, ctx->vol, &e);
  if (!ctx->d_psf_tmp) ctx->d_psf_tmp = dalloc<float>(ctx, ctx->vol, &e);
  if (!ctx->d_psf_fx || !ctx->d_psf_fy || !ctx->d_psf_normz || !ctx->d_image_psf || !ctx->d_corr || !ctx->d_psf_tmp)
    return fail(ctx, HRRT_ERR_NOMEM, "PSF buffers");
  CK(cudaStreamSynchronize(ctx->stream), "psf");
  ctx->psf_h = h;
  ctx->psf_on = true;
  ctx->have_sens = false;
  ctx->config_epoch++;
  return HRRT_OK;
}

int hrrt_psf_convolve(hrrt_ctx *ctx, const float *image_xyz, float *out_xyz) {
  if (!ctx || !image_xyz || !out_xyz) return HRRT_ERR_ARG;
  if (!ctx->psf_on) return fail(ctx, HRRT_ERR_STATE, "hrrt_set_psf must come first");
  cudaError_t e = cudaSuccess;
  if (!ctx->d_tmp_img) ctx->d_tmp_img = dalloc<float>(ctx, ctx->vol, &e);
  if (!ctx->d_tmp_img) return fail(ctx, HRRT_ERR_NOMEM, "scratch");
  CK(cudaMemcpyAsync(ctx->d_tmp_img, image_xyz, sizeof(float) * ctx->vol, cudaMemcpyHostToDevice, ctx->stream),
     "psf");
  CK(cudaMemsetAsync(ctx->d_corr, 0, sizeof(float) * ctx->vol, ctx->stream), "psf");
  if (int rc = run_psf(ctx, ctx->d_tmp_img, ctx->d_corr)) return rc;
  CK(cudaMemcpyAsync(out_xyz, ctx->d_corr, sizeof(float) * ctx->vol, cudaMemcpyDeviceToHost, ctx->stream), "psf");
  CK(cudaStreamSynchronize(ctx->stream), "psf");
  return HRRT_OK;
}

int hrrt_set_map(hrrt_ctx *ctx, int technique, float beta, int first_subset) {
  if (!ctx) return HRRT_ERR_ARG;
  // -b technique,beta (hrrt_osem3d.cpp:3360-3369): either 0 turns MAP off
  if (technique == 0 || beta == 0.f) {
    ctx->map_on = false;
    return HRRT_OK;
  }
  if (technique != 1)
    return fail(ctx, HRRT_ERR_ARG,
                "MAP: technique 1 only (technique 2 needs an MR image, and its voxel loop in dpfcalc.c:245 "
                "tests the wrong counter)");
  if (first_subset < 0) return fail(ctx, HRRT_ERR_ARG, "MAP: first subset must be >= 0");
  if (ctx->batch) return fail(ctx, HRRT_ERR_STATE, "MAP: not available while the context serves a batch");
  cudaError_t e = cudaSuccess;
  if (!ctx->d_corr) ctx->d_corr = dalloc<float>(ctx, ctx->vol, &e);
  if (!ctx->d_dpf) {
    ctx->d_dpf = dalloc<float>(ctx, ctx->vol, &e);
    // the prior is written on FOV columns only; the rest stays 0
    if (ctx->d_dpf) CK(cudaMemsetAsync(ctx->d_dpf, 0, sizeof(float) * ctx->vol, ctx->stream), "map");
  }
  if (!ctx->d_mapmax) ctx->d_mapmax = dalloc<unsigned int>(ctx, 1, &e);
  if (!ctx->d_corr || !ctx->d_dpf || !ctx->d_mapmax) return fail(ctx, HRRT_ERR_NOMEM, "MAP buffers");
  CK(cudaStreamSynchronize(ctx->stream), "map");
  ctx->map_on = true;
  ctx->map_beta = beta;
  ctx->map_first = first_subset;
  return HRRT_OK;
}

int hrrt_map_prior(hrrt_ctx *ctx, const float *image_xyz, float *prior_xyz) {
  if (!ctx || !image_xyz || !prior_xyz) return HRRT_ERR_ARG;
  if (!ctx->map_on) return fail(ctx, HRRT_ERR_STATE, "hrrt_set_map must come first");
  cudaError_t e = cudaSuccess;
  if (!ctx->d_tmp_img) ctx->d_tmp_img = dalloc<float>(ctx, ctx->vol, &e);
  if (!ctx->d_tmp_img) return fail(ctx, HRRT_ERR_NOMEM, "scratch");
  CK(cudaMemcpyAsync(ctx->d_tmp_img, image_xyz, sizeof(float) * ctx->vol, cudaMemcpyHostToDevice, ctx->stream),
     "map prior");
  {
    Launch L(ctx, "map_dpf_kernel");
    CK(launch_map_prior(ctx->dg, ctx->d_tmp_img, ctx->d_mapmax, ctx->d_dpf, ctx->stream), "map prior");
  }
  CK(cudaMemcpyAsync(prior_xyz, ctx->d_dpf, sizeof(float) * ctx->vol, cudaMemcpyDeviceToHost, ctx->stream),
     "map prior");
  CK(cudaStreamSynchronize(ctx->stream), "map prior");
  return HRRT_OK;
}

int hrrt_set_backprojector(hrrt_ctx *ctx, int mode) {
  if (!ctx) return HRRT_ERR_ARG;
  if (mode != HRRT_BP_REF && mode != HRRT_BP_ADJOINT) return fail(ctx, HRRT_ERR_ARG, "unknown back projector");
  if (mode != ctx->bp_mode) {
    ctx->have_sens = false;
    ctx->config_epoch++;
  }
  ctx->bp_mode = mode;
  return HRRT_OK;
}

int hrrt_bp_pair(hrrt_ctx *ctx, const float *prj, int view, float *imagebuf_xyz, int mode) {
  if (!ctx || !prj || !imagebuf_xyz) return HRRT_ERR_ARG;
  if (mode != HRRT_BP_REF && mode != HRRT_BP_ADJOINT) return fail(ctx, HRRT_ERR_ARG, "unknown back projector");
  const Geometry &g = ctx->geo;
  if (view < 0 || view >= g.nviews / 2) return fail(ctx, HRRT_ERR_ARG, "view must be < nviews/2");
  cudaError_t e = cudaSuccess;
  const size_t rows = (size_t)2 * g.segmentsize * g.nbins;
  if (!ctx->d_tmp_img) ctx->d_tmp_img = dalloc<float>(ctx, ctx->vol, &e);
  if (!ctx->d_rows) ctx->d_rows = ctx->d_tmp_img ? dalloc<float>(ctx, rows, &e) : nullptr;
  if (!ctx->d_rows) return fail(ctx, HRRT_ERR_NOMEM, "scratch");
  std::vector<QuadWork> work;
  for (int x = 1; x <= g.c; x++)
    if (g.cyl0[x] != g.cyl1[x]) work.push_back(QuadWork{0, (int16_t)x, (int16_t)view, 0});
  QuadWork *dw = dupload(ctx, work, &e);
  if (!dw) return cuda_fail(ctx, e, "work");
  CK(cudaMemcpyAsync(ctx->d_rows, prj, rows * 4, cudaMemcpyHostToDevice, ctx->stream), "bp_pair");
  CK(cudaMemsetAsync(ctx->d_ratio, 0, ctx->quad_pair * 4, ctx->stream), "bp_pair");
  if (mode == HRRT_BP_ADJOINT) {
    CK(launch_rows_to_quad(ctx->dg, g.nbins, ctx->d_rows, ctx->d_ratio, 0, ctx->stream), "pack");
    CK(cudaMemsetAsync(ctx->d_bc, 0, ctx->vol * 4, ctx->stream), "bp_pair");
    CK(cudaMemsetAsync(ctx->d_br, 0, ctx->vol * 4, ctx->stream), "bp_pair");
    {
      Launch L(ctx, "adj_kernel");
      CK(launch_adj(ctx->dg, ctx->d_ratio, ctx->quad_pair, dw, (int)work.size(), ctx->d_bc, ctx->d_br, ctx->vol, one_frame(),
                    ctx->stream),
         "adj_kernel");
    }
    CK(cudaMemsetAsync(ctx->d_tmp_img, 0, ctx->vol * 4, ctx->stream), "bp_pair");
    CK(cudaMemcpyAsync(ctx->d_view1, &view, sizeof(int), cudaMemcpyHostToDevice, ctx->stream), "bp_pair");
    CK(cudaStreamSynchronize(ctx->stream), "bp_pair");
    {
      Launch L(ctx, "adj_rotate_kernel");
      CK(launch_adj_rotate(ctx->dg, ctx->d_view1, 1, ctx->d_bc, ctx->d_br, ctx->vol, nullptr, nullptr,
                           ctx->d_tmp_img, 2, one_frame(), ctx->stream),
         "adj_rotate_kernel");
    }
    CK(cudaMemcpyAsync(imagebuf_xyz, ctx->d_tmp_img, ctx->vol * 4, cudaMemcpyDeviceToHost, ctx->stream), "bp_pair");
    CK(cudaStreamSynchronize(ctx->stream), "bp_pair");
    cudaFree(dw);
    ctx->allocs.erase(std::find(ctx->allocs.begin(), ctx->allocs.end(), (void *)dw));
    return device_status(ctx);
  }
  CK(launch_rows_to_quad(ctx->dg, g.nbins, ctx->d_rows, ctx->d_ratio, 1, ctx->stream), "pack");
  {
    Launch L(ctx, "bp_kernel");
    CK(launch_bp(ctx->dg, ctx->d_ratio, ctx->quad_pair, dw, (int)work.size(), ctx->d_bc, ctx->d_br, ctx->vol, ctx->tune, one_frame(),
                 ctx->stream),
       "bp_kernel");
  }
  CK(launch_add_partials(ctx->dg, ctx->d_bc, ctx->d_br, ctx->d_tmp_img, ctx->stream), "add");
  CK(cudaMemcpyAsync(imagebuf_xyz, ctx->d_tmp_img, ctx->vol * 4, cudaMemcpyDeviceToHost, ctx->stream), "bp_pair");
  CK(cudaStreamSynchronize(ctx->stream), "bp_pair");
  cudaFree(dw);
  ctx->allocs.erase(std::find(ctx->allocs.begin(), ctx->allocs.end(), (void *)dw));
  return HRRT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Back projection without allocation.
//
// Some callers cannot allocate device memory while they run: an acquisition
// loop that must not stall on cudaMalloc's implicit device synchronisation, or
// a host application that hands this library a fixed memory budget at
// start-up and forbids allocations after it.  hrrt_bp_pair_noalloc serves
// them.  It runs the reference back projector (the result of hrrt_bp_pair
// with HRRT_BP_REF, whatever back projector the context has selected).  Its
// only scratch -- the quad-layout copy of the input sinogram rows, scaled by
// the back projector's segment weights -- lives in the static device array
// below, so the call itself never allocates; the input rows and the output
// buffer are the caller's.
//
// The array is kNoAllocScratchBytes (16 MiB: the quad layout of an HRRT span-3
// view pair is 13.3 MB).  Every GPU on which the library is loaded holds it
// until the process exits.  The first call on a device looks up the array's
// device address there (cudaGetSymbolAddress), once.  All calls share the
// array and it keeps the last call's contents, so each call clears it first,
// and calls that overlap on the GPU (other streams, other host threads) race
// with each other.
// ---------------------------------------------------------------------------
constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchBytes / sizeof(float)];

namespace {
// device address of g_noalloc_scratch, resolved once per device (the host
// symbol is only a stand-in for it)
std::mutex g_noalloc_mu;
std::map<int, float *> g_noalloc_ptr;

cudaError_t noalloc_scratch(float **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  auto it = g_noalloc_ptr.find(dev);
  if (it != g_noalloc_ptr.end()) {
    *out = it->second;
    return cudaSuccess;
  }
  float *p = nullptr;
  e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
  if (e != cudaSuccess) return e;
  g_noalloc_ptr[dev] = p;
  *out = p;
  return cudaSuccess;
}
// the body of hrrt_bp_pair_noalloc, with ctx->device current
int noalloc_bp(hrrt_ctx *ctx, const float *d_prj, int view, float *d_imagebuf, void *stream, size_t need) {
  const Geometry &g = ctx->geo;
  float *scratch = nullptr;
  CK(noalloc_scratch(&scratch), "hrrt_bp_pair_noalloc: cudaGetSymbolAddress");
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  int x0 = 0, x1 = -1;  // the FOV quads are one run of x
  for (int x = 1; x <= g.c; x++)
    if (g.cyl0[x] != g.cyl1[x]) {
      if (x0 == 0) x0 = x;
      x1 = x;
    }
  // the segment pads of the quad layout must read as zero; the output
  // collects two atomically added partial sums per voxel
  CK(cudaMemsetAsync(scratch, 0, need, st), "hrrt_bp_pair_noalloc: clear scratch");
  CK(cudaMemsetAsync(d_imagebuf, 0, (size_t)ctx->vol * sizeof(float), st), "hrrt_bp_pair_noalloc: clear output");
  CK(launch_rows_to_quad(ctx->dg, g.nbins, d_prj, scratch, 1, st), "hrrt_bp_pair_noalloc: pack");
  CK(launch_bp_sum(ctx->dg, scratch, view, x0, x1 - x0 + 1, d_imagebuf, st), "hrrt_bp_pair_noalloc: bp");
  return HRRT_OK;
}
}  // namespace

extern "C" {

int hrrt_bp_pair_noalloc(hrrt_ctx *ctx, const float *d_prj, int view, float *d_imagebuf, void *stream) {
  if (!ctx || !d_prj || !d_imagebuf) return HRRT_ERR_ARG;
  const Geometry &g = ctx->geo;
  if (view < 0 || view >= g.nviews / 2) return fail(ctx, HRRT_ERR_ARG, "view must be < nviews/2");
  const size_t need = (size_t)ctx->quad_pair * sizeof(float);
  if (need > kNoAllocScratchBytes)
    return fail(ctx, HRRT_ERR_ARG,
                "hrrt_bp_pair_noalloc: this geometry needs " + std::to_string(need) +
                    " bytes of scratch; the static scratch holds " + std::to_string(kNoAllocScratchBytes));
  // the work runs on the context's device; the caller's current device is
  // put back on every return
  int caller_dev = -1;
  CK(cudaGetDevice(&caller_dev), "hrrt_bp_pair_noalloc: cudaGetDevice");
  if (caller_dev != ctx->device) CK(cudaSetDevice(ctx->device), "hrrt_bp_pair_noalloc: cudaSetDevice");
  const int rc = noalloc_bp(ctx, d_prj, view, d_imagebuf, stream, need);
  if (caller_dev != ctx->device) {
    const cudaError_t e = cudaSetDevice(caller_dev);
    if (e != cudaSuccess && rc == HRRT_OK) return cuda_fail(ctx, e, "hrrt_bp_pair_noalloc: restore the device");
  }
  return rc;
}

int hrrt_rotate_add(hrrt_ctx *ctx, const float *imagebuf_xyz, int view, float *corr_xyz) {
  if (!ctx || !imagebuf_xyz || !corr_xyz) return HRRT_ERR_ARG;
  const Geometry &g = ctx->geo;
  if (view < 0 || view >= g.nviews / 2) return fail(ctx, HRRT_ERR_ARG, "view must be < nviews/2");
  cudaError_t e = cudaSuccess;
  if (!ctx->d_tmp_img) ctx->d_tmp_img = dalloc<float>(ctx, ctx->vol, &e);
  if (!ctx->d_tmp_img) return fail(ctx, HRRT_ERR_NOMEM, "scratch");
  int *dv = dupload(ctx, std::vector<int>{view}, &e);
  if (!dv) return cuda_fail(ctx, e, "view");
  // corr in d_bc[1], imagebuf in d_bc[0]
  CK(cudaMemcpyAsync(ctx->d_bc, imagebuf_xyz, ctx->vol * 4, cudaMemcpyHostToDevice, ctx->stream), "rotate");
  CK(cudaMemcpyAsync(ctx->d_tmp_img, corr_xyz, ctx->vol * 4, cudaMemcpyHostToDevice, ctx->stream), "rotate");
  {
    Launch L(ctx, "rotback_kernel");
    CK(launch_rotback(ctx->dg, dv, 1, ctx->d_bc, nullptr, ctx->vol, nullptr, nullptr, ctx->d_tmp_img, 2, one_frame(), ctx->stream),
       "rotback");
  }
  CK(cudaMemcpyAsync(corr_xyz, ctx->d_tmp_img, ctx->vol * 4, cudaMemcpyDeviceToHost, ctx->stream), "rotate");
  CK(cudaStreamSynchronize(ctx->stream), "rotate");
  cudaFree(dv);
  ctx->allocs.erase(std::find(ctx->allocs.begin(), ctx->allocs.end(), (void *)dv));
  return HRRT_OK;
}

long long hrrt_geometry_table(const hrrt_geom *gp, const char *name, void *out, size_t bytes) {
  if (!gp || !name) return HRRT_ERR_ARG;
  ScannerParams p;
  p.nrings = gp->nrings;
  p.nelements = gp->nelements;
  p.nangles = gp->nangles;
  p.ring_radius = gp->ring_radius;
  p.plane_sep = gp->plane_sep;
  p.binsize = gp->binsize;
  p.span = gp->span;
  p.maxdel = gp->maxdel;
  p.subsets = gp->subsets;
  p.rel_fov = gp->rel_fov;
  Geometry g;
  if (!g.build(p).empty()) return HRRT_ERR_ARG;
  std::vector<char> buf;
  auto put = [&](const void *src, size_t n) {
    const char *c = (const char *)src;
    buf.insert(buf.end(), c, c + n);
  };
  const std::string n(name);
  if (n == "cylwiny") {
    for (int y = 0; y < g.ny; y++) {
      put(&g.cyl0[y], 2);
      put(&g.cyl1[y], 2);
    }
  } else if (n == "segments") {
    put(g.yr_bottom.data(), 4 * g.nseg);
    put(g.yr_top.data(), 4 * g.nseg);
    put(g.segment_offset.data(), 4 * g.nseg);
  } else if (n == "sin_theta") put(g.sin_theta.data(), 4 * g.nseg);
  else if (n == "cos_theta") put(g.cos_theta.data(), 4 * g.nseg);
  else if (n == "sin_psi") put(g.sin_psi.data(), 4 * g.nviews);
  else if (n == "cos_psi") put(g.cos_psi.data(), 4 * g.nviews);
  else if (n == "tantheta") put(g.tantheta.data(), 4 * g.tantheta.size());
  else if (n == "rescale") put(g.rescale.data(), 4 * g.rescale.size());
  else if (n == "flookup_zzi") put(g.fl_zzi.data(), 4 * g.fl_zzi.size());
  else if (n == "flookup_zzz0") put(g.fl_zzz0.data(), 4 * g.fl_zzz0.size());
  else if (n == "blookup") {
    for (size_t i = 0; i < g.bl_zsa.size(); i++) {
      put(&g.bl_zsa[i], 4);
      put(&g.bl_zea[i], 4);
      put(&g.bl_yra[i], 4);
    }
  } else if (n == "blookup_yr2a") put(g.bl_yr2a.data(), 4 * g.bl_yr2a.size());
  else if (n == "bp_scale") put(g.bp_scale.data(), 4 * g.bp_scale.size());
  else if (n == "order") put(g.order.data(), 2 * g.order.size());
  else return HRRT_ERR_ARG;
  if (out && bytes >= buf.size()) std::memcpy(out, buf.data(), buf.size());
  return (long long)buf.size();
}

int hrrt_set_profiling(hrrt_ctx *ctx, int enable) {
  if (!ctx) return HRRT_ERR_ARG;
  ctx->prof = enable != 0;
  return HRRT_OK;
}

int hrrt_kernel_stats(hrrt_ctx *ctx, const char *kernel, int *launches, double *total_ms) {
  if (!ctx || !kernel) return HRRT_ERR_ARG;
  drain_timers(ctx);
  auto it = ctx->kstats.find(kernel);
  if (launches) *launches = it == ctx->kstats.end() ? 0 : it->second.first;
  if (total_ms) *total_ms = it == ctx->kstats.end() ? 0.0 : it->second.second;
  return HRRT_OK;
}

int hrrt_reset_kernel_stats(hrrt_ctx *ctx) {
  if (!ctx) return HRRT_ERR_ARG;
  drain_timers(ctx);
  ctx->kstats.clear();
  return HRRT_OK;
}

}  // extern "C"
