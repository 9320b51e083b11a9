// kernels.cu -- sm_100a kernels of the hrrt_osem3d OSEM hot path.
//
// Compiled with -fmad=false: the reference (x86-64 SSE2 build) never fuses a
// multiply with an add, and every expression below keeps the reference's
// association, so the forward projector, the rotate-back and the update are
// bit-identical to the reference on the same inputs.
#include "kernels.cuh"

#include <cuda.h>  // CUtensorMap (the encoder is reached through the runtime's driver entry point)

#include <cfloat>
#include <cstring>
#include <type_traits>

namespace hrrt {

namespace {

__device__ __forceinline__ float4 f4(float v) { return make_float4(v, v, v, v); }
__device__ __forceinline__ float4 operator+(float4 a, float4 b) {
  return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
__device__ __forceinline__ float4 operator*(float4 a, float s) {
  return make_float4(a.x * s, a.y * s, a.z * s, a.w * s);
}
__device__ __forceinline__ float lane(const float4 &v, int l) {
  return l == 0 ? v.x : (l == 1 ? v.y : (l == 2 ? v.z : v.w));
}

// ---- storage-type helpers for the sinogram inputs ----
struct P4 { float v[4]; };
__device__ __forceinline__ P4 load_p4(const int16_t *p, size_t i) {
  const short4 s = reinterpret_cast<const short4 *>(p)[i];
  return P4{{(float)s.x, (float)s.y, (float)s.z, (float)s.w}};
}
__device__ __forceinline__ P4 load_p4(const __half *p, size_t i) {
  const uint2 u = reinterpret_cast<const uint2 *>(p)[i];
  const __half2 a = *reinterpret_cast<const __half2 *>(&u.x);
  const __half2 b = *reinterpret_cast<const __half2 *>(&u.y);
  return P4{{__low2float(a), __high2float(a), __low2float(b), __high2float(b)}};
}
__device__ __forceinline__ P4 load_p4(const float *p, size_t i) {
  const float4 f = reinterpret_cast<const float4 *>(p)[i];
  return P4{{f.x, f.y, f.z, f.w}};
}
__device__ __forceinline__ P4 load_p4(const __nv_bfloat16 *p, size_t i) {
  const uint2 u = reinterpret_cast<const uint2 *>(p)[i];
  const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162 *>(&u.x);
  const __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162 *>(&u.y);
  return P4{{__low2float(a), __high2float(a), __low2float(b), __high2float(b)}};
}
__device__ __forceinline__ void store_p4(int16_t *p, size_t i, const float *v) {
  reinterpret_cast<short4 *>(p)[i] = make_short4((short)v[0], (short)v[1], (short)v[2], (short)v[3]);
}
__device__ __forceinline__ void store_p4(__half *p, size_t i, const float *v) {
  __half2 a = __floats2half2_rn(v[0], v[1]), b = __floats2half2_rn(v[2], v[3]);
  uint2 u;
  u.x = *reinterpret_cast<uint32_t *>(&a);
  u.y = *reinterpret_cast<uint32_t *>(&b);
  reinterpret_cast<uint2 *>(p)[i] = u;
}
__device__ __forceinline__ void store_p4(float *p, size_t i, const float *v) {
  reinterpret_cast<float4 *>(p)[i] = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void store_p4(__nv_bfloat16 *p, size_t i, const float *v) {
  __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]), b = __floats2bfloat162_rn(v[2], v[3]);
  uint2 u;
  u.x = *reinterpret_cast<uint32_t *>(&a);
  u.y = *reinterpret_cast<uint32_t *>(&b);
  reinterpret_cast<uint2 *>(p)[i] = u;
}



// ---- packed pairs of IEEE single-precision values (sm_100 f32x2) ----
// Each op is element-wise round-to-nearest, exactly the scalar add/sub/mul of
// the reference, two values per instruction.  A quad value (4 lanes) is two
// pairs: lanes (0,1) and (2,3).
struct Q2 {
  uint64_t lo, hi;
};
__device__ __forceinline__ uint64_t pk(float a, float b) {
  uint64_t r;
  asm("mov.b64 %0, {%1,%2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float2 upk(uint64_t v) {
  float2 r;
  asm("mov.b64 {%0,%1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
  return r;
}
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
// a + p where p is a packed product.  The code generator contracts a packed
// multiply that feeds a packed add into a fused multiply-add (which rounds once
// instead of twice), even with -fmad=false and explicit .rn, and folds a
// multiply by a literal 1 away; a packed fused multiply-add of p by a run-time
// (1, 1) and a cannot absorb p's multiply and rounds p + a once, as the
// reference's add does (measured bit-identical on B200; two scalar adds, the
// alternative, cost one more instruction per pair).
__device__ __forceinline__ uint64_t addp(uint64_t a, uint64_t p, uint64_t one) {
  uint64_t r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(p), "l"(one), "l"(a));
  return r;
}
__device__ __forceinline__ Q2 ldq(const float4 *p) {
  const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(p);
  return Q2{v.x, v.y};
}
__device__ __forceinline__ Q2 qadd(Q2 a, Q2 b) { return Q2{add2(a.lo, b.lo), add2(a.hi, b.hi)}; }
__device__ __forceinline__ Q2 qmul(Q2 a, uint64_t s) { return Q2{mul2(a.lo, s), mul2(a.hi, s)}; }
__device__ __forceinline__ Q2 qaddp(Q2 a, Q2 p, uint64_t one) { return Q2{addp(a.lo, p.lo, one), addp(a.hi, p.hi, one)}; }
// packed a * b + c (one rounding), where no reference rounding order is to
// be kept: the back projector (held to the reference within 2e-6, its sums
// being incremental there and direct here) and the exact adjoint (held to
// the FP64 oracle)
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
__device__ __forceinline__ Q2 qfma(Q2 a, uint64_t b, Q2 c) { return Q2{fma2(a.lo, b, c.lo), fma2(a.hi, b, c.hi)}; }
__device__ __forceinline__ float4 q2f(Q2 q) {
  const float2 a = upk(q.lo), b = upk(q.hi);
  return make_float4(a.x, a.y, b.x, b.y);
}

// ---- TMA bulk copies + mbarrier (sm_90+ async proxy) ----
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// one box of a 4-D tensor (coordinates innermost first) into shared memory,
// completing on the mbarrier; the map is a __grid_constant__ kernel parameter
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
// bounded wait on an mbarrier phase; on timeout records the error and returns false
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err) {
  const uint32_t a = smem_u32(bar);
  for (int i = 0; i < (1 << 22); i++) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  if (err) atomicExch(err, 1);
  return false;
}

// Rotated-grid sample point (sbrt:1866-1871): position of rotated-frame voxel
// (a,b) in the image, as flat column index of its (ix,iy) corner and the four
// bilinear weights.  base < 0: outside (the reference zeroes that sample).
struct SamplePt {
  int base;
  float c0, c1, c2, c3;
};
__device__ __forceinline__ SamplePt sample_point(int a, int b, int c, int N, int zp, float cosv, float sinv) {
  SamplePt s;
  const float fa = (float)(a - c), fb = (float)(b - c), fc = (float)c;
  const float xx0 = fa * cosv - fb * sinv + fc;
  const float yy0 = fa * sinv + fb * cosv + fc;
  const float lim = (float)(N - 2);
  // the reference tests xx0 against the upper limit twice and never yy0
  if (xx0 < 0 || xx0 > lim || yy0 < 0 || xx0 > lim) {
    s.base = -1;
    s.c0 = s.c1 = s.c2 = s.c3 = 0.f;
    return s;
  }
  const int ix = (int)xx0, iy = (int)yy0;
  const float x1 = xx0 - ix, y1 = yy0 - iy;
  s.c0 = (1 - x1) * (1 - y1);
  s.c1 = x1 * (1 - y1);
  s.c2 = y1 * (1 - x1);
  s.c3 = y1 * x1;
  // contiguous [x][y][zp] addressing, as the reference's matrix3dm128 image
  if ((ix + 1) * N + iy + 1 >= N * N) {
    s.base = -1;
    return s;
  }
  s.base = (ix * N + iy) * zp;
  return s;
}
__device__ __forceinline__ float bilinear(const float *__restrict__ img, const SamplePt &s, int N, int zp, int z) {
  if (s.base < 0) return 0.f;
  const float r1 = __ldg(img + s.base + z);
  const float r2 = __ldg(img + s.base + N * zp + z);
  const float r3 = __ldg(img + s.base + zp + z);
  const float r4 = __ldg(img + s.base + N * zp + zp + z);
  return (r1 * s.c0 + r2 * s.c1) + (r3 * s.c2 + r4 * s.c3);
}

// ============================================================================
// Forward projection (+ fused OP ratio), one CTA per (view pair, quad x).
// Restates forward_proj3d_view1_thread (sbrt:1728-1978) for one x: the eight
// symmetric rotated-grid columns at row y are sampled once into shared memory
// (pam: lanes (x,y),(N-x,y),(N-y,x),(N-y,N-x); pam2: (x,N-y),(N-x,N-y),(y,x),
// (y,N-x)), then every thread accumulates its own (segment, plane-run) outputs
// for all four lanes, row by row in the reference's order.
// The consumers are bound by instruction issue and shared-load latency (64
// registers a thread at 1024 threads), not by shared-memory bandwidth.
// Measured on B200 at span 3 and not used: rows staged as bf16 (half the
// shared bytes, plus the widening: 1.89 -> 1.89 ms), consumer warps split
// into two or three groups with a row-ready barrier each (2.12, 2.23 ms), and
// two CTAs per quad with half the tasks each, two CTAs or one of 128
// registers per SM (2.01, 3.27 ms).
// ============================================================================
// named barriers (id 0 is __syncthreads); ids are immediates so the kernel
// reserves only the barriers it uses
template <int ID>
__device__ __forceinline__ void bar_sync_id(int count) {
  asm volatile("bar.sync %0, %1;" ::"n"(ID), "r"(count) : "memory");
}
template <int ID>
__device__ __forceinline__ void bar_arrive_id(int count) {
  asm volatile("bar.arrive %0, %1;" ::"n"(ID), "r"(count) : "memory");
}
// named barriers with immediate ids (a register id reserves all 16)
__device__ __forceinline__ void bar_sync(int id, int count) {
  switch (id) {
    case 1: bar_sync_id<1>(count); break;
    case 2: bar_sync_id<2>(count); break;
    case 3: bar_sync_id<3>(count); break;
    case 4: bar_sync_id<4>(count); break;
    case 5: bar_sync_id<5>(count); break;
    case 6: bar_sync_id<6>(count); break;
    case 7: bar_sync_id<7>(count); break;
    case 8: bar_sync_id<8>(count); break;
    case 9: bar_sync_id<9>(count); break;
    case 10: bar_sync_id<10>(count); break;
    case 11: bar_sync_id<11>(count); break;
    case 12: bar_sync_id<12>(count); break;
    default: bar_sync_id<13>(count); break;
  }
}
__device__ __forceinline__ void bar_arrive(int id, int count) {
  switch (id) {
    case 1: bar_arrive_id<1>(count); break;
    case 2: bar_arrive_id<2>(count); break;
    case 3: bar_arrive_id<3>(count); break;
    case 4: bar_arrive_id<4>(count); break;
    case 5: bar_arrive_id<5>(count); break;
    case 6: bar_arrive_id<6>(count); break;
    case 7: bar_arrive_id<7>(count); break;
    case 8: bar_arrive_id<8>(count); break;
    case 9: bar_arrive_id<9>(count); break;
    case 10: bar_arrive_id<10>(count); break;
    case 11: bar_arrive_id<11>(count); break;
    default: bar_arrive_id<12>(count); break;
  }
}
constexpr int kBarFull = 1;                 // + slot: sampled row ready (producers arrive, consumers wait)
constexpr int kBarEmpty = 1 + kFpSlots;     // + slot: sampled row consumed (consumers arrive, producers wait)
constexpr int kBarProd = 1 + 2 * kFpSlots;  // producers only: corner slot read by every producer
static_assert(kBarProd <= 13, "named barrier ids");

template <int MODE, int PL, int MW, typename PT, typename AT>
__global__ void __launch_bounds__(MW * 32, 1) fp_kernel(DevGeom g, const float *__restrict__ image,
                                                     const QuadWork *__restrict__ work,
                                                     const PT *__restrict__ prompts, const AT *__restrict__ add,
                                                     float4 *__restrict__ out, long long out_pair_stride,
                                                     int nprod_warps, FrameStrides fr,
                                                     const __grid_constant__ CUtensorMap cols, int use_cols) {
  // shared memory: [S slots][8 points][2 column pairs][2*zp] staged corner
  // columns, 2*cpair zeros (the corners of outside points), [S slots][2 halves]
  // [ZS] sampled rows, [ZS] centre column (S = kFpSlots)
  const uint64_t one = pk(g.unit, g.unit);
  extern __shared__ __align__(128) float4 smem[];
  const int ZS = g.zp + kFpZPad;
  const int zp = g.zp;
  const int cpair = 2 * zp;  // floats per column pair
  float *corners = reinterpret_cast<float *>(smem);
  // the four corner columns of a point arrive as one box of the image's
  // tensor map where the map is there and the slots are 128-byte aligned
  const bool box4 = use_cols && (smem_u32(corners) & 127u) == 0;
  const int zoff = kFpSlots * 8 * 2 * cpair;
  float *zcol = corners + zoff;
  float4 *rows = smem + (size_t)(kFpSlots * 8 * 2 + 2) * cpair / 4;  // [S][2][ZS]
  float4 *cen = rows + 2 * kFpSlots * ZS;
  __shared__ ulonglong2 s_w[kFpSlots][4][2];
  __shared__ int s_off[kFpSlots][8];
  // each row's middle-plane sampling entries (z, f, z2, f2 per group),
  // copied in with the row's columns.  Twice as many slots as rows in flight:
  // the entries of row r + S arrive while the consumers may still read those
  // of rows r - S + 1 .. r.  (3 KB: two CTAs per SM still fit at span 9.)
  __shared__ __align__(16) FpMid s_mid[2 * kFpSlots][kFpMaxGroups];
  __shared__ __align__(8) uint64_t s_bar[kFpSlots];

  const int nwork = gridDim.x / fr.n, frame = blockIdx.x / nwork, item = blockIdx.x - frame * nwork;
  const QuadWork w = work[item];
  const int fs = fr.map ? __ldg(fr.map + frame) : frame;
  image += (size_t)fs * fr.image;
  out += (size_t)frame * fr.ratio / 4;
  if (MODE == 1) {
    prompts += (size_t)fs * fr.input;
    add += (size_t)fs * fr.input;
  }
  const int x = w.x, v = w.view;
  const int N = g.nx, c = g.c;
  const float cosv = g.cos_psi[v], sinv = g.sin_psi[v];
  const int ystart = g.cyl0[x];
  const int nrows = c - ystart;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int nprod = nprod_warps * 32;   // producer threads: [ncons, nthr)
  const int ncons = nthr - nprod;        // consumer threads: one task each
  const bool producer = tid >= ncons;
  const int ptid = tid - ncons;

  // TMA issue (producer lanes 0-7, one sample point each): the two contiguous
  // column pairs (ix, iy..iy+1) and (ix+1, iy..iy+1) of each inside point
  auto issue_row = [&](int r) {
    const int sl = r % kFpSlots, y = ystart + r, l = ptid;
    int a, b;
    switch (l) {
      case 0: a = x; b = y; break;
      case 1: a = N - x; b = y; break;
      case 2: a = N - y; b = x; break;
      case 3: a = N - y; b = N - x; break;
      case 4: a = x; b = N - y; break;
      case 5: a = N - x; b = N - y; break;
      case 6: a = y; b = x; break;
      default: a = y; b = N - x; break;
    }
    const SamplePt pt = sample_point(a, b, c, N, zp, cosv, sinv);
    const bool inside = pt.base >= 0;
    // weights packed per lane pair: s_w[slot][point/2] = {(c0,c0'),(c1,c1')},{(c2,c2'),(c3,c3')}
    float *wf = reinterpret_cast<float *>(&s_w[sl][l >> 1][0]);
    const int e = l & 1;
    wf[0 + e] = pt.c0;
    wf[2 + e] = pt.c1;
    wf[4 + e] = pt.c2;
    wf[6 + e] = pt.c3;
    // outside points read the zero column pairs
    s_off[sl][l] = inside ? (sl * 8 + l) * 2 * cpair : zoff;
    const unsigned m = __ballot_sync(0xffu, inside);
    const int G = g.groupmax, es = r % (2 * kFpSlots);
    if (l == 0) {
      fence_proxy_async();
      mbar_arrive_tx(&s_bar[sl], (uint32_t)__popc(m) * 2u * cpair * 4u + (uint32_t)G * 16u);
    }
    __syncwarp(0xffu);
    if (l == 0) bulk_g2s(&s_mid[es][0], g.fpmid + (size_t)y * G, (uint32_t)G * 16u, &s_bar[sl]);
    if (inside) {
      float *dst = corners + ((size_t)(sl * 8 + l) * 2) * cpair;
      const int ix = pt.base / (N * zp), iy = pt.base / zp - ix * N;
      if (box4 && iy + 1 < N) {
        // columns (ix, iy..iy+1) and (ix+1, iy..iy+1): box {zp, 2, 2} at
        // (0, iy, ix, stored frame), laid out as the two pairs below
        tma_load_4d(dst, &cols, 0, iy, ix, fs, &s_bar[sl]);
      } else {
        // the pair (ix, N-1..N) runs on into column (ix+1, 0) in the
        // contiguous image, as the reference's flat addressing reads it
        bulk_g2s(dst, image + pt.base, cpair * 4u, &s_bar[sl]);
        bulk_g2s(dst + cpair, image + pt.base + (size_t)N * zp, cpair * 4u, &s_bar[sl]);
      }
    }
  };

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < kFpSlots; s++) mbar_init(&s_bar[s], 1);
    fence_mbar_init();
  }
  for (int i = tid; i < (2 * kFpSlots + 1) * kFpZPad; i += nthr) {
    const int col = i / kFpZPad, k = i % kFpZPad;
    rows[col * ZS + zp + k] = f4(0.f);
  }
  for (int i = tid; i < 2 * cpair; i += nthr) zcol[i] = 0.f;
  __syncthreads();
  if (producer && ptid < 8) {
    for (int r = 0; r < kFpSlots && r < nrows; r++) issue_row(r);
  }

  // centre column y = c (sbrt:1815-1853): lanes (x,c),(N-x,c),(c,x),(c,N-x)
  {
    SamplePt cp[4];
#pragma unroll
    for (int l = 0; l < 4; l++) {
      const int a = (l == 0) ? x : (l == 1) ? N - x : c;
      const int b = (l == 0 || l == 1) ? c : (l == 2) ? x : N - x;
      cp[l] = sample_point(a, b, c, N, zp, cosv, sinv);
    }
    for (int z = tid; z < zp; z += nthr)
      cen[z] = make_float4(bilinear(image, cp[0], N, zp, z), bilinear(image, cp[1], N, zp, z),
                           bilinear(image, cp[2], N, zp, z), bilinear(image, cp[3], N, zp, z));
  }
  for (int z = zp + tid; z < ZS; z += nthr) cen[z] = f4(0.f);
  __syncthreads();

  bool timed_out = false;
  if (producer) {
    // ---------------- producers: bilinear samples, kFpSlots rows ahead ----------------
    const int hsplit = nprod / 2;
    const int h_mine = ptid >= hsplit, z_mine = ptid - h_mine * hsplit;
    for (int r = 0; r < nrows; r++) {
      const int sl = r % kFpSlots;
      if (!mbar_wait(&s_bar[sl], (uint32_t)((r / kFpSlots) & 1), g.err)) timed_out = true;
      if (r >= kFpSlots) bar_sync(kBarEmpty + sl, nthr);  // consumers are done with row r-S
      {
        // lanes (0,1) and (2,3) of this half share nothing but the plane: each
        // lane pair is evaluated with packed pairs, its weights pre-packed
        float4 *rw = rows + (size_t)sl * 2 * ZS + h_mine * ZS;
        for (int z = z_mine; z < zp; z += hsplit) {
          uint64_t vv[2];
#pragma unroll
          for (int pp = 0; pp < 2; pp++) {
            const int pt = h_mine * 4 + 2 * pp;
            const ulonglong2 wa = s_w[sl][pt >> 1][0], wb = s_w[sl][pt >> 1][1];
            const float *qa = corners + s_off[sl][pt], *qb = corners + s_off[sl][pt + 1];
            // corner order of the reference: r1 (ix,iy), r2 (ix+1,iy), r3 (ix,iy+1), r4 (ix+1,iy+1)
            const uint64_t r1 = pk(qa[z], qb[z]), r2 = pk(qa[cpair + z], qb[cpair + z]);
            const uint64_t r3 = pk(qa[zp + z], qb[zp + z]), r4 = pk(qa[cpair + zp + z], qb[cpair + zp + z]);
            vv[pp] = add2(addp(mul2(r1, wa.x), mul2(r2, wa.y), one), addp(mul2(r3, wb.x), mul2(r4, wb.y), one));
          }
          *reinterpret_cast<ulonglong2 *>(rw + z) = make_ulonglong2(vv[0], vv[1]);
        }
      }
      bar_arrive(kBarFull + sl, nthr);
      // every producer has finished reading corner slot sl: refill it with row r+S
      bar_sync(kBarProd, nprod);
      if (ptid < 8 && r + kFpSlots < nrows) issue_row(r + kFpSlots);
    }
    if (timed_out) {
      // results are void (the host reports the status word); give copies
      // still in flight a bounded chance to land before the CTA exits
      for (int r = max(0, nrows - kFpSlots); r < nrows; r++)
        mbar_wait(&s_bar[r % kFpSlots], (uint32_t)((r / kFpSlots) & 1), nullptr);
    }
    return;
  }

  // ---------------- consumers: one task (segment, plane run) each ----------------
  // accumulators start at the centre sample of their plane (the reference
  // assigns the centre column before accumulating rows y < c)
  Q2 acc[PL];
  const FpTask tk = (tid < g.nfptasks) ? g.fptasks[tid] : FpTask{0, 0, 0, -1};
  {
    const int zb = (tk.type < 0) ? 0 : g.ybot[tk.seg] + tk.p0;
#pragma unroll
    for (int j = 0; j < PL; j++) acc[j] = ldq(cen + min(zb + j, ZS - 1));
  }
  const int gg = (tk.seg + 1) / 2 - 1;
  const bool odd = tk.seg & 1;  // segment 2k-1: pam2 at z, pam at z2
  const int pofs = tk.p0 - g.zshift;
  const int gs = gg < 0 ? 0 : gg;
  const int ns_t = (tk.type < 0) ? 0 : g.ytop[tk.seg] - g.ybot[tk.seg] + 1;
  const int li0 = gg * 2 * g.zshift + ((tk.p0 < g.zshift) ? tk.p0 : tk.p0 - ns_t + 2 * g.zshift);
  const int FS = g.groupmax * 2 * g.zshift;
  for (int r = 0; r < nrows; r++) {
    const int sl = r % kFpSlots, es = r % (2 * kFpSlots), y = ystart + r;
    bar_sync(kBarFull + sl, nthr);
    const float4 *pam = rows + (size_t)sl * 2 * ZS;
    const float4 *pam2 = pam + ZS;
    if (tk.type == 0) {
      // theta = 0 (sbrt:1907-1910)
#pragma unroll
      for (int j = 0; j < PL; j++) acc[j] = qadd(acc[j], qadd(ldq(pam + tk.p0 + j), ldq(pam2 + tk.p0 + j)));
    } else if (tk.type > 0) {
      const FpMid m = s_mid[es][gs];
      if (m.z >= 0) {  // else the group is skipped for this row (sbrt:1923-1924)
        // segment 2k accumulates pam at z and pam2 at z2; segment 2k-1 the converse
        const float4 *A = odd ? pam2 : pam;
        const float4 *B = odd ? pam : pam2;
        if (tk.type == 1) {
          // middle planes: z, z2 advance with the plane (sbrt:1933-1947)
          const float4 *Aw = A + m.z + pofs, *Bw = B + m.z2 + pofs;
          const uint64_t f = pk(m.f, m.f), f2 = pk(m.f2, m.f2);
          Q2 a0 = ldq(Aw), b0 = ldq(Bw);
#pragma unroll
          for (int j = 0; j < PL; j++) {
            const Q2 a1 = ldq(Aw + j + 1), b1 = ldq(Bw + j + 1);
            acc[j] = qadd(acc[j], qaddp(qmul(qadd(b1, a0), f2), qmul(qadd(a1, b0), f), one));
            a0 = a1;
            b0 = b1;
          }
        } else {
          // end planes: per-plane flookup entries (sbrt:1925-1931, :1948-1952)
          const int2 *fy = g.fl_zf + y * FS + li0, *fm = g.fl_zf + (N - y) * FS + li0;
#pragma unroll
          for (int j = 0; j < kFpEndPlanes; j++) {
            if (j < tk.n) {
              const int2 e1 = __ldg(fy + j), e2 = __ldg(fm + j);
              const int z = e1.x, z2 = e2.x;
              const float f = __int_as_float(e1.y), f2 = __int_as_float(e2.y);
              const uint64_t ff = pk(f, f), ff2 = pk(f2, f2);
              acc[j] = qadd(acc[j], qaddp(qmul(qadd(ldq(B + z2 + 1), ldq(A + z)), ff2),
                                          qmul(qadd(ldq(A + z + 1), ldq(B + z2)), ff), one));
            }
          }
        }
      }
    }
    if (r + kFpSlots < nrows) bar_arrive(kBarEmpty + sl, nthr);
  }

  // scale (sbrt:1953-1975), then either store the estimate or the OP ratio
  // (pt_update_est_w3, drv:2474-2520) pre-multiplied by the back projector's
  // segment weight (sbrt:1637-1649)
  if (tk.type < 0) return;
  const size_t qbase = (size_t)x * g.pplanes;
  const int sg = tk.seg;
#pragma unroll
  for (int j = 0; j < PL; j++) {
    if (j >= tk.n) continue;
    const int r = tk.p0 + j, yr = g.ybot[sg] + r;
    const float sc = (sg == 0) ? g.y_size : g.rescale[gg * g.nz + yr];
    const float4 est = q2f(qmul(acc[j], pk(sc, sc)));
    const size_t qi = qbase + g.poff[sg] + r;
    if (MODE == 0) {
      out[(size_t)w.slot * out_pair_stride + qi] = est;
    } else {
      const size_t ii = (size_t)v * g.nquads * g.pplanes + qi;
      const P4 p = load_p4(prompts, ii);
      const P4 ad = load_p4(add, ii);
      const float bs = g.bp_scale[sg];
      float rr[4];
#pragma unroll
      for (int l = 0; l < 4; l++) {
        const float den = lane(est, l) + ad.v[l];
        float q;
        if (p.v[l] == 0.f) q = 0.f;
        else if (den > g.eps3) q = p.v[l] / den;
        else q = 1.0f;
        rr[l] = q * bs;
      }
      out[(size_t)w.slot * out_pair_stride + qi] = make_float4(rr[0], rr[1], rr[2], rr[3]);
    }
  }
}

// ============================================================================
// Back projection, one CTA per (view pair, quad x).  Voxel-driven restatement
// of back_proj3d_view_n1thread (sbrt:4162-4668): the quad's four sinogram
// lanes sit in shared memory; each thread evaluates, for its rotated-grid row
// y and a run of kBpZ planes, the two 4-lane sums the reference builds
// incrementally (sumt1 for voxels (x,y),(N-x,y),(N-y,x),(N-y,N-x); sumt2 for
// (x,N-y),(N-x,N-y),(y,x),(y,N-x)) as direct linear interpolations of the
// zero-padded sinogram at yr = z + d.  Each voxel receives two partial sums,
// one from the ray of view p (its column quad) and one from the ray of view
// p+nviews/2 (its row quad); they go to Bc and Br and are added in the
// rotate-back, which is the reference's assign-then-accumulate order.
// ============================================================================
// The shared planes are stored swizzled: plane i at bsw(i), its position
// within its aligned group of 8 XORed with the group's index.  Threads of a
// warp take consecutive 8-plane runs of one row, so their loads of the same
// window offset are 8 planes (128 bytes) apart; the swizzle puts them in
// different 16-byte bank groups without the shared memory a padding would
// cost.
__device__ __forceinline__ int bsw(int i) { return i ^ ((i >> 3) & 7); }

template <int KB>
__device__ __forceinline__ void bp_lerp(Q2 (&s)[KB], const float4 *__restrict__ P, int pbase, const BpLut &bl,
                                        int z0) {
  // windows wholly outside [zs, ze] contribute nothing; a window that
  // straddles an end reads the segment's zero planes for its outside planes
  if (z0 + KB - 1 < bl.zs || z0 > bl.ze) return;
  const int i0 = pbase + z0 + bl.d;
  // the reference's p[yr] + f*(p[yr+1]-p[yr]) (sbrt:4312-4315) as
  // (1-f) p[yr] + f p[yr+1], added with two fused multiply-adds
  const uint64_t f = pk(bl.f, bl.f), g = pk(1.0f - bl.f, 1.0f - bl.f);
  Q2 a = ldq(P + bsw(i0));
#pragma unroll
  for (int j = 0; j < KB; j++) {
    const Q2 b = ldq(P + bsw(i0 + j + 1));
    s[j] = qfma(b, f, qfma(a, g, s[j]));
    a = b;
  }
}

template <int KB, bool ACC = false>
__device__ __forceinline__ void store_lane(float *__restrict__ dst, const Q2 (&s)[KB], int l) {
  float v[KB];
#pragma unroll
  for (int j = 0; j < KB; j++) {
    const float2 t = upk(l < 2 ? s[j].lo : s[j].hi);
    v[j] = (l & 1) ? t.y : t.x;
  }
  if (ACC) {
#pragma unroll
    for (int j = 0; j < KB; j++) atomicAdd(dst + j, v[j]);
  } else if constexpr (KB == 8) {
    // one 32-byte store (sm_100): a whole sector per lane, one line touched
    // per row of the warp's task tile instead of two stores to each
    asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(dst), "f"(v[0]), "f"(v[1]), "f"(v[2]),
                 "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
                 : "memory");
  } else {
#pragma unroll
    for (int j = 0; j < KB; j += 4)
      *reinterpret_cast<float4 *>(dst + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
  }
}

template <int KB, bool ACC = false, bool MULTI = false, int NT = 256>
__global__ void __launch_bounds__(NT, NT >= 384 ? 2 : kBpMinBlocks) bp_kernel(DevGeom g, const float4 *__restrict__ in, long long in_pair_stride,
                                                 const QuadWork *__restrict__ work, float *__restrict__ bc,
                                                 float *__restrict__ br, long long vol, FrameStrides fr,
                                                 int view0, int x0, int rlog) {
  extern __shared__ float4 P[];  // [bp_splanes]: segments with kBpPad zero planes each side
  // ACC: one view pair, quads x0 + blockIdx.x, both partial sums added into bc
  // (each voxel receives exactly two terms, so the atomic adds onto a zeroed
  // buffer give a + b whatever their order)
  // MULTI: several frames per launch (one frame: the frame arithmetic is
  // compiled out, which keeps the single-frame kernel free of spills)
  int item = blockIdx.x;
  if (MULTI) {
    const int nwork = gridDim.x / fr.n, frame = blockIdx.x / nwork;
    item = blockIdx.x - frame * nwork;
    in += (size_t)frame * fr.ratio / 4;
    bc += (size_t)frame * fr.bc;
    br += (size_t)frame * fr.bc;
  }
  const QuadWork w = ACC ? QuadWork{0, (int16_t)(x0 + blockIdx.x), (int16_t)view0, 0} : work[item];
  const int x = w.x, N = g.nx, c = g.c, zp = g.zp, G = g.groupmax;
  const bool masked = g.nzmask[w.view * g.nquads + x] == 0;
  const float4 *src = in + (size_t)w.slot * in_pair_stride + (size_t)x * g.pplanes;
  if (!masked)
    for (int i = threadIdx.x; i < g.bp_splanes; i += blockDim.x) {
      const int q = __ldg(g.bp_src + i);
      P[bsw(i)] = (q >= 0) ? src[q] : f4(0.f);
    }
  __syncthreads();

  // ACC: both partial sums go through bc (br is unused and may be null), so
  // the two destinations derive from one restrict pointer
  float *bcp = bc + (size_t)w.slot * vol;
  float *brp = (ACC ? bc : br) + (size_t)w.slot * vol;
  const int ystart = g.cyl0[x];
  const int nyq = c - ystart + 1, nzc = zp / KB;
  const int o0 = g.bp_soff[0];
  // task = (half, row, plane run); half 0 builds sumt1 (voxels (x,y),(N-x,y),
  // (N-y,x),(N-y,N-x)), half 1 sumt2 (voxels (x,N-y),(N-x,N-y),(y,x),(y,N-x)).
  // A warp's 32 tasks are a tile of R = 2^rlog consecutive plane runs of
  // 32/R consecutive rows.  Along the runs a warp's stores of a voxel column
  // are contiguous, and the swizzle spreads its shared loads over the banks;
  // along the rows the row entries differ, but windows at the same planes
  // and a slowly varying offset d(y) often coincide (broadcast).  Many
  // segment groups favour few runs, few groups (store-heavy) many.
  const int R = 1 << rlog, RW = 32 >> rlog;
  const int CT = (nzc + R - 1) >> rlog, RT = (nyq + RW - 1) / RW;
  const int per_half = RT * CT * 32;
  for (int task = threadIdx.x; task < 2 * per_half; task += blockDim.x) {
    const int half = task >= per_half;
    const int t2 = task - half * per_half;
    const int tile = t2 >> 5, l = t2 & 31, ty = tile / CT, tc = tile - ty * CT;
    const int yi = ty * RW + (l >> rlog), zc = (tc << rlog) + (l & (R - 1)), z0 = zc * KB;
    if (yi >= nyq || zc >= nzc) continue;
    const int y = ystart + yi;
    if (half && y == c) continue;  // the centre row has a single voxel set
    Q2 s[KB];
    if (masked) {
      // masked quads contribute zero (sbrt:4223-4258, :4595-4640)
#pragma unroll
      for (int j = 0; j < KB; j++) s[j] = Q2{0ull, 0ull};
    } else if (y == c) {
      // centre row (sbrt:4260-4284): rays pass plane yr = z exactly
#pragma unroll
      for (int j = 0; j < KB; j++) s[j] = ldq(P + bsw(o0 + z0 + j));
      for (int gg = 0; gg < G; gg++) {
        const int se = 2 * gg + 2, so = 2 * gg + 1;
        const int yb = g.ybot[se], yt = g.ytop[se];
        const int pe = g.bp_soff[se] - yb, po = g.bp_soff[so] - yb;
#pragma unroll
        for (int j = 0; j < KB; j++) {
          const int z = z0 + j;
          if (z >= yb && z <= yt) s[j] = qadd(s[j], qadd(ldq(P + bsw(pe + z)), ldq(P + bsw(po + z))));
        }
      }
    } else {
#pragma unroll
      for (int j = 0; j < KB; j++) s[j] = ldq(P + bsw(o0 + z0 + j));
      // bplut is [group][row]: the threads of a row read the same entries
      const BpLut *l1 = g.bplut + y, *l2 = g.bplut + (N - y);
      BpLut b1 = l1[0], b2 = l2[0];
      for (int gg = 0; gg < G; gg++) {
        const int se = 2 * gg + 2, so = 2 * gg + 1;
        const int yb = g.ybot[se];
        const int pe = g.bp_soff[se] - yb, po = g.bp_soff[so] - yb;
        const int gn = (gg + 1 < G) ? gg + 1 : gg;
        const BpLut n1 = l1[(size_t)gn * N], n2 = l2[(size_t)gn * N];  // next group, in flight
        // sumt1: segment 2k at +u and 2k-1 at -u; sumt2: the converse
        bp_lerp<KB>(s, P, half ? po : pe, b1, z0);
        bp_lerp<KB>(s, P, half ? pe : po, b2, z0);
        b1 = n1;
        b2 = n2;
      }
    }
    // the reference writes planes z < nz only
#pragma unroll
    for (int j = 0; j < KB; j++)
      if (z0 + j >= g.nz) s[j] = Q2{0ull, 0ull};
    const size_t cz = (size_t)z0;
    if (!half) {
      store_lane<KB, ACC>(bcp + ((size_t)x * N + y) * zp + cz, s, 0);
      store_lane<KB, ACC>(brp + ((size_t)(N - y) * N + x) * zp + cz, s, 2);
      if (x != c) {
        store_lane<KB, ACC>(bcp + ((size_t)(N - x) * N + y) * zp + cz, s, 1);
        store_lane<KB, ACC>(brp + ((size_t)(N - y) * N + N - x) * zp + cz, s, 3);
      }
    } else {
      store_lane<KB, ACC>(bcp + ((size_t)x * N + N - y) * zp + cz, s, 0);
      store_lane<KB, ACC>(brp + ((size_t)y * N + x) * zp + cz, s, 2);
      if (x != c) {
        store_lane<KB, ACC>(bcp + ((size_t)(N - x) * N + N - y) * zp + cz, s, 1);
        store_lane<KB, ACC>(brp + ((size_t)y * N + N - x) * zp + cz, s, 3);
      }
    }
  }
}

// ============================================================================
// Exact adjoint of the forward projector (no counterpart in the reference,
// whose back projector is not the transpose of its forward projector).
//
// adj_kernel: per (pair, quad x) the forward projector's z interpolation
// transposed -- every rotated-frame sample of the forward projection receives
// the rows it fed, weighted as it was weighted (sbrt:1914-1951 read backwards:
// the middle planes are two windows of the segment, the end planes one
// position each), with the rows first scaled as the forward projector scales
// them (sbrt:1953-1976).  The samples are the back projector's voxel roles, so
// the lanes go to the same column / row partials.
// adj_rotate_kernel: the bilinear sampling transposed as a gather: an image
// voxel collects from the <= 16 rotated-frame points around its inverse
// rotation whose sample footprint (recomputed with the forward projector's own
// float expressions) holds it, with that footprint's weight.
// ============================================================================


// One side of a segment group's middle planes transposed: for the task's
// planes z0 + j, s[j] += w0 * P[a0 + j - d0] + w1 * P[a0 + j - d1] over the
// window entries inside [lo, hi] (d0, d1 in {0, 1}).  Windows wholly inside
// the middle planes slide without checks; windows that straddle an end check
// each entry.
template <int KB>
__device__ __forceinline__ void adj_side(Q2 (&s)[KB], const float4 *__restrict__ P, int a0, int lo, int hi,
                                         uint64_t w_at, uint64_t w_below) {
  // w_at multiplies P[a0 + j], w_below multiplies P[a0 + j - 1]
  if (a0 - 1 >= lo && a0 + KB - 1 <= hi) {
    Q2 prev = ldq(P + a0 - 1);
#pragma unroll
    for (int j = 0; j < KB; j++) {
      const Q2 cur = ldq(P + a0 + j);
      s[j] = qfma(prev, w_below, qfma(cur, w_at, s[j]));
      prev = cur;
    }
  } else if (a0 + KB - 1 >= lo && a0 - 1 <= hi) {
#pragma unroll
    for (int j = 0; j < KB; j++) {
      const int ya = a0 + j;
      if (ya >= lo && ya <= hi) s[j] = qfma(ldq(P + ya), w_at, s[j]);
      if (ya - 1 >= lo && ya - 1 <= hi) s[j] = qfma(ldq(P + ya - 1), w_below, s[j]);
    }
  }
}

template <int KB>
__global__ void __launch_bounds__(256, 3) adj_kernel(DevGeom g, const float4 *__restrict__ in, long long in_pair_stride,
                                                  const QuadWork *__restrict__ work, float *__restrict__ bc,
                                                  float *__restrict__ br, long long vol, FrameStrides fr) {
  extern __shared__ float4 P[];
  const int nwork = gridDim.x / fr.n, frame = blockIdx.x / nwork, item = blockIdx.x - frame * nwork;
  const QuadWork w = work[item];
  in += (size_t)frame * fr.ratio / 4;
  bc += (size_t)frame * fr.bc;
  br += (size_t)frame * fr.bc;
  const int x = w.x, N = g.nx, c = g.c, zp = g.zp, G = g.groupmax, ZS = g.zshift, nz = g.nz;
  const bool masked = g.nzmask[w.view * g.nquads + x] == 0 || g.cyl0[x] == g.cyl1[x];
  const float4 *src = in + (size_t)w.slot * in_pair_stride + (size_t)x * g.pplanes;
  if (!masked)
    for (int i = threadIdx.x; i < g.bp_splanes; i += blockDim.x) {
      const int q = __ldg(g.bp_src + i);
      float4 v = f4(0.f);
      if (q >= 0) {
        const int sg = g.pplane_seg[q];
        const int yb = g.ybot[sg], yr = yb + (q - g.poff[sg]);
        float sc = g.y_size;
        if (sg > 0) {
          int zs = yr - yb;
          if (zs >= ZS) zs = g.ytop[sg] - yr;
          sc = g.rescale[((sg - 1) >> 1) * nz + (zs < ZS ? yr : yb + ZS)];
        }
        v = src[q] * sc;
      }
      P[i] = v;
    }
  __syncthreads();
  float *bcp = bc + (size_t)w.slot * vol;
  float *brp = br + (size_t)w.slot * vol;
  const int ystart = g.cyl0[x];
  const int nyq = c - ystart + 1, nzc = zp / KB;
  const float4 *P0 = P + g.bp_soff[0];
  // a warp's 32 tasks are 32 consecutive rows at one plane run: the rows'
  // table entries ([group][row]) are contiguous, the stores whole sectors
  const int per_half = nyq * nzc;
  for (int task = threadIdx.x; task < 2 * per_half; task += blockDim.x) {
    const int half = task >= per_half;
    const int t2 = task - half * per_half;
    const int zc = t2 / nyq, yi = t2 - zc * nyq, z0 = zc * KB;
    const int y = ystart + yi;
    if (half && y == c) continue;
    Q2 s[KB];
#pragma unroll
    for (int j = 0; j < KB; j++) s[j] = Q2{0ull, 0ull};
    if (!masked) {
#pragma unroll
      for (int j = 0; j < KB; j++) s[j] = ldq(P0 + z0 + j);
      if (y == c) {
        // centre row: every plane of every segment took the centre samples
        for (int gg = 0; gg < G; gg++) {
          const int se = 2 * gg + 2, so = 2 * gg + 1;
          const int yb = g.ybot[se], yt = g.ytop[se];
          const float4 *pe = P + g.bp_soff[se] - yb, *po = P + g.bp_soff[so] - yb;
#pragma unroll
          for (int j = 0; j < KB; j++) {
            const int z = z0 + j;
            if (z >= yb && z <= yt) s[j] = qadd(s[j], qadd(ldq(pe + z), ldq(po + z)));
          }
        }
      } else {
        const FpMid *mrow = g.fpmid_t + y;
        const int2 *e1 = g.fl_t + y, *e2 = g.fl_t + (N - y);
        for (int gg = 0; gg < G; gg++) {
          const FpMid m = mrow[(size_t)gg * c];
          if (m.z < 0) continue;  // the forward projector skipped this group for this row
          const int se = 2 * gg + 2, so = 2 * gg + 1;
          const int yb = g.ybot[se], yt = g.ytop[se], ym = yb + ZS, ye = yt - ZS;
          // A: the rows that read this sample at (z, z+1) with (f2, f); B:
          // the rows that read it at (z2+1, z2) with (f2, f)
          const float4 *A = P + g.bp_soff[half ? so : se] - yb, *B = P + g.bp_soff[half ? se : so] - yb;
          const uint64_t f = pk(m.f, m.f), f2 = pk(m.f2, m.f2);
          adj_side<KB>(s, A, z0 - m.z + ym, ym, ye, f2, f);
          adj_side<KB>(s, B, z0 - m.z2 + ym, ym, ye, f, f2);
          // end planes: one position per plane; an end whose entries touch
          // no plane of this task's run is skipped whole
          const size_t eb = (size_t)gg * 2 * ZS * N;
          const int4 er = __ldg(g.adj_endr + (size_t)gg * c + y);
          const bool bot = er.x < z0 + KB && er.y >= z0, top = er.z < z0 + KB && er.w >= z0;
          for (int i = bot ? 0 : ZS; i < (top ? 2 * ZS : ZS); i++) {
            const int2 u = __ldg(e1 + eb + (size_t)i * N), v = __ldg(e2 + eb + (size_t)i * N);
            const int za = u.x, zb = v.x;
            if ((za + 1 < z0 || za >= z0 + KB) && (zb + 1 < z0 || zb >= z0 + KB)) continue;
            const int yr = (i < ZS) ? yb + i : yt - 2 * ZS + 1 + i;
            const float fa = __int_as_float(u.y), fb = __int_as_float(v.y);
            const uint64_t pfa = pk(fa, fa), pfb = pk(fb, fb);
            const Q2 a = ldq(A + yr), b = ldq(B + yr);
#pragma unroll
            for (int j = 0; j < KB; j++) {
              const int z = z0 + j;
              if (z == za) s[j] = qfma(a, pfb, s[j]);
              if (z == za + 1) s[j] = qfma(a, pfa, s[j]);
              if (z == zb + 1) s[j] = qfma(b, pfb, s[j]);
              if (z == zb) s[j] = qfma(b, pfa, s[j]);
            }
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < KB; j++)
      if (z0 + j >= nz) s[j] = Q2{0ull, 0ull};
    const size_t cz = (size_t)z0;
    if (!half) {
      store_lane<KB>(bcp + ((size_t)x * N + y) * zp + cz, s, 0);
      store_lane<KB>(brp + ((size_t)(N - y) * N + x) * zp + cz, s, 2);
      if (x != c) {
        store_lane<KB>(bcp + ((size_t)(N - x) * N + y) * zp + cz, s, 1);
        store_lane<KB>(brp + ((size_t)(N - y) * N + N - x) * zp + cz, s, 3);
      }
    } else {
      store_lane<KB>(bcp + ((size_t)x * N + N - y) * zp + cz, s, 0);
      store_lane<KB>(brp + ((size_t)y * N + x) * zp + cz, s, 2);
      if (x != c) {
        store_lane<KB>(bcp + ((size_t)(N - x) * N + N - y) * zp + cz, s, 1);
        store_lane<KB>(brp + ((size_t)y * N + N - x) * zp + cz, s, 3);
      }
    }
  }
}

// For each pair slot and voxel column (every column for MODE 2, the FOV
// columns otherwise): the rotated-frame points (a, b) around the column's
// inverse rotation whose forward-projection sample footprint -- recomputed
// with the forward projector's own float expressions -- covers the column,
// with that footprint's weight, in scan order.  One thread per (pair, column);
// the rotate then reads these instead of every thread of a column repeating
// the 16 candidate footprints.
template <int MODE>
__global__ void __launch_bounds__(256) adj_cover_kernel(DevGeom g, const int *__restrict__ pair_views, int npairs) {
  const int N = g.nx, c = g.c;
  const long long ncols = (MODE == 2) ? (long long)N * N : g.fov_columns;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ncols * npairs) return;
  const int p = (int)(t / ncols);
  const int col = (int)(t - (long long)p * ncols);
  int i, j;
  if (MODE == 2) {
    i = col / N;
    j = col - i * N;
  } else {
    const short2 xy = g.fov_xy[col];
    i = xy.x;
    j = xy.y;
  }
  const int view = pair_views[p];
  const float cosv = g.cos_psi[view], sinv = g.sin_psi[view];
  const float di = (float)(i - c), dj = (float)(j - c);
  const int qx0 = (int)floorf(di * cosv + dj * sinv + (float)c) - 1;
  const int qy0 = (int)floorf(-di * sinv + dj * cosv + (float)c) - 1;
  int2 *ent = g.adj_ent + t * kAdjCover;
  int n = 0;
  for (int a = qx0; a < qx0 + 4; a++) {
    if (a < 0 || a >= N) continue;
    for (int b = qy0; b < qy0 + 4; b++) {
      if (b < 0 || b >= N) continue;
      const SamplePt pt = sample_point(a, b, c, N, g.zp, cosv, sinv);
      if (pt.base < 0) continue;
      const int ix = pt.base / (N * g.zp), iy = (pt.base / g.zp) - ix * N;
      const int dx = i - ix, dy = j - iy;
      if (dx < 0 || dx > 1 || dy < 0 || dy > 1) continue;
      const float wgt = dx ? (dy ? pt.c3 : pt.c1) : (dy ? pt.c2 : pt.c0);
      if (n < kAdjCover) ent[n] = make_int2(a * N + b, __float_as_int(wgt));
      n++;
    }
  }
  if (n > kAdjCover) atomicExch(g.err, 2);  // more covering points than the table holds: results void
  g.adj_cnt[t] = min(n, kAdjCover);
}

// MODE 0: OSEM update, 1: inverse sensitivity (both over the FOV columns, as
// the rotate-back), 2: out += adjoint over every image column.
template <int MODE>
__global__ void __launch_bounds__(256) adj_rotate_kernel(DevGeom g, const int *__restrict__ pair_views, int npairs,
                                                         const float *__restrict__ bc, const float *__restrict__ br,
                                                         long long vol, float *__restrict__ image,
                                                         float *__restrict__ nf_inv, float *__restrict__ out,
                                                         FrameStrides fr) {
  const int nq = g.zp / 4, N = g.nx;
  if (MODE == 0) {
    image += (size_t)(fr.map ? __ldg(fr.map + blockIdx.y) : (int)blockIdx.y) * fr.image;
    bc += (size_t)blockIdx.y * fr.bc;
    br += (size_t)blockIdx.y * fr.bc;
  }
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int col = (int)(t / nq), q = (int)(t - (long long)col * nq);
  int i, j;
  if (MODE == 2) {
    if (col >= N * N) return;
    i = col / N;
    j = col - i * N;
  } else {
    if (col >= g.fov_columns) return;
    const short2 xy = g.fov_xy[col];
    i = xy.x;
    j = xy.y;
  }
  // the covering points of this column, found once per pair by
  // adj_cover_kernel in this scan order
  const long long ncols = (MODE == 2) ? (long long)N * N : g.fov_columns;
  float4 acc = f4(0.f);
  for (int p = 0; p < npairs; p++) {
    const float4 *Bc = reinterpret_cast<const float4 *>(bc + (size_t)p * vol);
    const float4 *Br = reinterpret_cast<const float4 *>(br + (size_t)p * vol);
    const long long e0 = (long long)p * ncols + col;
    const int n = __ldg(g.adj_cnt + e0);
    const int2 *ent = g.adj_ent + e0 * kAdjCover;
    for (int k = 0; k < n; k++) {
      const int2 u = __ldg(ent + k);
      const size_t o = (size_t)u.x * nq + q;
      acc = acc + (__ldg(Bc + o) + __ldg(Br + o)) * __int_as_float(u.y);
    }
  }
  const size_t o = ((size_t)i * N + j) * nq + q;
  if (MODE == 0) {
    float4 *im = reinterpret_cast<float4 *>(image);
    const float4 nf = reinterpret_cast<const float4 *>(nf_inv)[o];
    float4 iv = im[o];
    float a[4] = {acc.x, acc.y, acc.z, acc.w}, b[4] = {iv.x, iv.y, iv.z, iv.w}, n[4] = {nf.x, nf.y, nf.z, nf.w};
#pragma unroll
    for (int l = 0; l < 4; l++) {
      const float lo = (0.01f > a[l]) ? 0.01f : a[l];
      const float cl = (100.0f < lo) ? 100.0f : lo;
      const float u = b[l] * (cl * n[l]);
      b[l] = (g.image_max < u) ? g.image_max : u;
    }
    im[o] = make_float4(b[0], b[1], b[2], b[3]);
  } else if (MODE == 1) {
    float a[4] = {acc.x, acc.y, acc.z, acc.w}, r[4];
#pragma unroll
    for (int l = 0; l < 4; l++) {
      const int z = q * 4 + l;
      r[l] = (z < g.nz && fabsf(a[l]) > g.eps1) ? (1.0f / a[l]) : 0.f;
    }
    reinterpret_cast<float4 *>(nf_inv)[o] = make_float4(r[0], r[1], r[2], r[3]);
  } else {
    float4 *dst = reinterpret_cast<float4 *>(out);
    dst[o] = dst[o] + acc;
  }
}

// ============================================================================
// Rotate-back of the summed partials of every pair (rotateimage2, sbrt:1137-
// 1186) fused with what consumes the correction image:
//   MODE 0: OSEM update pt_cal_updateimage (drv:2018-2059)
//   MODE 1: inverse sensitivity pt_normfac_calculate (drv:1852-1894)
//   MODE 2: corr_out += rotate-back (rotate_image_buf for one view)
// One thread per (FOV column, 4 planes); pairs are added in subset order.
// ============================================================================
template <int MODE>
__global__ void __launch_bounds__(256) rotback_kernel(DevGeom g, const int *__restrict__ pair_views, int npairs,
                                                      const float *__restrict__ bc, const float *__restrict__ br,
                                                      long long vol, float *__restrict__ image,
                                                      float *__restrict__ nf_inv, float *__restrict__ corr_out,
                                                      FrameStrides fr) {
  const int nq = g.zp / 4;
  if (MODE == 0) {
    image += (size_t)(fr.map ? __ldg(fr.map + blockIdx.y) : (int)blockIdx.y) * fr.image;
    bc += (size_t)blockIdx.y * fr.bc;
    if (br != nullptr) br += (size_t)blockIdx.y * fr.bc;
  }
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int col = (int)(t / nq), q = (int)(t - (long long)col * nq);
  if (col >= g.fov_columns) return;
  const short2 xy = g.fov_xy[col];
  const int N = g.nx;
  float4 acc = f4(0.f);
  for (int p = 0; p < npairs; p++) {
    const float2 pos = g.rotpos[(size_t)pair_views[p] * g.fov_columns + col];
    const int ix = (int)pos.x, iy = (int)pos.y;
    if (ix < 0 || ix > N - 2 || iy < 0 || iy > N - 2) continue;
    const float x1 = pos.x - ix, y1 = pos.y - iy;
    const float c1 = (1 - x1) * (1 - y1), c2 = x1 * (1 - y1), c3 = y1 * (1 - x1), c4 = y1 * x1;
    const float4 *Bc = reinterpret_cast<const float4 *>(bc + (size_t)p * vol);
    const size_t i1 = ((size_t)ix * N + iy) * nq + q, i2 = i1 + (size_t)N * nq, i3 = i1 + nq, i4 = i2 + nq;
    float4 b1 = __ldg(Bc + i1), b2 = __ldg(Bc + i2), b3 = __ldg(Bc + i3), b4 = __ldg(Bc + i4);
    if (br != nullptr) {
      const float4 *Br = reinterpret_cast<const float4 *>(br + (size_t)p * vol);
      b1 = b1 + __ldg(Br + i1);
      b2 = b2 + __ldg(Br + i2);
      b3 = b3 + __ldg(Br + i3);
      b4 = b4 + __ldg(Br + i4);
    }
    acc = acc + ((b1 * c1 + b2 * c2) + (b3 * c3 + b4 * c4));
  }
  const size_t o = ((size_t)xy.x * N + xy.y) * nq + q;
  if (MODE == 0) {
    float4 *im = reinterpret_cast<float4 *>(image);
    const float4 nf = reinterpret_cast<const float4 *>(nf_inv)[o];
    float4 iv = im[o];
    float a[4] = {acc.x, acc.y, acc.z, acc.w}, b[4] = {iv.x, iv.y, iv.z, iv.w}, n[4] = {nf.x, nf.y, nf.z, nf.w};
#pragma unroll
    for (int l = 0; l < 4; l++) {
      // _mm_max_ps(0.01, c), _mm_min_ps(100, .), _mm_min_ps(image_max, .):
      // each returns its second operand when either is NaN
      const float lo = (0.01f > a[l]) ? 0.01f : a[l];
      const float cl = (100.0f < lo) ? 100.0f : lo;
      const float u = b[l] * (cl * n[l]);
      b[l] = (g.image_max < u) ? g.image_max : u;
    }
    im[o] = make_float4(b[0], b[1], b[2], b[3]);
  } else if (MODE == 1) {
    float a[4] = {acc.x, acc.y, acc.z, acc.w}, r[4];
#pragma unroll
    for (int l = 0; l < 4; l++) {
      const int z = q * 4 + l;
      r[l] = (z < g.nz && fabsf(a[l]) > g.eps1) ? (1.0f / a[l]) : 0.f;
    }
    reinterpret_cast<float4 *>(nf_inv)[o] = make_float4(r[0], r[1], r[2], r[3]);
  } else if (MODE == 2) {
    float4 *co = reinterpret_cast<float4 *>(corr_out);
    co[o] = co[o] + acc;
  } else {
    reinterpret_cast<float4 *>(corr_out)[o] = acc;
  }
}

// rotate-back sample positions, incremented along y exactly as rotateimage2
// does (sbrt:1148-1184)
__global__ void rotpos_kernel(DevGeom g, float2 *__restrict__ rotpos, const int *__restrict__ row_start) {
  const int X = blockIdx.x * blockDim.x + threadIdx.x, vi = blockIdx.y;
  if (X >= g.nx) return;
  const int N = g.nx, h = N / 2;
  const float cosv = g.cos_psi[vi] / 1.0f;
  const float sinv = -g.sin_psi[vi] / 1.0f;
  const float xxx0 = (float)(-N / 2) * cosv + (float)h * sinv + (float)h;
  const float yyy0 = (float)(-N / 2) * sinv - (float)h * cosv + (float)h;
  const int ys = g.cyl0[X], ye = g.cyl1[X];
  float xx0 = xxx0 - (float)ys * sinv + (float)X * cosv;
  float yy0 = yyy0 + (float)ys * cosv + (float)X * sinv;
  float2 *dst = rotpos + (size_t)vi * g.fov_columns + row_start[X];
  for (int y = ys; y < ye; y++) {
    dst[y - ys] = make_float2(xx0, yy0);
    xx0 -= sinv;
    yy0 += cosv;
  }
}

// ============================================================================
// Input preparation + re-layout (prepare_norm/norm_ANW drv:796-1056,
// prepare_osem3dw3 drv:1649-1818, mul/add projection simd_operation.cpp:4-58)
// from the flat file layout into the quad layout.  One thread per (pair,
// quad, run of planes).
// ============================================================================
template <typename PT, typename AT>
__global__ void prep_kernel(DevGeom g, int nbins, const int16_t *__restrict__ prompts,
                            const float *__restrict__ randoms, const float *__restrict__ norm,
                            const float *__restrict__ atten, const float *__restrict__ scatter, int npskip,
                            float eps2, PT *__restrict__ qp, AT *__restrict__ qadd, AT *__restrict__ qmult,
                            int *__restrict__ mask_accum, int planes_per_thread, int plane0, int nplanes,
                            const int *__restrict__ pair_views, long long s_plane, long long s_half,
                            long long s_slot, long long pf_plane, long long pf_half) {
  // Input element of plane gp, lane l: base + (gp - plane0)*s_plane + h*s_half
  // + bin.  Flat-file chunk (pair_views null): pair = blockIdx.z, base =
  // pair*nbins, planes [plane0, plane0 + nplanes).  Pair-major staging: pair =
  // pair_views[blockIdx.z], base = blockIdx.z*s_slot, all planes.  With
  // pf_plane > 0 the prompts are the whole sinogram instead: element
  // gp*pf_plane + pair*nbins + h*pf_half + bin.
  const int x = blockIdx.x * blockDim.x + threadIdx.x;  // quad
  const int vi = pair_views ? pair_views[blockIdx.z] : (int)blockIdx.z;
  const long long base = pair_views ? (long long)blockIdx.z * s_slot : (long long)vi * nbins;
  if (x >= g.nquads) return;
  const int gp0 = plane0 + blockIdx.y * planes_per_thread;
  const int gp1 = min(gp0 + planes_per_thread, plane0 + nplanes);
  const int hl[4] = {0, 0, 1, 1};
  int bins[4] = {x, nbins - x, x, nbins - x};
  bool ok[4];
  for (int l = 0; l < 4; l++) ok[l] = (bins[l] >= 0 && bins[l] < nbins && x > 0);
  int any = 0;
  for (int gp = gp0; gp < gp1; gp++) {
    const int s = g.plane_seg[gp];
    const int segoff = g.poff[s] - 2 * s - 1;
    const int r = gp - segoff, ns = g.ytop[s] - g.ybot[s] + 1;
    const bool kill = (r < npskip || r + npskip >= ns);
    float pv[4], av[4], mv[4];
    for (int l = 0; l < 4; l++) {
      pv[l] = av[l] = mv[l] = 0.f;
      if (!ok[l]) continue;
      const size_t i = (size_t)(base + (long long)(gp - plane0) * s_plane + hl[l] * s_half + bins[l]);
      const float nz = norm ? (kill ? 0.f : __ldg(norm + i)) : 1.0f;
      const float araw = atten ? __ldg(atten + i) : 1.0f;
      const float ac = (araw < 1.0f) ? 1.0f : araw;
      float m;
      if (nz > 0.0f) {
        const float den = nz * ac;
        m = (den > eps2) ? 1.0f / den : 0.0f;
      } else {
        m = nz;
      }
      float a = __ldg(randoms + i) * nz;
      if (scatter) a = a + __ldg(scatter + i);
      a = a * araw;
      const size_t pi = pf_plane > 0 ? (size_t)((long long)gp * pf_plane + (long long)vi * nbins +
                                                hl[l] * pf_half + bins[l])
                                     : i;
      const float p = (nz == 0.0f) ? 0.f : (float)__ldg(prompts + pi);
      if (nz != 0.0f) any = 1;
      pv[l] = p;
      av[l] = a;
      mv[l] = m;
    }
    const size_t o = ((size_t)vi * g.nquads + x) * g.pplanes + g.poff[s] + r;
    if (std::is_same<AT, __half>::value) {
      // fp16 holds magnitudes up to 65504: a larger term is reported, not stored wrapped
      bool over = false;
      for (int l = 0; l < 4; l++) over |= fabsf(av[l]) > 65504.f || fabsf(mv[l]) > 65504.f;
      if (over) atomicOr(g.range_err, 1);
    }
    store_p4(qp, o, pv);
    store_p4(qadd, o, av);
    store_p4(qmult, o, mv);
  }
  if (any) atomicOr(mask_accum + vi * g.nquads + x, 1);
}

__global__ void finish_mask_kernel(DevGeom g, const int *__restrict__ accum, int16_t *__restrict__ nzmask) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (g.nviews / 2) * g.nquads) return;
  const int x = i % g.nquads;
  nzmask[i] = (x == 0) ? 1 : (accum[i] ? 1 : 0);
}

__global__ void init_image_kernel(DevGeom g, float *__restrict__ image) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)g.nx * g.nx * g.zp;
  if (t >= total) return;
  const int z = (int)(t % g.zp);
  const long long xy = t / g.zp;
  const int X = (int)(xy / g.nx), Y = (int)(xy % g.nx);
  const bool fov = g.cyl0[X] != g.cyl1[X] && Y >= g.cyl0[X] && Y < g.cyl1[X];
  image[t] = (fov && z >= g.z_min && z < g.z_max) ? 1.0f : 0.0f;
}

// post-iteration pass (drv:4288-4297) with an FP64 sum, deterministic:
// per-block partial sums, then one block adds them in order.
__global__ void post_iter_kernel(DevGeom g, float *__restrict__ image, double *__restrict__ partial,
                                 FrameStrides fr) {
  __shared__ double red[256];
  image += (size_t)(fr.map ? __ldg(fr.map + blockIdx.y) : (int)blockIdx.y) * fr.image;
  partial += (size_t)blockIdx.y * fr.partial;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nz = g.z_max - g.z_min;
  double s = 0.0;
  if (t < (long long)g.fov_columns * nz) {
    const int col = (int)(t / nz), z = g.z_min + (int)(t % nz);
    const short2 xy = g.fov_xy[col];
    float *p = image + ((size_t)xy.x * g.nx + xy.y) * g.zp + z;
    const float v = *p;
    s = (double)v;
    if ((double)v < 1e-16) *p = 0.f;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if ((int)threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}
// One block: each thread sums a contiguous run of partials, then a fixed
// tree adds the runs -- the same order on every call (deterministic).
__global__ void sum_partials_kernel(const double *__restrict__ partial, int n, double *__restrict__ out,
                                    long long frame_stride, const int *__restrict__ map) {
  __shared__ double red[1024];
  partial += (size_t)blockIdx.x * frame_stride;
  out += map ? map[blockIdx.x] : (int)blockIdx.x;
  const int t = threadIdx.x, T = blockDim.x;
  const int per = (n + T - 1) / T, b = t * per, e = min(b + per, n);
  double s = 0.0;
  for (int i = b; i < e; i++) s += partial[i];
  red[t] = s;
  __syncthreads();
  for (int k = T / 2; k > 0; k >>= 1) {
    if (t < k) red[t] += red[t + k];
    __syncthreads();
  }
  if (t == 0) *out = red[0];
}

__global__ void rows_to_quad_kernel(DevGeom g, int nbins, const float *__restrict__ rows, float4 *__restrict__ quad,
                                    int apply_bp_scale) {
  const int gp = blockIdx.y, x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= g.nquads || gp >= g.segmentsize) return;
  const int s = g.plane_seg[gp];
  const int segoff = g.poff[s] - 2 * s - 1;
  const int r = gp - segoff;
  const size_t P = g.segmentsize;
  const int xm = nbins - x;
  float v[4] = {0.f, 0.f, 0.f, 0.f};
  if (x > 0) {
    v[0] = rows[(size_t)gp * nbins + x];
    v[1] = rows[(size_t)gp * nbins + xm];
    v[2] = rows[(P + gp) * nbins + x];
    v[3] = rows[(P + gp) * nbins + xm];
  }
  if (apply_bp_scale) {
    const float bs = g.bp_scale[s];
    for (int l = 0; l < 4; l++) v[l] = v[l] * bs;
  }
  quad[(size_t)x * g.pplanes + g.poff[s] + r] = make_float4(v[0], v[1], v[2], v[3]);
}

__global__ void quad_to_rows_kernel(DevGeom g, int nbins, const float4 *__restrict__ quad,
                                    const QuadWork *__restrict__ work, float *__restrict__ rows) {
  const int gp = blockIdx.x * blockDim.x + threadIdx.x;
  const QuadWork w = work[blockIdx.y];
  if (gp >= g.segmentsize) return;
  const int s = g.plane_seg[gp];
  const int segoff = g.poff[s] - 2 * s - 1;
  const int r = gp - segoff;
  const size_t P = g.segmentsize;
  const int x = w.x, xm = nbins - x;
  const float4 q = quad[(size_t)x * g.pplanes + g.poff[s] + r];
  rows[(size_t)gp * nbins + x] = q.x;
  rows[(size_t)gp * nbins + xm] = q.y;
  rows[(P + gp) * nbins + x] = q.z;
  rows[(P + gp) * nbins + xm] = q.w;
}

__global__ void quad_to_file_kernel(DevGeom g, int nbins, const float4 *__restrict__ quad, long long stride,
                                    const QuadWork *__restrict__ work, float *__restrict__ sino) {
  const int gp = blockIdx.x * blockDim.x + threadIdx.x;
  const QuadWork w = work[blockIdx.y];
  if (gp >= g.segmentsize) return;
  const int s = g.plane_seg[gp];
  const int r = gp - (g.poff[s] - 2 * s - 1);
  const int x = w.x, xm = nbins - x, V = g.nviews;
  const float4 q = quad[(size_t)w.slot * stride + (size_t)x * g.pplanes + g.poff[s] + r];
  const size_t r0 = ((size_t)gp * V + w.view) * nbins, r1 = ((size_t)gp * V + w.view + V / 2) * nbins;
  sino[r0 + x] = q.x;
  sino[r0 + xm] = q.y;
  sino[r1 + x] = q.z;
  sino[r1 + xm] = q.w;
}

__global__ void add_partials_kernel(long long n4, const float4 *__restrict__ a, const float4 *__restrict__ b,
                                    float4 *__restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n4) out[i] = a[i] + b[i];
}

template <typename T>
__global__ void scale_pairs_kernel(DevGeom g, const T *__restrict__ src, const int *__restrict__ views,
                                   float4 *__restrict__ dst, long long dst_pair_stride) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per = (long long)g.nquads * g.pplanes;
  if (i >= per) return;
  const int slot = blockIdx.y;
  const int pp = (int)(i % g.pplanes);
  const int s = g.pplane_seg[pp];
  const P4 m = load_p4(src, (size_t)views[slot] * per + i);
  float4 o = f4(0.f);
  if (s >= 0) {
    const float bs = g.bp_scale[s];
    o = make_float4(m.v[0] * bs, m.v[1] * bs, m.v[2] * bs, m.v[3] * bs);
  }
  dst[(size_t)slot * dst_pair_stride + i] = o;
}

// The images the forward projector samples as a 4-D tensor (z, y, x, stored
// frame) with a box of the four corner columns of one sample point, {zp, 2,
// 2, 1}: one bulk tensor copy instead of two per point (the projector's row
// pipeline is bound by the number of copies, not their bytes).  Returns 0 (the
// kernel then copies column pairs) where the encoder is unavailable or
// refuses the shape.
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
int image_column_map(const DevGeom &g, const float *image, const FrameStrides &fr, CUtensorMap *map) {
  static EncodeTiledFn encode = [] {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (EncodeTiledFn) nullptr;
    }
    return reinterpret_cast<EncodeTiledFn>(fn);
  }();
  std::memset(map, 0, sizeof(*map));
  if (!encode || !image || (reinterpret_cast<uintptr_t>(image) & 15)) return 0;
  const cuuint64_t N = (cuuint64_t)g.nx, zp = (cuuint64_t)g.zp;
  const cuuint64_t fstride = fr.image > 0 ? (cuuint64_t)fr.image : N * N * zp;
  // stored frames: every frame a launch may name (the map bounds no access the
  // kernel makes; coordinates stay inside the frames that exist)
  const cuuint64_t frames = fr.image > 0 ? (cuuint64_t)1 << 16 : 1;
  const cuuint64_t dim[4] = {zp, N, N, frames};
  const cuuint64_t stride[3] = {zp * 4, N * zp * 4, fstride * 4};
  const cuuint32_t box[4] = {(cuuint32_t)zp, 2, 2, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  if (zp > 256 || (zp * 4) % 16 || (fstride * 4) % 16) return 0;
  const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float *>(image), dim, stride, box, es,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 1 : 0;
}

template <int MODE, int PL, int MW, typename PT, typename AT>
cudaError_t launch_fp_t(const DevGeom &g, const float *image, const QuadWork *work, int nwork, const void *prompts,
                        const void *add, float *out, long long out_pair_stride, int pwarps_req,
                        const FrameStrides &fr, cudaStream_t st) {
  // consumer warps: one task per thread; producer warps: enough to keep the
  // sampled rows ahead of the consumers (a row is ~2*zp bilinear quads)
  const int cwarps = (g.nfptasks + 31) / 32;
  const int pwarps = pwarps_req > 0 ? pwarps_req : min(6, max(2, MW - cwarps));
  if (pwarps < 2 || cwarps + pwarps > MW) return cudaErrorInvalidConfiguration;
  const int threads = (cwarps + pwarps) * 32;
  const int ZS = g.zp + kFpZPad;
  const size_t smem =
      (size_t)(kFpSlots * 8 * 2 + 2) * 2 * g.zp * sizeof(float) + (size_t)(2 * kFpSlots + 1) * ZS * sizeof(float4);
  auto k = fp_kernel<MODE, PL, MW, PT, AT>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  CUtensorMap cols;
  const int use_cols = image_column_map(g, image, fr, &cols);
  k<<<(unsigned)nwork * fr.n, threads, smem, st>>>(g, image, work, (const PT *)prompts, (const AT *)add,
                                                   reinterpret_cast<float4 *>(out), out_pair_stride / 4, pwarps, fr,
                                                   cols, use_cols);
  return cudaGetLastError();
}

template <int PL, int MW>
cudaError_t launch_fp_pl(const DevGeom &g, const float *image, const QuadWork *work, int nwork, int mode,
                         const void *prompts, const void *add, int storage, float *out, long long stride, int pwarps,
                         const FrameStrides &fr, cudaStream_t st) {
  if (mode == 0)
    return launch_fp_t<0, PL, MW, int16_t, float>(g, image, work, nwork, nullptr, nullptr, out, stride, pwarps, fr,
                                                  st);
  if (storage == 0)
    return launch_fp_t<1, PL, MW, int16_t, float>(g, image, work, nwork, prompts, add, out, stride, pwarps, fr, st);
  if (storage == 1)
    return launch_fp_t<1, PL, MW, int16_t, __nv_bfloat16>(g, image, work, nwork, prompts, add, out, stride, pwarps,
                                                          fr, st);
  return launch_fp_t<1, PL, MW, int16_t, __half>(g, image, work, nwork, prompts, add, out, stride, pwarps, fr, st);
}

}  // namespace

cudaError_t launch_fp(const DevGeom &g, const float *image, const QuadWork *work, int nwork, int mode,
                      const void *prompts, const void *add, int storage, float *out, long long out_pair_stride,
                      const ProjTune &tune, const FrameStrides &fr, cudaStream_t st) {
  if (nwork <= 0 || fr.n <= 0) return cudaSuccess;
  static_assert(kFpPlaneVariants[0] == 7 && kFpPlaneVariants[1] == 9 && kFpPlaneVariants[2] == 11, "variants");
  const int pl = tune.fp_planes > 0 ? tune.fp_planes : kFpPlanes;
  switch (pl) {
    case 7:
      return launch_fp_pl<7, kFpVariantWarps[0]>(g, image, work, nwork, mode, prompts, add, storage, out,
                                                 out_pair_stride, tune.fp_pwarps, fr, st);
    case 9:
      return launch_fp_pl<9, kFpVariantWarps[1]>(g, image, work, nwork, mode, prompts, add, storage, out,
                                                 out_pair_stride, tune.fp_pwarps, fr, st);
    case 11:
      return launch_fp_pl<11, kFpVariantWarps[2]>(g, image, work, nwork, mode, prompts, add, storage, out,
                                                  out_pair_stride, tune.fp_pwarps, fr, st);
    default:
      return cudaErrorInvalidValue;
  }
}

// log2 of the back projector's tile width (bp_kernel): the tuned one, else
// 2 runs where there are many segment groups and 4 where there are few
// (measured on B200 over 1..32: span 3 1.56 ms at 2, span 9 0.57 ms at 4);
// -1 if invalid
int bp_tile_log2(const DevGeom &g, const ProjTune &t) {
  const int r = t.bp_tile > 0 ? t.bp_tile : (g.groupmax > 12 ? 2 : 4);
  for (int l = 0; l <= 5; l++)
    if (r == 1 << l) return l;
  return -1;
}

template <int KB, int NT>
cudaError_t launch_bp_t(const DevGeom &g, const float *in, long long in_pair_stride, const QuadWork *work, int nwork,
                        float *bc, float *br, long long vol, const FrameStrides &fr, int rlog, cudaStream_t st) {
  static_assert(kBpPad >= KB, "a straddling window must stay inside the zero planes");
  const size_t smem = (size_t)g.bp_splanes * sizeof(float4);
  auto k = fr.n > 1 ? bp_kernel<KB, false, true, NT> : bp_kernel<KB, false, false, NT>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  k<<<(unsigned)nwork * fr.n, NT, smem, st>>>(g, reinterpret_cast<const float4 *>(in), in_pair_stride / 4, work, bc,
                                              br, vol, fr, 0, 0, rlog);
  return cudaGetLastError();
}

cudaError_t launch_bp(const DevGeom &g, const float *in, long long in_pair_stride, const QuadWork *work, int nwork,
                      float *bc, float *br, long long vol, const ProjTune &tune, const FrameStrides &fr,
                      cudaStream_t st) {
  if (nwork <= 0 || fr.n <= 0) return cudaSuccess;
  const int kb = tune.bp_planes > 0 ? tune.bp_planes : kBpZ;
  // 384 threads (two CTAs of 80 registers per SM) measured faster than 256
  // (three CTAs) at span 3 and 9 on B200: 1.58 vs 1.74 ms and 0.71 vs 0.74 ms
  const int nt = tune.bp_threads > 0 ? tune.bp_threads : 384;
  const int rl = bp_tile_log2(g, tune);
  if (rl < 0) return cudaErrorInvalidValue;
  if (kb == 8 && nt == 256) return launch_bp_t<8, 256>(g, in, in_pair_stride, work, nwork, bc, br, vol, fr, rl, st);
  if (kb == 8 && nt == 384) return launch_bp_t<8, 384>(g, in, in_pair_stride, work, nwork, bc, br, vol, fr, rl, st);
  if (kb == 4 && nt == 256) return launch_bp_t<4, 256>(g, in, in_pair_stride, work, nwork, bc, br, vol, fr, rl, st);
  if (kb == 4 && nt == 384) return launch_bp_t<4, 384>(g, in, in_pair_stride, work, nwork, bc, br, vol, fr, rl, st);
  return cudaErrorInvalidValue;
}

cudaError_t launch_adj(const DevGeom &g, const float *in, long long in_pair_stride, const QuadWork *work, int nwork,
                       float *bc, float *br, long long vol, const FrameStrides &fr, cudaStream_t st) {
  if (nwork <= 0 || fr.n <= 0) return cudaSuccess;
  const size_t smem = (size_t)g.bp_splanes * sizeof(float4);
  auto k = adj_kernel<kBpZ>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  k<<<(unsigned)nwork * fr.n, 256, smem, st>>>(g, reinterpret_cast<const float4 *>(in), in_pair_stride / 4, work, bc,
                                               br, vol, fr);
  return cudaGetLastError();
}

cudaError_t launch_adj_rotate(const DevGeom &g, const int *pair_views, int npairs, const float *bc, const float *br,
                              long long vol, float *image, float *nf_inv, float *out, int mode,
                              const FrameStrides &fr, cudaStream_t st) {
  if (fr.n <= 0) return cudaSuccess;
  if (mode != 0 && fr.n != 1) return cudaErrorInvalidValue;
  const long long cols = (mode == 2) ? (long long)g.nx * g.nx : (long long)g.fov_columns;
  if (npairs > g.adj_pairs || !g.adj_ent || !g.adj_cnt) return cudaErrorInvalidValue;
  const int threads = 256;
  {
    const long long m = cols * npairs;
    const unsigned cb = (unsigned)((m + threads - 1) / threads);
    if (mode == 2)
      adj_cover_kernel<2><<<cb, threads, 0, st>>>(g, pair_views, npairs);
    else
      adj_cover_kernel<0><<<cb, threads, 0, st>>>(g, pair_views, npairs);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  const long long n = cols * (g.zp / 4);
  const dim3 blocks((unsigned)((n + threads - 1) / threads), fr.n);
  if (mode == 0)
    adj_rotate_kernel<0><<<blocks, threads, 0, st>>>(g, pair_views, npairs, bc, br, vol, image, nf_inv, out, fr);
  else if (mode == 1)
    adj_rotate_kernel<1><<<blocks, threads, 0, st>>>(g, pair_views, npairs, bc, br, vol, image, nf_inv, out, fr);
  else
    adj_rotate_kernel<2><<<blocks, threads, 0, st>>>(g, pair_views, npairs, bc, br, vol, image, nf_inv, out, fr);
  return cudaGetLastError();
}

cudaError_t launch_bp_sum(const DevGeom &g, const float *quad, int view, int x0, int nquads, float *out,
                          cudaStream_t st) {
  if (nquads <= 0) return cudaSuccess;
  const size_t smem = (size_t)g.bp_splanes * sizeof(float4);
  auto k = bp_kernel<kBpZ, true>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  k<<<nquads, 256, smem, st>>>(g, reinterpret_cast<const float4 *>(quad), 0, nullptr, out, nullptr, 0, one_frame(), view,
                               x0, bp_tile_log2(g, default_tune()));
  return cudaGetLastError();
}

cudaError_t launch_rotback(const DevGeom &g, const int *pair_views, int npairs, const float *bc, const float *br,
                           long long vol, float *image, float *nf_inv, float *corr_out, int mode,
                           const FrameStrides &fr, cudaStream_t st) {
  if (fr.n <= 0) return cudaSuccess;
  if (mode != 0 && fr.n != 1) return cudaErrorInvalidValue;
  const long long n = (long long)g.fov_columns * (g.zp / 4);
  const int threads = 256;
  const dim3 blocks((unsigned)((n + threads - 1) / threads), fr.n);
  if (mode == 0)
    rotback_kernel<0><<<blocks, threads, 0, st>>>(g, pair_views, npairs, bc, br, vol, image, nf_inv, corr_out, fr);
  else if (mode == 1)
    rotback_kernel<1><<<blocks, threads, 0, st>>>(g, pair_views, npairs, bc, br, vol, image, nf_inv, corr_out, fr);
  else if (mode == 2)
    rotback_kernel<2><<<blocks, threads, 0, st>>>(g, pair_views, npairs, bc, br, vol, image, nf_inv, corr_out, fr);
  else
    rotback_kernel<3><<<blocks, threads, 0, st>>>(g, pair_views, npairs, bc, br, vol, image, nf_inv, corr_out, fr);
  return cudaGetLastError();
}

cudaError_t launch_rotpos(const DevGeom &g, float2 *rotpos, const int *row_start, cudaStream_t st) {
  dim3 grid((g.nx + 127) / 128, g.nviews / 2);
  rotpos_kernel<<<grid, 128, 0, st>>>(g, rotpos, row_start);
  return cudaGetLastError();
}

cudaError_t launch_prep(const DevGeom &g, int nbins, const int16_t *prompts, const float *randoms, const float *norm,
                        const float *atten, const float *scatter, int npskip, float eps2, int storage, void *q_prompts,
                        void *q_add, void *q_mult, int *quad_mask_accum, int plane0, int nplanes,
                        cudaStream_t st) {
  const int ppt = 16;
  dim3 grid((g.nquads + 127) / 128, (nplanes + ppt - 1) / ppt, g.nviews / 2);
  const long long sp = (long long)g.nviews * nbins, sh = (long long)(g.nviews / 2) * nbins;
  if (storage == 0)
    prep_kernel<int16_t, float><<<grid, 128, 0, st>>>(g, nbins, prompts, randoms, norm, atten, scatter, npskip, eps2,
                                                      (int16_t *)q_prompts, (float *)q_add, (float *)q_mult,
                                                      quad_mask_accum, ppt, plane0, nplanes, nullptr, sp, sh, 0, 0, 0);
  else if (storage == 1)
    prep_kernel<int16_t, __nv_bfloat16><<<grid, 128, 0, st>>>(
        g, nbins, prompts, randoms, norm, atten, scatter, npskip, eps2, (int16_t *)q_prompts, (__nv_bfloat16 *)q_add,
        (__nv_bfloat16 *)q_mult, quad_mask_accum, ppt, plane0, nplanes, nullptr, sp, sh, 0, 0, 0);
  else
    prep_kernel<int16_t, __half><<<grid, 128, 0, st>>>(
        g, nbins, prompts, randoms, norm, atten, scatter, npskip, eps2, (int16_t *)q_prompts, (__half *)q_add,
        (__half *)q_mult, quad_mask_accum, ppt, plane0, nplanes, nullptr, sp, sh, 0, 0, 0);
  return cudaGetLastError();
}

// SaveImage's layout (drv:4020-4043): out[z][y][x] = image[x][y][z] on FOV
// columns, planes < nz; zero elsewhere.  One thread per (z, y, x), x fastest.
__global__ void image_zyx_kernel(DevGeom g, const float *__restrict__ image, float *__restrict__ out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)g.nz * g.nx * g.nx;
  if (t >= n) return;
  const int x = (int)(t % g.nx), y = (int)((t / g.nx) % g.nx), z = (int)(t / ((long long)g.nx * g.nx));
  const bool in = y >= g.cyl0[x] && y < g.cyl1[x];
  out[t] = in ? __ldg(image + ((size_t)x * g.nx + y) * g.zp + z) : 0.f;
}

cudaError_t launch_image_zyx(const DevGeom &g, const float *image, float *out, cudaStream_t st) {
  const long long n = (long long)g.nz * g.nx * g.nx;
  image_zyx_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, image, out);
  return cudaGetLastError();
}

cudaError_t launch_prep_pairs(const DevGeom &g, int nbins, const int16_t *prompts, const float *randoms,
                              const float *norm, const float *atten, const float *scatter, int npskip, float eps2,
                              int storage, void *q_prompts, void *q_add, void *q_mult, int *quad_mask_accum,
                              const int *pair_views, int npairs, cudaStream_t st, bool flat_prompts) {
  const int ppt = 16;
  dim3 grid((g.nquads + 127) / 128, (g.segmentsize + ppt - 1) / ppt, npairs);
  const long long P = g.segmentsize, sp = nbins, sh = P * nbins, ss = 2 * P * nbins;
  const long long fp = flat_prompts ? (long long)g.nviews * nbins : 0, fh = (long long)(g.nviews / 2) * nbins;
  if (storage == 0)
    prep_kernel<int16_t, float><<<grid, 128, 0, st>>>(g, nbins, prompts, randoms, norm, atten, scatter, npskip, eps2,
                                                      (int16_t *)q_prompts, (float *)q_add, (float *)q_mult,
                                                      quad_mask_accum, ppt, 0, g.segmentsize, pair_views, sp, sh, ss, fp, fh);
  else if (storage == 1)
    prep_kernel<int16_t, __nv_bfloat16><<<grid, 128, 0, st>>>(
        g, nbins, prompts, randoms, norm, atten, scatter, npskip, eps2, (int16_t *)q_prompts, (__nv_bfloat16 *)q_add,
        (__nv_bfloat16 *)q_mult, quad_mask_accum, ppt, 0, g.segmentsize, pair_views, sp, sh, ss, fp, fh);
  else
    prep_kernel<int16_t, __half><<<grid, 128, 0, st>>>(
        g, nbins, prompts, randoms, norm, atten, scatter, npskip, eps2, (int16_t *)q_prompts, (__half *)q_add,
        (__half *)q_mult, quad_mask_accum, ppt, 0, g.segmentsize, pair_views, sp, sh, ss, fp, fh);
  return cudaGetLastError();
}

cudaError_t launch_scale_pairs(const DevGeom &g, const void *src, int storage, const int *views, int npairs,
                               float *dst, long long dst_pair_stride, cudaStream_t st) {
  const long long per = (long long)g.nquads * g.pplanes;
  dim3 grid((unsigned)((per + 255) / 256), npairs);
  if (storage == 0)
    scale_pairs_kernel<float><<<grid, 256, 0, st>>>(g, (const float *)src, views, reinterpret_cast<float4 *>(dst),
                                                    dst_pair_stride / 4);
  else if (storage == 1)
    scale_pairs_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>(g, (const __nv_bfloat16 *)src, views,
                                                            reinterpret_cast<float4 *>(dst), dst_pair_stride / 4);
  else
    scale_pairs_kernel<__half><<<grid, 256, 0, st>>>(g, (const __half *)src, views, reinterpret_cast<float4 *>(dst),
                                                     dst_pair_stride / 4);
  return cudaGetLastError();
}

cudaError_t launch_finish_mask(const DevGeom &g, const int *accum, int16_t *nzmask, cudaStream_t st) {
  const int n = (g.nviews / 2) * g.nquads;
  finish_mask_kernel<<<(n + 255) / 256, 256, 0, st>>>(g, accum, nzmask);
  return cudaGetLastError();
}

cudaError_t launch_init_image(const DevGeom &g, float *image, cudaStream_t st) {
  const long long n = (long long)g.nx * g.nx * g.zp;
  init_image_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, image);
  return cudaGetLastError();
}

cudaError_t launch_post_iteration(const DevGeom &g, float *image, double *partial, double *sum,
                                  const FrameStrides &fr, cudaStream_t st) {
  if (fr.n <= 0) return cudaSuccess;
  const long long n = (long long)g.fov_columns * (g.z_max - g.z_min);
  const int blocks = (int)((n + 255) / 256);
  if (fr.n > 1 && fr.partial < blocks) return cudaErrorInvalidValue;
  post_iter_kernel<<<dim3(blocks, fr.n), 256, 0, st>>>(g, image, partial, fr);
  sum_partials_kernel<<<fr.n, 1024, 0, st>>>(partial, blocks, sum, fr.partial, fr.map);
  return cudaGetLastError();
}

int post_iteration_blocks(const DevGeom &g) {
  const long long n = (long long)g.fov_columns * (g.z_max - g.z_min);
  return (int)((n + 255) / 256);
}

cudaError_t launch_rows_to_quad(const DevGeom &g, int nbins, const float *rows, float *quad, int apply_bp_scale,
                                cudaStream_t st) {
  dim3 grid((g.nquads + 127) / 128, g.segmentsize);
  rows_to_quad_kernel<<<grid, 128, 0, st>>>(g, nbins, rows, reinterpret_cast<float4 *>(quad), apply_bp_scale);
  return cudaGetLastError();
}

cudaError_t launch_quad_to_rows(const DevGeom &g, int nbins, const float *quad, const QuadWork *work, int nwork,
                                float *rows, cudaStream_t st) {
  if (nwork <= 0) return cudaSuccess;
  dim3 grid((g.segmentsize + 255) / 256, nwork);
  quad_to_rows_kernel<<<grid, 256, 0, st>>>(g, nbins, reinterpret_cast<const float4 *>(quad), work, rows);
  return cudaGetLastError();
}

cudaError_t launch_quad_to_file(const DevGeom &g, int nbins, const float *quad, long long quad_pair_stride,
                                const QuadWork *work, int nwork, float *sino, cudaStream_t st) {
  if (nwork <= 0) return cudaSuccess;
  dim3 grid((g.segmentsize + 255) / 256, nwork);
  quad_to_file_kernel<<<grid, 256, 0, st>>>(g, nbins, reinterpret_cast<const float4 *>(quad), quad_pair_stride / 4,
                                            work, sino);
  return cudaGetLastError();
}

cudaError_t launch_add_partials(const DevGeom &g, const float *bc, const float *br, float *out, cudaStream_t st) {
  const long long n4 = (long long)g.nx * g.nx * g.zp / 4;
  add_partials_kernel<<<(unsigned)((n4 + 255) / 256), 256, 0, st>>>(n4, reinterpret_cast<const float4 *>(bc),
                                                                     reinterpret_cast<const float4 *>(br),
                                                                     reinterpret_cast<float4 *>(out));
  return cudaGetLastError();
}

// ============================================================================
// PSF resolution modelling (psf.cpp), on the FOV columns of [x][y][zp] images.
// psf_x_kernel is convolvex (psf.cpp:163-206): taps mask in [-h, h) of the
// x kernel over the x positions inside the FOV of row y, the result divided
// by the sum of the taps used unless that sum is 0 or 1.  psf_yz_kernel is
// convolveyz (psf.cpp:350-460): the same along y (its tap sum kept, not
// applied), then along z over the planes [z_min, z_max) -- with the y
// kernel's taps, as the reference's loop reads them -- scaled by
// norm_z[z] / (y tap sum), norm_z the inverse of the z kernel taps that fall
// inside [z_min, z_max) (host-computed).  One CTA per FOV column, one thread
// per plane; sums in tap order, unfused.
// ============================================================================
__global__ void psf_x_kernel(DevGeom g, const float *__restrict__ in, float *__restrict__ out,
                             const float *__restrict__ filt, int h) {
  const int col = blockIdx.x, z = threadIdx.x;
  if (z >= g.zp) return;
  const short2 xy = g.fov_xy[col];
  const int x = xy.x, y = xy.y, N = g.nx;
  const int lo = g.cyl0[y], hi = g.cyl1[y];
  float acc = 0.f, norm = 0.f;
  for (int mask = -h; mask < h; mask++) {
    const int x2 = x + mask;
    if (x2 < lo || x2 >= hi) continue;
    const float c = __ldg(filt + mask + h);
    norm = norm + c;
    acc = acc + __ldg(in + ((size_t)x2 * N + y) * g.zp + z) * c;
  }
  if (norm != 1.0f && norm != 0.0f) acc = acc * (1.0f / norm);
  out[((size_t)x * N + y) * g.zp + z] = acc;
}

__global__ void psf_yz_kernel(DevGeom g, const float *__restrict__ in, float *__restrict__ out,
                              const float *__restrict__ filty, int h, const float *__restrict__ normz) {
  extern __shared__ float col[];  // [zp] the y-convolved column
  const int c = blockIdx.x, z = threadIdx.x;
  const short2 xy = g.fov_xy[c];
  const int x = xy.x, y = xy.y, N = g.nx, zp = g.zp;
  const int lo = g.cyl0[x], hi = g.cyl1[x];
  float acc = 0.f, norm = 0.f;
  for (int mask = -h; mask < h; mask++) {
    const int y2 = y + mask;
    if (y2 < lo || y2 >= hi) continue;
    const float f = __ldg(filty + mask + h);
    norm = norm + f;
    if (z < zp) acc = acc + __ldg(in + ((size_t)x * N + y2) * zp + z) * f;
  }
  if (z < zp) col[z] = acc;
  __syncthreads();
  if (z >= zp) return;
  float o = 0.f;
  if (norm != 0.0f) {
    for (int mask = -h; mask < h; mask++) {
      const int z2 = z + mask;
      if (z2 < g.z_min || z2 >= g.z_max || z >= g.nz) continue;
      o = o + col[z2] * __ldg(filty + mask + h);
    }
    o = o * (__ldg(normz + z) * (1.0f / norm));
  }
  out[((size_t)x * N + y) * zp + z] = o;
}

// The consumers of the correction image once it is a separate volume (the
// PSF path): MODE 0 the OSEM update, MODE 1 the inverse sensitivity; the
// arithmetic of rotback_kernel's modes 0 and 1.  MODE 2: the MAP update of
// pt_cal_updateimage_mapem (je_hrrt_osem3d/hrrt_osem3d.cpp:2031-2073),
// image = min(image_max, image * min(100, max(0.1, corr / (beta * dpf + 1 / nf_inv))))
// with SSE's min/max rule; the reference's _mm_rcp_ps approximation of
// 1 / nf_inv (relative error up to 1.5 * 2^-12) is the exact reciprocal here.
template <int MODE>
__global__ void __launch_bounds__(256) apply_corr_kernel(DevGeom g, const float *__restrict__ corr,
                                                         float *__restrict__ image, float *__restrict__ nf_inv,
                                                         const float *__restrict__ dpf, float beta) {
  const int nq = g.zp / 4;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int col = (int)(t / nq), q = (int)(t - (long long)col * nq);
  if (col >= g.fov_columns) return;
  const short2 xy = g.fov_xy[col];
  const size_t o = ((size_t)xy.x * g.nx + xy.y) * nq + q;
  const float4 acc = reinterpret_cast<const float4 *>(corr)[o];
  if (MODE == 0) {
    float4 *im = reinterpret_cast<float4 *>(image);
    const float4 nf = reinterpret_cast<const float4 *>(nf_inv)[o];
    float4 iv = im[o];
    float a[4] = {acc.x, acc.y, acc.z, acc.w}, b[4] = {iv.x, iv.y, iv.z, iv.w}, n[4] = {nf.x, nf.y, nf.z, nf.w};
#pragma unroll
    for (int l = 0; l < 4; l++) {
      const float lo = (0.01f > a[l]) ? 0.01f : a[l];
      const float cl = (100.0f < lo) ? 100.0f : lo;
      const float u = b[l] * (cl * n[l]);
      b[l] = (g.image_max < u) ? g.image_max : u;
    }
    im[o] = make_float4(b[0], b[1], b[2], b[3]);
  } else if (MODE == 2) {
    float4 *im = reinterpret_cast<float4 *>(image);
    const float4 nf = reinterpret_cast<const float4 *>(nf_inv)[o];
    const float4 dp = reinterpret_cast<const float4 *>(dpf)[o];
    float4 iv = im[o];
    float a[4] = {acc.x, acc.y, acc.z, acc.w}, b[4] = {iv.x, iv.y, iv.z, iv.w}, n[4] = {nf.x, nf.y, nf.z, nf.w},
          d[4] = {dp.x, dp.y, dp.z, dp.w};
#pragma unroll
    for (int l = 0; l < 4; l++) {
      const float den = __fadd_rn(__fmul_rn(beta, d[l]), __frcp_rn(n[l]));
      const float q = __fdiv_rn(a[l], den);
      const float lo = (0.1f > q) ? 0.1f : q;
      const float cl = (100.0f < lo) ? 100.0f : lo;
      const float u = __fmul_rn(b[l], cl);
      b[l] = (g.image_max < u) ? g.image_max : u;
    }
    im[o] = make_float4(b[0], b[1], b[2], b[3]);
  } else {
    float a[4] = {acc.x, acc.y, acc.z, acc.w}, r[4];
#pragma unroll
    for (int l = 0; l < 4; l++) {
      const int z = q * 4 + l;
      r[l] = (z < g.nz && fabsf(a[l]) > g.eps1) ? (1.0f / a[l]) : 0.f;
    }
    reinterpret_cast<float4 *>(nf_inv)[o] = make_float4(r[0], r[1], r[2], r[3]);
  }
}

cudaError_t launch_psf(const DevGeom &g, const float *in, float *tmp, float *out, const float *filt_x, int hx,
                       const float *filt_y, int hy, const float *normz, cudaStream_t st) {
  const int threads = ((g.zp + 31) / 32) * 32;
  psf_x_kernel<<<g.fov_columns, threads, 0, st>>>(g, in, tmp, filt_x, hx);
  psf_yz_kernel<<<g.fov_columns, threads, g.zp * sizeof(float), st>>>(g, tmp, out, filt_y, hy, normz);
  return cudaGetLastError();
}

// ============================================================================
// MAP, technique 1 of je_hrrt_osem3d (-b 1,beta): Green's one-step-late
// prior.  calculate_DPF_image (je_hrrt_osem3d/dpfcalc.c:23-31, :66-85,
// :266-300) and the update pt_cal_updateimage_mapem (hrrt_osem3d.cpp:
// 2031-2073).
//   map_max_kernel : the image maximum over the FOV columns and planes
//                    [0, nz), never below 0 (the float's bits, an unsigned
//                    maximum, order like the values for non-negative floats);
//   map_dpf_kernel : one thread per FOV voxel: delta = (1.2 max) / 20 and,
//                    for 1 <= x < nx-1 and 1 <= z < nz-1, the 6 face and
//                    (times sqrt(0.5)) 12 edge terms tanh((c - n) / delta) =
//                    (e - 1) / (e + 1), e = exp(2 (c - n) / delta), summed in
//                    the source's order in float, combined in double; 0
//                    elsewhere.  e is exp() in double rounded to float, the
//                    correctly rounded value.
//   MAP update     : apply_corr_kernel<2>.
// ============================================================================
__global__ void __launch_bounds__(256) map_max_kernel(DevGeom g, const float *__restrict__ img,
                                                      unsigned int *__restrict__ mx) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned int v = 0;
  if (t < (long long)g.fov_columns * g.nz) {
    const int col = (int)(t / g.nz), z = (int)(t - (long long)col * g.nz);
    const short2 xy = g.fov_xy[col];
    const float f = img[((size_t)xy.x * g.nx + xy.y) * g.zp + z];
    if (f > 0.f) v = __float_as_uint(f);
  }
  v = __reduce_max_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0 && v) atomicMax(mx, v);
}

__device__ __forceinline__ float map_tanh(float r, float delta) {
  const float e = __double2float_rn(exp((double)__fdiv_rn(__fmul_rn(2.0f, r), delta)));
  return __fdiv_rn(__fsub_rn(e, 1.0f), __fadd_rn(e, 1.0f));
}

__global__ void __launch_bounds__(256) map_dpf_kernel(DevGeom g, const float *__restrict__ img,
                                                      const unsigned int *__restrict__ mx, float *__restrict__ dpf) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)g.fov_columns * g.zp) return;
  const int col = (int)(t / g.zp), z = (int)(t - (long long)col * g.zp);
  const short2 xy = g.fov_xy[col];
  const int x = xy.x, y = xy.y, N = g.nx, zp = g.zp;
  float out = 0.f;
  if (x >= 1 && x < N - 1 && z >= 1 && z < g.nz - 1) {
    const float maxpet = __double2float_rn(1.2 * (double)__uint_as_float(*mx));
    const float delta = __double2float_rn((double)maxpet / 20.0);
    auto I = [&](int a, int b, int c) { return __ldg(img + ((size_t)a * N + b) * zp + c); };
    const float c = I(x, y, z);
    float a = map_tanh(__fsub_rn(c, I(x, y, z - 1)), delta);
    a = __fadd_rn(a, map_tanh(__fsub_rn(c, I(x, y, z + 1)), delta));
    a = __fadd_rn(a, map_tanh(__fsub_rn(c, I(x - 1, y, z)), delta));
    a = __fadd_rn(a, map_tanh(__fsub_rn(c, I(x + 1, y, z)), delta));
    a = __fadd_rn(a, map_tanh(__fsub_rn(c, I(x, y - 1, z)), delta));
    a = __fadd_rn(a, map_tanh(__fsub_rn(c, I(x, y + 1, z)), delta));
    float b = map_tanh(__fsub_rn(c, I(x - 1, y, z - 1)), delta);
    b = __fadd_rn(b, map_tanh(__fsub_rn(c, I(x, y - 1, z - 1)), delta));
    b = __fadd_rn(b, map_tanh(__fsub_rn(c, I(x + 1, y, z - 1)), delta));
    b = __fadd_rn(b, map_tanh(__fsub_rn(c, I(x, y + 1, z - 1)), delta));
    b = __fadd_rn(b, map_tanh(__fsub_rn(c, I(x - 1, y - 1, z)), delta));
    b = __fadd_rn(b, map_tanh(__fsub_rn(c, I(x - 1, y + 1, z)), delta));
    b = __fadd_rn(b, map_tanh(__fsub_rn(c, I(x + 1, y - 1, z)), delta));
    b = __fadd_rn(b, map_tanh(__fsub_rn(c, I(x + 1, y + 1, z)), delta));
    b = __fadd_rn(b, map_tanh(__fsub_rn(c, I(x - 1, y, z + 1)), delta));
    b = __fadd_rn(b, map_tanh(__fsub_rn(c, I(x, y - 1, z + 1)), delta));
    b = __fadd_rn(b, map_tanh(__fsub_rn(c, I(x + 1, y, z + 1)), delta));
    b = __fadd_rn(b, map_tanh(__fsub_rn(c, I(x, y + 1, z + 1)), delta));
    out = __double2float_rn(__dadd_rn((double)a, __dmul_rn(0.70710678118654752440, (double)b)));
  }
  dpf[((size_t)x * N + y) * zp + z] = out;
}

cudaError_t launch_map_prior(const DevGeom &g, const float *image, unsigned int *mx, float *dpf, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(mx, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess) return e;
  const long long n1 = (long long)g.fov_columns * g.nz, n2 = (long long)g.fov_columns * g.zp;
  map_max_kernel<<<(unsigned)((n1 + 255) / 256), 256, 0, st>>>(g, image, mx);
  map_dpf_kernel<<<(unsigned)((n2 + 255) / 256), 256, 0, st>>>(g, image, mx, dpf);
  return cudaGetLastError();
}

cudaError_t launch_apply_corr(const DevGeom &g, const float *corr, float *image, float *nf_inv, int mode,
                              cudaStream_t st, const float *dpf, float beta) {
  const long long n = (long long)g.fov_columns * (g.zp / 4);
  const unsigned blocks = (unsigned)((n + 255) / 256);
  if (mode == 0)
    apply_corr_kernel<0><<<blocks, 256, 0, st>>>(g, corr, image, nf_inv, nullptr, 0.f);
  else if (mode == 1)
    apply_corr_kernel<1><<<blocks, 256, 0, st>>>(g, corr, image, nf_inv, nullptr, 0.f);
  else
    apply_corr_kernel<2><<<blocks, 256, 0, st>>>(g, corr, image, nf_inv, dpf, beta);
  return cudaGetLastError();
}

}  // namespace hrrt
