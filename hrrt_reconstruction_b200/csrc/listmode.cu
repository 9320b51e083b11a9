// listmode.cu -- HRRT 64-bit listmode histogramming on the device.
//
// The reference (lmhistogram_mp/histogram_mp.cpp, LM_Rebinner_mp.cpp) reads
// the stream in packets of 1 Mi 64-bit events (LM_Reader_mp.hpp:39), decodes
// each packet from its first word -- an out-of-sync word pair advances the
// parse by one word, anything else by two (histogram_mp.cpp:1055-1066) --
// rebins events through a crystal-pair LUT, and increments 16-bit bins in
// stream order until a time tag ends the frame.
//
// Device design.  The word stream is cut into tiles of kTileWords words (a
// tile never straddles a packet); a block of 256 threads owns a tile, each
// thread 16 consecutive words.  Where a thread's parse starts depends on the
// words before it, but only through one bit: whether the previous event
// ended on the thread's first word or ran one word into it.  Each thread
// therefore parses its words twice (entering at offset 0 and at offset 1),
// which yields a 2-state map (entry -> exit) plus the number of time tags
// seen for each entry.  Maps compose associatively, so
//   lm_map_kernel   : block scan -> one composed map per tile;
//   lm_entry_kernel : one thread per packet walks its tiles -> tile entry
//                     offsets and per-tile time-tag offsets;
//   lm_scan_kernel  : exclusive scan of the per-packet tag counts;
//   lm_hist_kernel  : re-derives each thread's entry with the same block
//                     scan, parses its words once, writes the time tags in
//                     stream order and (below the frame limit) adds the
//                     events to the sinograms.
// The frame end is found on the host from the ordered time tags (the clock
// logic of process_tagword, histogram_mp.cpp:225-260); when a frame length
// is given the histogram pass runs after it with the limit.
//
// Bins are 16-bit and wrap (the reference's short sinogram).  Two bins share
// a 32-bit word; an increment of the low half that wraps carries into the
// high half, which the thread that caused it takes back with a second atomic
// -- the sum of all updates is exact modulo 2^16 per bin whatever the order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/hrrt_gpu.h"
#include "lm_tables.h"

namespace {

constexpr int kThreads = 256;
constexpr int kSub = 16;                       // words per thread
constexpr int kTileWords = kThreads * kSub;    // 4096
constexpr long long kPacketWords = 2LL << 20;  // 1 Mi 64-bit events
static_assert(kPacketWords % kTileWords == 0, "tiles must not straddle packets");
constexpr int kSinoPlane = 256 * 288;
// Three ways to the same sinograms.  Direct (the default): 16-bit bins updated
// with atomics whose old value is checked for a carry.  Wide: 32-bit counters
// updated with reductions that return nothing, folded into the 16-bit bins at
// the end.  Partitioned: events scattered by 64 MB partition and added
// partition by partition in L2.  On B200, for 2.5e8 events: direct 14.3 ms,
// wide 17.0 ms (the random read-modify-write of a DRAM sector per event bounds
// both; the wide path adds a clear and a fold of 4-byte counters), partitioned
// 21.0 ms (two extra parses), so the other two run only when asked for.  A
// fourth way, rebinning every event into a 4-byte record in stream order and
// adding the records in a separate pass with 30 registers a thread (eight
// blocks per SM, more adds in flight), measured 19.1 ms: the adds are bound
// by the DRAM sectors they read and write, not by how many are in flight.
constexpr bool kPartitionedByDefault = false;
constexpr long long kPartitionMinWords = 1LL << 24;
constexpr bool kWideByDefault = false;
constexpr long long kWideMinWords = 1LL << 26;
// EWTYPES (geometry_info.h:76) packed two bits per entry: index =
// (ew1 >> 30) << 2 | (ew2 >> 30); 0 prompt, 1 delayed, 2 tag, 3 out of sync
constexpr uint32_t kEwTypes = (3u << 0) | (3u << 2) | (1u << 4) | (0u << 6) | (3u << 8) | (3u << 10) | (2u << 12) |
                              (2u << 14) | 0xFFFF0000u;

struct LmDev {
  const hrrt::LmSol *sol;   // [21][144][144]
  const float *zpos, *zpos2;  // [104]
  const int *segz0, *segzmax, *segzoff;  // [nsegs]
  int nsegs;
  long long sino_size;
  // head curve (HRRT_LM_HEAD_CURVE; null otherwise): prompts / delayed of the
  // events before time tag i (after tag i-1) in ivl[2i], ivl[2i+1]; block
  // singles tags (position, value) appended to sing
  unsigned long long *ivl;
  longlong2 *sing;
  unsigned int *sing_n;
  long long sing_cap;
  // coincidence histogram (HRRT_LM_CRYSTAL_COUNTS; null otherwise): prompt
  // then delayed counts per crystal [layer 2][ring 104][head 8][x 72]
  unsigned int *ccounts;
};

// head pairs of the 20 coincidence combinations (geometry_info.h:68-75)
__constant__ int c_pair_heads[21][2] = {{-1, -1}, {0, 2}, {0, 3}, {0, 4}, {0, 5}, {0, 6}, {1, 3}, {1, 4},
                                        {1, 5},   {1, 6}, {1, 7}, {2, 4}, {2, 5}, {2, 6}, {2, 7}, {3, 5},
                                        {3, 6},   {3, 7}, {4, 6}, {4, 7}, {5, 7}};

enum : int { kStPrompts, kStDelayed, kStTimetags, kStTags, kStInvalid, kStUnmapped, kStDoiOther, kStDoi7, kStResync,
             kStCount };

__device__ __forceinline__ int ewtype(uint32_t ew1, uint32_t ew2) {
  return (kEwTypes >> (2 * (((ew1 >> 30) << 2) | (ew2 >> 30)))) & 3;
}

// A thread's parse summary: bit e of `map` = exit offset when entering at e;
// c0 / c1 = time tags seen when entering at 0 / 1.
struct Sub {
  uint32_t map, c0, c1;
};
__device__ __forceinline__ Sub compose(const Sub &a, const Sub &b) {  // a then b
  const uint32_t a0 = a.map & 1, a1 = (a.map >> 1) & 1;
  Sub h;
  h.map = ((b.map >> a0) & 1) | (((b.map >> a1) & 1) << 1);
  h.c0 = a.c0 + (a0 ? b.c1 : b.c0);
  h.c1 = a.c1 + (a1 ? b.c1 : b.c0);
  return h;
}
__device__ __forceinline__ bool is_timetag(uint32_t ew1, uint32_t ew2) {
  const uint32_t tag = (ew1 & 0xffff) | ((ew2 & 0xffff) << 16);
  return (tag & 0xE0000000u) == 0x80000000u;
}

// Parse positions [s + e, s + kSub) of the staged tile; `pend` is where the
// packet (or the stream) ends, relative to the tile.
__device__ __forceinline__ void sub_parse(const uint32_t *w, int s, int e, int pend, uint32_t &exit_off,
                                          uint32_t &ntags) {
  int pos = s + e;
  ntags = 0;
  while (pos < s + kSub) {
    if (pos + 1 >= pend) {  // the packet's last word has no partner
      exit_off = 0;
      return;
    }
    const uint32_t a = w[pos], b = w[pos + 1];
    const int t = ewtype(a, b);
    if (t == 2 && is_timetag(a, b)) ntags++;
    pos += (t == 3) ? 1 : 2;
  }
  exit_off = (uint32_t)(pos - (s + kSub));
}

__device__ __forceinline__ Sub sub_summary(const uint32_t *w, int s, int pend) {
  Sub r;
  uint32_t x0, x1;
  sub_parse(w, s, 0, pend, x0, r.c0);
  sub_parse(w, s, 1, pend, x1, r.c1);
  r.map = x0 | (x1 << 1);
  return r;
}

__device__ __forceinline__ Sub shfl_up_sub(const Sub &v, int d) {
  Sub o;
  o.map = __shfl_up_sync(0xffffffffu, v.map, d);
  o.c0 = __shfl_up_sync(0xffffffffu, v.c0, d);
  o.c1 = __shfl_up_sync(0xffffffffu, v.c1, d);
  return o;
}

// Inclusive block scan of Sub (composition in thread order); also returns
// the exclusive prefix of this thread.  Identity: map 0b10 (0->0, 1->1).
__device__ void block_scan(Sub v, Sub &incl, Sub &excl, Sub *warp_tot) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  Sub x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const Sub o = shfl_up_sub(x, d);
    if (lane >= d) x = compose(o, x);
  }
  if (lane == 31) warp_tot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    Sub t = lane < kThreads / 32 ? warp_tot[lane] : Sub{2u, 0u, 0u};
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const Sub o = shfl_up_sub(t, d);
      if (lane >= d) t = compose(o, t);
    }
    if (lane < kThreads / 32) warp_tot[lane] = t;  // inclusive over warps
  }
  __syncthreads();
  incl = (wid > 0) ? compose(warp_tot[wid - 1], x) : x;
  const Sub prev_lane = shfl_up_sub(x, 1);
  const Sub in_warp = (lane > 0) ? prev_lane : Sub{2u, 0u, 0u};
  excl = (wid > 0) ? compose(warp_tot[wid - 1], in_warp) : in_warp;
}

// Stage the tile (plus one halo word) in shared memory; returns `pend`.
__device__ __forceinline__ int stage_tile(const uint32_t *__restrict__ words, long long n, long long t0, uint32_t *w) {
  const long long pkt_end = (t0 / kPacketWords + 1) * kPacketWords;
  const long long lim = pkt_end < n ? pkt_end : n;
  const long long avail = lim - t0;
  const int pend = (int)(avail < kTileWords + 1 ? avail : (long long)kTileWords + 1);
  const uint4 *src = reinterpret_cast<const uint4 *>(words + t0);
  const int nvec = (pend >= kTileWords) ? kTileWords / 4 : pend / 4;
  for (int i = threadIdx.x; i < nvec; i += kThreads) reinterpret_cast<uint4 *>(w)[i] = __ldg(src + i);
  for (int i = nvec * 4 + threadIdx.x; i < pend; i += kThreads) w[i] = __ldg(words + t0 + i);
  for (int i = pend + threadIdx.x; i < kTileWords + 1; i += kThreads) w[i] = 0u;
  __syncthreads();
  return pend;
}

__global__ void __launch_bounds__(kThreads) lm_map_kernel(const uint32_t *__restrict__ words, long long n,
                                                          unsigned long long *__restrict__ tile_sum) {
  __shared__ __align__(16) uint32_t w[kTileWords + 4];
  __shared__ Sub wt[32];
  const long long t0 = (long long)blockIdx.x * kTileWords;
  const int pend = stage_tile(words, n, t0, w);
  const Sub v = sub_summary(w, threadIdx.x * kSub, pend);
  Sub incl, excl;
  block_scan(v, incl, excl, wt);
  if (threadIdx.x == kThreads - 1)
    tile_sum[blockIdx.x] = (unsigned long long)incl.map | ((unsigned long long)incl.c0 << 16) |
                           ((unsigned long long)incl.c1 << 40);
}

// One warp per packet: tile entries and tag offsets within the packet.  Each
// lane composes the summaries of its run of tiles, a warp scan gives every
// run its entry (a packet is parsed from its first word: entry 0) and tag
// offset, and the lane walks its run again to write them.
constexpr int kEntryThreads = 128;
__global__ void __launch_bounds__(kEntryThreads) lm_entry_kernel(const unsigned long long *__restrict__ tile_sum,
                                                                 long long ntiles, int tiles_per_packet,
                                                                 long long npackets, uint8_t *__restrict__ tile_entry,
                                                                 unsigned int *__restrict__ tile_tagoff,
                                                                 unsigned long long *__restrict__ packet_tags) {
  const long long p = ((long long)blockIdx.x * kEntryThreads + threadIdx.x) >> 5;  // the same in the whole warp
  const int lane = threadIdx.x & 31;
  if (p >= npackets) return;
  const long long t_begin = p * tiles_per_packet;
  const long long t_end = min(t_begin + tiles_per_packet, ntiles);
  const int per = (tiles_per_packet + 31) / 32;
  const long long lb = min(t_begin + (long long)lane * per, t_end), le = min(lb + per, t_end);
  auto tile = [](unsigned long long s) {
    return Sub{(uint32_t)(s & 3u), (uint32_t)((s >> 16) & 0xFFFFFF), (uint32_t)((s >> 40) & 0xFFFFFF)};
  };
  Sub run{2u, 0u, 0u};  // identity: 0 -> 0, 1 -> 1
  for (long long t = lb; t < le; t++) run = compose(run, tile(tile_sum[t]));
  Sub incl = run;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const Sub o = shfl_up_sub(incl, d);
    if (lane >= d) incl = compose(o, incl);
  }
  const Sub prev = shfl_up_sub(incl, 1);
  const Sub excl = lane > 0 ? prev : Sub{2u, 0u, 0u};
  uint32_t e = excl.map & 1u;  // entering the packet at offset 0
  unsigned long long off = excl.c0;
  for (long long t = lb; t < le; t++) {
    const unsigned long long s = tile_sum[t];
    tile_entry[t] = (uint8_t)e;
    tile_tagoff[t] = (unsigned int)off;
    off += e ? ((s >> 40) & 0xFFFFFF) : ((s >> 16) & 0xFFFFFF);
    e = (uint32_t)((s >> e) & 1);
  }
  if (lane == 31) packet_tags[p] = incl.c0;
}

// Exclusive scan of the per-packet tag counts (one block).
__global__ void lm_scan_kernel(unsigned long long *__restrict__ v, long long n, unsigned long long *__restrict__ total) {
  __shared__ unsigned long long part[1024];
  const int t = threadIdx.x, T = blockDim.x;
  const long long per = (n + T - 1) / T, b = t * per, e = min(b + per, n);
  unsigned long long s = 0;
  for (long long i = b; i < e; i++) s += v[i];
  part[t] = s;
  __syncthreads();
  if (t == 0) {
    unsigned long long run = 0;
    for (int i = 0; i < T; i++) {
      const unsigned long long x = part[i];
      part[i] = run;
      run += x;
    }
    *total = run;
  }
  __syncthreads();
  unsigned long long run = part[t];
  for (long long i = b; i < e; i++) {
    const unsigned long long x = v[i];
    v[i] = run;
    run += x;
  }
}

__device__ __forceinline__ void bump16(uint32_t *__restrict__ bins, long long addr, bool minus) {
  uint32_t *w = bins + (addr >> 1);
  const uint32_t hi = (uint32_t)(addr & 1);
  const uint32_t inc = minus ? 0xFFFFu : 1u;
  const uint32_t old = atomicAdd(w, inc << (16 * hi));
  if (!hi && (old & 0xFFFFu) + inc > 0xFFFFu) atomicSub(w, 0x10000u);  // undo the carry into the high bin
}

// Tables every histogram block stages in shared memory.
constexpr int kMaxSegs = 64;
struct LmShared {
  float zp[104], zp2[104];                         // m_c_zpos, m_c_zpos2
  int z0[kMaxSegs], zmax[kMaxSegs], zoff[kMaxSegs];  // m_segz0, m_segzmax, m_segzoffset
};

// rebin_event (LM_Rebinner_mp.cpp:188-219) in two halves: the LUT entry of a
// crystal pair, then the address (or -1) from that entry.
__device__ __forceinline__ size_t sol_index(int mp, int al, int ax, int bl, int bx) {
  return ((size_t)mp * 144 + ax + 72 * al) * 144 + bx + 72 * bl;
}
__device__ __forceinline__ long long rebin_address(const LmDev &g, const LmShared &t, const hrrt::LmSol &s, int ay,
                                                   int by) {
  if (s.nsino == -1) return -1;
  const float cay = t.zp2[ay];
  const float dz2 = __fsub_rn(t.zp[by], t.zp[ay]);
  const int plane = (int)__fadd_rn(cay, __fmul_rn(s.z, dz2));
  const float seg = (float)(0.5 + (double)__fmul_rn(dz2, s.d));
  int segnum = (int)seg;
  segnum = (seg < 0) ? 1 - 2 * segnum : 2 * segnum;
  if (segnum >= g.nsegs) return -1;
  if (plane < 0 || plane > 206) return -1;
  if (plane < t.z0[segnum] || plane > t.zmax[segnum]) return -1;
  return (long long)(plane + t.zoff[segnum]) * kSinoPlane + s.nsino;
}

// Partitions of the histogram for the L2-resident pass: 32 Mi bins (64 MB of
// 16-bit bins) each, prompts-side partitions first.
constexpr int kPartShift = 25;
constexpr int kMaxParts = 64;

// Walk one thread's words from its entry offset: count the statistics (kStats),
// record time tags in stream order (when tags != null), and hand every
// histogrammed event to emit(address, sinogram 0/1, subtract) -- the
// coincidence events together, to emit_events(addresses, live, sinogram-1
// and subtract bit masks).  The parse
// runs first and notes where the thread's coincidence events start (at most
// kSub/2 of them); the events are then decoded and rebinned in an unrolled
// pass whose LUT loads are independent of one another.  Emission order does
// not matter: the bins are sums modulo 2^16 and the statistics counts.
template <bool kStats, typename Emit, typename EmitEvents>
__device__ __forceinline__ void walk_events(const LmDev &g, const LmShared &t, const uint32_t *w, int s, int e,
                                            int pend, long long t0, long long limit, int mode, int flags,
                                            uint32_t (&c)[kStCount], unsigned long long tagpos, long long tag_cap,
                                            longlong2 *__restrict__ tags, Emit emit, EmitEvents emit_events) {
  const bool doi = (flags & HRRT_LM_NO_DOI) == 0;
  const bool border = (flags & HRRT_LM_IGNORE_BORDER_CRYSTAL) != 0;
  const int xhigh = border ? 71 : 72;
  uint32_t evmask = 0;  // bit k: an event (below the limit) starts at word s + k
  uint32_t ttmask = 0;  // bit k: a time tag starts at word s + k (head curve)
  const unsigned long long tagpos0 = tagpos;
  int pos = s + e;
  while (pos < s + kSub) {
    if (pos + 1 >= pend) break;
    const long long gp = t0 + pos;
    const uint32_t ew1 = w[pos], ew2 = w[pos + 1];
    const int type = ewtype(ew1, ew2);
    if (type == 3) {
      if (kStats && gp < limit) c[kStResync]++;
      pos += 1;
      continue;
    }
    pos += 2;
    if (type == 2) {
      const uint32_t tag = (ew1 & 0xffff) | ((ew2 & 0xffff) << 16);
      const bool timetag = (tag & 0xE0000000u) == 0x80000000u;
      if (timetag) {
        if (tags && (long long)tagpos < tag_cap) tags[tagpos] = make_longlong2(gp, (long long)tag);
        tagpos++;
        ttmask |= 1u << (pos - 2 - s);
      } else if (tags && g.sing && (tag & 0xE0000000u) == 0xA0000000u) {
        // block singles (process_tagword, histogram_mp.cpp:260-270), in stream order later
        const unsigned int k = atomicAdd(g.sing_n, 1u);
        if ((long long)k < g.sing_cap) g.sing[k] = make_longlong2(gp, (long long)tag);
      }
      if (gp >= limit) continue;
      if (kStats) {
        c[kStTags]++;
        if (timetag) c[kStTimetags]++;
      }
      if (tag & 0x80000000u) continue;
      // a tag value with bit 31 clear reads as an event word
      const bool prompt = (tag & 0x40000000u) != 0;
      if (kStats) {
        if (prompt)
          c[kStPrompts]++;
        else
          c[kStDelayed]++;
        if (g.ivl) atomicAdd(g.ivl + 2 * tagpos + (prompt ? 0 : 1), 1ull);
      }
      const long long addr = tag & 0x3fffffff;
      if (addr < g.sino_size) {
        if (mode == HRRT_LM_PROMPTS_AND_DELAYED)
          emit(addr, prompt ? 0 : 1, false);
        else
          emit(addr, 0, !prompt);
      }
      continue;
    }
    if (gp >= limit) continue;
    evmask |= 1u << (pos - 2 - s);
  }
  if (!evmask) return;
  // coincidence events (rebin_packet, histogram_mp.cpp:1114-1225): decode,
  // reject, LUT entry ...
  constexpr int kEv = kSub / 2;
  size_t idx[kEv];
  uint32_t need = 0, delayed = 0;  // bit k: event k is rebinned / is delayed
  int ays[kEv], bys[kEv];
  uint32_t m = evmask;
#pragma unroll
  for (int k = 0; k < kEv; k++) {
    idx[k] = 0;
    ays[k] = bys[k] = 0;
    if (!m) continue;
    const int p = __ffs(m) - 1;
    m &= m - 1;
    const uint32_t ew1 = w[s + p], ew2 = w[s + p + 1];
    const int type = ewtype(ew1, ew2);
    const int mpe = ((ew1 >> 16) & 7) | (((ew2 >> 16) & 7) << 3);
    const int ax = ew1 & 0xff, ay = (ew1 >> 8) & 0xff, bx = ew2 & 0xff, by = (ew2 >> 8) & 0xff;
    const int doia = doi ? (int)((ew1 >> 22) & 7) : 1, doib = doi ? (int)((ew2 >> 22) & 7) : 1;
    if (mpe < 1 || mpe > 20 || ax >= 72 || ay >= 104 || bx >= 72 || by >= 104) {
      if (kStats) c[kStInvalid]++;
      continue;
    }
    if (doia == 7 || doib == 7) {
      if (kStats) c[kStDoi7]++;
      continue;
    }
    if (doia > 1 || doib > 1) {
      if (kStats) c[kStDoiOther]++;
      continue;
    }
    if (kStats && g.ccounts) {
      // the coincidence histogram counts both crystals of every emission
      // event with DOI 0/1, mapped or not (rebin_packet, histogram_mp.cpp:1212-1223)
      const int ah = c_pair_heads[mpe][0], bh = c_pair_heads[mpe][1];
      unsigned int *cc = g.ccounts + (type ? 119808 : 0);
      atomicAdd(cc + doia * 59904 + ah * 72 + ax + ay * 576, 1u);
      atomicAdd(cc + doib * 59904 + bh * 72 + bx + by * 576, 1u);
    }
    if ((border && (ax * bx == 0 || ax == xhigh || bx == xhigh)) || (mode == HRRT_LM_PROMPTS_ONLY && type != 0)) {
      if (kStats) c[kStUnmapped]++;
      continue;
    }
    idx[k] = sol_index(mpe, doia, ax, doib, bx);
    ays[k] = ay;
    bys[k] = by;
    need |= 1u << k;
    if (type != 0) delayed |= 1u << k;
  }
  // ... the LUT entries, all loads in flight together ...
  hrrt::LmSol sol[kEv];
#pragma unroll
  for (int k = 0; k < kEv; k++)
    if ((need >> k) & 1) sol[k] = g.sol[idx[k]];
  // ... and the addresses, handed over together
  long long addr[kEv];
  uint32_t live = 0, sel = 0, minus = 0;
  // head curve: each event counts towards the interval of the time tags
  // before it, accumulated while the interval stays the same
  unsigned long long hc_iv = ~0ull, hc_p = 0, hc_d = 0;
  uint32_t m2 = evmask;
#pragma unroll
  for (int k = 0; k < kEv; k++) {
    addr[k] = 0;
    const int p = m2 ? __ffs(m2) - 1 : 0;
    if (m2) m2 &= m2 - 1;
    if (!((need >> k) & 1)) continue;
    const long long a = rebin_address(g, t, sol[k], ays[k], bys[k]);
    if (a < 0) {
      if (kStats) c[kStUnmapped]++;
      continue;
    }
    const bool dly = (delayed >> k) & 1;
    if (kStats) {
      if (dly)
        c[kStDelayed]++;
      else
        c[kStPrompts]++;
      if (g.ivl) {
        const unsigned long long iv = tagpos0 + __popc(ttmask & ((1u << p) - 1u));
        if (iv != hc_iv) {
          if (hc_iv != ~0ull) {
            if (hc_p) atomicAdd(g.ivl + 2 * hc_iv, hc_p);
            if (hc_d) atomicAdd(g.ivl + 2 * hc_iv + 1, hc_d);
          }
          hc_iv = iv;
          hc_p = hc_d = 0;
        }
        if (dly)
          hc_d++;
        else
          hc_p++;
      }
    }
    addr[k] = a;
    live |= 1u << k;
    if (mode == HRRT_LM_PROMPTS_AND_DELAYED) {
      if (dly) sel |= 1u << k;
    } else if (dly) {
      minus |= 1u << k;
    }
  }
  if (kStats && g.ivl && hc_iv != ~0ull) {
    if (hc_p) atomicAdd(g.ivl + 2 * hc_iv, hc_p);
    if (hc_d) atomicAdd(g.ivl + 2 * hc_iv + 1, hc_d);
  }
  if (live) emit_events(addr, live, sel, minus);
}

// The direct histogram of a thread's events: every add issued before any
// carry is checked, so the read-modify-writes are in flight together.
template <int kEv>
__device__ __forceinline__ void bump16_events(uint32_t *__restrict__ sino, uint32_t *__restrict__ dly,
                                              const long long (&addr)[kEv], uint32_t live, uint32_t sel,
                                              uint32_t minus) {
  // a high-half bin's carry leaves the 32-bit word (the sum modulo 2^16 the
  // bin keeps), so its add returns nothing; only a low-half bin's old value is
  // needed, to take back a carry into its neighbour
  uint32_t old[kEv];
#pragma unroll
  for (int k = 0; k < kEv; k++) {
    old[k] = 0;
    if (!((live >> k) & 1)) continue;
    uint32_t *w = (((sel >> k) & 1) ? dly : sino) + (addr[k] >> 1);
    const uint32_t inc = ((minus >> k) & 1) ? 0xFFFFu : 1u;
    if (addr[k] & 1)
      atomicAdd(w, inc << 16);
    else
      old[k] = atomicAdd(w, inc);
  }
#pragma unroll
  for (int k = 0; k < kEv; k++) {
    if (!((live >> k) & 1) || (addr[k] & 1)) continue;
    const uint32_t inc = ((minus >> k) & 1) ? 0xFFFFu : 1u;
    if ((old[k] & 0xFFFFu) + inc > 0xFFFFu) atomicSub((((sel >> k) & 1) ? dly : sino) + (addr[k] >> 1), 0x10000u);
  }
}

// kMode 0: time tags only; 1: histogram directly (atomics into the 16-bit
// bins); 2: count events per histogram partition; 3: scatter packed event
// records (address | sinogram << 29 | subtract << 30) partition-major; 4:
// histogram into 32-bit counters with reductions that return nothing (no
// carry to check, so no read-modify-write round trip per event), folded into
// the 16-bit bins afterwards.  Statistics are counted by modes 1, 2 and 4.
#ifndef HRRT_LM_MIN_BLOCKS
#define HRRT_LM_MIN_BLOCKS 3  // 4 and 5 (64 and 48 registers, with spills) measured slower on B200
#endif
template <int kMode>
__global__ void __launch_bounds__(kThreads, HRRT_LM_MIN_BLOCKS) lm_hist_kernel(
    LmDev g, const uint32_t *__restrict__ words, long long n, const uint8_t *__restrict__ tile_entry,
    const unsigned int *__restrict__ tile_tagoff, const unsigned long long *__restrict__ packet_tagoff,
    int tiles_per_packet, long long limit, int mode, int flags, long long tag_cap, longlong2 *__restrict__ tags,
    uint32_t *__restrict__ sino, uint32_t *__restrict__ dly, unsigned long long *__restrict__ stats,
    unsigned long long *__restrict__ part_cursor, uint32_t *__restrict__ records, int parts_per_sino) {
  __shared__ __align__(16) uint32_t w[kTileWords + 4];
  __shared__ Sub wt[32];
  __shared__ LmShared tb;
  __shared__ unsigned long long st[kStCount];
  __shared__ unsigned int pcount[kMaxParts];
  __shared__ unsigned long long pbase[kMaxParts];
  if (threadIdx.x < 104) {
    tb.zp[threadIdx.x] = g.zpos[threadIdx.x];
    tb.zp2[threadIdx.x] = g.zpos2[threadIdx.x];
  }
  if (threadIdx.x < g.nsegs) {
    tb.z0[threadIdx.x] = g.segz0[threadIdx.x];
    tb.zmax[threadIdx.x] = g.segzmax[threadIdx.x];
    tb.zoff[threadIdx.x] = g.segzoff[threadIdx.x];
  }
  if (threadIdx.x < kStCount) st[threadIdx.x] = 0;
  if (threadIdx.x < kMaxParts) pcount[threadIdx.x] = 0;
  const long long tile = blockIdx.x;
  const long long t0 = tile * kTileWords;
  const int pend = stage_tile(words, n, t0, w);
  const int s = threadIdx.x * kSub;
  const Sub v = sub_summary(w, s, pend);
  Sub incl, excl;
  block_scan(v, incl, excl, wt);
  const uint32_t te = tile_entry[tile];
  const int e = (int)((excl.map >> te) & 1);
  const unsigned long long tagpos =
      packet_tagoff[tile / tiles_per_packet] + tile_tagoff[tile] + (te ? excl.c1 : excl.c0);
  longlong2 *tg = tag_cap > 0 ? tags : nullptr;
  uint32_t c[kStCount] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  auto part_of = [&](long long addr, int sel) { return sel * parts_per_sino + (int)(addr >> kPartShift); };
  // a per-event emitter applied to every event of a thread's batch
  auto each = [](auto f) {
    return [f](const auto &a, uint32_t live, uint32_t sel, uint32_t minus) {
#pragma unroll
      for (int k = 0; k < kSub / 2; k++)
        if ((live >> k) & 1) f(a[k], (int)((sel >> k) & 1), ((minus >> k) & 1) != 0);
    };
  };
  if (kMode == 0) {
    auto none = [](long long, int, bool) {};
    walk_events<false>(g, tb, w, s, e, pend, t0, limit, mode, flags, c, tagpos, tag_cap, tg, none, each(none));
  } else if (kMode == 1) {
    walk_events<true>(g, tb, w, s, e, pend, t0, limit, mode, flags, c, tagpos, tag_cap, tg,
                      [&](long long addr, int sel, bool minus) { bump16(sel ? dly : sino, addr, minus); },
                      [&](const long long (&a)[kSub / 2], uint32_t live, uint32_t sel, uint32_t minus) {
                        bump16_events<kSub / 2>(sino, dly, a, live, sel, minus);
                      });
  } else if (kMode == 4) {
    int *cs = reinterpret_cast<int *>(records), *cd = cs + g.sino_size;
    auto wide = [&](long long addr, int sel, bool minus) { atomicAdd((sel ? cd : cs) + addr, minus ? -1 : 1); };
    walk_events<true>(g, tb, w, s, e, pend, t0, limit, mode, flags, c, tagpos, tag_cap, tg, wide, each(wide));
  } else if (kMode == 2) {
    auto count = [&](long long addr, int sel, bool) { atomicAdd(&pcount[part_of(addr, sel)], 1u); };
    walk_events<true>(g, tb, w, s, e, pend, t0, limit, mode, flags, c, tagpos, tag_cap, tg, count, each(count));
    __syncthreads();
    if (threadIdx.x < 2 * parts_per_sino && pcount[threadIdx.x])
      atomicAdd(&part_cursor[threadIdx.x], (unsigned long long)pcount[threadIdx.x]);
  } else {
    auto count = [&](long long addr, int sel, bool) { atomicAdd(&pcount[part_of(addr, sel)], 1u); };
    walk_events<false>(g, tb, w, s, e, pend, t0, limit, mode, flags, c, tagpos, 0, nullptr, count, each(count));
    __syncthreads();
    if (threadIdx.x < 2 * parts_per_sino) {
      const unsigned int k = pcount[threadIdx.x];
      pbase[threadIdx.x] = k ? atomicAdd(&part_cursor[threadIdx.x], (unsigned long long)k) : 0ull;
      pcount[threadIdx.x] = 0;
    }
    __syncthreads();
    auto scatter = [&](long long addr, int sel, bool minus) {
      const int p = part_of(addr, sel);
      const unsigned int k = atomicAdd(&pcount[p], 1u);
      records[pbase[p] + k] = (uint32_t)addr | ((uint32_t)sel << 29) | ((uint32_t)minus << 30);
    };
    walk_events<false>(g, tb, w, s, e, pend, t0, limit, mode, flags, c, tagpos, 0, nullptr, scatter,
                       each(scatter));
  }
  if (kMode == 1 || kMode == 2 || kMode == 4) {
    // block reduction of the counters
#pragma unroll
    for (int k = 0; k < kStCount; k++) {
      uint32_t x = c[k];
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
      if ((threadIdx.x & 31) == 0 && x) atomicAdd(&st[k], (unsigned long long)x);
    }
    __syncthreads();
    if (threadIdx.x < kStCount && st[threadIdx.x]) atomicAdd(&stats[threadIdx.x], st[threadIdx.x]);
  }
}

// Partition counts -> start offsets (exclusive scan; one thread, <= 64 entries).
__global__ void lm_part_scan_kernel(unsigned long long *__restrict__ cursor, int nparts,
                                    unsigned long long *__restrict__ starts) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  unsigned long long run = 0;
  for (int p = 0; p < nparts; p++) {
    const unsigned long long k = cursor[p];
    starts[p] = run;
    cursor[p] = run;
    run += k;
  }
  starts[nparts] = run;
}

// The records in partition order, contiguous chunks per block: the blocks
// resident at any moment touch one or two 64 MB partitions, which stay in L2.
constexpr int kRecPerThread = 16;
__global__ void __launch_bounds__(kThreads) lm_part_hist_kernel(const uint32_t *__restrict__ records,
                                                                const unsigned long long *__restrict__ total,
                                                                uint32_t *__restrict__ sino, uint32_t *__restrict__ dly) {
  const unsigned long long n = *total;
  const unsigned long long b0 = (unsigned long long)blockIdx.x * kThreads * kRecPerThread;
#pragma unroll 4
  for (int k = 0; k < kRecPerThread; k++) {
    const unsigned long long i = b0 + (unsigned long long)k * kThreads + threadIdx.x;
    if (i >= n) break;
    const uint32_t r = __ldg(records + i);
    bump16(((r >> 29) & 1) ? dly : sino, r & 0x1FFFFFFFu, ((r >> 30) & 1) != 0);
  }
}

// Smoothed randoms: compute_delays (gen_delays_lib/gen_delays_lib.cpp:89-153)
// for every head pair at once.  Thread = (head pair, crystal A (layer, y, x),
// layer of crystal B, run of 8 crystal-B x positions); for each B crystal and
// every B ring within maxrd + 6 rings of A the crystal pair is rebinned
// exactly as an event is (rebin_address) and singles(A) * singles(B) * 2 tau
// * T is added to its bin.  Crystal A's singles use the index of
// gen_delays_fromarchive.cpp:191 (layer, y, head, x): the library copy at
// gen_delays_lib.cpp:117 multiplies y by a whole layer and reads past the
// singles array.
constexpr int kDelayBxRun = 8;
__global__ void __launch_bounds__(128) lm_delays_kernel(LmDev g, const float *__restrict__ csings, float tauftime,
                                                        int maxrd, float *__restrict__ out) {
  __shared__ LmShared tb;
  if (threadIdx.x < 104) {
    tb.zp[threadIdx.x] = g.zpos[threadIdx.x];
    tb.zp2[threadIdx.x] = g.zpos2[threadIdx.x];
  }
  if (threadIdx.x < g.nsegs) {
    tb.z0[threadIdx.x] = g.segz0[threadIdx.x];
    tb.zmax[threadIdx.x] = g.segzmax[threadIdx.x];
    tb.zoff[threadIdx.x] = g.segzoff[threadIdx.x];
  }
  __syncthreads();
  constexpr int kRuns = 72 / kDelayBxRun;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int run = (int)(t % kRuns);
  t /= kRuns;
  const int bl = (int)(t % 2);
  t /= 2;
  const int ax = (int)(t % 72);
  t /= 72;
  const int ay = (int)(t % 104);
  t /= 104;
  const int al = (int)(t % 2);
  const int mp = (int)(t / 2) + 1;
  if (mp > 20) return;
  const int ahead = c_pair_heads[mp][0], bhead = c_pair_heads[mp][1];
  const float awt = csings[al * 59904 + ay * 576 + ahead * 72 + ax] * tauftime;
  if (awt == 0) return;
  // B rings with |ay - by| < maxrd + 6
  const int bs = max(0, ay - (maxrd + 5)), be = min(103, ay + maxrd + 5);
  for (int bx = run * kDelayBxRun; bx < (run + 1) * kDelayBxRun; bx++) {
    const hrrt::LmSol sol = g.sol[sol_index(mp, al, ax, bl, bx)];
    if (sol.nsino == -1) continue;
    const float *sb = csings + bl * 59904 + bhead * 72 + bx;
    for (int by = bs; by <= be; by++) {
      const long long a = rebin_address(g, tb, sol, ay, by);
      if (a >= 0) atomicAdd(out + a, sb[576 * by] * awt);
    }
  }
}

// The 32-bit counts of mode 4 added into the 16-bit bins modulo 2^16 (the
// reference's short bins wrap the same way), two bins (one 32-bit word) per
// thread.
__global__ void lm_fold_kernel(const int2 *__restrict__ counts, uint32_t *__restrict__ bins, long long npairs) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npairs) return;
  const int2 c = counts[i];
  const uint32_t b = bins[i];
  const uint32_t lo = (b + (uint32_t)c.x) & 0xFFFFu, hi = ((b >> 16) + (uint32_t)c.y) & 0xFFFFu;
  bins[i] = lo | (hi << 16);
}

// The span-3 -> span-9 fold of the trues sinogram (convert_span9 after the
// prompts - delayed subtraction of write_sino, lmhistogram_mp.cpp:650-676):
// one thread per 8 bins (16 bytes) of a span-9 plane adds, in 16-bit lanes
// that wrap like the reference's shorts, prompts - delayed of the plane's
// (up to three) span-3 source planes.  Grid: x over the 9216 16-byte words
// of a plane, y over the span-9 planes.  HBM-bound: 16 B read per source
// plane and input, 16 B written.
__global__ void __launch_bounds__(256) lm_span9_kernel(const uint4 *__restrict__ prompts,
                                                       const uint4 *__restrict__ delayed,
                                                       const int4 *__restrict__ src, uint4 *__restrict__ out) {
  constexpr int kWords = 256 * 288 / 8;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kWords) return;
  const int4 s = src[blockIdx.y];
  const int sp[3] = {s.x, s.y, s.z};
  uint4 acc = make_uint4(0, 0, 0, 0);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (sp[k] < 0) continue;
    const size_t at = (size_t)sp[k] * kWords + i;
    uint4 v = __ldcs(prompts + at);
    if (delayed) {
      const uint4 d = __ldcs(delayed + at);
      v.x = __vsub2(v.x, d.x);
      v.y = __vsub2(v.y, d.y);
      v.z = __vsub2(v.z, d.z);
      v.w = __vsub2(v.w, d.w);
    }
    acc.x = __vadd2(acc.x, v.x);
    acc.y = __vadd2(acc.y, v.y);
    acc.z = __vadd2(acc.z, v.z);
    acc.w = __vadd2(acc.w, v.w);
  }
  __stcs(out + (size_t)blockIdx.y * kWords + i, acc);
}

}  // namespace

// ============================================================================
// C ABI
// ============================================================================
struct hrrt_lm {
  hrrt::LmTables tab;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  LmDev dev{};
  std::vector<void *> allocs;
  // scratch grown on demand
  void *scratch = nullptr;
  size_t scratch_bytes = 0;
  uint32_t *h_words_dev = nullptr;  // host-API staging
  // host API, streamed: two chunk buffers filled on their own stream while
  // the previous chunk is histogrammed (chunk_words: 0 default, < 0 never)
  long long chunk_words = 0;
  uint32_t *chunk_dev[2] = {nullptr, nullptr};
  long long chunk_cap = 0;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_copied[2] = {nullptr, nullptr};
  size_t h_words_cap = 0;
  uint16_t *h_sino_dev = nullptr;   // host-API sinograms (prompts, delayed)
  longlong2 *tagbuf = nullptr;      // ordered time tags (position, value)
  long long tag_cap = 0;
  uint32_t *records = nullptr;      // partitioned path: packed event records
  long long rec_cap = 0;
  // head curve of the last call (HRRT_LM_HEAD_CURVE)
  unsigned long long *ivl = nullptr;
  long long ivl_cap = 0;
  longlong2 *sing = nullptr;
  unsigned int *sing_n = nullptr;
  long long sing_cap = 0;
  unsigned int *ccounts = nullptr;  // coincidence histogram of the last call
  int4 *span9_src = nullptr;        // span-9 plane -> span-3 source planes
  int span9_planes = 0;
  std::vector<hrrt_lm_second> hc;
  std::vector<int> block_rates;
  long long hc_prompts = 0, hc_randoms = 0;
  // clock carried across frames (process_tagword's statics)
  long long current_time = -1, current_time_msec = -1, prev_time = 0;
  int clock_reset = 0;
  ~hrrt_lm() {
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(device);
    for (void *p : allocs) cudaFree(p);
    if (scratch) cudaFree(scratch);
    if (tagbuf) cudaFree(tagbuf);
    if (records) cudaFree(records);
    if (ivl) cudaFree(ivl);
    if (sing) cudaFree(sing);
    if (sing_n) cudaFree(sing_n);
    if (ccounts) cudaFree(ccounts);
    if (span9_src) cudaFree(span9_src);
    if (h_words_dev) cudaFree(h_words_dev);
    for (int b = 0; b < 2; b++) {
      if (chunk_dev[b]) cudaFree(chunk_dev[b]);
      if (ev_copied[b]) cudaEventDestroy(ev_copied[b]);
    }
    if (copy_stream) cudaStreamDestroy(copy_stream);
    if (h_sino_dev) cudaFree(h_sino_dev);
    if (stream) cudaStreamDestroy(stream);
    cudaSetDevice(cur);
  }
};

namespace {

int lm_fail(hrrt_lm *h, int code, const std::string &m) {
  if (h) h->err = m;
  return code;
}
int lm_cuda(hrrt_lm *h, cudaError_t e, const char *where) {
  return lm_fail(h, HRRT_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

template <typename T>
T *lm_upload(hrrt_lm *h, const std::vector<T> &v, cudaError_t *e) {
  T *p = nullptr;
  *e = cudaMalloc(&p, sizeof(T) * std::max<size_t>(v.size(), 1));
  if (*e != cudaSuccess) return nullptr;
  h->allocs.push_back(p);
  *e = cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice);
  return p;
}

// process_tagword's time-tag branch (histogram_mp.cpp:225-260) over the
// ordered time tags; returns the index of the tag that ends the frame or -1.
struct ClockState {
  long long time, msec, prev;
  int reset;
};

// The head curve and block singles of one frame (process_tagword,
// histogram_mp.cpp:225-303, replayed in stream order from the clock as the
// frame found it): at every change of second a record (time in ms, prompts
// and delayed events since the previous record, the sum over blocks of their
// latest singles sample), the singles tags updating each block's latest
// sample, total and sample count.  ivl[2i], ivl[2i+1]: the events before time
// tag i; sing: (position, tag) of the block singles tags.
void build_head_curve(hrrt_lm *h, ClockState c, long long frame_start, const std::vector<longlong2> &tags,
                      long long end_tag, const std::vector<unsigned long long> &ivl, std::vector<longlong2> sing,
                      int duration, int flags, long long limit) {
  constexpr int kBlocks = 936;  // GeometryInfo::NBLOCKS
  std::sort(sing.begin(), sing.end(), [](const longlong2 &a, const longlong2 &b) { return a.x < b.x; });
  struct Blk {
    long long last = 0, total = 0, n = 0;
  };
  std::vector<Blk> blk(kBlocks);
  auto take = [&](uint32_t tag) {
    const int b = (int)((tag & 0x1ff80000u) >> 19);
    if (b >= 0 && b < kBlocks) {
      blk[b].last = tag & 0x0007ffff;
      blk[b].total += tag & 0x0007ffff;
      blk[b].n++;
    }
  };
  h->hc.clear();
  long long pacc = 0, racc = 0, tp = 0, tr = 0;
  size_t si = 0;
  const long long n = (long long)tags.size(), last = end_tag >= 0 ? end_tag : n - 1;
  for (long long i = 0; i <= last; i++) {
    pacc += (long long)ivl[2 * i];
    racc += (long long)ivl[2 * i + 1];
    while (si < sing.size() && sing[si].x < tags[i].x) take((uint32_t)sing[si++].y);
    const uint32_t tag = (uint32_t)tags[i].y;
    if (flags & HRRT_LM_TIME_FROM_COUNT)
      c.msec++;
    else
      c.msec = tag & 0x3fffffff;
    if (c.prev > c.msec && !c.reset) {
      c.time = c.msec / 1000;
      c.reset = 1;
      continue;
    }
    c.prev = c.msec;
    if (c.time != c.msec / 1000) {
      long long singles = 0;
      for (const Blk &b : blk) singles += b.last;
      h->hc.push_back(hrrt_lm_second{c.msec, pacc, racc, singles});
      tp += pacc;
      tr += racc;
      pacc = racc = 0;
      c.time = c.msec / 1000;
      if (frame_start < 0) frame_start = c.time;
      if (duration > 0 && c.time - frame_start >= duration) break;
    }
  }
  if (end_tag < 0)  // the frame ran to the end of the stream
    while (si < sing.size() && sing[si].x < limit) take((uint32_t)sing[si++].y);
  h->block_rates.assign(kBlocks, 0);
  for (int b = 0; b < kBlocks; b++) h->block_rates[b] = blk[b].n ? (int)(blk[b].total / blk[b].n) : 0;
  h->hc_prompts = tp;
  h->hc_randoms = tr;
}

long long replay_clock(hrrt_lm *h, const longlong2 *tags, long long ntags, int duration, int flags,
                       long long *frame_start) {
  for (long long i = 0; i < ntags; i++) {
    const uint32_t tag = (uint32_t)tags[i].y;
    if (flags & HRRT_LM_TIME_FROM_COUNT)
      h->current_time_msec++;
    else
      h->current_time_msec = tag & 0x3fffffff;
    if (h->prev_time > h->current_time_msec && !h->clock_reset) {
      h->current_time = h->current_time_msec / 1000;
      h->clock_reset = 1;
      continue;
    }
    h->prev_time = h->current_time_msec;
    if (h->current_time != h->current_time_msec / 1000) {
      h->current_time = h->current_time_msec / 1000;
      if (*frame_start < 0) *frame_start = h->current_time;
      if (duration > 0 && h->current_time - *frame_start >= duration) return i;
    }
  }
  return -1;
}

}  // namespace

extern "C" {

int hrrt_lm_create(int span, int maxrd, int device, hrrt_lm **out) {
  if (!out) return HRRT_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<hrrt_lm> h(new hrrt_lm());
  std::string m = h->tab.build(span, maxrd);
  if (!m.empty()) {
    hrrt_lm *raw = h.release();
    raw->err = m;
    *out = raw;
    return HRRT_ERR_ARG;
  }
  h->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  LmDev &d = h->dev;
  if (e == cudaSuccess) d.sol = lm_upload(h.get(), h->tab.sol, &e);
  if (e == cudaSuccess) d.zpos = lm_upload(h.get(), h->tab.zpos, &e);
  if (e == cudaSuccess) d.zpos2 = lm_upload(h.get(), h->tab.zpos2, &e);
  if (e == cudaSuccess) d.segz0 = lm_upload(h.get(), h->tab.segz0, &e);
  if (e == cudaSuccess) d.segzmax = lm_upload(h.get(), h->tab.segzmax, &e);
  if (e == cudaSuccess) d.segzoff = lm_upload(h.get(), h->tab.segzoffset, &e);
  d.nsegs = h->tab.nsegs;
  if (d.nsegs > kMaxSegs) {
    hrrt_lm *raw = h.release();
    raw->err = "hrrt_lm_create: too many segments";
    *out = raw;
    return HRRT_ERR_ARG;
  }
  d.sino_size = h->tab.sino_size();
  if (e != cudaSuccess) {
    hrrt_lm *raw = h.release();
    lm_cuda(raw, e, "hrrt_lm_create");
    *out = raw;
    return HRRT_ERR_CUDA;
  }
  *out = h.release();
  return HRRT_OK;
}

void hrrt_lm_destroy(hrrt_lm *h) { delete h; }

const char *hrrt_lm_last_error(const hrrt_lm *h) { return h ? h->err.c_str() : "null listmode context"; }

long long hrrt_lm_sino_size(const hrrt_lm *h) { return h ? h->tab.sino_size() : -1; }

void *hrrt_lm_get_stream(const hrrt_lm *h) { return h ? (void *)h->stream : nullptr; }

int hrrt_lm_reset_clock(hrrt_lm *h) {
  if (!h) return HRRT_ERR_ARG;
  h->current_time = -1;
  h->current_time_msec = -1;
  h->prev_time = 0;
  h->clock_reset = 0;
  return HRRT_OK;
}

}  // extern "C"

namespace {

// One histogram call over d_words.  *frame_start_io carries the frame's start
// (s, -1 before the first time tag) into and out of the call, so that the
// chunks of one frame can be histogrammed call by call; `last`: the words end
// the stream here, so an unterminated frame takes its rounded end time
// (histogram_mp.cpp:1390-1396).
int lm_hist_call(hrrt_lm *h, const uint32_t *d_words, long long nwords, int mode, int duration, int flags,
                 uint16_t *d_sino, uint16_t *d_delayed, hrrt_lm_stats *out, void *stream, long long *frame_start_io,
                 bool last) {
  if (!h) return HRRT_ERR_ARG;
  if (nwords < 0 || (nwords > 0 && !d_words) || !d_sino || !out)
    return lm_fail(h, HRRT_ERR_ARG, "hrrt_lm_histogram: null buffer or negative length");
  if (mode != HRRT_LM_TRUES && mode != HRRT_LM_PROMPTS_AND_DELAYED && mode != HRRT_LM_PROMPTS_ONLY)
    return lm_fail(h, HRRT_ERR_ARG, "hrrt_lm_histogram: unknown mode");
  if (mode == HRRT_LM_PROMPTS_AND_DELAYED && !d_delayed)
    return lm_fail(h, HRRT_ERR_ARG, "hrrt_lm_histogram: the delayed sinogram is required in this mode");
  if (((uintptr_t)d_words & 15) || ((uintptr_t)d_sino & 3) || ((uintptr_t)d_delayed & 3))
    return lm_fail(h, HRRT_ERR_ARG, "hrrt_lm_histogram: words need 16-byte, sinograms 4-byte alignment");
  memset(out, 0, sizeof(*out));
  cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return lm_cuda(h, e, "hrrt_lm_histogram");
  long long frame_start = *frame_start_io;
  if (nwords == 0) {
    out->frame_start = frame_start;
    return HRRT_OK;
  }
  const long long ntiles = (nwords + kTileWords - 1) / kTileWords;
  const int tpp = (int)(kPacketWords / kTileWords);
  const long long npackets = (nwords + kPacketWords - 1) / kPacketWords;
  // scratch: tile sums (8), entries (1), tag offsets (4) per tile; packet
  // offsets (8) per packet; stats.  The time tags get their own buffer once
  // the scan has counted them.
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t b_sum = al(8 * ntiles), b_ent = al(ntiles), b_off = al(4 * ntiles), b_pk = al(8 * (npackets + 1)),
               b_st = al(8 * (kStCount + 1 + 2 * kMaxParts + 1));
  const size_t need = b_sum + b_ent + b_off + b_pk + b_st;
  if (h->scratch_bytes < need) {
    if (h->scratch) cudaFree(h->scratch);
    h->scratch = nullptr;
    h->scratch_bytes = 0;
    e = cudaMalloc(&h->scratch, need);
    if (e != cudaSuccess) return lm_fail(h, HRRT_ERR_NOMEM, "hrrt_lm_histogram: scratch");
    h->scratch_bytes = need;
  }
  char *p = (char *)h->scratch;
  auto *tile_sum = (unsigned long long *)p;
  auto *tile_entry = (uint8_t *)(p + b_sum);
  auto *tile_tagoff = (unsigned int *)(p + b_sum + b_ent);
  auto *pk = (unsigned long long *)(p + b_sum + b_ent + b_off);
  auto *stats = (unsigned long long *)(p + b_sum + b_ent + b_off + b_pk);
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEventCreate(&ev0);
  cudaEventCreate(&ev1);
  cudaEventRecord(ev0, st);
  e = cudaMemsetAsync(stats, 0, 8 * (kStCount + 1), st);
  if (e == cudaSuccess) {
    lm_map_kernel<<<(unsigned)ntiles, kThreads, 0, st>>>(d_words, nwords, tile_sum);
    lm_entry_kernel<<<(unsigned)((npackets * 32 + kEntryThreads - 1) / kEntryThreads), kEntryThreads, 0, st>>>(
        tile_sum, ntiles, tpp, npackets, tile_entry, tile_tagoff, pk);
    lm_scan_kernel<<<1, 1024, 0, st>>>(pk, npackets, stats + kStCount);
    e = cudaGetLastError();
  }
  unsigned long long ntags = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&ntags, stats + kStCount, 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess && (long long)ntags > h->tag_cap) {
    if (h->tagbuf) cudaFree(h->tagbuf);
    h->tagbuf = nullptr;
    h->tag_cap = 0;
    const long long cap = std::max<long long>((long long)ntags, 1024);
    e = cudaMalloc(&h->tagbuf, sizeof(longlong2) * (size_t)cap);
    if (e != cudaSuccess) {
      h->tagbuf = nullptr;
      cudaEventDestroy(ev0);
      cudaEventDestroy(ev1);
      return lm_fail(h, HRRT_ERR_NOMEM, "hrrt_lm_histogram: time tags");
    }
    h->tag_cap = cap;
  }
  longlong2 *tags = h->tagbuf;
  const long long tag_cap = h->tag_cap;
  // Histogram path: directly (atomics into the full sinograms) for short
  // streams, partitioned (events scattered by 64 MB partition, then
  // histogrammed partition by partition in L2) for long ones.
  const int pps = (int)((h->dev.sino_size + (1LL << kPartShift) - 1) >> kPartShift);
  bool partitioned = kPartitionedByDefault && nwords >= kPartitionMinWords;
  bool wide = kWideByDefault && nwords >= kWideMinWords;
  if (flags & HRRT_LM_FORCE_DIRECT) partitioned = wide = false;
  if (flags & HRRT_LM_FORCE_PARTITIONED) {
    partitioned = true;
    wide = false;
  }
  if (flags & HRRT_LM_FORCE_WIDE) {
    wide = true;
    partitioned = false;
  }
  if (2 * pps > kMaxParts) partitioned = false;
  unsigned long long *cursor = stats + kStCount + 1;          // [kMaxParts]
  unsigned long long *starts = cursor + kMaxParts;            // [kMaxParts + 1]
  if ((partitioned || wide) && e == cudaSuccess) {
    // partitioned: one packed record per event; wide: 32-bit counters for
    // both sinograms
    const long long cap = partitioned ? nwords / 2 + 1 : 2 * h->dev.sino_size;
    if (cap > h->rec_cap) {
      if (h->records) cudaFree(h->records);
      h->records = nullptr;
      h->rec_cap = 0;
      e = cudaMalloc(&h->records, sizeof(uint32_t) * (size_t)cap);
      if (e != cudaSuccess) {
        h->records = nullptr;
        partitioned = wide = false;  // not enough memory: fall back to the direct path
        e = cudaSuccess;
        cudaGetLastError();
      } else {
        h->rec_cap = cap;
      }
    }
  }
  if (partitioned && e == cudaSuccess) e = cudaMemsetAsync(cursor, 0, 8 * kMaxParts, st);
  if (wide && e == cudaSuccess) e = cudaMemsetAsync(h->records, 0, sizeof(uint32_t) * 2 * h->dev.sino_size, st);
  LmDev dv = h->dev;  // this call's copy: the head-curve buffers when asked for
  auto launch = [&](int kmode, long long lim, long long tcap) {
    const unsigned nb = (unsigned)ntiles;
    uint32_t *sn = (uint32_t *)d_sino, *dl = (uint32_t *)d_delayed;
    switch (kmode) {
      case 0:
        lm_hist_kernel<0><<<nb, kThreads, 0, st>>>(dv, d_words, nwords, tile_entry, tile_tagoff, pk, tpp, lim,
                                                   mode, flags, tcap, tags, sn, dl, stats, cursor, h->records, pps);
        break;
      case 1:
        lm_hist_kernel<1><<<nb, kThreads, 0, st>>>(dv, d_words, nwords, tile_entry, tile_tagoff, pk, tpp, lim,
                                                   mode, flags, tcap, tags, sn, dl, stats, cursor, h->records, pps);
        break;
      case 2:
        lm_hist_kernel<2><<<nb, kThreads, 0, st>>>(dv, d_words, nwords, tile_entry, tile_tagoff, pk, tpp, lim,
                                                   mode, flags, tcap, tags, sn, dl, stats, cursor, h->records, pps);
        break;
      case 4:
        lm_hist_kernel<4><<<nb, kThreads, 0, st>>>(dv, d_words, nwords, tile_entry, tile_tagoff, pk, tpp, lim,
                                                   mode, flags, tcap, tags, sn, dl, stats, cursor, h->records, pps);
        break;
      default:
        lm_hist_kernel<3><<<nb, kThreads, 0, st>>>(dv, d_words, nwords, tile_entry, tile_tagoff, pk, tpp, lim,
                                                   mode, flags, tcap, tags, sn, dl, stats, cursor, h->records, pps);
    }
    return cudaGetLastError();
  };
  // pass 1: the ordered time tags (and, without a frame length, the counts
  // or the histogram itself)
  // head curve: the tags pass also collects the block singles tags, and the
  // histogram pass counts events per time-tag interval
  const bool hc = (flags & HRRT_LM_HEAD_CURVE) != 0;
  if (hc && e == cudaSuccess) {
    auto grow = [&](void **p, long long *cap, long long want, size_t elem) {
      if (want <= *cap) return cudaSuccess;
      if (*p) cudaFree(*p);
      *p = nullptr;
      *cap = 0;
      cudaError_t r = cudaMalloc(p, elem * (size_t)want);
      if (r == cudaSuccess) *cap = want;
      return r;
    };
    e = grow((void **)&h->ivl, &h->ivl_cap, 2 * ((long long)ntags + 1), sizeof(unsigned long long));
    if (e == cudaSuccess) e = grow((void **)&h->sing, &h->sing_cap, std::max<long long>(4096, 2 * (long long)ntags), 16);
    if (e == cudaSuccess && !h->sing_n) e = cudaMalloc(&h->sing_n, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemsetAsync(h->ivl, 0, sizeof(unsigned long long) * 2 * (ntags + 1), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->sing_n, 0, sizeof(unsigned int), st);
    dv.sing = h->sing;
    dv.sing_n = h->sing_n;
    dv.sing_cap = h->sing_cap;
  }
  if ((flags & HRRT_LM_CRYSTAL_COUNTS) && e == cudaSuccess) {
    if (!h->ccounts) e = cudaMalloc(&h->ccounts, sizeof(unsigned int) * 2 * hrrt::kCrystals);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->ccounts, 0, sizeof(unsigned int) * 2 * hrrt::kCrystals, st);
  }
  const bool one_pass = duration <= 0 && !hc;
  const int hist_mode = partitioned ? 2 : (wide ? 4 : 1);
  if (one_pass && (flags & HRRT_LM_CRYSTAL_COUNTS)) dv.ccounts = h->ccounts;
  if (e == cudaSuccess) e = launch(one_pass ? hist_mode : 0, one_pass ? nwords : -1, tag_cap);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  unsigned int nsing = 0;
  if (hc && e == cudaSuccess) {
    e = cudaMemcpy(&nsing, h->sing_n, sizeof(unsigned int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && (long long)nsing > h->sing_cap) {  // more singles tags than room: again, sized
      cudaFree(h->sing);
      h->sing = nullptr;
      h->sing_cap = 0;
      e = cudaMalloc(&h->sing, 16 * (size_t)nsing);
      if (e == cudaSuccess) {
        h->sing_cap = nsing;
        dv.sing = h->sing;
        dv.sing_cap = h->sing_cap;
        e = cudaMemsetAsync(h->sing_n, 0, sizeof(unsigned int), st);
        if (e == cudaSuccess) e = launch(0, -1, tag_cap);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      }
    }
    dv.sing = nullptr;
    dv.ivl = h->ivl;
  }
  // the crystal counts are taken in the histogram pass only
  auto hist_dev = [&]() {
    if (flags & HRRT_LM_CRYSTAL_COUNTS) dv.ccounts = h->ccounts;
  };
  std::vector<longlong2> htags;
  if (e == cudaSuccess && ntags > 0) {
    htags.resize(ntags);
    e = cudaMemcpyAsync(htags.data(), tags, 16 * ntags, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  if (e != cudaSuccess) {
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    return lm_cuda(h, e, "hrrt_lm_histogram");
  }
  const ClockState clock0{h->current_time, h->current_time_msec, h->prev_time, h->clock_reset};
  const long long frame_start0 = frame_start;
  const long long end_tag = replay_clock(h, htags.data(), (long long)ntags, duration, flags, &frame_start);
  long long limit = nwords;
  if (end_tag >= 0) limit = htags[end_tag].x;
  if (!one_pass) {
    hist_dev();
    e = launch(hist_mode, limit, 0);
  }
  if (wide && e == cudaSuccess) {
    const long long np = h->dev.sino_size / 2;  // bin pairs (sinogram sizes are multiples of 4)
    const unsigned nb = (unsigned)((np + 255) / 256);
    const int2 *cs = reinterpret_cast<const int2 *>(h->records);
    lm_fold_kernel<<<nb, 256, 0, st>>>(cs, (uint32_t *)d_sino, np);
    if (mode == HRRT_LM_PROMPTS_AND_DELAYED) lm_fold_kernel<<<nb, 256, 0, st>>>(cs + np, (uint32_t *)d_delayed, np);
    e = cudaGetLastError();
  }
  if (partitioned && e == cudaSuccess) {
    lm_part_scan_kernel<<<1, 32, 0, st>>>(cursor, 2 * pps, starts);
    e = launch(3, limit, 0);
    if (e == cudaSuccess) {
      const long long blocks = (nwords / 2 + 1 + (long long)kThreads * kRecPerThread - 1) / ((long long)kThreads * kRecPerThread);
      lm_part_hist_kernel<<<(unsigned)blocks, kThreads, 0, st>>>(h->records, starts + 2 * pps, (uint32_t *)d_sino,
                                                                 (uint32_t *)d_delayed);
      e = cudaGetLastError();
    }
  }
  std::vector<unsigned long long> hivl;
  std::vector<longlong2> hsing;
  if (hc && e == cudaSuccess) {
    hivl.resize(2 * (ntags + 1));
    hsing.resize(nsing);
    e = cudaMemcpyAsync(hivl.data(), h->ivl, 8 * hivl.size(), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && nsing)
      e = cudaMemcpyAsync(hsing.data(), h->sing, 16 * (size_t)nsing, cudaMemcpyDeviceToHost, st);
  }
  unsigned long long hs[kStCount] = {};
  cudaEventRecord(ev1, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hs, stats, 8 * kStCount, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  float ms = 0;
  cudaEventElapsedTime(&ms, ev0, ev1);
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  if (e != cudaSuccess) return lm_cuda(h, e, "hrrt_lm_histogram");
  // the time tags below the limit, and the tag that ends the frame itself
  out->prompts = (long long)hs[kStPrompts];
  out->delayed = (long long)hs[kStDelayed];
  out->timetags = (long long)hs[kStTimetags] + (end_tag >= 0 ? 1 : 0);
  out->tags = (long long)hs[kStTags] + (end_tag >= 0 ? 1 : 0);
  out->invalid = (long long)hs[kStInvalid];
  out->unmapped = (long long)hs[kStUnmapped];
  out->doi_other = (long long)hs[kStDoiOther];
  out->doi7 = (long long)hs[kStDoi7];
  out->resyncs = (long long)hs[kStResync];
  out->terminated = end_tag >= 0;
  out->words_used = end_tag >= 0 ? limit + 2 : nwords;
  if (end_tag < 0 && last) h->current_time = (h->current_time_msec + 500) / 1000;
  *frame_start_io = frame_start;
  out->frame_start = frame_start;
  out->duration = h->current_time - frame_start;
  out->ms = ms;
  if (hc) build_head_curve(h, clock0, frame_start0, htags, end_tag, hivl, std::move(hsing), duration, flags, limit);
  return HRRT_OK;
}

}  // namespace

extern "C" {

int hrrt_lm_histogram_device(hrrt_lm *h, const uint32_t *d_words, long long nwords, int mode, int duration, int flags,
                             uint16_t *d_sino, uint16_t *d_delayed, hrrt_lm_stats *out, void *stream) {
  if (!h) return HRRT_ERR_ARG;
  long long frame_start = h->current_time >= 0 ? h->current_time : -1;
  return lm_hist_call(h, d_words, nwords, mode, duration, flags, d_sino, d_delayed, out, stream, &frame_start, true);
}

int hrrt_lm_head_curve(hrrt_lm *h, hrrt_lm_second *out, int capacity) {
  if (!h) return HRRT_ERR_ARG;
  const int n = (int)h->hc.size();
  if (out)
    for (int i = 0; i < n && i < capacity; i++) out[i] = h->hc[i];
  return n;
}

int hrrt_lm_crystal_counts(hrrt_lm *h, uint32_t *counts) {
  if (!h || !counts) return HRRT_ERR_ARG;
  if (!h->ccounts) return lm_fail(h, HRRT_ERR_STATE, "no call with HRRT_LM_CRYSTAL_COUNTS yet");
  cudaError_t e = cudaSetDevice(h->device);
  if (e == cudaSuccess)
    e = cudaMemcpy(counts, h->ccounts, sizeof(uint32_t) * 2 * hrrt::kCrystals, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return lm_cuda(h, e, "hrrt_lm_crystal_counts");
  return HRRT_OK;
}

int hrrt_lm_block_singles(hrrt_lm *h, int *rates, long long *total_prompts, long long *total_randoms) {
  if (!h) return HRRT_ERR_ARG;
  if (rates)
    for (size_t b = 0; b < h->block_rates.size(); b++) rates[b] = h->block_rates[b];
  if (total_prompts) *total_prompts = h->hc_prompts;
  if (total_randoms) *total_randoms = h->hc_randoms;
  return (int)h->block_rates.size();
}

long long hrrt_lm_table(int span, int maxrd, const char *name, void *out, size_t bytes) {
  if (!name) return HRRT_ERR_ARG;
  hrrt::LmTables t;
  if (!t.build(span, maxrd).empty()) return HRRT_ERR_ARG;
  const void *src = nullptr;
  size_t n = 0;
  const std::string k(name);
  if (k == "sol") {
    src = t.sol.data();
    n = t.sol.size() * sizeof(hrrt::LmSol);
  } else if (k == "zpos") {
    src = t.zpos.data();
    n = t.zpos.size() * sizeof(float);
  } else if (k == "zpos2") {
    src = t.zpos2.data();
    n = t.zpos2.size() * sizeof(float);
  } else if (k == "segz0") {
    src = t.segz0.data();
    n = t.segz0.size() * sizeof(int);
  } else if (k == "segzmax") {
    src = t.segzmax.data();
    n = t.segzmax.size() * sizeof(int);
  } else if (k == "segzoffset") {
    src = t.segzoffset.data();
    n = t.segzoffset.size() * sizeof(int);
  } else {
    return HRRT_ERR_ARG;
  }
  if (out && bytes >= n) std::memcpy(out, src, n);
  return (long long)n;
}

}  // extern "C"

namespace {

constexpr long long kDefaultChunkWords = 32 * kPacketWords;  // 64 Mi words, 256 MB

// hrrt_lm_histogram_at over a long host stream, streamed: chunks of whole
// packets (the first one led by the packet-phase filler) go up on a copy
// stream into two device buffers while the previous chunk is histogrammed.
// The chunks of one frame share its start and the clock; only the chunk that
// ends the stream rounds an unterminated frame's end time, so the result is
// that of one call over the whole stream.
int lm_histogram_chunked(hrrt_lm *h, const uint32_t *words, long long nwords, long long phase, long long C, int mode,
                         int duration, int flags, uint16_t *sino, uint16_t *delayed, hrrt_lm_stats *out) {
  const long long S = h->tab.sino_size();
  cudaError_t e = cudaSuccess;
  if (h->chunk_cap < C) {
    for (int b = 0; b < 2; b++) {
      if (h->chunk_dev[b]) cudaFree(h->chunk_dev[b]);
      h->chunk_dev[b] = nullptr;
    }
    h->chunk_cap = 0;
    for (int b = 0; b < 2 && e == cudaSuccess; b++) e = cudaMalloc(&h->chunk_dev[b], sizeof(uint32_t) * (size_t)C);
    if (e != cudaSuccess) return lm_fail(h, HRRT_ERR_NOMEM, "hrrt_lm_histogram: event chunks");
    h->chunk_cap = C;
  }
  if (!h->copy_stream) {
    e = cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking);
    for (int b = 0; b < 2 && e == cudaSuccess; b++)
      e = cudaEventCreateWithFlags(&h->ev_copied[b], cudaEventDisableTiming);
    if (e != cudaSuccess) return lm_cuda(h, e, "hrrt_lm_histogram: copy stream");
  }
  cudaStream_t st = h->stream, cs = h->copy_stream;
  e = cudaMemsetAsync(h->h_sino_dev, 0, sizeof(uint16_t) * 2 * (size_t)S, st);
  if (e != cudaSuccess) return lm_cuda(h, e, "hrrt_lm_histogram");
  // chunk k holds the caller's words [lo(k), hi(k)); chunk 0 after `phase`
  // filler words
  const long long first = C - phase;
  const int nchunks = (int)(1 + (nwords - first + C - 1) / C);
  auto lo = [&](int k) { return k == 0 ? 0 : first + (long long)(k - 1) * C; };
  auto hi = [&](int k) { return std::min(nwords, k == 0 ? first : first + (long long)k * C); };
  auto issue = [&](int k) {
    const int b = k & 1;
    cudaError_t r = cudaSuccess;
    uint32_t *dst = h->chunk_dev[b];
    if (k == 0 && phase > 0) {
      r = cudaMemsetAsync(dst, 0x80, sizeof(uint32_t) * phase, cs);
      dst += phase;
    }
    if (r == cudaSuccess)
      r = cudaMemcpyAsync(dst, words + lo(k), sizeof(uint32_t) * (hi(k) - lo(k)), cudaMemcpyHostToDevice, cs);
    if (r == cudaSuccess) r = cudaEventRecord(h->ev_copied[b], cs);
    return r;
  };
  memset(out, 0, sizeof(*out));
  long long frame_start = h->current_time >= 0 ? h->current_time : -1;
  int rc = HRRT_OK;
  e = issue(0);
  for (int k = 0; k < nchunks && e == cudaSuccess && rc == HRRT_OK; k++) {
    // the buffer of chunk k + 1 held chunk k - 1, whose call has returned
    if (k + 1 < nchunks) e = issue(k + 1);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, h->ev_copied[k & 1], 0);
    if (e != cudaSuccess) break;
    const long long n = hi(k) - lo(k) + (k == 0 ? phase : 0);
    hrrt_lm_stats c;
    rc = lm_hist_call(h, h->chunk_dev[k & 1], n, mode, duration, flags, h->h_sino_dev, h->h_sino_dev + S, &c, st,
                      &frame_start, k + 1 == nchunks);
    if (rc != HRRT_OK) break;
    out->prompts += c.prompts;
    out->delayed += c.delayed;
    out->timetags += c.timetags;
    out->tags += c.tags;
    out->invalid += c.invalid;
    out->unmapped += c.unmapped;
    out->doi_other += c.doi_other;
    out->doi7 += c.doi7;
    out->resyncs += c.resyncs - (k == 0 ? phase : 0);
    out->ms += c.ms;
    out->frame_start = c.frame_start;
    out->duration = c.duration;
    if (c.terminated) {
      out->terminated = 1;
      out->words_used = lo(k) + c.words_used - (k == 0 ? phase : 0);
      break;
    }
    out->words_used = hi(k);
  }
  const cudaError_t e2 = cudaStreamSynchronize(cs);
  if (rc != HRRT_OK) return rc;
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaMemcpyAsync(sino, h->h_sino_dev, sizeof(uint16_t) * S, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && delayed && mode == HRRT_LM_PROMPTS_AND_DELAYED)
    e = cudaMemcpyAsync(delayed, h->h_sino_dev + S, sizeof(uint16_t) * S, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return lm_cuda(h, e, "hrrt_lm_histogram");
  return HRRT_OK;
}

}  // namespace

extern "C" {

int hrrt_lm_set_chunk(hrrt_lm *h, long long words) {
  if (!h) return HRRT_ERR_ARG;
  if (words > 0 && words % kPacketWords != 0)
    return lm_fail(h, HRRT_ERR_ARG, "hrrt_lm_set_chunk: a chunk is a whole number of 2 Mi-word packets");
  h->chunk_words = words;
  return HRRT_OK;
}

int hrrt_lm_histogram(hrrt_lm *h, const uint32_t *words, long long nwords, int mode, int duration, int flags,
                      uint16_t *sino, uint16_t *delayed, hrrt_lm_stats *out) {
  return hrrt_lm_histogram_at(h, words, nwords, 0, mode, duration, flags, sino, delayed, out);
}

// Packets count from the file start: the staging buffer holds `phase`
// filler words before the caller's words, each a word whose top bits (10)
// make it out of sync whatever follows (EWTYPES, histogram_mp.cpp:1056-1062),
// so the parse steps over them one by one and meets words[0] in sync, where
// the reference's parse stands after the previous frame.  The filler shows
// in no output but the resync count and the words used, which are corrected.
int hrrt_lm_histogram_at(hrrt_lm *h, const uint32_t *words, long long nwords, long long file_offset, int mode,
                         int duration, int flags, uint16_t *sino, uint16_t *delayed, hrrt_lm_stats *out) {
  if (!h) return HRRT_ERR_ARG;
  if (nwords < 0 || file_offset < 0 || (nwords > 0 && !words) || !sino || !out)
    return lm_fail(h, HRRT_ERR_ARG, "hrrt_lm_histogram: null buffer or negative length");
  if (mode == HRRT_LM_PROMPTS_AND_DELAYED && !delayed)
    return lm_fail(h, HRRT_ERR_ARG, "hrrt_lm_histogram: the delayed sinogram is required in this mode");
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return lm_cuda(h, e, "hrrt_lm_histogram");
  const long long S = h->tab.sino_size();
  if (!h->h_sino_dev) {
    e = cudaMalloc(&h->h_sino_dev, sizeof(uint16_t) * 2 * (size_t)S);
    if (e != cudaSuccess) {
      h->h_sino_dev = nullptr;
      return lm_fail(h, HRRT_ERR_NOMEM, "hrrt_lm_histogram: sinograms");
    }
  }
  const long long phase = file_offset % kPacketWords, staged = nwords + phase;
  // streamed in chunks where every output is additive across chunks (the
  // head curve and the coincidence histogram are per call; the wide and
  // partitioned paths clear and fold per call)
  const long long chunk = h->chunk_words == 0 ? kDefaultChunkWords : h->chunk_words;
  const int whole_call = HRRT_LM_HEAD_CURVE | HRRT_LM_CRYSTAL_COUNTS | HRRT_LM_FORCE_WIDE | HRRT_LM_FORCE_PARTITIONED;
  if (h->chunk_words >= 0 && !(flags & whole_call) && !kWideByDefault && !kPartitionedByDefault && staged > chunk)
    return lm_histogram_chunked(h, words, nwords, phase, chunk, mode, duration, flags, sino, delayed, out);
  if ((size_t)staged > h->h_words_cap) {
    if (h->h_words_dev) cudaFree(h->h_words_dev);
    h->h_words_dev = nullptr;
    h->h_words_cap = 0;
    e = cudaMalloc(&h->h_words_dev, sizeof(uint32_t) * std::max<long long>(staged, 4));
    if (e != cudaSuccess) return lm_fail(h, HRRT_ERR_NOMEM, "hrrt_lm_histogram: event staging");
    h->h_words_cap = (size_t)staged;
  }
  cudaStream_t st = h->stream;
  e = cudaMemsetAsync(h->h_sino_dev, 0, sizeof(uint16_t) * 2 * (size_t)S, st);
  if (e == cudaSuccess && phase > 0) e = cudaMemsetAsync(h->h_words_dev, 0x80, sizeof(uint32_t) * phase, st);
  if (e == cudaSuccess && nwords > 0)
    e = cudaMemcpyAsync(h->h_words_dev + phase, words, sizeof(uint32_t) * nwords, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return lm_cuda(h, e, "hrrt_lm_histogram");
  int rc = hrrt_lm_histogram_device(h, h->h_words_dev, staged, mode, duration, flags, h->h_sino_dev,
                                    h->h_sino_dev + S, out, st);
  if (rc != HRRT_OK) return rc;
  out->words_used -= phase;
  out->resyncs -= phase;
  e = cudaMemcpyAsync(sino, h->h_sino_dev, sizeof(uint16_t) * S, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && delayed && mode == HRRT_LM_PROMPTS_AND_DELAYED)
    e = cudaMemcpyAsync(delayed, h->h_sino_dev + S, sizeof(uint16_t) * S, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return lm_cuda(h, e, "hrrt_lm_histogram");
  return HRRT_OK;
}

int hrrt_lm_crystal_singles(const int32_t *delayed_counts, float scan_duration, float tau, float *singles) {
  if (!delayed_counts || !singles) return HRRT_ERR_ARG;
  return hrrt::singles_from_delayed(delayed_counts, tau > 0 ? tau : 6.0e-9f, scan_duration > 0 ? scan_duration : 1.0f,
                                    singles);
}

int hrrt_lm_smooth_randoms(hrrt_lm *h, const int32_t *coinc_hist, float scan_duration, float tau, float *sino,
                           int *iterations) {
  if (!h) return HRRT_ERR_ARG;
  if (!coinc_hist || !sino) return lm_fail(h, HRRT_ERR_ARG, "hrrt_lm_smooth_randoms: null buffer");
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return lm_cuda(h, e, "hrrt_lm_smooth_randoms");
  // gen_delays: the delayed half of the histogram gives the crystal singles
  // (g_tau 6 ns and g_ftime 1 s unless given, gen_delays_lib.cpp:322-323)
  const float t = tau > 0 ? tau : 6.0e-9f, ft = scan_duration > 0 ? scan_duration : 1.0f;
  std::vector<float> cs(hrrt::kCrystals);
  const int it = hrrt::singles_from_delayed(coinc_hist + hrrt::kCrystals, t, ft, cs.data());
  if (iterations) *iterations = it;
  const long long S = h->dev.sino_size;
  cudaStream_t st = h->stream;
  float *d_cs = nullptr, *d_out = nullptr;
  e = cudaMallocAsync(&d_cs, sizeof(float) * hrrt::kCrystals, st);
  if (e == cudaSuccess) e = cudaMallocAsync(&d_out, sizeof(float) * S, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_cs, cs.data(), sizeof(float) * hrrt::kCrystals, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_out, 0, sizeof(float) * S, st);
  if (e == cudaSuccess) {
    const long long threads = 20LL * 2 * 104 * 72 * 2 * (72 / kDelayBxRun);
    lm_delays_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(h->dev, d_cs, t * ft, h->tab.maxrd, d_out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(sino, d_out, sizeof(float) * S, cudaMemcpyDeviceToHost, st);
  if (d_cs) cudaFreeAsync(d_cs, st);
  if (d_out) cudaFreeAsync(d_out, st);
  const cudaError_t e2 = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = e2;
  if (e != cudaSuccess) return lm_cuda(h, e, "hrrt_lm_smooth_randoms");
  return HRRT_OK;
}

int hrrt_lm_seek(hrrt_lm *h, const uint32_t *words, long long nwords, long long file_offset, int target_s, int flags,
                 long long *consumed) {
  if (!h) return HRRT_ERR_ARG;
  if (nwords < 0 || file_offset < 0 || (nwords > 0 && !words) || !consumed)
    return lm_fail(h, HRRT_ERR_ARG, "hrrt_lm_seek: null buffer or negative length");
  *consumed = 0;
  if ((flags & HRRT_LM_TIME_FROM_COUNT) && target_s == 0) return HRRT_OK;
  for (long long p0 = -(file_offset % kPacketWords); p0 < nwords; p0 += kPacketWords) {
    const long long end = std::min(p0 + kPacketWords, nwords);
    long long i = std::max(p0, 0LL);
    while (i + 1 < end) {
      const uint32_t ew1 = words[i], ew2 = words[i + 1];
      const int t = (int)((kEwTypes >> (2 * (((ew1 >> 30) << 2) | (ew2 >> 30)))) & 3);
      if (t == 3) {
        i++;
        continue;
      }
      i += 2;
      if (t != 2) continue;
      const uint32_t tag = (ew1 & 0xffff) | ((ew2 & 0xffff) << 16);
      if ((tag & 0xE0000000u) != 0x80000000u) continue;
      const long long ms = tag & 0x3fffffff;
      if (ms == 0 && target_s == 0) {
        h->current_time = 0;
        *consumed = i;
        return HRRT_OK;
      }
      if (h->current_time != ms / 1000) {
        h->current_time = ms / 1000;
        if (h->current_time == target_s) {
          *consumed = i;
          return HRRT_OK;
        }
      }
    }
  }
  return lm_fail(h, HRRT_ERR_NOT_FOUND, "hrrt_lm_seek: the stream ends before the requested time");
}

long long hrrt_lm_convert_span9(const int16_t *span3, const int16_t *delayed, int16_t *span9, int maxrd) {
  std::vector<int32_t> src;
  const int planes9 = hrrt::span9_plane_sources(maxrd, hrrt::LmTables::kYCrys, &src);
  if (planes9 < 0 || !span3 || !span9) return HRRT_ERR_ARG;
  constexpr long long kPix = 256LL * 288;
  auto fold = [&](int p0, int p1) {
    for (int p = p0; p < p1; p++) {
      uint16_t *o = (uint16_t *)span9 + p * kPix;
      std::memset(o, 0, sizeof(uint16_t) * kPix);
      for (int k = 0; k < 3; k++) {
        const int32_t sp = src[(size_t)p * 3 + k];
        if (sp < 0) continue;
        const uint16_t *a = (const uint16_t *)span3 + sp * kPix;
        const uint16_t *d = delayed ? (const uint16_t *)delayed + sp * kPix : nullptr;
        for (long long j = 0; j < kPix; j++) o[j] = (uint16_t)(o[j] + a[j] - (d ? d[j] : 0));
      }
    }
  };
  const int nt = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; t++) pool.emplace_back(fold, planes9 * t / nt, planes9 * (t + 1) / nt);
  for (auto &th : pool) th.join();
  return planes9;
}

int hrrt_lm_trues_span9_device(hrrt_lm *h, const uint16_t *d_prompts, const uint16_t *d_delayed, int16_t *d_span9,
                               void *stream) {
  if (!h) return HRRT_ERR_ARG;
  if (h->tab.span != 3) return lm_fail(h, HRRT_ERR_ARG, "hrrt_lm_trues_span9_device: the handle is not span 3");
  if (!d_prompts || !d_span9) return lm_fail(h, HRRT_ERR_ARG, "hrrt_lm_trues_span9_device: null buffer");
  if (((uintptr_t)d_prompts | (uintptr_t)d_delayed | (uintptr_t)d_span9) & 15)
    return lm_fail(h, HRRT_ERR_ARG, "hrrt_lm_trues_span9_device: buffers must be 16-byte aligned");
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return lm_cuda(h, e, "hrrt_lm_trues_span9_device");
  if (!h->span9_src) {
    std::vector<int32_t> src;
    const int planes9 = hrrt::span9_plane_sources(h->tab.maxrd, hrrt::LmTables::kYCrys, &src);
    if (planes9 < 0) return lm_fail(h, HRRT_ERR_ARG, "hrrt_lm_trues_span9_device: maxrd has no span-9 fold");
    std::vector<int4> packed(planes9);
    for (int p = 0; p < planes9; p++) packed[p] = make_int4(src[3 * p], src[3 * p + 1], src[3 * p + 2], -1);
    e = cudaMalloc(&h->span9_src, sizeof(int4) * planes9);
    if (e == cudaSuccess)
      e = cudaMemcpy(h->span9_src, packed.data(), sizeof(int4) * planes9, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return lm_cuda(h, e, "hrrt_lm_trues_span9_device: tables");
    h->span9_planes = planes9;
  }
  cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
  const dim3 grid((256 * 288 / 8 + 255) / 256, (unsigned)h->span9_planes);
  lm_span9_kernel<<<grid, 256, 0, st>>>((const uint4 *)d_prompts, (const uint4 *)d_delayed, h->span9_src,
                                         (uint4 *)d_span9);
  e = cudaGetLastError();
  if (e != cudaSuccess) return lm_cuda(h, e, "hrrt_lm_trues_span9_device");
  return HRRT_OK;
}

}  // extern "C"
