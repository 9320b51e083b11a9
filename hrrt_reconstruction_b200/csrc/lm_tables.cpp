// lm_tables.cpp -- see lm_tables.h.  Built with -ffp-contract=off.
//
// Reference files (within the reference project):
//   gen_delays_lib/geometry_info.{h,cpp}          crystal geometry
//   gen_delays_lib/segment_info_fromarchive.cpp   segment tables
//   gen_delays_lib/lor_sinogram_map.cpp           init_phy_to_pro / init_sol
//   hrrt_rebinner_lut/hrrt_rebinner_lut.cpp       crystal depth 1.0, maxrd 67
#include "lm_tables.h"

#include <array>
#include <cmath>

namespace hrrt {

namespace {

constexpr double kPi = 3.14159265358979323846;  // M_PI

// Head pairs of the 20 coincidence combinations (geometry_info.h:70-75).
constexpr int kPairHeads[21][2] = {{-1, -1}, {0, 2}, {0, 3}, {0, 4}, {0, 5}, {0, 6}, {1, 3}, {1, 4},
                                   {1, 5},   {1, 6}, {1, 7}, {2, 4}, {2, 5}, {2, 6}, {2, 7}, {3, 5},
                                   {3, 6},   {3, 7}, {4, 6}, {4, 7}, {5, 7}};
// span-3 segment -> span-9 segment (segment_info_fromarchive.cpp:23-26)
constexpr int kSpan9Of[45] = {0, 0, 0,  1,  2, 1,  2, 1,  2,  3,  4,  3,  4,  3,  4,  5,  6,  5,  6,  5,  6,  7,  8,
                              7, 8, 7,  8,  9, 10, 9, 10, 9,  10, 11, 12, 11, 12, 11, 12, 13, 14, 13, 14, 13, 14};

// Block geometry in cm (geometry_info.h:50-56): `const float` initialised
// from double expressions.
struct Head {
  float csize = 0.22f, cgap = 0.02f, bgap = 0.05f;
  float bsize = (float)(8.0 * csize + 7 * cgap);
  float xhsize = (float)(9.0 * bsize + 8 * bgap);
  double radius = 46.9f / 2.0;  // RDIAM / 2
  float depth = 1.0f;           // layer thickness (LTHICK)
  std::array<double, 8> s{}, c{};
  Head() {
    for (int i = 0; i < 8; i++) {
      s[i] = std::sin(i * 2.0 * kPi / 8);
      c[i] = std::cos(i * 2.0 * kPi / 8);
    }
  }
  // calc_det_to_phy (geometry_info.cpp:137-163)
  void position(int head, int layer, int detx, int dety, float out[3]) const {
    const float along = (detx / 8) * (bsize + bgap) + (detx % 8) * (csize + cgap);
    const double x = along - xhsize / 2.0 + csize / 2.0;
    const double y = radius + depth * (1 - layer) + 0.5 * depth;
    const float axial = (dety / 8) * (bsize + bgap) + (dety % 8) * (csize + cgap);
    out[0] = (float)(x * c[head] + y * s[head]);
    out[1] = (float)(-x * s[head] + y * c[head]);
    out[2] = (float)(double)axial;
  }
};

}  // namespace

std::string LmTables::build(int span_, int maxrd_) {
  if (span_ != 3 && span_ != 9) return "listmode span must be 3 or 9";
  if (maxrd_ < span_ || maxrd_ > 2 * kYCrys - 2) return "listmode maximum ring difference out of range";
  span = span_;
  maxrd = maxrd_;
  const Head hd;
  const float pitch = 0.24375f;
  const double plane_sep = pitch / 2.0, binsize = pitch / 2.0;
  const int np = 2 * kYCrys - 1;

  // output-span plane offsets (init_seginfo) and the span-3 segments the
  // rebinner works in (init_seginfo2), segment_info_fromarchive.cpp:35-141
  auto segments = [&](int sp, std::vector<int> &z0, std::vector<int> &zmax, std::vector<int> &off) {
    const int n = 2 * (maxrd / sp) + 1;
    z0.assign(n, 0);
    zmax.assign(n, 0);
    off.assign(n, 0);
    int start = 0;
    for (int i = 0; i < n; i++) {
      z0[i] = (i == 0) ? 0 : (sp + 1) / 2 + sp * ((i - 1) / 2);
      const int nz = np - 2 * z0[i];
      zmax[i] = z0[i] + nz - 1;
      off[i] = start - z0[i];
      start += nz;
    }
    return start;
  };
  std::vector<int> oz0, ozmax, ooff;
  const int out_planes = segments(span, oz0, ozmax, ooff);
  nplanes = segments(3, segz0, segzmax, segzoffset);
  nsegs = (int)segz0.size();
  if (span == 9) {
    nplanes = out_planes;
    for (int i = 0; i < nsegs; i++) segzoffset[i] = ooff[kSpan9Of[i]];
  }
  d_tan_theta = 3 * plane_sep / hd.radius;

  // crystal-pair LUT (init_sol / init_phy_to_pro): positions at ring 0
  std::vector<std::array<float, 3>> ring0((size_t)kHeads * kXD);
  for (int h = 0; h < kHeads; h++)
    for (int l = 0; l < kLayers; l++)
      for (int x = 0; x < kXCrys; x++) hd.position(h, l, x, 0, ring0[(size_t)h * kXD + x + kXCrys * l].data());
  sol.assign((size_t)21 * kXD * kXD, LmSol{0, 0.f, 0.f});
  const float fpi = (float)kPi;
  for (int mp = 1; mp <= kPairs; mp++) {
    const int ha = kPairHeads[mp][0], hb = kPairHeads[mp][1];
    for (int a = 0; a < kXD; a++) {
      const float *pa = ring0[(size_t)ha * kXD + a].data();
      for (int b = 0; b < kXD; b++) {
        const float *pb = ring0[(size_t)hb * kXD + b].data();
        const double dy = pa[1] - pb[1];
        const double dx = pa[0] - pb[0];
        double d = std::sqrt(dx * dx + dy * dy);
        float r = (float)((pa[1] * pb[0] - pa[0] * pb[1]) / d);
        float phi = (float)std::atan2(dx, dy);
        if (phi < 0.0) {
          phi += fpi;
          r = -r;
          d = -d;
        }
        if (phi >= kPi) {
          phi = 0.0f;
          r = -r;
          d = -d;
        }
        int view = (int)(kViews * phi / kPi);
        if (view >= kViews || view <= -1) view = 0;
        const float zt = (float)((pa[0] * dx + pa[1] * dy) / (d * d));
        const int bin = (int)(kBins / 2 + (r / binsize + 0.5));
        LmSol &e = sol[((size_t)mp * kXD + a) * kXD + b];
        e.nsino = (bin < 0 || bin > kBins - 1) ? -1 : bin + view * kBins;
        e.d = (float)(1.0 / d / d_tan_theta);
        e.z = (float)(zt / plane_sep);
      }
    }
  }
  zpos.assign(kYCrys, 0.f);
  zpos2.assign(kYCrys, 0.f);
  for (int y = 0; y < kYCrys; y++) {
    float p[3];
    hd.position(0, 0, 0, y, p);
    zpos[y] = p[2];
    zpos2[y] = (float)(p[2] / plane_sep + 0.5);
  }
  return std::string();
}

// ---- crystal singles from delayed coincidences (gen_delays_lib.cpp:163-255) ----
// Crystal index i = x + 72*head + 576*y + 59904*layer (compute_drate, :175).

void pair_heads(int mp, int *ahead, int *bhead) {
  *ahead = kPairHeads[mp][0];
  *bhead = kPairHeads[mp][1];
}

namespace {

constexpr int kNH = LmTables::kHeads, kNX = LmTables::kXCrys, kNY = LmTables::kYCrys, kND = LmTables::kLayers;
constexpr int kPerLayer = kNH * kNX * kNY;

int crystal(int head, int layer, int cx, int cy) { return kNX * head + cx + kNX * kNH * cy + kPerLayer * layer; }

// per-head singles totals in the reference's summation order (layer, x, y)
void head_sums(const float *srate, float *hsum) {
  for (int head = 0; head < kNH; head++) {
    hsum[head] = 0.0f;
    for (int layer = 0; layer < kND; layer++)
      for (int cx = 0; cx < kNX; cx++)
        for (int cy = 0; cy < kNY; cy++) hsum[head] += srate[crystal(head, layer, cx, cy)];
  }
}

// the five heads facing `head` (heads head+2 .. head+6)
float facing_sum(const float *hsum, int head) {
  float s = 0.0f;
  for (int j = 0; j < 5; j++) s += hsum[(head + j + 2) % kNH];
  return s;
}

// compute_drate (:163-193): expected delayed rate of every crystal
void drate_of(const float *srate, float tau, float *drate) {
  float hsum[kNH];
  head_sums(srate, hsum);
  for (int head = 0; head < kNH; head++) {
    const float oh = facing_sum(hsum, head);
    for (int layer = 0; layer < kND; layer++)
      for (int cx = 0; cx < kNX; cx++)
        for (int cy = 0; cy < kNY; cy++) {
          const int i = crystal(head, layer, cx, cy);
          drate[i] = srate[i] * tau * oh;
        }
  }
}

// estimate_srate (:195-222): halfway towards the rates that explain drate
void update_srate(const float *drate, float tau, float *srate) {
  float hsum[kNH];
  head_sums(srate, hsum);
  for (int head = 0; head < kNH; head++) {
    const float oh = facing_sum(hsum, head);
    for (int layer = 0; layer < kND; layer++)
      for (int cx = 0; cx < kNX; cx++)
        for (int cy = 0; cy < kNY; cy++) {
          const int i = crystal(head, layer, cx, cy);
          srate[i] = (srate[i] + drate[i] / (tau * oh)) / 2.0f;
        }
  }
}

}  // namespace

int singles_from_delayed(const int32_t *dcoins, float tau, float dt, float *srates) {
  std::vector<float> drates(kCrystals), xrates(kCrystals);
  for (int i = 0; i < kCrystals; i++) drates[i] = dcoins[i] / dt;
  // compute_initial_srate (:224-232)
  float dtotal = 0.0f;
  for (int i = 0; i < kCrystals; i++) dtotal += drates[i];
  const float stotal = (float)(8.0 * std::sqrt(dtotal / (40. * tau)));
  for (int i = 0; i < kCrystals; i++) srates[i] = drates[i] * stotal / dtotal;
  int iter;
  for (iter = 0; iter < 100; iter++) {
    drate_of(srates, tau, xrates.data());
    // errtotal (:234-243): squared rounding error of the predicted counts, in
    // the reference's int arithmetic (wrapping, as its build does)
    uint32_t err = 0;
    for (int i = 0; i < kCrystals; i++) {
      const uint32_t d = (uint32_t)(int)(dcoins[i] - (0.5 + xrates[i] * dt));
      err += d * d;
    }
    if (iter && err == 0) break;
    update_srate(drates.data(), tau, srates);
  }
  return iter;
}

// convert_span9 folds in place: span-9 segment 0 is span-3 segment 0 plus
// segments -1 / +1 at their plane offset; span-9 segment -k / +k starts as
// a copy of span-3 segment -(3k-1) / +(3k-1) and adds -(3k) / +(3k) and
// -(3k+1) / +(3k+1) at theirs.  Every read is ahead of every write, so the
// fold equals this gather of the input planes.
int span9_plane_sources(int maxrd, int nrings, std::vector<int32_t> *src) {
  const int nseg = (2 * maxrd + 1) / 3, nseg9 = (2 * maxrd + 1) / 9;
  if (nseg9 < 1 || nseg != 3 * nseg9 || nseg % 2 == 0) return -1;
  std::vector<int> nplns(nseg), move(nseg, 0);
  for (int i = 0; i < nseg; i++) {
    const int seg = (i + 1) / 2, seg9 = (i + 3) / 6;
    nplns[i] = seg > 0 ? 2 * nrings - 3 * (2 * seg - 1) - 2 : 2 * nrings - 1;
    const int n9 = seg > 1 ? 2 * nrings - 9 * (2 * seg9 - 1) - 2 : 2 * nrings - 1;
    if (seg > 0) move[i] = (n9 - nplns[i]) / 2;
  }
  std::vector<int> start(nseg + 1, 0);
  for (int i = 0; i < nseg; i++) start[i + 1] = start[i] + nplns[i];
  int planes9 = nplns[0];
  for (int k = 1; 2 * k - 1 < nseg9; k++) planes9 += 2 * nplns[6 * k - 3];
  src->assign((size_t)planes9 * 3, -1);
  auto add = [&](int dst_plane, int slot, int seg) {
    for (int q = 0; q < nplns[seg]; q++) (*src)[(size_t)(dst_plane + q) * 3 + slot] = start[seg] + q;
  };
  add(0, 0, 0);
  add(move[1], 1, 1);
  add(move[2], 2, 2);
  int pos9 = nplns[0];
  for (int first = 3; first < nseg; first += 6) {
    const int nout = nplns[first];
    for (int k = 0; k < 6; k++) {
      const int seg = first + k;
      const int base = pos9 + (k % 2 ? nout : 0);
      add(base + (k < 2 ? 0 : move[seg]), k / 2, seg);
    }
    pos9 += 2 * nout;
  }
  return planes9;
}

}  // namespace hrrt
