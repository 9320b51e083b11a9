// lm_tables.h -- HRRT listmode rebinning tables (host).
//
// The crystal-pair lookup the reference's hrrt_rebinner_lut writes and
// lmhistogram_mp reads (lor_sinogram_map.cpp:99-221), the axial crystal
// positions, and the span-3 segment tables with the output span's plane
// offsets (segment_info_fromarchive.cpp:35-141).  Computed with the same
// float/double operand types and order as the reference so that every
// event lands in the reference's bin.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace hrrt {

struct LmSol {
  int32_t nsino;  // bin + view * 256, -1 outside the sinogram
  float d;        // 1 / (transaxial length * d_tan_theta), signed by orientation
  float z;        // axial parameter / plane separation
};

struct LmTables {
  static constexpr int kHeads = 8, kLayers = 2, kXCrys = 72, kYCrys = 104, kPairs = 20;
  static constexpr int kXD = kXCrys * kLayers;  // crystal x index with layer
  static constexpr int kBins = 256, kViews = 288;
  int span = 3, maxrd = 67;
  int nsegs = 0;         // span-3 segments (45 at maxrd 67)
  int nplanes = 0;       // planes of the output sinogram (6367 / 2209)
  double d_tan_theta = 0;
  std::vector<LmSol> sol;        // [21][144][144], head pair 0 unused
  std::vector<float> zpos, zpos2;  // [104]: z (cm) and z / plane_sep + 0.5
  std::vector<int> segz0, segzmax, segzoffset;  // [nsegs]
  long long sino_size() const { return (long long)nplanes * kBins * kViews; }
  // empty string on success
  std::string build(int span, int maxrd);
};

// Crystal singles rates from the delayed coincidence counts of a
// coincidence histogram (compute_csings_from_drates and its helpers,
// gen_delays_lib/gen_delays_lib.cpp:163-255): `dcoins` and `srates` are
// [layer 2][y 104][head 8][x 72]; `dt` the scan duration (s), `tau` the
// coincidence window (s).  Returns the iterations run (at most 100).
int singles_from_delayed(const int32_t *dcoins, float tau, float dt, float *srates);
constexpr int kCrystals = LmTables::kLayers * LmTables::kYCrys * LmTables::kHeads * LmTables::kXCrys;  // 119808
// head pair mp (1..20) -> (head a, head b)
void pair_heads(int mp, int *ahead, int *bhead);

// The span-3 -> span-9 plane fold of convert_span9
// (lmhistogram_mp/convert_span9.cpp:13-150) as a gather: for every span-9
// plane the (up to three) span-3 planes that sum into it, -1 for none.
// Returns the span-9 plane count (2209 at maxrd 67, 104 rings), or -1 when
// maxrd does not give whole span-9 segments.
int span9_plane_sources(int maxrd, int nrings, std::vector<int32_t> *src /* [planes9][3] */);

}  // namespace hrrt
