// lmhist_ref_main.cpp -- a command-line harness around the reference's OWN
// listmode code, compiled unmodified from its sources by oracle/Makefile
// (target "ref", executable oracle/_ref/lmhist_ref):
//   lmhistogram_mp/histogram_mp.cpp   rebin_packet, histogram, process_tagword,
//                                     check_end_of_frame, coincidence map
//   lmhistogram_mp/LM_Reader_mp.cpp   the packet reader (load_buffer_64/32)
//   lmhistogram_mp/LM_Rebinner_mp.cpp rebin_event
//   lmhistogram_mp/convert_span9.cpp  the span-3 -> span-9 fold
//   gen_delays_lib/lor_sinogram_map.cpp init_sol / init_phy_to_pro (the LUT)
//   gen_delays_lib/geometry_info.cpp  crystal positions (calc_det_to_phy)
//   gen_delays_lib/segment_info_fromarchive.cpp init_segment_info
//   gen_delays_lib/gen_delays_lib.cpp compute_csings_from_drates (crystal
//                                     singles from delayed coincidences)
// TEST INFRASTRUCTURE: the checker of oracle/lm_oracle.c and of the device
// histogrammer; nothing in the product links or runs it.
//
// What the harness supplies, because the reference's own set-up cannot run
// here (LM_Rebinner::init_rebinner needs the gm328.ini gantry file and a LUT
// file written by hrrt_rebinner_lut, which does not compile):
//   * the geometry state init_geometry_hrrt sets for the HRRT (LR_0), with
//     calc_det_to_phy called for every crystal as its loop intends (the loop
//     counter is never initialised there, geometry_info.cpp:206-214);
//   * the segment tables: the archive's init_segment_info (the pre-rewrite
//     semantics; the rewrite's writes through reserve()d vectors,
//     segment_info.cpp:50-70) copied into the rewrite's SegmentInfo globals
//     that lor_sinogram_map.cpp and LM_Rebinner_mp.cpp read;
//   * the LUT built in memory by the reference's own lor_sinogram::init_sol
//     with those tables (what hrrt_rebinner_lut would write, then
//     init_lut_sol read back);
//   * the packet containers and the input stream of the reader (lm64_reader
//     reads into its containers before allocating them, LM_Reader_mp.cpp:128).
//   * link-time definitions of functions that only the skipped set-up and
//     file helpers call (GantryInfo, hrrt_util file opening and writing, the
//     rewrite's init_segment_info); none of them runs.
//
// Subcommands (binary files, native endianness):
//   tables    <span> <maxrd> <out.bin>   SOL [21][144][144] {int32 nsino, float d, float z},
//                                        c_zpos [104], c_zpos2 [104], segplane [63][207] int16
//   rebin     <span> <maxrd> <in.bin> <out.bin>   int32 [n][7] (mp, al, ax, ay, bl, bx, by) -> int32 [n]
//   span9     <maxrd> <nrings> <inout.bin>        int16 span-3 sinogram folded in place
//   singles   <tau> <dt> <dcoins.bin> <out.bin>   int32 [119808] delayed crystal counts ->
//                                                 float [119808] singles rates, then int32 iterations
//   histogram <span> <maxrd> <mode> <duration> <flags> <words.l64> <sino.bin> <hc.txt> <stats.txt> [<coinc.bin>]
//             mode 0 trues, 1 prompts + delayed, 2 prompts only; flags 1 ignore border crystals,
//             2 no DOI, 4 time from the tag count.  sino.bin: int16 [2][sino_size]
//             (prompts or trues, then delayed); coinc.bin: uint32 [2][2*59904 + 104*7488],
//             the coincidence maps indexed as rebin_packet indexes them.  The frame must end (duration > 0) before the
//             file does: the reader exits the process on a read past the end
//             (LM_Reader_mp.cpp:179-182).  Runs as lmhistogram -v does (see
//             cmd_histogram).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "LM_Reader_mp.hpp"
#include "LM_Rebinner_mp.hpp"
#include "convert_span9.hpp"
#include "gen_delays_lib.hpp"
#include "geometry_info.h"
#include "gantryinfo.hpp"
#include "histogram_mp.hpp"
#include "hrrt_util.hpp"
#include "lor_sinogram_map.h"
#include "segment_info.h"

// ---- the reference translation units' symbols this harness drives ----
namespace GeometryInfo {
void calc_det_to_phy(int head, int layer, int detx, int dety, float location[3]);
}
int init_segment_info(int *nsegs, int *nplanes, double *d_tan_theta, int maxrd, int span, int NYCRYS,
                      double crystal_radius, double plane_sep);  // segment_info_fromarchive.cpp
extern int *m_segz0, *m_segzmax, *m_segzoffset;                    // segment_info_fromarchive.cpp
extern L64EventPacket *g_l64_container;                            // LM_Reader_mp.cpp
extern L32EventPacket *g_l32_container;

// ---- definitions the rewrite's headers declare and no compiled file defines ----
double SegmentInfo::m_d_tan_theta = 0.0;
double SegmentInfo::m_d_tan_theta_tx = 0.0;
int SegmentInfo::m_nsegs = 0;
std::vector<int> SegmentInfo::conversiontable;
std::vector<int> SegmentInfo::m_segz0;
std::vector<int> SegmentInfo::m_segzmax;
std::vector<int> SegmentInfo::m_segzoffset_span9;
std::vector<int> SegmentInfo::m_segzoffset;
int SegmentInfo::init_segment_info(int *, int *, double *, int, int, int, double, double) { return 0; }
namespace cps {
int GantryInfo::load(int) { return 0; }
int GantryInfo::get(const char *, int &) { return 0; }
int GantryInfo::get(const char *, float &) { return 0; }
int GantryInfo::get(const char *, int, int &) { return 0; }
}  // namespace cps
// gen_delays_lib.cpp's input and output file names (declared by the stand-in
// gen_delays.hpp; the checked function takes its data as arguments)
boost::filesystem::path g_coincidence_histogram_file, g_crystal_singles_file, g_delayed_coincidence_file,
    g_output_csings_file;
int compute_csings_from_drates(int *dcoins, float tau, float dt, float *srates);  // gen_delays_lib.cpp:235
// the gen_delays program's parameters, defaults of gen_delays.cpp:67-76
// (the checked function takes tau and the duration as arguments)
int g_num_elems = GeometryInfo::NUM_ELEMS, g_num_views = GeometryInfo::NUM_VIEWS, g_span = 9,
    g_max_ringdiff = GeometryInfo::MAX_RINGDIFF;
float g_pitch = 0.0f, g_diam = 0.0f, g_thick = 0.0f, g_tau = 6.0e-9f, g_ftime = 1.0f;

namespace hrrt_util {
int open_istream(std::ifstream &, const boost::filesystem::path &, std::ios_base::openmode) { return 1; }
int open_ostream(std::ofstream &, const boost::filesystem::path &, std::ios_base::openmode) { return 1; }
template <typename T>
int write_binary_file(T *, int, boost::filesystem::path const &, std::string const &) {
  return 1;
}
template int write_binary_file<float>(float *, int, boost::filesystem::path const &, std::string const &);
}  // namespace hrrt_util

namespace {

void setup(int span, int maxrd) {
  using namespace GeometryInfo;
  // init_geometry_hrrt(0, 0, 0) for LR_0 (geometry_info.cpp:168-218)
  const float pitch = PITCH, rdiam = RDIAM, lthick = LTHICK;
  for (int i = 0; i < NHEADS; i++) {
    sin_head_[i] = sin(i * 2.0 * M_PI / NHEADS);
    cos_head_[i] = cos(i * 2.0 * M_PI / NHEADS);
  }
  crystal_radius_ = rdiam / 2.0;
  crystal_x_pitch_ = crystal_y_pitch_ = pitch;
  const LR_Geom geom = lr_geometries_.at(LR_Type::LR_0);
  nprojs_ = geom.nprojs;
  nviews_ = geom.nviews;
  binsize_ = pitch / 2.0;
  plane_sep_ = pitch / 2.0;
  head_crystal_depth_.fill(lthick);
  maxrd_ = maxrd;
  float pos[3];
  int i = 0;
  for (int head = 0; head < NHEADS; head++)
    for (int layer = 0; layer < NDOIS; layer++)
      for (int xcrys = 0; xcrys < NXCRYS; xcrys++)
        for (int ycrys = 0; ycrys < NYCRYS; ycrys++, i++) {
          calc_det_to_phy(head, layer, xcrys, ycrys, pos);
          crystal_xpos_[i] = pos[0];
          crystal_ypos_[i] = pos[1];
          crystal_zpos_[i] = pos[2];
        }
  // init_rebinner's segment set-up (LM_Rebinner_mp.cpp:146), archive semantics
  int nsegs = 0, nplanes = 0;
  double dt = 0;
  init_segment_info(&nsegs, &nplanes, &dt, maxrd, span, NYCRYS, crystal_radius_, plane_sep_);
  SegmentInfo::m_nsegs = nsegs;
  SegmentInfo::m_d_tan_theta = dt;
  SegmentInfo::m_segz0.assign(m_segz0, m_segz0 + nsegs);
  SegmentInfo::m_segzmax.assign(m_segzmax, m_segzmax + nsegs);
  SegmentInfo::m_segzoffset.assign(m_segzoffset, m_segzoffset + nsegs);
  // the LUT (hrrt_rebinner_lut: init_sol with the segment tables above)
  lor_sinogram::init_sol(SegmentInfo::m_segzoffset.data());
}

long sino_size(int span) {
  const int planes = span == 3 ? 6367 : 2209;
  return (long)planes * GeometryInfo::nprojs_ * GeometryInfo::nviews_;
}

template <class T>
std::vector<T> read_all(const char *fn) {
  std::vector<T> v;
  FILE *f = fopen(fn, "rb");
  if (!f) return v;
  fseek(f, 0, SEEK_END);
  const long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  v.resize(n / sizeof(T));
  if (!v.empty() && fread(v.data(), sizeof(T), v.size(), f) != v.size()) v.clear();
  fclose(f);
  return v;
}

template <class T>
bool write_all(FILE *f, const T *p, size_t n) {
  return fwrite(p, sizeof(T), n, f) == n;
}

int cmd_tables(int span, int maxrd, const char *out) {
  setup(span, maxrd);
  FILE *f = fopen(out, "wb");
  if (!f) return 2;
  const int nx = GeometryInfo::NUM_CRYSTALS_X_DOIS;
  std::vector<lor_sinogram::SOL> zero(nx);
  for (int mp = 0; mp <= 20; mp++)
    for (int a = 0; a < nx; a++)
      write_all(f, mp == 0 ? zero.data() : lor_sinogram::solution_[mp][a], nx);
  write_all(f, lor_sinogram::m_c_zpos, GeometryInfo::NYCRYS);
  write_all(f, lor_sinogram::m_c_zpos2, GeometryInfo::NYCRYS);
  for (int s = 0; s < 63; s++) write_all(f, lor_sinogram::m_segplane[s], 2 * GeometryInfo::NYCRYS - 1);
  fclose(f);
  return 0;
}

int cmd_rebin(int span, int maxrd, const char *in, const char *out) {
  setup(span, maxrd);
  const std::vector<int32_t> ev = read_all<int32_t>(in);
  const size_t n = ev.size() / 7;
  std::vector<int32_t> addr(n);
  for (size_t k = 0; k < n; k++) {
    const int32_t *e = &ev[k * 7];
    addr[k] = rebin_event(e[0], e[1], e[2], e[3], e[4], e[5], e[6]);
  }
  FILE *f = fopen(out, "wb");
  if (!f) return 2;
  write_all(f, addr.data(), n);
  fclose(f);
  return 0;
}

int cmd_span9(int maxrd, int nrings, const char *fn) {
  GeometryInfo::nprojs_ = 256;
  GeometryInfo::nviews_ = 288;
  std::vector<int16_t> s = read_all<int16_t>(fn);
  if (s.empty()) return 2;
  convert_span9(s.data(), maxrd, nrings);
  FILE *f = fopen(fn, "wb");
  if (!f) return 2;
  write_all(f, s.data(), s.size());
  fclose(f);
  return 0;
}

int cmd_singles(float tau, float dt, const char *in, const char *out) {
  std::vector<int32_t> dc = read_all<int32_t>(in);
  if (dc.size() != (size_t)GeometryInfo::NUM_CRYSTALS_X_Y_HEADS_DOIS) return 2;
  std::vector<float> sr(dc.size(), 0.f);
  const int32_t it = compute_csings_from_drates(dc.data(), tau, dt, sr.data());
  FILE *f = fopen(out, "wb");
  if (!f) return 2;
  write_all(f, sr.data(), sr.size());
  write_all(f, &it, 1);
  fclose(f);
  return 0;
}

int cmd_histogram(int span, int maxrd, int mode, int duration, int flags, const char *words, const char *sino_fn,
                  const char *hc_fn, const char *stats_fn, const char *coinc_fn) {
  setup(span, maxrd);
  // lmhistogram's option handling (lmhistogram_mp.cpp:328-353)
  g_hist_mode = mode == 1 ? HISTOGRAM_MODE::PRO_RAN : mode == 2 ? HISTOGRAM_MODE::PRO : HISTOGRAM_MODE::TRU;
  if (flags & 1) eg_rebinner_method |= IGNORE_BORDER_CRYSTAL;
  if (flags & 2) eg_rebinner_method |= NODOI_PROCESSING;
  if (flags & 4) timetag_processing = 0;
  // -v (lmhistogram_fromarchive.cpp:412): rebin_packet rejects an invalid
  // head pair only in verbose mode (histogram_mp.cpp:1124-1127, the log line
  // in between is commented out); otherwise rebin_event indexes the LUT with
  // it, outside the 20 pairs the LUT holds.  Verbose mode changes nothing
  // else on this path (its other uses only log).
  verbose = 1;
  g_max_rd = maxrd;
  // the coincidence maps: rebin_packet steps a crystal row by
  // NUM_CRYSTALS_X_Y (histogram_mp.cpp:1049, :1218) where the earlier program
  // steps it by NHEADS * NXCRYS (histogram_mp_fromarchive.cpp:916), so its
  // indexes reach past the NUM_CRYSTALS_X_Y_HEADS_DOIS entries lmhistogram
  // allocates (lmhistogram_mp.cpp:501); room for every index it forms
  const size_t ncrys = (size_t)GeometryInfo::NDOIS * GeometryInfo::NUM_CRYSTALS_X_Y_HEADS +
                       (size_t)GeometryInfo::NYCRYS * GeometryInfo::NUM_CRYSTALS_X_Y;
  std::vector<unsigned> pmap(ncrys, 0), dmap(ncrys, 0);
  g_p_coinc_map = pmap.data();
  g_d_coinc_map = dmap.data();
  // the reader's state (lm64_reader, LM_Reader_mp.cpp:124-138, allocating first)
  L64EventPacket::in_fname = words;
  L64EventPacket::in_fp.open(words, std::ios::in | std::ios::binary);
  if (!L64EventPacket::in_fp.is_open()) return 2;
  g_l64_container = new L64EventPacket[2];
  g_l32_container = new L32EventPacket;
  const long S = sino_size(span);
  std::vector<int16_t> sino((size_t)2 * S, 0);
  std::ofstream hc(hc_fn);
  int dur = duration;
  const int start = histogram<short>(sino.data(), nullptr, (int)S, dur, hc);
  hc.close();
  FILE *f = fopen(sino_fn, "wb");
  if (!f) return 2;
  write_all(f, sino.data(), sino.size());
  fclose(f);
  FILE *st = fopen(stats_fn, "w");
  if (!st) return 2;
  fprintf(st, "frame_start %d\nduration %d\nprompts %lld\nrandoms %lld\n", start, dur, (long long)total_prompts(),
          (long long)total_randoms());
  for (int b = 0; b < GeometryInfo::NBLOCKS; b++) fprintf(st, "singles %d %d\n", b, singles_rate(b));
  fclose(st);
  if (coinc_fn) {
    FILE *c = fopen(coinc_fn, "wb");
    if (!c) return 2;
    write_all(c, pmap.data(), ncrys);
    write_all(c, dmap.data(), ncrys);
    fclose(c);
  }
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 2) return 1;
  const std::string cmd = argv[1];
  if (cmd == "tables" && argc == 5) return cmd_tables(atoi(argv[2]), atoi(argv[3]), argv[4]);
  if (cmd == "rebin" && argc == 6) return cmd_rebin(atoi(argv[2]), atoi(argv[3]), argv[4], argv[5]);
  if (cmd == "span9" && argc == 5) return cmd_span9(atoi(argv[2]), atoi(argv[3]), argv[4]);
  if (cmd == "singles" && argc == 6) return cmd_singles((float)atof(argv[2]), (float)atof(argv[3]), argv[4], argv[5]);
  if (cmd == "histogram" && (argc == 11 || argc == 12))
    return cmd_histogram(atoi(argv[2]), atoi(argv[3]), atoi(argv[4]), atoi(argv[5]), atoi(argv[6]), argv[7], argv[8],
                         argv[9], argv[10], argc == 12 ? argv[11] : nullptr);
  fprintf(stderr, "usage: lmhist_ref tables|rebin|span9|singles|histogram ...\n");
  return 1;
}
