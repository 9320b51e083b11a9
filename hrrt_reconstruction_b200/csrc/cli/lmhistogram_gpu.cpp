// lmhistogram_gpu -- the lmhistogram command line on libhrrt_gpu.
//
// Reads a 64-bit HRRT listmode file and its Interfile header (<stem>.l64.hdr)
// and writes, frame by frame, what lmhistogram_mp writes for an emission
// scan (lmhistogram_mp.cpp:574-736, 936-1118): the sinogram (.s) with its
// header (.s.hdr), in -PR mode the trues folded into span 9 (.tr.s,
// convert_span9) and with -ra the delayed (.ra.s), the coincidence
// histogram (.ch, write_coin_map in histogram_mp.cpp:646-690), the head
// curve (_lm.hc, process_tagword in histogram_mp.cpp:225-260) and for more
// than one frame the .dyn list.
//
// Options (boost::program_options in the reference, lmhistogram_mp.cpp:427-
// 478; one or two dashes): <in.l64> | -i, -o, --span 3|9, --PR, -P, --ra,
// --notimetag, --nodoi, --EB, -d <D> | <D,skip> | <D*N> (repeatable).
// Transmission scans, --add, --mock, --count, --start, --scan and -L are
// refused with a message.
//
// Where the reference's rewrite cannot run as written, the earlier
// lmhistogram (the *_fromarchive.cpp sources) gives the behaviour:
//   * -d: "D", "D,skip" and "D*N" (lmhistogram_fromarchive.cpp:452-470);
//     the header's "Frame definition" is a list of "D" and "D*N" separated
//     by ", " (:1104-1140);
//   * the frame files are <stem>_frame<N>.s, their trues / randoms /
//     coincidence histograms <stem>_frame<N>.tr.s / .ra.s / .ch, the .dyn
//     file the frame count and then one frame file per line;
//   * the head curve has one line per second;
//   * the dose delay is study date+time minus dose assay date+time
//     (get_dose_delay, :978-996);
//   * -ra writes the whole delayed sinogram.
#include <sys/mman.h>
#include <sys/stat.h>
#include <fcntl.h>
#include <unistd.h>

#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "hrrt_gpu.h"

namespace {

[[noreturn]] void die(const char *fmt, const char *a = "", const char *b = "") {
  std::fprintf(stderr, "lmhistogram_gpu: ");
  std::fprintf(stderr, fmt, a, b);
  std::fprintf(stderr, "\n");
  std::exit(1);
}

// HISTOGRAM_MODE (histogram_mp.hpp:41-46)
enum Mode { kTrues = 0, kPromptsRandoms = 1, kPrompts = 2, kTransmission = 7 };
// the rebinner method flags written to the header (histogram_mp.hpp:130)
enum { kSwRebinner = 0x2, kIgnoreBorder = 0x4, kNoDoi = 0x8 };
constexpr int kNumSinos3 = 6367, kNumSinos9 = 2209;  // NUM_SINOS (lmhistogram_mp.cpp:105-116)
constexpr int kBlocks = 936;
constexpr int kDefaultLld = 400;
constexpr long long kCrystals = 2LL * 104 * 8 * 72;

struct Options {
  std::string in, out;
  int span = 9;
  bool span_set = false;
  int mode = kTrues;
  bool ra = false, notimetag = false, nodoi = false, eb = false;
  std::vector<int> durations, skips;
  int device = 0;
};

void usage() {
  std::fprintf(stdout,
               "usage: lmhistogram_gpu <file.l64> [-o out.s] [--span 3|9] [--PR | -P] [--ra] [--notimetag]\n"
               "       [--nodoi] [--EB] [-d D | -d D,skip | -d D*N ...] [--device N]\n"
               "  reads <file>.l64.hdr; writes <out>.s + .s.hdr (per frame <out>_frame<N>.s), _lm.hc, .ch;\n"
               "  --PR: prompts in .s, trues (span 9 for span 3) in .tr.s, --ra: delayed in .ra.s\n");
}

// "D", "D,skip", "D*N" (lmhistogram_fromarchive.cpp:452-470)
void add_duration(Options &o, const char *s) {
  int d = 0, n = 0, skip = 0;
  char tail = 0;
  if (std::sscanf(s, "%d*%d%c", &d, &n, &tail) == 2) {
    if (d <= 0 || n <= 0) die("invalid frame duration argument: -d %s", s);
    for (int k = 0; k < n; k++) {
      o.durations.push_back(d);
      o.skips.push_back(0);
    }
    return;
  }
  const int got = std::sscanf(s, "%d,%d%c", &d, &skip, &tail);
  if (got < 1 || got > 2 || d < 0 || skip < 0) die("invalid frame duration argument: -d %s", s);
  o.durations.push_back(d);
  o.skips.push_back(got == 2 ? skip : 0);
}

void parse(int argc, char **argv, Options &o) {
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    if (a.size() < 2 || a[0] != '-') {
      if (!o.in.empty()) die("unexpected argument '%s'", a.c_str());
      o.in = a;
      continue;
    }
    const std::string name = a.substr(a[1] == '-' ? 2 : 1);
    auto val = [&]() -> std::string {
      if (i + 1 >= argc) die("option %s needs a value", a.c_str());
      return argv[++i];
    };
    if (name == "h" || name == "help") {
      usage();
      std::exit(0);
    } else if (name == "o" || name == "out") {
      o.out = val();
    } else if (name == "i" || name == "infile") {
      o.in = val();
    } else if (name == "span") {
      const std::string v = val();
      if (std::sscanf(v.c_str(), "%d", &o.span) != 1 || (o.span != 3 && o.span != 9)) die("span must be 3 or 9");
      o.span_set = true;
    } else if (name == "PR") {
      o.mode = kPromptsRandoms;
    } else if (name == "P" || name == "prompts") {
      o.mode = kPrompts;
    } else if (name == "ra") {
      o.ra = true;
    } else if (name == "notimetag") {
      o.notimetag = true;
    } else if (name == "nodoi") {
      o.nodoi = true;
    } else if (name == "EB") {
      o.eb = true;
    } else if (name == "d" || name == "duration") {
      add_duration(o, val().c_str());
      while (i + 1 < argc && argv[i + 1][0] != '-') add_duration(o, argv[++i]);  // multitoken
    } else if (name == "device") {
      if (std::sscanf(val().c_str(), "%d", &o.device) != 1) die("error decoding --device");
    } else if (name == "V" || name == "verbosity" || name == "l" || name == "log" || name == "model") {
      (void)val();
    } else if (name == "add" || name == "mock" || name == "count" || name == "start" || name == "L" ||
               name == "lr_type") {
      die("option %s is not supported", a.c_str());
    } else if (name == "scan") {
      die("--scan is not supported: the head curve is written with every histogram");
    } else {
      usage();
      die("unknown option '%s'", a.c_str());
    }
  }
  if (o.in.empty()) die("no input listmode file");
}

// ---- Interfile header: an ordered list of "key := value" tags (CHeader,
// cheader_lib/CHeader.cpp:130-330); writing a tag updates it in place or
// appends it ----
struct Header {
  std::vector<std::pair<std::string, std::string>> tags;

  static std::string rtrim(std::string s) {
    while (!s.empty() && (s.back() == ' ' || s.back() == '\t' || s.back() == '\r' || s.back() == '\n')) s.pop_back();
    return s;
  }
  bool read(const std::string &path) {
    FILE *f = std::fopen(path.c_str(), "rt");
    if (!f) return false;
    char buf[4096];
    while (std::fgets(buf, sizeof buf, f)) {
      std::string line = rtrim(buf);
      // "key := value": the last " := " splits key and value
      const size_t at = line.rfind(" :=");
      if (at == std::string::npos || at == 0) continue;
      size_t ks = line.find_first_not_of(" \t");
      std::string key = rtrim(line.substr(ks, at - ks));
      std::string value = line.substr(at + 3);
      const size_t vs = value.find_first_not_of(" \t");
      value = vs == std::string::npos ? std::string() : value.substr(vs);
      if (!key.empty()) tags.emplace_back(key, value);
    }
    std::fclose(f);
    return true;
  }
  const std::string *find(const std::string &key) const {
    for (const auto &t : tags)
      if (t.first == key) return &t.second;
    return nullptr;
  }
  bool get_int(const std::string &key, int *v) const {
    const std::string *s = find(key);
    return s && std::sscanf(s->c_str(), "%d", v) == 1;
  }
  bool get_float(const std::string &key, float *v) const {
    const std::string *s = find(key);
    return s && std::sscanf(s->c_str(), "%f", v) == 1;
  }
  void set(const std::string &key, const std::string &value) {
    for (auto &t : tags)
      if (t.first == key) {
        t.second = value;
        return;
      }
    tags.emplace_back(key, value);
  }
  void set_int(const std::string &key, long long v) { set(key, std::to_string(v)); }
  void set_float(const std::string &key, float v) {
    char b[64];
    std::snprintf(b, sizeof b, "%f", (double)v);
    set(key, b);
  }
  void write(const std::string &path) const {
    FILE *f = std::fopen(path.c_str(), "wt");
    if (!f) die("cannot write %s: %s", path.c_str(), std::strerror(errno));
    std::fprintf(f, "!INTERFILE\n");
    for (const auto &t : tags) std::fprintf(f, "%s := %s\n", t.first.c_str(), t.second.c_str());
    if (std::fclose(f) != 0) die("error writing %s", path.c_str());
  }
};

// days since 1970-01-01 of a proleptic Gregorian date
long long days_from_civil(int y, int m, int d) {
  y -= m <= 2;
  const long long era = (y >= 0 ? y : y - 399) / 400;
  const unsigned yoe = (unsigned)(y - era * 400);
  const unsigned doy = (153 * (m + (m > 2 ? -3 : 9)) + 2) / 5 + d - 1;
  const unsigned doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
  return era * 146097 + (long long)doe - 719468;
}

// seconds of "dd:mm:yyyy" + "hh:mm:ss", -1 when either does not parse
long long date_time(const std::string *date, const std::string *time) {
  int dd, mo, yy, hh, mi, ss;
  if (!date || !time) return -1;
  if (std::sscanf(date->c_str(), "%d:%d:%d", &dd, &mo, &yy) != 3) return -1;
  if (std::sscanf(time->c_str(), "%d:%d:%d", &hh, &mi, &ss) != 3) return -1;
  return days_from_civil(yy, mo, dd) * 86400 + hh * 3600 + mi * 60 + ss;
}

const std::string *find_any(const Header &h, const char *a, const char *b) {
  const std::string *s = h.find(a);
  return s ? s : h.find(b);
}

// get_dose_delay (lmhistogram_fromarchive.cpp:978-996): study minus dose
// assay, 0 when either is missing or the study is not later
int dose_delay(const Header &h) {
  const long long t0 = date_time(find_any(h, "dose_assay_date (dd:mm:yryr)", "dose assay date (dd:mm:yryr)"),
                                 find_any(h, "dose_assay_time (hh:mm:ss)", "dose assay time (hh:mm:ss)"));
  const long long t1 = date_time(find_any(h, "!study date (dd:mm:yryr)", "study date (dd:mm:yryr)"),
                                 find_any(h, "!study time (hh:mm:ss)", "study time (hh:mm:ss)"));
  if (t0 < 0 || t1 < 0 || t1 <= t0) return 0;
  return (int)(t1 - t0);
}

// GetDTC (lmhistogram_mp/dtc.cpp): exp(energy level x singles per block),
// the level interpolated between the LLD settings 250, 300, 350 and 400.
// Below 250 the reference leaves the level unset; 1 (no correction) here.
float dead_time_factor(int lld, long singles_per_block) {
  double e;
  if (lld < 250) return 1.0f;
  if (lld == 250) e = 6.9378e-6;
  else if (lld < 300) e = ((double)lld - 250.0) / 50.0 * (7.0677e-6 - 6.9378e-6) + 6.9378e-6;
  else if (lld == 300) e = 7.0677e-6;
  else if (lld < 350) e = ((double)lld - 300.0) / 50.0 * (7.7004e-6 - 7.0677e-6) + 7.0677e-6;
  else if (lld == 350) e = 7.7004e-6;
  else if (lld < 400) e = ((double)lld - 350.0) / 50.0 * (8.94e-6 - 7.7004e-6) + 7.7004e-6;
  else e = 8.94e-6;
  return (float)std::exp(e * (double)singles_per_block);
}

// "Frame definition" of the header: "D" and "D*N" items separated by ", "
// (lmhistogram_fromarchive.cpp:1104-1140)
void frames_from_header(Options &o, const std::string &def) {
  std::string s = def;
  for (char &c : s)
    if (c == ',') c = ' ';
  size_t p = 0;
  while (p < s.size()) {
    const size_t q = s.find(' ', p);
    const std::string item = s.substr(p, q == std::string::npos ? std::string::npos : q - p);
    p = q == std::string::npos ? s.size() : q + 1;
    if (item.empty()) continue;
    int d = 0, n = 0;
    if (std::sscanf(item.c_str(), "%d*%d", &d, &n) == 2) {
      if (d <= 0) break;
      for (int k = 0; k < n; k++) {
        o.durations.push_back(d);
        o.skips.push_back(0);
      }
    } else if (std::sscanf(item.c_str(), "%d", &d) == 1 && d > 0) {
      o.durations.push_back(d);
      o.skips.push_back(0);
    } else {
      break;
    }
  }
}

std::string strip_ext(const std::string &p, const char *ext) {
  const size_t n = std::strlen(ext);
  if (p.size() > n && p.compare(p.size() - n, n, ext) == 0) return p.substr(0, p.size() - n);
  const size_t dot = p.rfind('.'), slash = p.rfind('/');
  if (dot != std::string::npos && (slash == std::string::npos || dot > slash)) return p.substr(0, dot);
  return p;
}

std::string base_name(const std::string &p) {
  const size_t s = p.rfind('/');
  return s == std::string::npos ? p : p.substr(s + 1);
}

void write_file(const std::string &path, const void *data, size_t bytes, const char *mode = "wb") {
  FILE *f = std::fopen(path.c_str(), mode);
  if (!f) die("cannot write %s: %s", path.c_str(), std::strerror(errno));
  if (bytes && std::fwrite(data, 1, bytes, f) != bytes) die("error writing %s", path.c_str());
  if (std::fclose(f) != 0) die("error writing %s", path.c_str());
}

struct Mapped {
  const uint32_t *words = nullptr;
  long long n = 0;
  size_t bytes = 0;
  ~Mapped() {
    if (words) munmap(const_cast<uint32_t *>(words), bytes);
  }
};

void map_file(const std::string &path, Mapped &m) {
  const int fd = open(path.c_str(), O_RDONLY);
  if (fd < 0) die("%s: %s", path.c_str(), std::strerror(errno));
  struct stat st;
  if (fstat(fd, &st) != 0) die("%s: %s", path.c_str(), std::strerror(errno));
  m.bytes = (size_t)st.st_size;
  m.n = (long long)(m.bytes / 4);
  if (m.bytes > 0) {
    void *p = mmap(nullptr, m.bytes, PROT_READ, MAP_PRIVATE, fd, 0);
    if (p == MAP_FAILED) die("%s: mmap: %s", path.c_str(), std::strerror(errno));
    m.words = (const uint32_t *)p;
  }
  close(fd);
}

}  // namespace

int main(int argc, char **argv) {
  Options o;
  parse(argc, argv, o);
  struct stat st;
  if (stat(o.in.c_str(), &st) != 0 || !S_ISREG(st.st_mode)) die("%s: File not found", o.in.c_str());
  const std::string in_stem = strip_ext(o.in, ".l64");
  const std::string hdr_in = in_stem + ".l64.hdr";
  Header hdr;
  if (!hdr.read(hdr_in)) die("header %s not found", hdr_in.c_str());

  // set_tx_source_speed, set_lld, set_histogramming_mode, set_isotope_halflife,
  // get_dose_delay, set_span (lmhistogram_mp.cpp:849-935)
  if (const std::string *t = hdr.find("!PET data type"))
    if (Header::rtrim(*t) == "transmission") die("transmission scans are not supported");
  int lld = kDefaultLld;
  if (!hdr.get_int("lower level", &lld)) lld = kDefaultLld;
  int sino_mode = 0;
  if (hdr.get_int("Sinogram Mode", &sino_mode)) {
    if (sino_mode != kTrues && sino_mode != kPromptsRandoms && sino_mode != kPrompts)
      die("Sinogram Mode %s is not supported", std::to_string(sino_mode).c_str());
    o.mode = sino_mode;
  }
  float halflife = 0.f;
  hdr.get_float("isotope halflife", &halflife);
  if (halflife == 0.f) die("No isotope halflife");
  const float decay_rate = halflife;
  const int delay = dose_delay(hdr);
  int axial = 0;
  if (hdr.get_int("axial compression", &axial)) {
    if (!o.span_set && axial > 0)
      o.span = axial;
    else
      hdr.set_int("axial compression", o.span);
  }
  if (o.span != 3 && o.span != 9) die("span %s is not supported (3 or 9)", std::to_string(o.span).c_str());
  if (o.durations.empty())
    if (const std::string *def = hdr.find("Frame definition")) frames_from_header(o, *def);
  if (o.durations.empty()) {  // one frame over the whole stream
    o.durations.push_back(0);
    o.skips.push_back(0);
  }
  const int nframes = (int)o.durations.size();
  const int nsinos = o.span == 3 ? kNumSinos3 : kNumSinos9;

  // create_hrrt_sinogram_header, do_init_rebinner (lmhistogram_mp.cpp:1025-1077)
  std::string stem = o.out.empty() ? in_stem : strip_ext(o.out, ".s");
  const unsigned method = kSwRebinner | (o.nodoi ? kNoDoi : 0) | (o.eb ? kIgnoreBorder : 0);
  hdr.set("!originating system", "HRRT");
  hdr.set("!name of data file", stem + ".s");
  hdr.set_int("number of dimensions", 3);
  hdr.set_int("matrix size [1]", 256);
  hdr.set_int("matrix size [2]", 288);
  hdr.set_int("matrix size [3]", nsinos);
  hdr.set("data format", "sinogram");
  hdr.set("number format", "signed integer");
  hdr.set_int("number of bytes per pixel", 2);
  hdr.set("!lmhistogram version", "HRRT_U 1.1");
  hdr.set("!lmhistogram build ID", std::string(__DATE__) + " " + __TIME__);
  hdr.set("!histogrammer revision", "2.0");
  hdr.set_float("scaling factor (mm/pixel) [1]", 10.0f * 0.121875f);
  hdr.set_int("scaling factor [2]", 1);
  hdr.set_float("scaling factor (mm/pixel) [3]", 10.0f * 0.121875f);
  hdr.set_int("!LM rebinner method", method);
  hdr.set_int("axial compression", o.span);
  hdr.set_int("maximum ring difference", 67);

  Mapped m;
  map_file(o.in, m);
  hrrt_lm *lm = nullptr;
  if (hrrt_lm_create(o.span, 67, o.device, &lm) != HRRT_OK) die("cannot create the listmode histogrammer");
  const long long S = hrrt_lm_sino_size(lm);
  std::vector<uint16_t> sino((size_t)S), delayed(o.mode == kPromptsRandoms ? (size_t)S : 0);
  std::vector<uint32_t> coinc(2 * kCrystals);
  std::vector<hrrt_lm_second> hc;
  std::vector<int> rates(kBlocks);
  int flags = HRRT_LM_HEAD_CURVE | HRRT_LM_CRYSTAL_COUNTS;
  if (o.eb) flags |= HRRT_LM_IGNORE_BORDER_CRYSTAL;
  if (o.nodoi) flags |= HRRT_LM_NO_DOI;
  if (o.notimetag) flags |= HRRT_LM_TIME_FROM_COUNT;
  const int lm_mode = o.mode == kPromptsRandoms ? HRRT_LM_PROMPTS_AND_DELAYED
                      : o.mode == kPrompts      ? HRRT_LM_PROMPTS_ONLY
                                                : HRRT_LM_TRUES;

  const std::string hc_path = in_stem + "_lm.hc";
  FILE *hcf = std::fopen(hc_path.c_str(), "wt");
  if (!hcf) die("cannot write %s: %s", hc_path.c_str(), std::strerror(errno));
  std::string dyn;
  if (nframes > 1) dyn = std::to_string(nframes) + "\n";

  long long pos = 0;
  long long current_time = -1;
  for (int f = 0; f < nframes; f++) {
    const std::string fstem = nframes > 1 ? stem + "_frame" + std::to_string(f) : stem;
    const std::string sino_path = fstem + ".s";
    if (nframes > 1) dyn += base_name(sino_path) + "\n";
    // position the stream (do_histogram_frame, lmhistogram_mp.cpp:969-986)
    const int target = o.skips[f] > 0 ? o.skips[f] : 0;
    if (o.skips[f] > 0 || current_time < 0) {
      long long used = 0;
      const int rc = hrrt_lm_seek(lm, m.words + pos, m.n - pos, pos, target, flags, &used);
      if (rc == HRRT_ERR_NOT_FOUND) {
        if (target > 0) die("Unable to locate requested time %s", std::to_string(target).c_str());
        die("Unable to locate time reset");
      }
      if (rc != HRRT_OK) die("seek: %s", hrrt_lm_last_error(lm));
      pos += used;
    }
    hrrt_lm_stats stt;
    int rc = hrrt_lm_histogram_at(lm, m.words + pos, m.n - pos, pos, lm_mode, o.durations[f], flags, sino.data(),
                                  delayed.empty() ? nullptr : delayed.data(), &stt);
    if (rc != HRRT_OK) die("histogram: %s", hrrt_lm_last_error(lm));
    pos += stt.words_used;
    const int n_hc = hrrt_lm_head_curve(lm, nullptr, 0);
    hc.resize((size_t)std::max(n_hc, 0));
    if (n_hc > 0) hrrt_lm_head_curve(lm, hc.data(), n_hc);
    long long line_prompts = 0, line_randoms = 0;
    if (hrrt_lm_block_singles(lm, rates.data(), &line_prompts, &line_randoms) != kBlocks ||
        hrrt_lm_crystal_counts(lm, coinc.data()) != HRRT_OK)
      die("frame statistics: %s", hrrt_lm_last_error(lm));
    std::fprintf(hcf, "Singles,Randoms,Prompts,Time(ms)\n");
    for (const hrrt_lm_second &l : hc)
      std::fprintf(hcf, "%lld,%lld,%lld,%lld\n", l.total_singles, l.randoms, l.prompts, l.time_ms);

    // histogram() returns the frame start and sets the frame's duration
    // (histogram_mp.cpp:1390-1397)
    const int relative_start = (int)stt.frame_start;
    const int duration = (int)stt.duration;
    if (duration <= 0) die("Invalid frame duration %s", std::to_string(duration).c_str());
    current_time = relative_start + duration;

    // write_sino (lmhistogram_mp.cpp:574-736)
    hdr.set_int("image duration", duration);
    hdr.set_int("image relative start time", relative_start);
    const int decay_time = relative_start + delay;
    float dcf1 = 1.0f, dcf2 = 1.0f;
    if (decay_rate > 0.0f) {
      dcf1 = std::pow(2.0f, decay_time / decay_rate);
      dcf2 = (float)((std::log(2.0) * duration) /
                     (decay_rate * (1.0 - std::pow(2.0f, -1.0f * duration / decay_rate))));
    }
    hdr.set_float("decay correction factor", dcf1);
    hdr.set_float("decay correction factor2", dcf2);
    hdr.set_int("frame", f);
    // the per-second totals plus the events after the last line
    // (histogram_mp.cpp:1387-1388): every event of the frame
    hdr.set_int("Total Prompts", stt.prompts);
    hdr.set_int("Total Randoms", stt.delayed);
    hdr.set_int("Total Net Trues", stt.prompts - stt.delayed);
    long long av = 0;
    for (int b = 0; b < kBlocks; b++) {
      hdr.set_int("block singles " + std::to_string(b), rates[b]);
      av += rates[b];
    }
    av /= kBlocks;
    hdr.set_int("average singles per block", av);
    hdr.set_float("Dead time correction factor", dead_time_factor(lld, (long)av));
    hdr.set("!name of data file", sino_path);
    hdr.set("Sinogram data type", o.mode == kTrues ? "true" : "prompt");
    if (o.mode == kPromptsRandoms) hdr.set("!name of true data file", fstem + ".tr.s");
    write_file(sino_path, sino.data(), sizeof(uint16_t) * (size_t)S);
    hdr.write(sino_path + ".hdr");
    if (o.mode == kPromptsRandoms) {
      // trues = prompts - delayed, folded into span 9 from span 3
      const std::string tr_path = fstem + ".tr.s";
      std::vector<int16_t> tr;
      if (o.span == 3) {
        tr.resize((size_t)kNumSinos9 * 256 * 288);
        if (hrrt_lm_convert_span9((const int16_t *)sino.data(), (const int16_t *)delayed.data(), tr.data(), 67) !=
            kNumSinos9)
          die("convert_span9 failed");
      } else {
        tr.resize((size_t)S);
        for (long long j = 0; j < S; j++) tr[j] = (int16_t)(uint16_t)(sino[j] - delayed[j]);
      }
      hdr.set("!name of data file", tr_path);
      hdr.set("Sinogram data type", "true");
      hdr.set_int("axial compression", 9);
      hdr.set_int("matrix size [3]", kNumSinos9);
      write_file(tr_path, tr.data(), sizeof(int16_t) * tr.size());
      hdr.write(tr_path + ".hdr");
      hdr.set_int("axial compression", o.span);
      hdr.set_int("matrix size [3]", nsinos);
      if (o.ra) {
        const std::string ra_path = fstem + ".ra.s";
        hdr.set("!name of data file", ra_path);
        hdr.set("Sinogram data type", "delayed");
        write_file(ra_path, delayed.data(), sizeof(uint16_t) * (size_t)S);
        hdr.write(ra_path + ".hdr");
      }
    }
    // write_coin_map: prompt then delayed crystal counts
    write_file(fstem + ".ch", coinc.data(), sizeof(uint32_t) * coinc.size());
    std::fprintf(stdout, "frame %d: start %d s, duration %d s, prompts %lld, delayed %lld -> %s\n", f,
                 relative_start, duration, stt.prompts, stt.delayed, sino_path.c_str());
  }
  if (std::fclose(hcf) != 0) die("error writing %s", hc_path.c_str());
  if (nframes > 1) write_file(stem + ".dyn", dyn.data(), dyn.size(), "wt");
  hrrt_lm_destroy(lm);
  return 0;
}
