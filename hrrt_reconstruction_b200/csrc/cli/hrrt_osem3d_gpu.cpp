// hrrt_osem3d_gpu -- the hrrt_osem3d command line on libhrrt_gpu.
//
// Takes the reference's flags and flat files (hrrt_osem3d_span3.cpp:3154-3355,
// usage :466-530) for the OP-OSEM path (-W 3) and writes the same outputs:
// the image as flat float [z][y][x] (SaveImage, :4020-4043) with its
// Interfile header (write_image_header.cpp:185-265), and with -h the forward
// projection of the final image as a flat float sinogram.
//
// Supported: -p -d -n -a -s -o -O -i -h -I -S -W 3 -m -f -k -e -u -Q -F -T -N
// -D -L -v -X 256 -M 999 -g -B, -z 1, -Z 1, and je_hrrt_osem3d's -b 1,beta
// (MAP, hrrt_osem3d.cpp:3360-3369).  The attenuation may be the span-9 file
// of a span-3 reconstruction (Atten3D_Span9, :1762-1796), the scatter a 2D
// segment with span-9 scale factors, the randoms a coincidence histogram
// (.ch).  Options for paths outside OP-OSEM (-t trues, -P/-R pre-corrected /
// 4-byte scans, -A MAP-EM gradient variant, -U mu-map, -C compression, -w)
// are refused with a message.
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "hrrt_gpu.h"

namespace {

struct Options {
  std::string prompt, delayed, norm, atten, scatter, out, init, out3d;
  bool save_each = false, float_prompts = false;
  int iterations = 1, subsets = 16, weighting = 2, span = 9, maxdel = 67, npskip = 0, verbose = 0, device = 0;
  bool psf = false;
  float psf_fwhm1 = 0.f, psf_fwhm2 = 0.f, psf_ratio = 0.f;
  int map_technique = 0;
  float map_beta = 0.f;
  int in_flip = 0, out_flip = 0, trim = 0;
  float rel_fov = 0.95f, image_max = 1.e4f, eps1 = 5.e-2f, eps2 = 1.e-2f, eps3 = 1.e-10f;
  int z_min = 6, z_max = 200;
  bool npskip_set = false;
};

[[noreturn]] void die(const char *fmt, const char *a = "", const char *b = "") {
  std::fprintf(stderr, "hrrt_osem3d_gpu: ");
  std::fprintf(stderr, fmt, a, b);
  std::fprintf(stderr, "\n");
  std::exit(1);
}

void usage() {
  std::fprintf(stdout,
               "usage: hrrt_osem3d_gpu -p prompts -d delayed [-n norm] [-a atten] [-s scatter] -o image|-O image\n"
               "       [-i initial_image] [-h out_3D_scan] -W 3 [-I iterations] [-S subsets] [-m span,maxdel]\n"
               "       [-f rel_fov,trim,zmin,zmax] [-k npskip] [-e eps1,eps2,eps3] [-u image_max] [-Q]\n"
               "       [-F in_flip,out_flip] [-T threads] [-N] [-D dir] [-L log] [-v level] [-X 256]\n"
               "  -p  3D flat integer (int16) prompt scan; -Q: float prompt scan of integer counts\n"
               "  -d  3D flat float delayed (smoothed randoms), or a coincidence histogram (.ch) from which the\n"
               "      smoothed randoms are computed over the scan duration in the prompt sinogram's .hdr\n"
               "  -n  3D flat normalisation, -a attenuation (span 9 accepted for span 3), -s scatter\n"
               "      (3D, or the unscaled 2D segment followed by 2209 span-9 plane scale factors)\n"
               "  -o  output image (flat float [z][y][x] + .hdr), -O also after each iteration\n"
               "  -h  output the forward projection of the final image (flat float scan)\n"
               "  -B  fwhm1,fwhm2,ratio: PSF resolution modelling (0,0,0: the HRRT defaults)\n"
               "  -b  technique,beta: MAP with the one-step-late prior of je_hrrt_osem3d (technique 1)\n");
}

bool parse(int argc, char **argv, Options &o) {
  for (int i = 1; i < argc; i++) {
    const char *a = argv[i];
    if (a[0] != '-' || a[1] == 0) die("unexpected argument '%s'", a);
    const char c = a[1];
    auto val = [&]() -> const char * {
      if (a[2]) return a + 2;
      if (i + 1 >= argc) die("option -%s needs a value", a + 1);
      return argv[++i];
    };
    switch (c) {
      case 'p': o.prompt = val(); break;
      case 'd': o.delayed = val(); break;
      case 'n': o.norm = val(); break;
      case 'a': o.atten = val(); break;
      case 's': o.scatter = val(); break;
      case 'o': o.out = val(); break;
      case 'O': o.out = val(); o.save_each = true; break;
      case 'i': o.init = val(); break;
      case 'h': o.out3d = val(); break;
      case 'Q': o.float_prompts = true; break;
      case 'N': break;                  // sensitivity images stay in device memory
      case 'D': (void)val(); break;     // no normfac.i is written
      case 'L': (void)val(); break;     // log to stdout/stderr
      case 'T': (void)val(); break;     // one GPU, no host threads to set
      case 'I': if (std::sscanf(val(), "%d", &o.iterations) != 1) die("error decoding -I"); break;
      case 'S': if (std::sscanf(val(), "%d", &o.subsets) != 1) die("error decoding -S"); break;
      case 'W': if (std::sscanf(val(), "%d", &o.weighting) != 1) die("error decoding -W"); break;
      case 'v': if (std::sscanf(val(), "%d", &o.verbose) != 1) die("error decoding -v"); break;
      case 'm': if (std::sscanf(val(), "%d,%d", &o.span, &o.maxdel) != 2) die("error decoding -m"); break;
      case 'k': if (std::sscanf(val(), "%d", &o.npskip) != 1) die("error decoding -k"); o.npskip_set = true; break;
      case 'u': if (std::sscanf(val(), "%f", &o.image_max) != 1) die("error decoding -u"); break;
      case 'e':
        if (std::sscanf(val(), "%f,%f,%f", &o.eps1, &o.eps2, &o.eps3) != 3) die("error decoding -e");
        break;
      case 'f':
        if (std::sscanf(val(), "%f,%d,%d,%d", &o.rel_fov, &o.trim, &o.z_min, &o.z_max) != 4) die("error decoding -f");
        break;
      case 'F':
        if (std::sscanf(val(), "%d,%d", &o.in_flip, &o.out_flip) != 2) die("error decoding -F");
        break;
      case 'X': {
        int x = 0;
        if (std::sscanf(val(), "%d", &x) != 1 || x != 256) die("-X: the HRRT image is 256 wide");
        break;
      }
      case 'M': {
        int m = 0;
        if (std::sscanf(val(), "%d", &m) != 1 || m != 999) die("-M: only the HRRT (model 999) is supported");
        break;
      }
      case 'g': (void)val(); break;  // all segment groups are reconstructed
      case 'z':
      case 'Z': {
        float z = 0;
        if (std::sscanf(val(), "%f", &z) != 1 || z != 1.0f) die("-%s: zoom 1 only", c == 'z' ? "z" : "Z");
        break;
      }
      case 't': die("-t (trues input) is outside the OP-OSEM path; use -p and -d");
      case 'P': case 'R': die("-%s: pre-corrected / 4-byte scans are outside the OP-OSEM path", a + 1);
      case 'B':
        if (std::sscanf(val(), "%f,%f,%f", &o.psf_fwhm1, &o.psf_fwhm2, &o.psf_ratio) != 3) die("error decoding -B");
        o.psf = true;
        break;
      case 'A': die("-A (the MAP-EM gradient variant) is not supported; -b 1,beta gives je_hrrt_osem3d's MAP");
      case 'b':
        // -b technique,beta (je_hrrt_osem3d/hrrt_osem3d.cpp:3360-3369)
        if (std::sscanf(val(), "%d,%f", &o.map_technique, &o.map_beta) != 2) die("error decoding -b");
        if (o.map_technique == 0) o.map_beta = 0.f;
        if (o.map_beta == 0.f) o.map_technique = 0;
        if (o.map_technique != 0 && o.map_technique != 1) die("-b: MAP technique 1 only");
        break;
      case 'U': die("-U (mu-map reconstruction) is not supported");
      case 'C': die("-C (sinogram compression) is not supported");
      case 'w': die("-w is not supported");
      default:
        usage();
        die("unknown option '%s'", a);
    }
  }
  if (o.prompt.empty() || o.delayed.empty()) die("-p prompts and -d delayed are required");
  if (o.out.empty()) die("-o or -O output image is required");
  if (o.weighting != 3) die("only -W 3 (OP-OSEM) is implemented on the GPU");
  return true;
}

long long file_size(const std::string &path) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) die("cannot open %s: %s", path.c_str(), std::strerror(errno));
  std::fseek(f, 0, SEEK_END);
  const long long n = std::ftell(f);
  std::fclose(f);
  return n;
}

template <typename T>
std::vector<T> read_flat(const std::string &path, size_t count) {
  std::vector<T> v(count);
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) die("cannot open %s: %s", path.c_str(), std::strerror(errno));
  if (std::fread(v.data(), sizeof(T), count, f) != count) die("short read on %s", path.c_str());
  std::fclose(f);
  return v;
}

void write_flat(const std::string &path, const void *p, size_t bytes) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) die("cannot create %s: %s", path.c_str(), std::strerror(errno));
  if (std::fwrite(p, 1, bytes, f) != bytes) die("write error on %s", path.c_str());
  std::fclose(f);
}

const char *base(const std::string &p) {
  const size_t k = p.find_last_of("/\\");
  return k == std::string::npos ? p.c_str() : p.c_str() + k + 1;
}

// write_image_header (write_image_header.cpp:185-265) for an OP image
void write_header(const Options &o, const hrrt_info &info, float voxel_mm, float plane_mm, int iterations) {
  const std::string name = o.out + ".hdr";
  FILE *f = std::fopen(name.c_str(), "wt");
  if (!f) die("cannot create %s", name.c_str());
  std::fprintf(f, "!INTERFILE\n");
  std::fprintf(f, "name of data file := %s\n", o.out.c_str());
  std::fprintf(f, "data format := image\n");
  std::fprintf(f, "number format := float\n");
  std::fprintf(f, "number of bytes per pixel := 4\n");
  std::fprintf(f, "number of dimensions := 3\n");
  std::fprintf(f, "matrix size [1] := %d\n", info.nx);
  std::fprintf(f, "matrix size [2] := %d\n", info.ny);
  std::fprintf(f, "matrix size [3] := %d\n", info.nz);
  std::fprintf(f, "scaling factor (mm/pixel) [1] := %f\n", voxel_mm);
  std::fprintf(f, "scaling factor (mm/pixel) [2] := %f\n", voxel_mm);
  std::fprintf(f, "scaling factor (mm/pixel) [3] := %f\n", plane_mm);
  std::fprintf(f, o.psf ? "reconstruction method := inki-2006-may-OSEM3D-OP-PSF\n"
                        : "reconstruction method := inki-2006-may-OSEM3D-OP\n");
  std::fprintf(f, "reconstruction version := hrrt_osem3d_gpu\n");
  std::fprintf(f, "prompt file used := %s\n", base(o.prompt));
  std::fprintf(f, "delayed file used := %s\n", base(o.delayed));
  if (!o.norm.empty()) std::fprintf(f, "norm file used := %s\n", base(o.norm));
  if (!o.atten.empty()) std::fprintf(f, "atten file used := %s\n", base(o.atten));
  if (!o.scatter.empty()) std::fprintf(f, "scatter file used := %s\n", base(o.scatter));
  std::fprintf(f, "number of iterations := %d\n", iterations);
  std::fprintf(f, "number of subsets := %d\n", o.subsets);
  // lines of the prompt scan's header that the image header does not restate
  FILE *in = std::fopen((o.prompt + ".hdr").c_str(), "r");
  if (in) {
    static const char *skip[] = {"!INTERFILE", "!Interfile", "!interfile", "name of data file", "data format",
                                 "number format", "number of bytes per", "number of dimensions", "matrix size",
                                 "scaling factor", "reconstruction method", "true file used", "prompt file used",
                                 "delayed file used", "norm file used", "atten file used", "scatter file used",
                                 "number of iterations", "number of subsets", "CPSCC-OSEM3D build",
                                 "CPSCC-Server build"};
    char line[1024];
    while (std::fgets(line, sizeof line, in)) {
      bool drop = false;
      for (const char *s : skip)
        if (std::strstr(line, s)) drop = true;
      if (!drop) std::fputs(line, f);
    }
    std::fclose(in);
  }
  std::fclose(f);
}

// Span-9 attenuation for a span-3 reconstruction (Atten3D_Span9,
// hrrt_osem3d_span3.cpp:1762-1796): span-3 segment s of group h takes the
// span-9 segment of group (h+1)/3 with the same sign, at the same axial
// planes.
std::vector<float> expand_span9_atten(const std::vector<float> &a9, const hrrt_geom &g3, int nrings) {
  auto segs = [&](int span, std::vector<int> &yb, std::vector<int> &off, std::vector<int> &np) {
    const int G = (g3.maxdel - (span - 1) / 2) / span, nz = 2 * nrings - 1;
    yb.assign(2 * G + 1, 0);
    np.assign(2 * G + 1, nz);
    for (int gr = 1; gr <= G; gr++) {
      const int zmin = (span + 1) / 2 + (gr - 1) * span;
      yb[2 * gr - 1] = yb[2 * gr] = zmin;
      np[2 * gr - 1] = np[2 * gr] = nz - 2 * zmin;
    }
    off.assign(2 * G + 1, 0);
    for (size_t s = 1; s < yb.size(); s++) off[s] = off[s - 1] + np[s - 1];
    return off.back() + np.back();
  };
  std::vector<int> yb3, off3, np3, yb9, off9, np9;
  const int P3 = segs(3, yb3, off3, np3), P9 = segs(9, yb9, off9, np9);
  const size_t plane = (size_t)g3.nangles * g3.nelements;
  if (a9.size() != (size_t)P9 * plane) die("span-9 attenuation has the wrong size");
  std::vector<float> a3((size_t)P3 * plane);
  for (size_t s = 0; s < yb3.size(); s++) {
    const int h = (int)(s + 1) / 2, gr = (h + 1) / 3;  // span-3 group, span-9 group
    const int src = (gr == 0) ? 0 : (s % 2 == 1 ? 2 * gr - 1 : 2 * gr);
    for (int p = 0; p < np3[s]; p++) {
      const int p9 = p + yb3[s] - yb9[src];
      std::memcpy(&a3[(size_t)(off3[s] + p) * plane], &a9[(size_t)(off9[src] + p9) * plane], plane * sizeof(float));
    }
  }
  return a3;
}

// 3D scatter from the unscaled 2D segment (nz planes) followed by the
// span-9 per-plane scale factors (the s2DFlag file form, drv:4407-4421):
// convert_s9_s3 (drv:1136-1162) turns the factors into span-3 ones, and
// apply_scale_factors (drv:1169-1179) scales 2D plane yr_bottom+yr into
// plane yr of each segment.  Both are restated as the reference runs them,
// including convert_s9_s3's walk over the span-3 segments three at a time.
std::vector<float> expand_scatter_2d(const std::vector<float> &file, const hrrt_geom &g, int nz, size_t plane) {
  const long long tb = hrrt_geometry_table(&g, "segments", nullptr, 0);
  if (tb <= 0) die("scatter: segment table");
  std::vector<int> seg((size_t)tb / sizeof(int));
  hrrt_geometry_table(&g, "segments", seg.data(), (size_t)tb);
  const int nseg = (int)seg.size() / 3;
  const int *yb = seg.data(), *yt = seg.data() + nseg, *off = seg.data() + 2 * nseg;
  const int P = off[nseg - 1] + yt[nseg - 1] - yb[nseg - 1] + 1;
  const int P9 = 2209;
  const float *sc2d = file.data(), *sf9 = file.data() + (size_t)nz * plane;
  std::vector<float> sf(P, 0.f);
  if (g.span == 9) {
    std::copy(sf9, sf9 + P9, sf.begin());
  } else {
    int i = 0, j = 0;
    for (int th = 0; th < nseg; th += 3) {
      int n = yt[th] - yb[th] + 1;
      if (j + n > P9 || i + n > P) die("scatter: scale factors do not fit this span");
      for (int p = 0; p < n; p++) sf[i++] = sf9[j++] / 3.0f;
      for (int k = 1; k <= 2 && th + k < nseg; k++) {
        const int so = yb[th + k] - yb[th + k - 1];
        const int m = n - 2 * so;
        if (m < 0 || i + m > P) die("scatter: scale factors do not fit this span");
        std::memmove(&sf[i], &sf[i - n + so], (size_t)m * sizeof(float));
        n = m;
        i += n;
      }
    }
  }
  std::vector<float> out((size_t)P * plane);
  for (int s = 0; s < nseg; s++)
    for (int yr = 0; yr <= yt[s] - yb[s]; yr++) {
      const float f = sf[off[s] + yr];
      const float *src = sc2d + (size_t)(yb[s] + yr) * plane;
      float *dst = out.data() + (size_t)(off[s] + yr) * plane;
      for (size_t k = 0; k < plane; k++) dst[k] = src[k] * f;
    }
  return out;
}

// get_scan_duration (hrrt_osem_utils.cpp:8-25): "image duration := <s>" in
// the prompt sinogram's .hdr
bool scan_duration_of(const std::string &sino, float *out) {
  FILE *f = std::fopen((sino + ".hdr").c_str(), "rt");
  if (!f) return false;
  char line[256];
  bool found = false;
  while (!found && std::fgets(line, sizeof line, f)) {
    const char *p = std::strstr(line, "image duration");
    if (p && (p = std::strstr(p, ":=")) && std::sscanf(p + 2, "%g", out) == 1) found = true;
  }
  std::fclose(f);
  return found;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 2) {
    usage();
    return 1;
  }
  Options o;
  parse(argc, argv, o);
  hrrt_geom g;
  hrrt_geom_default(&g);
  g.span = o.span;
  g.maxdel = o.maxdel;
  g.subsets = o.subsets;
  g.rel_fov = o.rel_fov;
  g.z_min = o.z_min;
  g.z_max = o.z_max;
  if (o.npskip_set) g.npskip = o.npskip;
  g.epsilon1 = o.eps1;
  g.epsilon2 = o.eps2;
  g.epsilon3 = o.eps3;
  g.image_max = o.image_max;
  const auto t0 = std::chrono::steady_clock::now();
  hrrt_ctx *ctx = nullptr;
  if (hrrt_ctx_create(&g, o.device, &ctx) != HRRT_OK) die("%s", hrrt_last_error(ctx));
  hrrt_info info;
  hrrt_get_info(ctx, &info);
  const size_t nbins = (size_t)info.segmentsize * info.nviews * info.nbins;

  // inputs (sizes checked as the reference does, drv:4407-4499)
  std::vector<int16_t> prompts;
  if (o.float_prompts) {
    if (file_size(o.prompt) != (long long)(nbins * 4)) die("%s: not a float scan of this span", o.prompt.c_str());
    const std::vector<float> pf = read_flat<float>(o.prompt, nbins);
    prompts.resize(nbins);
    for (size_t i = 0; i < nbins; i++) {
      const float v = pf[i];
      if (v != std::floor(v) || v < -32768.f || v > 32767.f)
        die("%s: -Q prompts must be integer counts within 16 bits", o.prompt.c_str());
      prompts[i] = (int16_t)v;
    }
  } else {
    if (file_size(o.prompt) != (long long)(nbins * 2)) die("%s: not an int16 scan of this span", o.prompt.c_str());
    prompts = read_flat<int16_t>(o.prompt, nbins);
  }
  auto read_scan = [&](const std::string &p) {
    if (p.empty()) return std::vector<float>();
    if (file_size(p) != (long long)(nbins * 4)) die("%s: not a float scan of this span", p.c_str());
    return read_flat<float>(p, nbins);
  };
  const std::vector<float> norm = read_scan(o.norm);
  std::vector<float> delayed;
  // a coincidence histogram (.ch: int32 counts per crystal and DOI
  // combination, drv:4424-4471) stands for the smoothed randoms gen_delays
  // computes from it, over the prompt sinogram's scan duration
  const long long ch_bytes = (long long)2 * 2 * 104 * 8 * 72 * 4;
  if (file_size(o.delayed) == ch_bytes) {
    float duration = 0.f;
    if (!scan_duration_of(o.prompt, &duration))
      die("Error: scan duration not found in sinogram %s header", o.prompt.c_str());
    const std::vector<int32_t> ch = read_flat<int32_t>(o.delayed, (size_t)ch_bytes / 4);
    hrrt_lm *lm = nullptr;
    if (hrrt_lm_create(o.span, o.maxdel, o.device, &lm) != HRRT_OK) die("%s", hrrt_lm_last_error(lm));
    if ((size_t)hrrt_lm_sino_size(lm) != nbins) die("smoothed randoms: sinogram size mismatch");
    delayed.resize(nbins);
    int iters = 0;
    if (hrrt_lm_smooth_randoms(lm, ch.data(), duration, 0.f, delayed.data(), &iters) != HRRT_OK)
      die("%s", hrrt_lm_last_error(lm));
    hrrt_lm_destroy(lm);
    if (o.verbose) std::printf("smoothed randoms from %s (%g s, %d singles iterations)\n", o.delayed.c_str(),
                               duration, iters);
  } else {
    delayed = read_scan(o.delayed);
  }
  std::vector<float> scatter;
  if (!o.scatter.empty()) {
    const size_t plane = (size_t)info.nviews * info.nbins;
    const long long sz = file_size(o.scatter);
    if (sz == (long long)((plane * info.nz + 2209) * 4))
      scatter = expand_scatter_2d(read_flat<float>(o.scatter, plane * info.nz + 2209), g, info.nz, plane);
    else
      scatter = read_scan(o.scatter);
  }
  std::vector<float> atten;
  if (!o.atten.empty()) {
    const long long sz = file_size(o.atten);
    if (sz == (long long)(nbins * 4)) {
      atten = read_flat<float>(o.atten, nbins);
    } else if (o.span == 3 && sz == (long long)2209 * info.nviews * info.nbins * 4) {
      atten = expand_span9_atten(read_flat<float>(o.atten, (size_t)2209 * info.nviews * info.nbins), g, g.nrings);
    } else {
      die("%s: attenuation size matches neither this span nor span 9", o.atten.c_str());
    }
  }
  if (hrrt_upload_inputs(ctx, prompts.data(), delayed.data(), norm.empty() ? nullptr : norm.data(),
                         atten.empty() ? nullptr : atten.data(), scatter.empty() ? nullptr : scatter.data(),
                         HRRT_STORE_F32) != HRRT_OK)
    die("%s", hrrt_last_error(ctx));
  if (o.psf && hrrt_set_psf(ctx, 1, o.psf_fwhm1, o.psf_fwhm2, o.psf_ratio) != HRRT_OK)
    die("%s", hrrt_last_error(ctx));
  // MAP from the sixth subset of the first iteration on (i_min_MAP,
  // je_hrrt_osem3d/hrrt_osem3d.cpp:4332-4341)
  if (o.map_technique && hrrt_set_map(ctx, o.map_technique, o.map_beta, 5) != HRRT_OK)
    die("MAP: %s", hrrt_last_error(ctx));
  if (hrrt_sensitivity(ctx) != HRRT_OK) die("%s", hrrt_last_error(ctx));
  const size_t vox = (size_t)info.nx * info.ny * info.nz;
  std::vector<float> img(vox);
  if (!o.init.empty()) {
    if (file_size(o.init) != (long long)(vox * 4)) die("%s: initial image size", o.init.c_str());
    img = read_flat<float>(o.init, vox);
    if (o.in_flip) {  // [z][y][x] stored transposed in x/y (-F)
      std::vector<float> t(vox);
      for (int z = 0; z < info.nz; z++)
        for (int y = 0; y < info.ny; y++)
          for (int x = 0; x < info.nx; x++)
            t[((size_t)z * info.ny + y) * info.nx + x] = img[((size_t)z * info.ny + x) * info.nx + y];
      img.swap(t);
    }
  }
  if (hrrt_init_image(ctx, o.init.empty() ? nullptr : img.data()) != HRRT_OK) die("%s", hrrt_last_error(ctx));

  const float voxel_mm = 1.21875f, plane_mm = 1.21875f;
  auto save = [&](int iters) {
    if (hrrt_get_image(ctx, img.data()) != HRRT_OK) die("%s", hrrt_last_error(ctx));
    if (o.out_flip) {
      std::vector<float> t(vox);
      for (int z = 0; z < info.nz; z++)
        for (int y = 0; y < info.ny; y++)
          for (int x = 0; x < info.nx; x++)
            t[((size_t)z * info.ny + y) * info.nx + x] = img[((size_t)z * info.ny + x) * info.nx + y];
      img.swap(t);
    }
    write_flat(o.out, img.data(), vox * 4);
    write_header(o, info, voxel_mm, plane_mm, iters);
  };
  for (int it = 0; it < o.iterations; it++) {
    hrrt_stats st;
    if (hrrt_osem(ctx, 1, &st) != HRRT_OK) die("%s", hrrt_last_error(ctx));
    std::printf("  Iteration %d: image sum %.6g, %.1f ms on the GPU\n", it + 1, st.sum_image, st.ms_total);
    if (o.save_each && it + 1 < o.iterations) save(it + 1);
  }
  save(o.iterations);
  if (!o.out3d.empty()) {
    std::vector<float> xyz((size_t)info.nx * info.ny * info.zp);
    std::vector<float> sino(nbins);
    if (hrrt_get_image_xyz(ctx, xyz.data()) != HRRT_OK || hrrt_forward_project(ctx, xyz.data(), sino.data()) != HRRT_OK)
      die("%s", hrrt_last_error(ctx));
    write_flat(o.out3d, sino.data(), nbins * 4);
  }
  hrrt_ctx_destroy(ctx);
  const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::printf("  hrrt_osem3d_gpu done in %.2f s\n", s);
  return 0;
}
