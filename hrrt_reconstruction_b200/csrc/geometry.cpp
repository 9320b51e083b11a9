// geometry.cpp -- see geometry.h.  Built with -ffp-contract=off: every float
// expression below is evaluated as separate IEEE single-precision operations in
// the order the reference writes them, as the reference's SSE2 build does.
#include "geometry.h"

#include <cmath>
#include <cstdlib>

namespace hrrt {

namespace {
// The reference code base assumes a predefined single-precision PI.
constexpr float kPi = 3.14159265358979f;

// get_info (sbrt:159-191): plane range of a segment group
void group_planes(int nrings, int span, int group, int *zmin, int *zmax) {
  if (group == 0) {
    *zmin = 0;
    *zmax = 2 * nrings - 2;
  } else {
    *zmin = (span + 1) / 2 + (group - 1) * span;
    *zmax = 2 * nrings - 2 - *zmin;
  }
}
}  // namespace

std::string Geometry::build(const ScannerParams &p) {
  sp = p;
  if (p.span < 3 || (p.span % 2) == 0) return "span must be odd and >= 3";
  if (p.nelements < 8 || (p.nelements % 4) != 0) return "radial bins must be a positive multiple of 4";
  if (p.nangles % p.subsets != 0) return "views must be a multiple of subsets";
  if (p.nangles % 2 != 0) return "views must be even";
  // GetScannerParameter (drv:3452-3551)
  nz = p.nrings * 2 - 1;
  zp = (nz % 4 == 0) ? nz : (nz / 4 + 1) * 4;
  ring_spacing = 2.0f * p.plane_sep;
  groupmax = (p.maxdel - (p.span - 1) / 2) / p.span;
  if (groupmax < 1) return "maxdel too small for span";
  nbins = p.nelements;
  nviews = p.nangles;
  // dependencies (sbrt:199-800), zoom = newzoom = 1, max_g = -1
  maxdel = groupmax * p.span + (p.span - 1) / 2;
  nx = ny = nbins;
  c = nx / 2;
  const float sino_sampling = p.binsize;
  x_size = (sino_sampling * nbins) / (1.0f * nx);
  y_size = x_size;
  z_size = ring_spacing / 2.0f;
  sviews = nviews / p.subsets;
  if ((sviews % 2) != 0) return "views per subset must be even (view pairs)";
  nseg = 2 * groupmax + 1;
  zshift = p.span - 1;
  rfov = p.rel_fov * x_size * nx / 2.0f;

  // cylindrical FOV mask cylwiny[y][0..1] (sbrt:339-356)
  cyl0.assign(ny, 0);
  cyl1.assign(ny, 0);
  fov_columns = 0;
  for (int y = 0; y < ny; y++) {
    int flag = 0;
    for (int x = 0; x < nx; x++) {
      const int dx = x - c, dy = y - c;
      const float r2 = dx * x_size * dx * x_size + dy * y_size * dy * y_size;
      if (std::sqrt(r2) <= rfov) {
        if (flag == 0) cyl0[y] = (int16_t)x;
        flag = 1;
        fov_columns++;
      } else {
        if (flag == 1) cyl1[y] = (int16_t)x;
        flag = 0;
      }
    }
  }

  // segment angles (sbrt:427-444)
  sin_theta.assign(nseg, 0.f);
  cos_theta.assign(nseg, 0.f);
  vcos.assign((size_t)groupmax * zshift, 0.f);
  vsin.assign((size_t)groupmax * zshift, 0.f);
  sin_theta[0] = 0.0f;
  cos_theta[0] = 1.0f;
  for (int g = 1; g <= groupmax; g++) {
    float t = g * p.span * ring_spacing;
    t = std::sqrt(t * t + (2 * p.ring_radius) * (2 * p.ring_radius));
    sin_theta[2 * g - 1] = g * p.span * ring_spacing / t;
    cos_theta[2 * g - 1] = (2.0f * p.ring_radius) / t;
    sin_theta[2 * g] = -sin_theta[2 * g - 1];
    cos_theta[2 * g] = cos_theta[2 * g - 1];
    for (int z = 0; z < zshift; z++) {
      const int zmin = p.span * g - (p.span - 1) / 2;
      const int mean_rd = zmin + (z + 1) / 2;
      float u = mean_rd * ring_spacing;
      u = std::sqrt(u * u + (2 * p.ring_radius) * (2 * p.ring_radius));
      vcos[(size_t)(g - 1) * zshift + z] = (2.0f * p.ring_radius) / u;
      vsin[(size_t)(g - 1) * zshift + z] = mean_rd * ring_spacing / u;
    }
  }

  // plane ranges and offsets (sbrt:446-468)
  yr_bottom.assign(nseg, 0);
  yr_top.assign(nseg, 0);
  segment_offset.assign(nseg, 0);
  yr_bottom[0] = 0;
  yr_top[0] = nz - 1;
  for (int g = 1; g <= groupmax; g++) {
    int zmin, zmax;
    group_planes(p.nrings, p.span, g, &zmin, &zmax);
    if (zmax - zmin + 1 < 2 * zshift + 1) return "segment too short for its end-plane corrections";
    yr_bottom[2 * g] = yr_bottom[2 * g - 1] = zmin;
    yr_top[2 * g] = yr_top[2 * g - 1] = zmax;
  }
  segmentsize = 0;
  for (int s = 0; s < nseg; s++) {
    segment_offset[s] = segmentsize;
    segmentsize += yr_top[s] - yr_bottom[s] + 1;
  }

  // view angles (sbrt:476-486)
  sin_psi.assign(nviews, 0.f);
  cos_psi.assign(nviews, 0.f);
  sin_psi[0] = 0.0f;
  cos_psi[0] = 1.0f;
  sin_psi[nviews / 2] = 1.0f;
  cos_psi[nviews / 2] = 0.0f;
  const float dpsi = kPi / nviews;
  for (int v = 1; v < nviews / 2; v++) {
    sin_psi[v] = std::sin(v * dpsi);                                   // single-precision sin
    cos_psi[v] = (float)std::sqrt(1. - (double)(sin_psi[v] * sin_psi[v]));  // double sqrt
    sin_psi[nviews - v] = sin_psi[v];
    cos_psi[nviews - v] = -cos_psi[v];
  }

  // subsets (sbrt:144-152) and subset order (drv:535-580)
  vieworder.assign((size_t)p.subsets * sviews, 0);
  for (int i = 0; i < p.subsets; i++)
    for (int k = 0; k < sviews; k++) vieworder[(size_t)i * sviews + k] = i + p.subsets * k;
  order.assign(p.subsets, 0);
  {
    std::vector<int> done(p.subsets, 0);
    order[0] = 0;
    done[0] = 1;
    for (int i = 1; i < p.subsets; ++i) {
      int ibest = 0, dbest = 0, j = 0;
      while (j < p.subsets) {
        while (j < p.subsets && done[j] == 1) j += 1;
        if (j < p.subsets) {
          const int k = order[i - 1];
          int d = std::abs(j - k);
          if ((p.subsets - std::abs(j - k)) < d) d = p.subsets - std::abs(j - k);
          if (d > dbest) { dbest = d; ibest = j; }
          j += 1;
        }
      }
      order[i] = (int16_t)ibest;
      done[ibest] = 1;
    }
  }

  // tantheta and rescalearray with end-plane corrections (sbrt:529-542)
  tantheta.assign((size_t)groupmax * nz, 0.f);
  rescale.assign((size_t)groupmax * nz, 0.f);
  for (int th = 2, g = 0; th < nseg; th += 2, g++) {
    for (int yr = yr_bottom[th]; yr <= yr_top[th]; yr++) {
      float t = sin_theta[th] / cos_theta[th];
      float r = y_size / std::fabs(cos_theta[th]);
      int zs = yr - yr_bottom[th];
      if (zs >= zshift) zs = yr_top[th] - yr;
      if (zs < zshift) {
        t = vsin[(size_t)g * zshift + zs] / vcos[(size_t)g * zshift + zs];
        t = -t;
        r = y_size / std::fabs(vcos[(size_t)g * zshift + zs]);
      }
      t = -t / 1.0f;
      tantheta[(size_t)g * nz + yr] = t;
      rescale[(size_t)g * nz + yr] = r;
    }
  }

  // forward-projection end-plane lookup flookup (sbrt:545-578)
  const int fs = flookup_stride();
  fl_zzi.assign((size_t)ny * fs, 0);
  fl_zzz0.assign((size_t)ny * fs, 0.f);
  for (int y = 0; y < ny; y++) {
    for (int th = 2, g = 0; th < nseg; th += 2, g++) {
      int yri = 0;
      for (int yr = yr_bottom[th]; yr < yr_bottom[th] + zshift; yr++, yri++) {
        float zz = yr + ((y - c) * tantheta[(size_t)g * nz + yr]);
        const int z = (int)zz;
        fl_zzz0[(size_t)y * fs + g * zshift * 2 + yri] = zz - z;
        fl_zzi[(size_t)y * fs + g * zshift * 2 + yri] = z;
      }
      for (int yr = yr_top[th] - zshift + 1; yr <= yr_top[th]; yr++, yri++) {
        float zz = yr + ((y - c) * tantheta[(size_t)g * nz + yr]);
        const int z = (int)zz;
        fl_zzz0[(size_t)y * fs + g * zshift * 2 + yri] = zz - z;
        fl_zzi[(size_t)y * fs + g * zshift * 2 + yri] = z;
      }
    }
  }

  // back-projection lookup blookup (sbrt:672-700)
  bl_zsa.assign((size_t)ny * groupmax, 0);
  bl_zea.assign((size_t)ny * groupmax, 0);
  bl_yra.assign((size_t)ny * groupmax, 0);
  bl_yr2a.assign((size_t)ny * groupmax, 0.f);
  for (int y = 0; y < ny; y++) {
    for (int th = 2, g = 0; th < nseg; th += 2, g++) {
      const float tb = -sin_theta[th] / cos_theta[th];
      const float yr0 = -(y - c) * tb;
      const float yr1 = yr0;
      float yr2 = std::fabs(yr0) - (int)std::fabs(yr0);
      int yri2 = (int)yr1;
      if (yr1 < 0) {
        yr2 = 1 - yr2;
        yri2 -= 1;
      }
      int zs = yr_bottom[th] - 1 - yri2;
      int ze = yr_top[th] - yri2;
      int yr = yr_bottom[th] - 1;
      if (zs < 0) {
        yr = yr - zs;
        zs = 0;
      }
      if (ze > nz - 1) ze = nz - 1;
      const size_t i = (size_t)y * groupmax + g;
      bl_zsa[i] = zs;
      bl_zea[i] = ze;
      bl_yra[i] = yr;
      bl_yr2a[i] = yr2;
    }
  }

  // per-segment back-projection weight (sbrt:1637-1649)
  bp_scale.assign(nseg, 0.f);
  for (int k = 0; k < nseg; k++)
    bp_scale[k] = cos_theta[k] * cos_theta[k] * cos_theta[k] * p.span * ring_spacing / (2 * p.ring_radius);

  // default norm_zero_mask (sbrt:333): all quads active
  norm_zero_mask.assign((size_t)(nviews / 2) * (nx / 2 + 1), 1);
  return std::string();
}

}  // namespace hrrt
