// geometry.h -- HRRT scanner / sinogram / image geometry tables.
//
// Host-side restatement of the reference's dependencies()
// (hrrt_osem3d/hrrt_osem3dv_sbrt_span3.cpp:199-800), get_info (:159-191),
// calculatevieworder (:144-152), GetScannerParameter
// (hrrt_osem3d/hrrt_osem3d_span3.cpp:3452-3551) and sequence() (:535-580).
// Every table is computed with the same single-precision expressions, in the
// same order, as the reference, so that the device kernels sample the image
// and the sinogram at bit-identical positions.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace hrrt {

struct ScannerParams {
  int nrings = 104;          // direct planes (scanner_model.cpp:124)
  int nelements = 256;       // radial bins
  int nangles = 288;         // views
  float ring_radius = 234.5f;
  float plane_sep = 1.21875f;
  float binsize = 1.21875f;
  int span = 9;
  int maxdel = 67;
  int subsets = 16;
  float rel_fov = 0.95f;
  int z_min = 6, z_max = 200, npskip = 3;   // drv:232, :289
  float epsilon1 = 5.E-2f, epsilon2 = 1.E-2f, epsilon3 = 1.E-10f, image_max = 1.E4f;  // drv:371-374
};

struct Geometry {
  ScannerParams sp;
  // image
  int nx = 0, ny = 0, nz = 0, zp = 0, c = 0;   // zp = z padded to a multiple of 4
  float x_size = 0, y_size = 0, z_size = 0, ring_spacing = 0, rfov = 0;
  // sinogram
  int nbins = 0, nviews = 0, groupmax = 0, maxdel = 0, nseg = 0, zshift = 0, segmentsize = 0;
  int sviews = 0;
  std::vector<int> yr_bottom, yr_top, segment_offset;   // [nseg]
  std::vector<float> sin_theta, cos_theta;              // [nseg]
  std::vector<float> sin_psi, cos_psi;                  // [nviews]
  std::vector<float> vcos, vsin;                        // [groupmax][zshift]
  std::vector<int16_t> cyl0, cyl1;                      // cylwiny[y][0..1]
  std::vector<float> tantheta, rescale;                 // [groupmax][nz]
  std::vector<int> fl_zzi;                              // flookup[y][g*2*zshift+i].zzi
  std::vector<float> fl_zzz0;                           //   .zzz0
  std::vector<int> bl_zsa, bl_zea, bl_yra;              // blookup[y][g]
  std::vector<float> bl_yr2a;
  std::vector<float> bp_scale;                          // [nseg] cos^3 * span * ring_spacing / 2R
  std::vector<int16_t> norm_zero_mask;                  // [nviews/2][nx/2+1]
  std::vector<int> vieworder;                           // [subsets][sviews]
  std::vector<int16_t> order;                           // [subsets]
  int fov_columns = 0;

  // returns empty string on success, else a message
  std::string build(const ScannerParams &p);
  int flookup_stride() const { return groupmax * 2 * zshift; }
  // first plane of segment s in the quad layout (padded by one plane on each side)
  int padded_offset(int s) const { return segment_offset[s] + 2 * s + 1; }
  int padded_planes() const { return segmentsize + 2 * nseg; }
};

}  // namespace hrrt
