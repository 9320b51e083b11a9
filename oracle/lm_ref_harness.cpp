// lm_ref_harness.cpp -- exposes, through a C interface, the parts of the
// reference's listmode geometry that build from their own sources:
//   gen_delays_lib/geometry_info.cpp           calc_det_to_phy (crystal positions)
//   gen_delays_lib/segment_info_fromarchive.cpp init_segment_info (segment tables)
// TEST INFRASTRUCTURE: used only to pin oracle/lm_oracle.c.  The reference
// sources are compiled where they lie (oracle/Makefile, target "ref"); none
// is copied.
//
// init_geometry_hrrt (geometry_info.cpp:168-218) indexes its position arrays
// with a loop counter that it never initialises, so it is not called; the
// state it sets for the default HRRT (LR_0) is set here and calc_det_to_phy
// is called for every crystal, as that loop does.
#include <array>
#include <cmath>
#include <cstring>
#include <vector>

#include "geometry_info.h"

namespace GeometryInfo {
void calc_det_to_phy(int head, int layer, int detx, int dety, float location[3]);
}

int init_segment_info(int *nsegs, int *nplanes, double *d_tan_theta, int maxrd, int span, int NYCRYS,
                      double crystal_radius, double plane_sep);
extern int *m_segz0, *m_segzmax, *m_segzoffset;

extern "C" {

/* crystal positions [head 8][layer 2][x 72][y 104][xyz], depth 1.0 cm */
int lmref_crystals(float *xyz) {
  using namespace GeometryInfo;
  const float pitch = PITCH, rdiam = RDIAM, lthick = LTHICK;
  for (int i = 0; i < NHEADS; i++) {
    sin_head_[i] = sin(i * 2.0 * M_PI / NHEADS);
    cos_head_[i] = cos(i * 2.0 * M_PI / NHEADS);
  }
  crystal_radius_ = rdiam / 2.0;
  crystal_x_pitch_ = crystal_y_pitch_ = pitch;
  binsize_ = pitch / 2.0;
  plane_sep_ = pitch / 2.0;
  head_crystal_depth_.fill(lthick);
  size_t k = 0;
  for (int h = 0; h < NHEADS; h++)
    for (int l = 0; l < NDOIS; l++)
      for (int x = 0; x < NXCRYS; x++)
        for (int y = 0; y < NYCRYS; y++, k += 3) calc_det_to_phy(h, l, x, y, xyz + k);
  return 0;
}

/* segment tables of init_segment_info for (maxrd, span) with the HRRT's
 * radius and plane separation */
int lmref_segments(int span, int maxrd, int *segz0, int *segzmax, int *segzoffset, int *nsegs, int *nplanes,
                   double *d_tan_theta) {
  const double radius = 46.9f / 2.0, plane_sep = 0.24375f / 2.0;
  int n = 0, np = 0;
  double dt = 0;
  init_segment_info(&n, &np, &dt, maxrd, span, 104, radius, plane_sep);
  for (int i = 0; i < n; i++) {
    segz0[i] = m_segz0[i];
    segzmax[i] = m_segzmax[i];
    segzoffset[i] = m_segzoffset[i];
  }
  *nsegs = n;
  *nplanes = np;
  *d_tan_theta = dt;
  return 0;
}

}  // extern "C"
