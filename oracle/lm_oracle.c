/*
 * lm_oracle.c -- CPU restatement of HRRT listmode histogramming.
 *
 * TEST INFRASTRUCTURE ONLY (see lm_oracle.h).  Plain C99, -ffp-contract=off:
 * every float and double expression below has the operand types and the
 * order of the reference's C++ (x86-64 SSE2, no fused multiply-add).
 *
 * Reference files cited, within the reference project:
 *   gi   = gen_delays_lib/geometry_info.{h,cpp}      crystal positions
 *   si   = gen_delays_lib/segment_info_fromarchive.cpp  segment tables
 *   lsm  = gen_delays_lib/lor_sinogram_map.cpp       LUT (init_sol)
 *   lut  = hrrt_rebinner_lut/hrrt_rebinner_lut.cpp   how the LUT file is made
 *   reb  = lmhistogram_mp/LM_Rebinner_mp.cpp         rebin_event
 *   hist = lmhistogram_mp/histogram_mp.cpp           decode, tags, histogram
 *   rdr  = lmhistogram_mp/LM_Reader_mp.{hpp,cpp}     packets
 */
#include "lm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* gi.h:31-66 */
#define NDOIS 2
#define NXCRYS 72
#define NYCRYS 104
#define NHEADS 8
#define NMPAIRS 20
#define NPROJS 256
#define NVIEWS 288
#define NXD (NXCRYS * NDOIS)
/* rdr.hpp:39: 1024*1024 64-bit events per packet */
#define PACKET_WORDS (2 * 1024 * 1024)

static const int HRRT_MPAIRS[21][2] = {{-1, -1}, {0, 2}, {0, 3}, {0, 4}, {0, 5}, {0, 6}, {1, 3}, {1, 4}, {1, 5}, {1, 6},
                                       {1, 7},   {2, 4}, {2, 5}, {2, 6}, {2, 7}, {3, 5}, {3, 6}, {3, 7}, {4, 6}, {4, 7},
                                       {5, 7}};
static const int EWTYPES[16] = {3, 3, 1, 0, 3, 3, 2, 2, 3, 3, 3, 3, 3, 3, 3, 3};
/* span-3 to span-9 segment map (si:23-26) */
static const int CONVERSION[45] = {0, 0,  0,  1,  2,  1,  2,  1,  2,  3,  4,  3,  4,  3,  4,  5,  6,  5,  6,  5,  6,  7,  8,
                                   7, 8,  7,  8,  9,  10, 9,  10, 9,  10, 11, 12, 11, 12, 11, 12, 13, 14, 13, 14, 13, 14};

struct lm_tables {
  int span, nsegs, nplanes_out;
  double d_tan_theta, plane_sep, binsize, crystal_radius;
  float xyz[NHEADS][NDOIS][NXCRYS][NYCRYS][3];
  float c_zpos[NYCRYS], c_zpos2[NYCRYS];
  int segz0[63], segzmax[63], segzoffset[63];
  short segplane[63][2 * NYCRYS - 1];
  lm_sol *sol; /* [21][NXD][NXD], entry 0 unused */
};

/* gi.h:50-66 constants, evaluated with the reference's types */
static float c_csize(void) { return 0.22f; }
static float c_cgap(void) { return 0.02f; }
static float c_bsize(void) { return (float)(8.0 * c_csize() + 7 * c_cgap()); }
static float c_bgap(void) { return 0.05f; }
static float c_xhsize(void) { return (float)(9.0 * c_bsize() + 8 * c_bgap()); }

/* calc_det_to_phy (gi.cpp:137-163), head_crystal_depth = 1.0 */
static void det_to_phy(const double *sin_head, const double *cos_head, double crystal_radius, int head, int layer,
                       int detx, int dety, float pos[3]) {
  const float BSIZE = c_bsize(), BGAP = c_bgap(), CSIZE = c_csize(), CGAP = c_cgap(), XHSIZE = c_xhsize();
  const float depth = 1.0f;
  const double sint = sin_head[head], cost = cos_head[head];
  int bcrys = detx % 8, blk = detx / 8;
  const float xf = blk * (BSIZE + BGAP) + bcrys * (CSIZE + CGAP);
  const double x = xf - XHSIZE / 2.0 + CSIZE / 2.0;
  const double y = crystal_radius + depth * (1 - layer) + 0.5 * depth;
  bcrys = dety % 8;
  blk = dety / 8;
  const float zf = blk * (BSIZE + BGAP) + bcrys * (CSIZE + CGAP);
  const double z = zf;
  const double xpos = x * cost + y * sint;
  const double ypos = -x * sint + y * cost;
  pos[0] = (float)xpos;
  pos[1] = (float)ypos;
  pos[2] = (float)z;
}

/* init_phy_to_pro (lsm:99-138) */
static void phy_to_pro(const lm_tables *t, const float deta[3], const float detb[3], lm_sol *sol) {
  const float pi = (float)M_PI;
  double dy = deta[1] - detb[1];
  double dx = deta[0] - detb[0];
  double d = sqrt(dx * dx + dy * dy);
  float r = (float)((deta[1] * detb[0] - deta[0] * detb[1]) / d);
  float phi = (float)(atan2(dx, dy));
  if (phi < 0.0) {
    phi += pi;
    r = -r;
    d = -d;
  }
  if (phi >= M_PI) {
    phi = 0.0;
    r = -r;
    d = -d;
  }
  int view = (int)(NVIEWS * phi / M_PI);
  if (view >= 288) view = 0;
  if (view <= -1) view = 0;
  const float z = (float)((deta[0] * dx + deta[1] * dy) / (d * d));
  const int bin = (int)(NPROJS / 2 + (r / t->binsize + 0.5));
  if (bin < 0 || bin > NPROJS - 1)
    sol->nsino = -1;
  else
    sol->nsino = bin + view * NPROJS;
  sol->d = (float)(1.0 / d / t->d_tan_theta);
  sol->z = (float)(z / t->plane_sep);
}

lm_tables *lm_create(int span, int maxrd) {
  if ((span != 3 && span != 9) || maxrd < span || maxrd > 103) return NULL;
  lm_tables *t = (lm_tables *)calloc(1, sizeof(lm_tables));
  if (!t) return NULL;
  t->span = span;
  /* init_geometry_hrrt (gi.cpp:168-218), LR_0, loop counter from 0 */
  const float pitch = 0.24375f, rdiam = 46.9f;
  double sin_head[NHEADS], cos_head[NHEADS];
  for (int i = 0; i < NHEADS; i++) {
    sin_head[i] = sin(i * 2.0 * M_PI / NHEADS);
    cos_head[i] = cos(i * 2.0 * M_PI / NHEADS);
  }
  t->crystal_radius = rdiam / 2.0;
  t->binsize = pitch / 2.0;
  t->plane_sep = pitch / 2.0;
  for (int h = 0; h < NHEADS; h++)
    for (int l = 0; l < NDOIS; l++)
      for (int x = 0; x < NXCRYS; x++)
        for (int y = 0; y < NYCRYS; y++) det_to_phy(sin_head, cos_head, t->crystal_radius, h, l, x, y, t->xyz[h][l][x][y]);

  /* init_segment_info (si:113-141): span-3 segment planes; offsets of the
   * output span (span 9 through the conversion table) */
  const int np = 2 * NYCRYS - 1;
  int seg9off[63] = {0};
  {
    const int maxseg = maxrd / span, nsegs = 2 * maxseg + 1, sp2 = (span + 1) / 2;
    int segz0 = 0, segnz = 0, segzoff = 0, prev_nz = 0;
    for (int i = 0; i < nsegs; i++) {
      segz0 = (i == 0) ? 0 : sp2 + span * ((i - 1) / 2);
      segnz = np - 2 * segz0;
      segzoff = (i == 0) ? 0 : segzoff + prev_nz;
      prev_nz = segnz;
      seg9off[i] = -segz0 + segzoff;
      t->nplanes_out = segzoff + segnz;
    }
    t->d_tan_theta = span * t->plane_sep / t->crystal_radius;
  }
  {
    const int maxseg = maxrd / 3, sp2 = 2;
    t->nsegs = 2 * maxseg + 1;
    int segzoff = 0, prev_nz = 0, total = 0;
    for (int i = 0; i < t->nsegs; i++) {
      t->segz0[i] = (i == 0) ? 0 : sp2 + 3 * ((i - 1) / 2);
      const int segnz = np - 2 * t->segz0[i];
      segzoff = (i == 0) ? 0 : segzoff + prev_nz;
      prev_nz = segnz;
      t->segzmax[i] = t->segz0[i] + segnz - 1;
      t->segzoffset[i] = -t->segz0[i] + segzoff;
      total = segzoff + segnz;
    }
    t->d_tan_theta = 3 * t->plane_sep / t->crystal_radius;
    if (span == 3) t->nplanes_out = total;
    if (span == 9)
      for (int i = 0; i < t->nsegs && i < 45; i++) t->segzoffset[i] = seg9off[CONVERSION[i]];
  }

  /* init_sol (lsm:141-221) */
  t->sol = (lm_sol *)calloc((size_t)21 * NXD * NXD, sizeof(lm_sol));
  if (!t->sol) {
    free(t);
    return NULL;
  }
  for (int i = 1; i <= NMPAIRS; i++) {
    const int ahead = HRRT_MPAIRS[i][0], bhead = HRRT_MPAIRS[i][1];
    for (int al = 0; al < NDOIS; al++)
      for (int ax = 0; ax < NXCRYS; ax++) {
        const int axx = ax + NXCRYS * al;
        for (int bl = 0; bl < NDOIS; bl++)
          for (int bx = 0; bx < NXCRYS; bx++) {
            const int bxx = bx + NXCRYS * bl;
            phy_to_pro(t, t->xyz[ahead][al][ax][0], t->xyz[bhead][bl][bx][0],
                       &t->sol[((size_t)i * NXD + axx) * NXD + bxx]);
          }
      }
  }
  for (int i = 0; i < NYCRYS; i++) {
    const float *p = t->xyz[0][0][0][i];
    t->c_zpos[i] = p[2];
    t->c_zpos2[i] = (float)(p[2] / t->plane_sep + 0.5);
  }
  for (int i = 0; i < 63; i++)
    for (int plane = 0; plane < np; plane++) {
      short v = 0;
      if (i > t->nsegs - 1 || plane < t->segz0[i] || plane > t->segzmax[i])
        v = -1;
      else
        v = (short)(plane + t->segzoffset[i]);
      t->segplane[i][plane] = v;
    }
  return t;
}

void lm_destroy(lm_tables *t) {
  if (!t) return;
  free(t->sol);
  free(t);
}

long long lm_sino_size(const lm_tables *t) { return (long long)t->nplanes_out * NPROJS * NVIEWS; }
int lm_nplanes(const lm_tables *t) { return t->nplanes_out; }
double lm_d_tan_theta(const lm_tables *t) { return t->d_tan_theta; }
void lm_get_sol(const lm_tables *t, lm_sol *sol) { memcpy(sol, t->sol, sizeof(lm_sol) * 21 * NXD * NXD); }
void lm_get_zpos(const lm_tables *t, float *a, float *b) {
  memcpy(a, t->c_zpos, sizeof(t->c_zpos));
  memcpy(b, t->c_zpos2, sizeof(t->c_zpos2));
}
void lm_get_seg(const lm_tables *t, int *z0, int *zmax, int *off, int *nsegs) {
  memcpy(z0, t->segz0, sizeof(int) * t->nsegs);
  memcpy(zmax, t->segzmax, sizeof(int) * t->nsegs);
  memcpy(off, t->segzoffset, sizeof(int) * t->nsegs);
  *nsegs = t->nsegs;
}
void lm_get_crystals(const lm_tables *t, float *xyz) { memcpy(xyz, t->xyz, sizeof(t->xyz)); }

/* rebin_event (reb:188-219).  A plane outside [0, 2*104-2] would index
 * m_segplane outside its row in the reference; here it has no address. */
int lm_rebin_event(const lm_tables *t, int mp, int alayer, int ax, int ay, int blayer, int bx, int by) {
  const int axx = ax + NXCRYS * alayer, bxx = bx + NXCRYS * blayer;
  const lm_sol *s = &t->sol[((size_t)mp * NXD + axx) * NXD + bxx];
  const int sino_addr = s->nsino;
  if (sino_addr == -1) return -1;
  const float cay = t->c_zpos2[ay];
  const float dz2 = t->c_zpos[by] - t->c_zpos[ay];
  const float z = s->z, d = s->d;
  const int plane = (int)(cay + z * dz2);
  const float seg = (float)(0.5 + dz2 * d);
  int segnum = (int)seg;
  if (seg < 0)
    segnum = 1 - 2 * segnum;
  else
    segnum = 2 * segnum;
  if (segnum >= t->nsegs) return -1;
  if (plane < 0 || plane > 2 * NYCRYS - 2) return -1;
  if (t->segplane[segnum][plane] == -1) return -1;
  return (plane + t->segzoffset[segnum]) * NPROJS * NVIEWS + sino_addr;
}

void lm_rebin_events(const lm_tables *t, long long n, const int32_t *ev, int32_t *addr) {
  for (long long k = 0; k < n; k++) {
    const int32_t *e = ev + 7 * k;
    addr[k] = lm_rebin_event(t, e[0], e[1], e[2], e[3], e[4], e[5], e[6]);
  }
}

void lm_clock_init(lm_clock *c) {
  c->current_time = -1;
  c->current_time_msec = -1;
  c->prev_time = 0;
  c->clock_reset = 0;
  c->pad = 0;
}

/* process_tagword time-tag branch (hist:225-260); returns 1 when the frame
 * ends at this tag */
/* head curve and block singles of a frame (process_tagword, hist:225-303) */
#define NBLOCKS 936
typedef struct {
  lm_second *out;
  int cap, n;
  long long prompts, randoms, t_prompts, t_randoms;
  long long last[NBLOCKS], total[NBLOCKS], nsamples[NBLOCKS];
} hc_state;

static int time_tag(lm_clock *c, unsigned tag, int duration, int flags, long long *frame_start, hc_state *hc) {
  if (hc && (tag & 0xE0000000u) == 0xA0000000u) { /* block singles (hist:260-270) */
    const int block = (int)((tag & 0x1ff80000u) >> 19);
    const long long v = tag & 0x0007ffff;
    if (block >= 0 && block < NBLOCKS) {
      hc->last[block] = v;
      hc->total[block] += v;
      hc->nsamples[block]++;
    }
    return 0;
  }
  if ((tag & 0xE0000000u) != 0x80000000u) return 0;
  if (flags & LM_TIME_FROM_COUNT)
    c->current_time_msec++;
  else
    c->current_time_msec = tag & 0x3fffffff;
  if (c->prev_time > c->current_time_msec) {
    if (!c->clock_reset) {
      c->current_time = c->current_time_msec / 1000;
      c->clock_reset = 1;
      return 0;
    }
  }
  c->prev_time = c->current_time_msec;
  if (c->current_time != c->current_time_msec / 1000) {
    if (hc) { /* the head-curve line (hist:241-258) */
      long long singles = 0;
      for (int b = 0; b < NBLOCKS; b++) singles += hc->last[b];
      if (hc->n < hc->cap) hc->out[hc->n] = (lm_second){c->current_time_msec, hc->prompts, hc->randoms, singles};
      hc->n++;
      hc->t_prompts += hc->prompts;
      hc->t_randoms += hc->randoms;
      hc->prompts = hc->randoms = 0;
    }
    c->current_time = c->current_time_msec / 1000;
    if (*frame_start < 0) *frame_start = c->current_time;
    if (duration > 0 && (c->current_time - *frame_start) >= duration) return 1;
  }
  return 0;
}

static void bump(uint16_t *h, long long a, int delta) { h[a] = (uint16_t)(h[a] + delta); }

/* Emission decode (rebin_packet, hist:1026-1233) and histogram (hist:1301-
 * 1372), in stream order.  Packets of PACKET_WORDS words are parsed from
 * their own first word: a word left over at a packet end is dropped
 * (`(src_pos + 1) < count`).  The reference's reader exits on a short last
 * packet; here the last packet is parsed like the others. */
static int histogram_impl(const lm_tables *t, const uint32_t *w, long long n, long long offset, int mode,
                          int duration, int flags, lm_clock *clk, uint16_t *sino, uint16_t *delayed, lm_stats *st,
                          hc_state *hc, uint32_t *ccounts) {
  memset(st, 0, sizeof(*st));
  const long long sino_size = lm_sino_size(t);
  const int ignore_border = flags & LM_IGNORE_BORDER_CRYSTAL;
  const int doi_processing = (flags & LM_NO_DOI) == 0;
  const int xhigh = ignore_border ? NXCRYS - 1 : NXCRYS;
  /* reset_statistics (hist:196-216) */
  long long frame_start = (clk->current_time >= 0) ? clk->current_time : -1;
  int terminated = 0;
  long long pos = 0;
  /* packets are counted from the start of the file: words[0] sits at
   * `offset` words into it */
  for (long long p0 = -(offset % PACKET_WORDS); p0 < n && !terminated; p0 += PACKET_WORDS) {
    const long long count = (n - p0 < PACKET_WORDS) ? n - p0 : PACKET_WORDS;
    long long sp = p0 < 0 ? -p0 : 0;
    while (sp + 1 < count && !terminated) {
      const unsigned ew1 = w[p0 + sp], ew2 = w[p0 + sp + 1];
      const int type = EWTYPES[((ew2 & 0xc0000000u) >> 30) | ((ew1 & 0xc0000000u) >> 28)];
      long long address = -1;
      unsigned word32 = 0;
      int have = 0;
      if (type == 3) {
        sp++;
        st->resyncs++;
        continue;
      }
      if (type == 2) {
        sp += 2;
        st->tags++;
        word32 = (ew1 & 0xffff) | ((ew2 & 0xffff) << 16);
        have = 1;
      } else {
        sp += 2;
        int doia = 1, doib = 1, err = 0;
        const int mpe = ((ew1 & 0x00070000) >> 16) | ((ew2 & 0x00070000) >> 13);
        const int ax = ew1 & 0xff, ay = (ew1 & 0xff00) >> 8, bx = ew2 & 0xff, by = (ew2 & 0xff00) >> 8;
        if (doi_processing) {
          doia = (ew1 & 0x01C00000) >> 22;
          doib = (ew2 & 0x01C00000) >> 22;
        }
        if (mpe < 1 || mpe > NMPAIRS) err++;
        if (ax >= NXCRYS || ay >= NYCRYS) err++;
        if (bx >= NXCRYS || by >= NYCRYS) err++;
        if (err) {
          st->invalid++;
          continue;
        }
        if (doia == 7 || doib == 7) {
          /* the transmission branch: in an emission stream the reference
           * looks the event up in a TX table that only a transmission run
           * builds; such events are not histogrammed */
          st->doi7++;
          continue;
        }
        if ((doia == 1 || doia == 0) && (doib == 1 || doib == 0) && ccounts) {
          /* the coincidence histogram (hist:1212-1223), with a crystal row
           * NHEADS * NXCRYS wide as in histogram_mp_fromarchive.cpp:916,
           * :1092-1096 (the rewrite's row of NUM_CRYSTALS_X_Y, hist:1049,
           * indexes past the map it allocates) */
          uint32_t *cc = ccounts + (type ? NXCRYS * NYCRYS * NHEADS * NDOIS : 0);
          cc[doia * NXCRYS * NYCRYS * NHEADS + HRRT_MPAIRS[mpe][0] * NXCRYS + ax + ay * NXCRYS * NHEADS]++;
          cc[doib * NXCRYS * NYCRYS * NHEADS + HRRT_MPAIRS[mpe][1] * NXCRYS + bx + by * NXCRYS * NHEADS]++;
        }
        if ((doia == 1 || doia == 0) && (doib == 1 || doib == 0)) {
          if (ignore_border && (ax * bx == 0 || ax == xhigh || bx == xhigh)) {
            address = -1;
          } else if (mode == LM_PROMPTS_ONLY && type != 0) {
            address = -1;
          } else {
            address = lm_rebin_event(t, mpe, doia, ax, ay, doib, bx, by);
            if (address >= 0 && type == 0) address |= 0x40000000;
          }
        } else {
          st->doi_other++;
        }
        if (address < 0) {
          if ((doia == 1 || doia == 0) && (doib == 1 || doib == 0)) st->unmapped++;
          continue;
        }
        word32 = (unsigned)address;
        have = 1;
      }
      if (!have) continue;
      /* next_event_32 (hist:334-382) and histogram (hist:1316-1362) */
      if (word32 & 0x80000000u) {
        st->timetags += ((word32 & 0xE0000000u) == 0x80000000u);
        if (time_tag(clk, word32, duration, flags, &frame_start, hc)) terminated = 1;
        continue;
      }
      const int prompt = (word32 & 0x40000000u) != 0;
      const long long value = word32 & 0x3fffffff;
      if (prompt)
        st->prompts++;
      else
        st->delayed++;
      if (hc) {
        if (prompt)
          hc->prompts++;
        else
          hc->randoms++;
      }
      if (value >= 0 && value < sino_size) {
        if (mode == LM_PROMPTS_AND_DELAYED) {
          if (prompt)
            bump(sino, value, 1);
          else if (delayed)
            bump(delayed, value, 1);
        } else {
          bump(sino, value, prompt ? 1 : -1);
        }
      }
    }
    pos = p0 + sp;
  }
  st->words_used = terminated ? pos : n;
  st->terminated = terminated;
  if (!terminated) clk->current_time = (clk->current_time_msec + 500) / 1000;
  st->frame_start = frame_start;
  st->duration = clk->current_time - frame_start;
  return 0;
}

int lm_histogram(const lm_tables *t, const uint32_t *w, long long n, int mode, int duration, int flags, lm_clock *clk,
                 uint16_t *sino, uint16_t *delayed, lm_stats *st) {
  return histogram_impl(t, w, n, 0, mode, duration, flags, clk, sino, delayed, st, NULL, NULL);
}

int lm_histogram_at(const lm_tables *t, const uint32_t *w, long long n, long long offset, int mode, int duration,
                    int flags, lm_clock *clk, uint16_t *sino, uint16_t *delayed, lm_stats *st) {
  return histogram_impl(t, w, n, offset, mode, duration, flags, clk, sino, delayed, st, NULL, NULL);
}

int lm_histogram_hc(const lm_tables *t, const uint32_t *w, long long n, long long offset, int mode, int duration,
                    int flags, lm_clock *clk, uint16_t *sino, uint16_t *delayed, lm_stats *st, lm_second *hc_out,
                    int hc_cap, int *block_rates, long long *totals, uint32_t *ccounts) {
  hc_state *hc = (hc_state *)calloc(1, sizeof(hc_state));
  hc->out = hc_out;
  hc->cap = hc_cap;
  if (ccounts) memset(ccounts, 0, sizeof(uint32_t) * 2 * NXCRYS * NYCRYS * NHEADS * NDOIS);
  const int r = histogram_impl(t, w, n, offset, mode, duration, flags, clk, sino, delayed, st, hc, ccounts);
  for (int b = 0; b < NBLOCKS; b++) block_rates[b] = hc->nsamples[b] ? (int)(hc->total[b] / hc->nsamples[b]) : 0;
  totals[0] = hc->t_prompts;
  totals[1] = hc->t_randoms;
  const int lines = hc->n;
  free(hc);
  return r < 0 ? r : lines;
}

/* ---- smoothed randoms (gen_delays_lib/gen_delays_lib.cpp) ---------------- */
/* crystal index of the coincidence histogram and of the singles:
 * x + 72 head + 576 y + 59904 layer (compute_drate, gdl:175) */
#define NCRYS (NDOIS * NYCRYS * NHEADS * NXCRYS)
static int crys(int head, int layer, int cx, int cy) {
  return NXCRYS * head + cx + NXCRYS * NHEADS * cy + NXCRYS * NYCRYS * NHEADS * layer;
}
static void head_sums(const float *srate, float *hsum) {
  for (int head = 0; head < NHEADS; head++) {
    hsum[head] = 0.0f;
    for (int layer = 0; layer < NDOIS; layer++)
      for (int cx = 0; cx < NXCRYS; cx++)
        for (int cy = 0; cy < NYCRYS; cy++) hsum[head] += srate[crys(head, layer, cx, cy)];
  }
}
static float facing(const float *hsum, int head) {
  float s = 0.0f;
  for (int j = 0; j < 5; j++) s += hsum[(head + j + 2) % NHEADS];
  return s;
}

/* compute_csings_from_drates with compute_initial_srate, compute_drate,
 * errtotal and estimate_srate (gdl:163-255) */
int lm_crystal_singles(const int32_t *dcoins, float tau, float dt, float *srates) {
  float *drates = (float *)malloc(sizeof(float) * NCRYS), *xrates = (float *)malloc(sizeof(float) * NCRYS);
  float hsum[NHEADS];
  for (int i = 0; i < NCRYS; i++) drates[i] = dcoins[i] / dt;
  float dtotal = 0.0f;
  for (int i = 0; i < NCRYS; i++) dtotal += drates[i];
  const float stotal = (float)(8.0 * sqrt(dtotal / (40. * tau)));
  for (int i = 0; i < NCRYS; i++) srates[i] = drates[i] * stotal / dtotal;
  int iter;
  for (iter = 0; iter < 100; iter++) {
    head_sums(srates, hsum);
    for (int head = 0; head < NHEADS; head++) {
      const float oh = facing(hsum, head);
      for (int layer = 0; layer < NDOIS; layer++)
        for (int cx = 0; cx < NXCRYS; cx++)
          for (int cy = 0; cy < NYCRYS; cy++) {
            const int i = crys(head, layer, cx, cy);
            xrates[i] = srates[i] * tau * oh;
          }
    }
    uint32_t err = 0; /* int arithmetic of errtotal, wrapping */
    for (int i = 0; i < NCRYS; i++) {
      const uint32_t d = (uint32_t)(int)(dcoins[i] - (0.5 + xrates[i] * dt));
      err += d * d;
    }
    if (iter && err == 0) break;
    head_sums(srates, hsum);
    for (int head = 0; head < NHEADS; head++) {
      const float oh = facing(hsum, head);
      for (int layer = 0; layer < NDOIS; layer++)
        for (int cx = 0; cx < NXCRYS; cx++)
          for (int cy = 0; cy < NYCRYS; cy++) {
            const int i = crys(head, layer, cx, cy);
            srates[i] = (srates[i] + drates[i] / (tau * oh)) / 2.0f;
          }
    }
  }
  free(drates);
  free(xrates);
  return iter;
}

/* gen_delays (gdl:285-548) on one thread: singles from the delayed half of
 * the histogram, then compute_delays (gdl:89-153) for head pairs 1..20 in
 * turn, crystal A's singles indexed as gen_delays_fromarchive.cpp:191 does.
 * sino: lm_sino_size() floats, overwritten. */
int lm_smooth_randoms(const lm_tables *t, const int32_t *coinc_hist, float scan_duration, float tau, int maxrd,
                      float *sino) {
  const float tt = tau > 0 ? tau : 6.0e-9f, ft = scan_duration > 0 ? scan_duration : 1.0f;
  float *cs = (float *)malloc(sizeof(float) * NCRYS);
  const int it = lm_crystal_singles(coinc_hist + NCRYS, tt, ft, cs);
  memset(sino, 0, sizeof(float) * (size_t)lm_sino_size(t));
  const float tauftime = tt * ft;
  for (int mp = 1; mp <= NMPAIRS; mp++) {
    const int ahead = HRRT_MPAIRS[mp][0], bhead = HRRT_MPAIRS[mp][1];
    for (int al = 0; al < NDOIS; al++)
      for (int ay = 0; ay < NYCRYS; ay++) {
        int bs = 1000, be = -1000;
        for (int by = 0; by < NYCRYS; by++) {
          const int rd = ay > by ? ay - by : by - ay;
          if (rd < maxrd + 6) {
            if (bs > by) bs = by;
            if (be < by) be = by;
          }
        }
        for (int ax = 0; ax < NXCRYS; ax++) {
          const float aw = cs[al * NHEADS * NXCRYS * NYCRYS + ay * NHEADS * NXCRYS + ahead * NXCRYS + ax];
          const float awt = aw * tauftime;
          if (awt == 0) continue;
          for (int bl = 0; bl < NDOIS; bl++)
            for (int bx = 0; bx < NXCRYS; bx++)
              for (int by = bs; by <= be; by++) {
                const int a = lm_rebin_event(t, mp, al, ax, ay, bl, bx, by);
                if (a < 0) continue;
                sino[a] += cs[bl * NHEADS * NXCRYS * NYCRYS + bhead * NXCRYS + bx + NHEADS * NXCRYS * by] * awt;
              }
        }
      }
  }
  free(cs);
  return it;
}

/* convert_span9 (lmhistogram_mp/convert_span9.cpp:13-150): the span-3 trues
 * sinogram folded in place into span 9.  Span-9 segment 0 is span-3 segment
 * 0 plus segments -1 and +1 shifted by their plane offset; every further
 * span-9 segment -k / +k is the copy of span-3 segment -(3k-1) / +(3k-1)
 * plus segments -(3k) / +(3k) and -(3k+1) / +(3k+1) shifted by theirs.  The
 * sums are 16-bit (they wrap); the first 2209 planes hold the result. */
void lm_convert_span9(int16_t *sino, int maxrd, int nrings) {
  const int nseg = (2 * maxrd + 1) / 3, nseg9 = (2 * maxrd + 1) / 9;
  const long long npix = 256LL * 288;
  int nplns[64], nplns9[64], move[64];
  if (nseg > 64) return;
  for (int i = 0; i < nseg; i++) {
    const int seg = (i + 1) / 2, seg9 = (i + 3) / 6;
    nplns[i] = nplns9[i] = 207;
    move[i] = 0;
    if (seg > 0) nplns[i] = 2 * nrings - 3 * (2 * seg - 1) - 2;
    if (seg > 1) nplns9[i] = 2 * nrings - 9 * (2 * seg9 - 1) - 2;
    if (seg > 0) move[i] = (nplns9[i] - nplns[i]) / 2;
  }
  int iseg = 0, iseg9 = 0;
  long long pos3 = 0, pos9 = 0;
  while (iseg9 < nseg9) {
    const int nout = nplns[iseg];
    if (iseg9 == 0) {
      /* segment 0 stays; add -1 and +1 */
      int16_t *out = sino + move[1] * npix;
      for (int k = 1; k <= 2; k++) {
        pos3 += nplns[k - 1];
        const int16_t *in = sino + pos3 * npix;
        const long long n = npix * nplns[1];
        for (long long j = 0; j < n; j++) out[j] = (int16_t)(out[j] + in[j]);
      }
      pos9 = nout;
      iseg = 3;
      iseg9 = 1;
    } else {
      int16_t *neg = sino + pos9 * npix;
      int16_t *pos = neg + (long long)nout * npix;
      for (int k = 0; k < 6; k++, iseg++) {
        pos3 += nplns[iseg - 1];
        const int16_t *in = sino + pos3 * npix;
        const long long n = npix * nplns[iseg];
        int16_t *out = (k % 2 == 0 ? neg : pos) + (k < 2 ? 0 : (long long)move[iseg] * npix);
        if (k < 2)
          memcpy(out, in, sizeof(int16_t) * n);
        else
          for (long long j = 0; j < n; j++) out[j] = (int16_t)(out[j] + in[j]);
      }
      pos9 += 2LL * nout;
      iseg9 += 2;
    }
  }
}

/* goto_event (histogram_mp.cpp:384-425, 619-623) over the l64 words: the
 * parse of histogram_impl, every time tag setting the clock's second, up to
 * and including the tag that reaches `target` s (for target 0: the tag that
 * reads 0 ms).  Returns the words consumed, or -1 when the stream ends
 * first.  Without time-tag processing a seek to 0 is a no-op. */
long long lm_seek(const uint32_t *w, long long n, long long offset, int target, int flags, lm_clock *clk) {
  if ((flags & LM_TIME_FROM_COUNT) && target == 0) return 0;
  for (long long p0 = -(offset % PACKET_WORDS); p0 < n; p0 += PACKET_WORDS) {
    const long long count = (n - p0 < PACKET_WORDS) ? n - p0 : PACKET_WORDS;
    long long sp = p0 < 0 ? -p0 : 0;
    while (sp + 1 < count) {
      const unsigned ew1 = w[p0 + sp], ew2 = w[p0 + sp + 1];
      const int type = EWTYPES[((ew2 & 0xc0000000u) >> 30) | ((ew1 & 0xc0000000u) >> 28)];
      if (type == 3) {
        sp++;
        continue;
      }
      sp += 2;
      if (type != 2) continue;
      const unsigned tag = (ew1 & 0xffff) | ((ew2 & 0xffff) << 16);
      if ((tag & 0xE0000000u) != 0x80000000u) continue;
      const long long ms = tag & 0x3fffffff;
      if (ms == 0 && target == 0) {
        clk->current_time = 0;
        return p0 + sp;
      }
      if (clk->current_time != ms / 1000) {
        clk->current_time = ms / 1000;
        if (clk->current_time == target) return p0 + sp;
      }
    }
  }
  return -1;
}
