/*
 * lm_oracle.h -- CPU restatement of HRRT 64-bit listmode histogramming
 * (lmhistogram_mp) into span-3 or span-9 sinograms.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the device histogrammer.
 *
 * Parity: the reference's lmhistogram_mp does not build from its own files
 * (Boost, an unfinished rewrite, and a LUT that it reads from a file written
 * by hrrt_rebinner_lut); the restatement computes the LUT the way
 * hrrt_rebinner_lut does and follows the decode, rebin and histogram code
 * line by line.  Pinned by hand-computed known answers in tests/ (every
 * EWTYPES class, invalid crystals, DOI values, packet resync, time-tag frame
 * end, 16-bit wrap).
 */
#ifndef HRRT_LM_ORACLE_H
#define HRRT_LM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lm_tables lm_tables;

/* one LUT entry: sinogram bin + view*256, 1/(d*d_tan_theta), z/plane_sep */
typedef struct {
  int32_t nsino;
  float d;
  float z;
} lm_sol;

/* clock state carried from one frame to the next */
typedef struct {
  long long current_time;      /* s, -1 before the first time tag */
  long long current_time_msec; /* ms, -1 before the first time tag */
  long long prev_time;         /* ms of the previous time tag */
  int clock_reset;
  int pad;
} lm_clock;

typedef struct {
  long long words_used;  /* words consumed: up to and including the frame's last tag, or all */
  long long prompts;     /* prompt events histogrammed (counted as next_event_32 counts them) */
  long long delayed;     /* delayed events */
  long long timetags;    /* time tags processed */
  long long tags;        /* tag words of every kind */
  long long invalid;     /* events rejected by the head-pair / crystal checks */
  long long unmapped;    /* valid events with no sinogram address */
  long long doi_other;   /* events with a DOI value other than 0, 1 (not 7) */
  long long doi7;        /* transmission-flagged events in an emission stream */
  long long resyncs;     /* out-of-sync words skipped */
  long long frame_start; /* s */
  long long duration;    /* s, histogrammed time */
  int terminated;        /* the frame ended on a time tag */
  int pad;
} lm_stats;

/* hist modes (lmhistogram -P / -PR / default) */
enum { LM_TRUES = 0, LM_PROMPTS_AND_DELAYED = 1, LM_PROMPTS_ONLY = 2 };
/* flags */
enum { LM_IGNORE_BORDER_CRYSTAL = 1, LM_NO_DOI = 2, LM_TIME_FROM_COUNT = 4 };

lm_tables *lm_create(int span, int maxrd);
void lm_destroy(lm_tables *t);
long long lm_sino_size(const lm_tables *t);
int lm_nplanes(const lm_tables *t);
/* the tables, for the device build and for tests */
void lm_get_sol(const lm_tables *t, lm_sol *sol /* [21][144][144] */);
void lm_get_zpos(const lm_tables *t, float *c_zpos, float *c_zpos2 /* [104] */);
void lm_get_seg(const lm_tables *t, int *segz0, int *segzmax, int *segzoffset /* [45] */, int *nsegs);
void lm_get_crystals(const lm_tables *t, float *xyz /* [8][2][72][104][3] */);
double lm_d_tan_theta(const lm_tables *t);
/* rebin_event: sinogram address of one coincidence or -1 */
int lm_rebin_event(const lm_tables *t, int mp, int alayer, int ax, int ay, int blayer, int bx, int by);
/* the same for n rows (mp, alayer, ax, ay, blayer, bx, by) of ev */
void lm_rebin_events(const lm_tables *t, long long n, const int32_t *ev, int32_t *addr);

void lm_clock_init(lm_clock *c);
/* histogram one frame of the word stream (32-bit words, little-endian pairs
 * ew1, ew2) into `sino` (prompts, or trues in LM_TRUES mode) and `delayed`
 * (LM_PROMPTS_AND_DELAYED; may be NULL otherwise), each lm_sino_size() 16-bit
 * bins that the call adds to.  duration <= 0: the whole stream. */
int lm_histogram(const lm_tables *t, const uint32_t *words, long long nwords, int mode, int duration, int flags,
                 lm_clock *clock, uint16_t *sino, uint16_t *delayed, lm_stats *st);
/* lm_histogram of words that sit `offset` words into the file: its packets
 * of 2 Mi words count from the file start */
int lm_histogram_at(const lm_tables *t, const uint32_t *words, long long nwords, long long offset, int mode,
                    int duration, int flags, lm_clock *clock, uint16_t *sino, uint16_t *delayed, lm_stats *st);

/* one head-curve line: time (ms), prompts and delayed since the previous
 * line, sum of the blocks' latest singles samples */
typedef struct {
  long long time_ms, prompts, randoms, total_singles;
} lm_second;
/* lm_histogram of words that sit `offset` words into the file (packets
 * count from the file start) that also writes the frame's head curve
 * (returns the number of lines, up to hc_cap stored), the blocks' average
 * singles rates [936], the
 * totals of the lines' prompts and randoms [2] and, when ccounts is not
 * NULL, the coincidence histogram [2][119808] */
int lm_histogram_hc(const lm_tables *t, const uint32_t *words, long long nwords, long long offset, int mode,
                    int duration, int flags, lm_clock *clock, uint16_t *sino, uint16_t *delayed, lm_stats *st,
                    lm_second *hc_out, int hc_cap, int *block_rates, long long *totals, uint32_t *ccounts);
/* goto_event: the words consumed up to and including the time tag that
 * reaches `target` s (the 0-ms tag for target 0), the clock's second set on
 * the way; -1 when the stream ends first.  `offset`: position of words[0]
 * in the file (packets of 2 Mi words count from the file start). */
long long lm_seek(const uint32_t *words, long long nwords, long long offset, int target, int flags, lm_clock *clock);

/* smoothed randoms (gen_delays): crystal singles from the 119808 delayed
 * crystal counts (returns the iterations), and the randoms sinogram from a
 * coincidence histogram [2][119808] (prompt then delayed counts), both as
 * gen_delays_lib.cpp computes them */
int lm_crystal_singles(const int32_t *dcoins, float tau, float dt, float *srates);
int lm_smooth_randoms(const lm_tables *t, const int32_t *coinc_hist, float scan_duration, float tau, int maxrd,
                      float *sino);

/* convert_span9: a span-3 trues sinogram (45 segments, maxrd 67) folded in
 * place into span 9; the first 2209 planes hold the result */
void lm_convert_span9(int16_t *sino, int maxrd, int nrings);

#ifdef __cplusplus
}
#endif
#endif
