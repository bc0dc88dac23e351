/*
 * CPU oracle for the delta-encoded Ising anneal path.  TEST INFRASTRUCTURE ONLY:
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg call this file as the
 * checker (and as the timed CPU restatement).  The product path never links it.
 *
 * Every function restates a reference algorithm in plain C, with the reference file:line
 * it follows.  Paths are relative to the reference project root (skethz/Arpeggio).
 *
 *  orc_philox_batch  Philox4x32-10 (Salmon et al., SC'11), as arpeggio/mimo/chordfx.py:39-49
 *                    and arpeggio/rtl/cycle_checks/rtl_a59/src/arpeggio_ref59.py:14-21.
 *  orc_anneal_dd     integer anneal on the compressed dDI coupling G (D x D):
 *                    policy 0 = first accept (arpeggio_ref59.py:41-85 mode 'arpeggio',
 *                    the contract of arpeggio/sim/arpeggio_fx.cu:35-100), policy 1 = Chord's
 *                    snapshot round (arpeggio_ref59.py:72-82 mode 'par', plus the Onsager term
 *                    of arpeggio/mimo/chordfx.py:105).
 *  orc_anneal_chord_hw the Chord round on compressed G with the random numbers of the reference's C++
 *                    engine model without Philox (arpeggio/sim/x3model/engine_model.cpp, philox = 0).
 *  orc_anneal_chord  Chord on a full N x N int16 coupling: arpeggio/mimo/chordfx.py:80-118
 *                    (chord_fx), modes 'chains' and 'best'.
 *  orc_anneal_dd_f32 the same two policies with FP32 fields (no reference kernel exists; the
 *                    rule is the integer rule of arpeggio_ref59.py:62 with the float decision
 *                    of arpeggio/sim/arpx55.py:65, written out operation by operation below).
 *  orc_anneal_full_f32 both policies with FP32 fields on a full symmetric J (the RI map of
 *                    arpeggio/mimo/mimo.py:132-149), the float rule of arpx55.py:28-99 with Philox draws.
 *
 * Parity pins: tests/golden (KATs of chordfx.py:53-56, outputs of arpeggio_ref59.anneal and
 * chordfx.chord_fx produced by importing the reference, generator committed beside them).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_M0 0xD2511F53u
#define ORC_M1 0xCD9E8D57u
#define ORC_W0 0x9E3779B9u
#define ORC_W1 0xBB67AE85u

static void philox10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int i = 0; i < 10; i++) {
    if (i) {
      k0 += ORC_W0;
      k1 += ORC_W1;
    }
    uint64_t p0 = (uint64_t)ORC_M0 * c[0];
    uint64_t p1 = (uint64_t)ORC_M1 * c[2];
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
    c[1] = (uint32_t)p1;
    c[3] = (uint32_t)p0;
    c[0] = n0;
    c[2] = n2;
  }
}

static uint32_t philox_word(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                            int w) {
  uint32_t c[4] = {c0, c1, c2, c3};
  philox10(c, k0, k1);
  return c[w];
}

/* in: n x 6 words (counter c0..c3, key k0, k1) -> out: n x 4 words. */
int orc_philox_batch(const uint32_t* in, uint32_t* out, int n) {
  for (int t = 0; t < n; t++) {
    uint32_t c[4] = {in[6 * t], in[6 * t + 1], in[6 * t + 2], in[6 * t + 3]};
    philox10(c, in[6 * t + 4], in[6 * t + 5]);
    memcpy(out + 4 * t, c, sizeof c);
  }
  return 0;
}

/* The i-th P-bit word with P/2 ones, counted in increasing order (arpeggio_ref59.py:31-38). */
static int bal_pat(int P, uint32_t i) {
  uint32_t n = 0;
  for (int v = 0; v < (1 << P); v++)
    if (__builtin_popcount(v) == P / 2) {
      if (n == i) return v;
      n++;
    }
  return 0;
}

static int bal_count(int P) { return P == 2 ? 2 : (P == 4 ? 6 : 20); }

/* ------------------------------------------------------------------ thread pool over anneals */
typedef void (*orc_job_fn)(void* ctx, long idx);
typedef struct {
  orc_job_fn fn;
  void* ctx;
  long n;
  long next;
  pthread_mutex_t mu;
} orc_pool;

static void* orc_worker(void* a) {
  orc_pool* p = (orc_pool*)a;
  for (;;) {
    pthread_mutex_lock(&p->mu);
    long i = p->next++;
    pthread_mutex_unlock(&p->mu);
    if (i >= p->n) break;
    p->fn(p->ctx, i);
  }
  return NULL;
}

static void orc_run(orc_job_fn fn, void* ctx, long n, int nthreads) {
  if (nthreads <= 1 || n <= 1) {
    for (long i = 0; i < n; i++) fn(ctx, i);
    return;
  }
  orc_pool p = {fn, ctx, n, 0, PTHREAD_MUTEX_INITIALIZER};
  pthread_t th[256];
  if (nthreads > 256) nthreads = 256;
  for (int t = 0; t < nthreads; t++) pthread_create(&th[t], NULL, orc_worker, &p);
  for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------ integer anneal, compressed G */
typedef struct {
  const int32_t *G, *h, *T, *c;
  int B, D, P, R, L;
  int32_t q;
  const uint32_t* inst;
  uint32_t k0, k1;
  int start, policy;
  int8_t* out_s;
  int64_t *out_de, *out_st;
  const int8_t* m0; /* start == 2: given spin sums (B, D) */
  int warm_r;       /* start == 2: anneals r >= warm_r start from m = 0 */
  const uint32_t* cdf; /* start == 2, or NULL: thresholds (B, D, 2) of sampled starts for anneals 0 < r < warm_r */
  const int32_t* ra;   /* or NULL: per-problem anneal counts (B); anneals r >= ra[b] are skipped */
  int64_t* out_n1;     /* or NULL: Chord rounds with at least one flip per anneal (B, R) */
} dd_ctx;

/* Start spins of one anneal (arpeggio_ref59.py:44-49, arpeggio_fx.cu:48-57). s is P x D. */
static void start_spins(int start, int P, int D, uint32_t r, uint32_t inst, uint32_t k0, uint32_t k1,
                        const int8_t* m0, const uint32_t* cdf, int8_t* s) {
  if (start == 2) { /* given spin sums: m = 0 takes the 'bal' pattern, m != 0 sets copies p < (m + P) / 2 */
    uint64_t C = (uint64_t)bal_count(P);
    for (int j = 0; j < D; j++) {
      uint32_t w0 = philox_word(0xFFFFFFFFu, (uint32_t)j, r, inst, k0, k1, 0);
      int m = m0[j];
      if (cdf) { /* sampled start: word 1 of the same block against the coordinate's thresholds */
        uint32_t w1 = philox_word(0xFFFFFFFFu, (uint32_t)j, r, inst, k0, k1, 1);
        m = w1 < cdf[2 * j] ? -2 : (w1 > cdf[2 * j + 1] ? 2 : 0);
      }
      m = m < -P ? -P : (m > P ? P : m);
      int pat = m == 0 ? bal_pat(P, (uint32_t)(((uint64_t)w0 * C) >> 32)) : (1 << ((m + P) / 2)) - 1;
      for (int p = 0; p < P; p++) s[p * D + j] = ((pat >> p) & 1) ? 1 : -1;
    }
  } else if (start == 0) {
    for (int p = 0; p < P; p++)
      for (int j = 0; j < D; j++)
        s[p * D + j] = philox_word(0xFFFFFFFFu, (uint32_t)(p * D + j), r, inst, k0, k1, 0) >= 0x80000000u ? 1 : -1;
  } else {
    uint64_t C = (uint64_t)bal_count(P);
    for (int j = 0; j < D; j++) {
      uint32_t w0 = philox_word(0xFFFFFFFFu, (uint32_t)j, r, inst, k0, k1, 0);
      int pat = bal_pat(P, (uint32_t)(((uint64_t)w0 * C) >> 32));
      for (int p = 0; p < P; p++) s[p * D + j] = ((pat >> p) & 1) ? 1 : -1;
    }
  }
}

static void dd_job(void* vctx, long t) {
  const dd_ctx* x = (const dd_ctx*)vctx;
  const int D = x->D, P = x->P, R = x->R;
  const long b = t / R;
  const uint32_t r = (uint32_t)(t % R), inst = x->inst[b];
  const int32_t* G = x->G + (size_t)b * D * D; /* G[i * D + j] */
  const int32_t* h = x->h + (size_t)b * D;
  int8_t s[6 * 128], bs[6 * 128];
  uint8_t pf[6 * 128];
  int64_t w[128];
  uint8_t F[128];
  static const int8_t zeros[128] = {0};
  if (x->ra) { /* a skipped anneal reports the guess: zero spin sums, best energy INT64_MAX, no tests */
    int rb = x->ra[b] < 1 ? 1 : (x->ra[b] > R ? R : x->ra[b]);
    if ((int)r >= rb) {
      memset(x->out_s + (size_t)t * P * D, 0, (size_t)P * D);
      x->out_de[t] = INT64_MAX;
      x->out_st[2 * t] = 0;
      x->out_st[2 * t + 1] = 0;
      return;
    }
  }
  start_spins(x->start, P, D, r, inst, x->k0, x->k1,
              x->m0 ? ((int)r < x->warm_r ? x->m0 + (size_t)b * D : zeros) : NULL,
              (x->cdf && r > 0 && (int)r < x->warm_r) ? x->cdf + (size_t)b * D * 2 : NULL, s);
  memcpy(bs, s, (size_t)P * D);
  memset(pf, 0, sizeof pf);
  for (int i = 0; i < D; i++) { /* w_i = h_i - 2 sum_j G_ij m_j (arpeggio_ref59.py:50-51) */
    int64_t acc = 0;
    for (int j = 0; j < D; j++) {
      int m = 0;
      for (int p = 0; p < P; p++) m += s[p * D + j];
      acc += (int64_t)G[i * D + j] * m;
    }
    w[i] = h[i] - 2 * acc;
  }
  int64_t de = 0, best = (int64_t)1 << 62, flips = 0, tests = 0, n1 = 0;
  for (int k = 0; k < x->L; k++) {
    const int p = k % P;
    const uint32_t n = (uint32_t)(k / P);
    const __int128 A = (__int128)4 * x->T[k];
    const int64_t Bk = (int64_t)x->q + 2 * (int64_t)x->T[k];
    int8_t* sp = s + p * D;
    if (x->policy == 0) { /* first accept: a flip updates every field before the next lane (:59-71) */
      int64_t tt = 1;
      for (int j = 0; j < D; j++) {
        uint32_t u = philox_word(n >> 2, (uint32_t)(p * D + j), r, inst, x->k0, x->k1, (int)(n & 3));
        int64_t dj = G[j * D + j];
        __int128 lhs = (__int128)u * A;
        __int128 rhs = ((__int128)sp[j] * w[j] + 2 * (__int128)dj + Bk) * ((__int128)1 << 32);
        if (lhs > rhs) {
          int so = sp[j];
          de += 4 * (int64_t)so * w[j] + 8 * dj;
          for (int i = 0; i < D; i++) w[i] += 4 * (int64_t)so * G[i * D + j];
          sp[j] = (int8_t)(-so);
          flips++;
          if (j < D - 1) tt++;
        }
      }
      tests += tt;
    } else { /* Chord's round: every lane tests the snapshot, then the flips commit in order (:72-82) */
      const int64_t ck = x->c ? (int64_t)x->c[k] : 0;
      for (int j = 0; j < D; j++) {
        uint32_t u = philox_word(n >> 2, (uint32_t)(p * D + j), r, inst, x->k0, x->k1, (int)(n & 3));
        int64_t dj = G[j * D + j];
        int64_t sgn = pf[p * D + j] ? -1 : 1;
        __int128 lhs = (__int128)u * A;
        __int128 rhs = ((__int128)sp[j] * w[j] + 2 * (__int128)dj + Bk - ck * sgn) * ((__int128)1 << 32);
        F[j] = lhs > rhs;
      }
      memset(pf, 0, (size_t)P * D);
      for (int j = 0; j < D; j++)
        if (F[j]) { /* n1: the round flips (arpeggio_ref59.py:74) */
          n1++;
          break;
        }
      for (int j = 0; j < D; j++) {
        if (!F[j]) continue;
        int so = sp[j];
        int64_t dj = G[j * D + j];
        de += 4 * (int64_t)so * w[j] + 8 * dj;
        for (int i = 0; i < D; i++) w[i] += 4 * (int64_t)so * G[i * D + j];
        sp[j] = (int8_t)(-so);
        pf[p * D + j] = 1;
        flips++;
      }
      tests += 1;
    }
    if (de < best) { /* best state after each pass (:83-84) */
      best = de;
      memcpy(bs, s, (size_t)P * D);
    }
  }
  memcpy(x->out_s + (size_t)t * P * D, bs, (size_t)P * D);
  x->out_de[t] = best;
  x->out_st[2 * t] = flips;
  x->out_st[2 * t + 1] = tests;
  if (x->out_n1) x->out_n1[t] = n1;
}

/* G (B, D, D) row-major G[b][i][j]; h (B, D); T (L) one temperature per pass (pass k tests copy k % P);
 * c (L) Onsager terms or NULL (policy 1 only); start 0 = 'rand', 1 = 'bal'; policy 0 = first accept,
 * 1 = Chord round.  Outputs: best spins (B, R, P*D) copy-major, best energy change (B, R), and
 * (flips, tests) per anneal (B, R, 2). */
int orc_anneal_dd(const int32_t* G, const int32_t* h, int B, int D, int P, int R, const int32_t* T,
                  const int32_t* c, int L, int32_t q, const uint32_t* inst, uint32_t k0, uint32_t k1, int start,
                  int policy, int8_t* out_s, int64_t* out_de, int64_t* out_st, int nthreads) {
  if (D < 1 || D > 128 || !(P == 2 || P == 4 || P == 6 || (P == 1 && start == 0)) || L < 1 || R < 1 || B < 0)
    return 1;
  dd_ctx x = {G, h, T, c, B, D, P, R, L, q, inst, k0, k1, start, policy, out_s, out_de, out_st, NULL, 0, NULL, NULL};
  orc_run(dd_job, &x, (long)B * R, nthreads);
  return 0;
}

/* orc_anneal_dd's Chord round (policy 1) that also counts, per anneal, the rounds with at least one flip (n1 of
 * arpeggio_ref59.anneal, rtl_a59/src/arpeggio_ref59.py:74): out_n1 (B, R). */
int orc_anneal_chord_dd_n1(const int32_t* G, const int32_t* h, int B, int D, int P, int R, const int32_t* T,
                           const int32_t* c, int L, int32_t q, const uint32_t* inst, uint32_t k0, uint32_t k1,
                           int start, int8_t* out_s, int64_t* out_de, int64_t* out_st, int64_t* out_n1,
                           int nthreads) {
  if (D < 1 || D > 128 || !(P == 2 || P == 4 || P == 6) || L < 1 || R < 1 || B < 0) return 1;
  dd_ctx x = {G, h, T, c, B, D, P, R, L, q, inst, k0, k1, start, 1, out_s, out_de, out_st, NULL, 0, NULL, NULL,
              out_n1};
  orc_run(dd_job, &x, (long)B * R, nthreads);
  return 0;
}

/* First accept from given spin sums m0 (B, D) (start 2 of start_spins) for anneals r < warm_r, from m = 0 for
 * the others; with cdf (B, D, 2) (or NULL) anneals 0 < r < warm_r draw their spin sums from those thresholds
 * instead of taking m0; with ra (B) (or NULL) problem b runs anneals r < ra[b] only.  The caller permutes the problem into scan order first (the device's flip-test order
 * is a relabelling of the coordinates). */
int orc_anneal_dd_warm(const int32_t* G, const int32_t* h, int B, int D, int P, int R, const int32_t* T, int L,
                       int32_t q, const uint32_t* inst, uint32_t k0, uint32_t k1, const int8_t* m0, int warm_r,
                       const uint32_t* cdf, const int32_t* ra, int8_t* out_s, int64_t* out_de, int64_t* out_st,
                       int nthreads) {
  if (D < 1 || D > 128 || !(P == 2 || P == 4 || P == 6) || L < 1 || R < 1 || B < 0 || !m0) return 1;
  if (cdf && P != 2) return 1;
  dd_ctx x = {G, h, T, NULL, B, D, P, R, L, q, inst, k0, k1, 2, 0, out_s, out_de, out_st, m0, warm_r, cdf, ra};
  orc_run(dd_job, &x, (long)B * R, nthreads);
  return 0;
}

/* ------------------------------------------------------------------ Chord with the engine's own numbers
 * The Chord round of orc_anneal_dd (policy 1) with the random numbers of the reference's C++ engine model when it
 * runs without Philox (philox = 0 of arpeggio/sim/x3model/engine_model.cpp, the mode of its production scripts
 * arpeggio/sim/x3_prod.py:105-106 and run_a516.py:135-136):
 *  - per anneal a seed chain of three murmur-style mixing rounds over (key low ^ inst), key high and r (the
 *    seeder's pop :185-194 and B chain :170-178), whose result + phi seeds the lanes;
 *  - lane j: mix(seed + j phi) (lane groups :179-184, stage B :165-167), finalised, zero replaced by phi, then one
 *    xorshift32 step (stage C :142-163): that word is the lane's generator state and its bits 31, 30, ... are the
 *    start spins of copies 0, 1, ...;
 *  - every step advances every lane's state by one xorshift32 step and takes its top 16 bits u (decision D1
 *    :242-257); the test is u 4 T > (s w_j + 2 G_jj + q - c + 2 T) 2^16 (D2 :229-240);
 *  - the best state starts at 2^35 - 1 (:46) and is taken after every step (D0 :264, the final check :128).  */
static inline uint32_t hw_mix_a(uint32_t v) { return (v ^ (v >> 16)) * 0x85EBCA6Bu; }
static inline uint32_t hw_mix_b(uint32_t v) { return (v ^ (v >> 13)) * 0xC2B2AE35u; }
static inline uint32_t hw_fin(uint32_t v) { return v ^ (v >> 16); }
static inline uint32_t hw_xs32(uint32_t x) {
  x ^= x << 13;
  x ^= x >> 17;
  x ^= x << 5;
  return x;
}

typedef struct {
  const int32_t *G, *h, *T, *c;
  int B, D, P, R, L;
  int32_t q;
  const uint32_t* inst;
  uint64_t key;
  int8_t* out_s;
  int64_t *out_de, *out_st;
} hw_ctx;

static void hw_job(void* vctx, long t) {
  const hw_ctx* x = (const hw_ctx*)vctx;
  const int D = x->D, P = x->P, R = x->R;
  const long b = t / R;
  const uint32_t r = (uint32_t)(t % R), PHI = 0x9E3779B9u;
  const int32_t* G = x->G + (size_t)b * D * D;
  const int32_t* h = x->h + (size_t)b * D;
  uint32_t f = hw_fin(hw_mix_b(hw_mix_a((uint32_t)x->key ^ x->inst[b])));
  f = hw_fin(hw_mix_b(hw_mix_a(f ^ (uint32_t)(x->key >> 32))));
  f = hw_fin(hw_mix_b(hw_mix_a(f ^ r)));
  const uint32_t seed = f + PHI;
  uint32_t rng[128];
  int8_t s[6 * 128], bs[6 * 128];
  int64_t w[128];
  uint8_t F[128];
  for (int j = 0; j < D; j++) {
    uint32_t v = hw_fin(hw_mix_b(hw_mix_a(seed + (uint32_t)j * PHI)));
    if (v == 0) v = PHI;
    rng[j] = hw_xs32(v);
    for (int p = 0; p < P; p++) s[p * D + j] = ((rng[j] >> (31 - p)) & 1u) ? 1 : -1;
  }
  memcpy(bs, s, (size_t)P * D);
  for (int i = 0; i < D; i++) { /* w_i = h_i - 2 sum_j G_ij m_j */
    int64_t acc = 0;
    for (int j = 0; j < D; j++) {
      int m = 0;
      for (int p = 0; p < P; p++) m += s[p * D + j];
      acc += (int64_t)G[i * D + j] * m;
    }
    w[i] = h[i] - 2 * acc;
  }
  int64_t de = 0, best = ((int64_t)1 << 35) - 1, flips = 0;
  for (int k = 0; k < x->L; k++) {
    const int p = k % P;
    const __int128 A = (__int128)4 * x->T[k];
    const int64_t Bk = (int64_t)x->q - (x->c ? (int64_t)x->c[k] : 0) + 2 * (int64_t)x->T[k];
    int8_t* sp = s + p * D;
    for (int j = 0; j < D; j++) {
      rng[j] = hw_xs32(rng[j]);
      const uint32_t u = rng[j] >> 16;
      const __int128 rhs = ((__int128)sp[j] * w[j] + 2 * (__int128)G[j * D + j] + Bk) * ((__int128)1 << 16);
      F[j] = (__int128)u * A > rhs;
    }
    for (int j = 0; j < D; j++) {
      if (!F[j]) continue;
      const int so = sp[j];
      de += 4 * (int64_t)so * w[j] + 8 * (int64_t)G[j * D + j];
      for (int i = 0; i < D; i++) w[i] += 4 * (int64_t)so * G[j * D + i];
      sp[j] = (int8_t)(-so);
      flips++;
    }
    if (de < best) {
      best = de;
      memcpy(bs, s, (size_t)P * D);
    }
  }
  memcpy(x->out_s + (size_t)t * P * D, bs, (size_t)P * D);
  x->out_de[t] = best;
  x->out_st[2 * t] = flips;
  x->out_st[2 * t + 1] = x->L;
}

/* G (B, D, D), h (B, D); T, c (L) per step (c may be NULL); q; inst (B); the 64-bit key.  Outputs as
 * orc_anneal_dd: best spins (B, R, P*D) copy-major, best energy change (B, R), (flips, steps) per anneal. */
int orc_anneal_chord_hw(const int32_t* G, const int32_t* h, int B, int D, int P, int R, const int32_t* T,
                        const int32_t* c, int L, int32_t q, const uint32_t* inst, uint64_t key, int8_t* out_s,
                        int64_t* out_de, int64_t* out_st, int nthreads) {
  if (D < 1 || D > 128 || P < 1 || P > 6 || L < 1 || R < 1 || B < 0) return 1;
  hw_ctx x = {G, h, T, c, B, D, P, R, L, q, inst, key, out_s, out_de, out_st};
  orc_run(hw_job, &x, (long)B * R, nthreads);
  return 0;
}

/* ------------------------------------------------------------------ Chord on a full int16 J (chord_fx) */
typedef struct {
  const int16_t* J;
  const int32_t *h, *h0, *T, *c;
  int q, S, P, R, N, B;
  uint32_t k0, k1, inst0;
  int64_t* e_all;  /* (B, R) */
  int8_t* s_all;   /* (B, R, N) */
} ch_ctx;

static void ch_job(void* vctx, long t) {
  const ch_ctx* x = (const ch_ctx*)vctx;
  const int N = x->N, P = x->P, R = x->R;
  const long b = t / R;
  const uint32_t r = (uint32_t)(t % R), m = x->inst0 + (uint32_t)b;
  const int16_t* J = x->J + (size_t)b * N * N;
  const int32_t* h = x->h + (size_t)b * N;
  const int32_t* h0 = x->h0 + (size_t)b * N;
  int8_t s[256], bs[256], pf[256], fl[256];
  int64_t u[256];
  for (int i = 0; i < N; i++) /* start (chordfx.py:93-94) */
    s[i] = philox_word(0xFFFFFFFFu, (uint32_t)i, r, m, x->k0, x->k1, 0) >= 0x80000000u ? 1 : -1;
  for (int i = 0; i < N; i++) { /* u = h + 2 J s (:95-96), row i of J */
    int64_t acc = 0;
    for (int j = 0; j < N; j++) acc += (int64_t)J[i * N + j] * s[j];
    u[i] = h[i] + 2 * acc;
  }
  memset(pf, 0, sizeof pf);
  memcpy(bs, s, (size_t)N);
  int64_t best = (int64_t)1 << 62;
  const int per = N / P;
  for (int k = 0; k < x->S; k++) {
    const int p = k % P, n = k / P;
    const __int128 A = (__int128)4 * x->T[k];
    for (int i = 0; i < N; i++) { /* decision (:104-106) */
      uint32_t xr = philox_word((uint32_t)(n / 4), (uint32_t)i, r, m, x->k0, x->k1, n % 4);
      int64_t z = (int64_t)s[i] * u[i] + x->q - (int64_t)x->c[k] * (pf[i] ? -1 : 1);
      fl[i] = ((__int128)xr * A > ((__int128)z + 2 * (__int128)x->T[k]) * ((__int128)1 << 32)) && (i / per == p);
    }
    for (int i = 0; i < N; i++) { /* s flips; u = h + 2 J s follows exactly by column updates */
      pf[i] = fl[i];
      if (!fl[i]) continue;
      int so = s[i];
      s[i] = (int8_t)(-so);
      for (int a = 0; a < N; a++) u[a] -= 4 * (int64_t)so * J[a * N + i];
    }
    int64_t e = 0; /* 2 E0 = sum s (h - 2 h0 - u) (:110) */
    for (int i = 0; i < N; i++) e += (int64_t)s[i] * ((int64_t)h[i] - 2 * (int64_t)h0[i] - u[i]);
    if (e < best) {
      best = e;
      memcpy(bs, s, (size_t)N);
    }
  }
  x->e_all[t] = best;
  memcpy(x->s_all + (size_t)t * N, bs, (size_t)N);
}

/* Contract of chordfx.chord_fx (arpeggio/mimo/chordfx.py:80-118).  mode 0 ('chains'): out_e (B, R),
 * out_s (B, R, N); mode 1 ('best'): the first anneal with the lowest energy, out_e (B), out_s (B, N). */
int orc_anneal_chord(const int16_t* J, const int32_t* h, const int32_t* h0, const int32_t* T, const int32_t* c,
                     int q, int S, int P, int R, int N, int B, uint32_t k0, uint32_t k1, uint32_t inst0, int mode,
                     int64_t* out_e, int8_t* out_s, int nthreads) {
  if (N < 1 || N > 256 || P < 1 || N % P || S < 1 || R < 1) return 1;
  int64_t* e_all = out_e;
  int8_t* s_all = out_s;
  if (mode == 1) {
    e_all = (int64_t*)malloc(sizeof(int64_t) * (size_t)B * R);
    s_all = (int8_t*)malloc((size_t)B * R * N);
  }
  ch_ctx x = {J, h, h0, T, c, q, S, P, R, N, B, k0, k1, inst0, e_all, s_all};
  orc_run(ch_job, &x, (long)B * R, nthreads);
  if (mode == 1) {
    for (int b = 0; b < B; b++) {
      int im = 0;
      for (int r = 1; r < R; r++)
        if (e_all[(size_t)b * R + r] < e_all[(size_t)b * R + im]) im = r;
      out_e[b] = e_all[(size_t)b * R + im];
      memcpy(out_s + (size_t)b * N, s_all + ((size_t)b * R + im) * N, (size_t)N);
    }
    free(e_all);
    free(s_all);
  }
  return 0;
}

/* ------------------------------------------------------------------ FP32 fields, compressed G */
/* The float rule, one IEEE single operation per line (no contraction; compile with
 * -ffp-contract=off):
 *   rr   = (float)(x >> 8) * 2^-24                    exact, in [0, 1)
 *   thr  = (rr - 0.5f) * (4 T_k)                      one rounding
 *   z    = ((s * w_j) + 2 G_jj) + q_k                 two roundings (q_k = q - c_k sgn for Chord)
 *   flip iff z < thr
 *   de  += (4 s w_j) + 8 G_jj                         two roundings
 *   w_i += (4 s) G_ij  (i = 0..D-1)                   one rounding each
 * Fields start as w_i = h_i - 2 sum_j G_ij m_j, summed in j order. */
typedef struct {
  const float *G, *h, *T, *c;
  int B, D, P, R, L;
  float q;
  const uint32_t* inst;
  uint32_t k0, k1;
  int start, policy;
  int8_t* out_s;
  float* out_de;
  int64_t* out_st;
} f32_ctx;

static float orc_thr(uint32_t x, float A) {
  volatile float rr = (float)(x >> 8) * 5.9604644775390625e-08f;
  volatile float d = rr - 0.5f;
  volatile float t = d * A;
  return t;
}

static void f32_job(void* vctx, long t) {
  const f32_ctx* x = (const f32_ctx*)vctx;
  const int D = x->D, P = x->P, R = x->R;
  const long b = t / R;
  const uint32_t r = (uint32_t)(t % R), inst = x->inst[b];
  const float* G = x->G + (size_t)b * D * D;
  const float* h = x->h + (size_t)b * D;
  int8_t s[6 * 128], bs[6 * 128];
  uint8_t pf[6 * 128], F[128];
  float w[128];
  start_spins(x->start, P, D, r, inst, x->k0, x->k1, NULL, NULL, s);
  memcpy(bs, s, (size_t)P * D);
  memset(pf, 0, sizeof pf);
  for (int i = 0; i < D; i++) {
    volatile float acc = 0.0f;
    for (int j = 0; j < D; j++) {
      int m = 0;
      for (int p = 0; p < P; p++) m += s[p * D + j];
      volatile float prod = G[i * D + j] * (float)m; /* exact: |m| <= 6 */
      acc = acc + prod;
    }
    volatile float two = 2.0f * acc;
    w[i] = h[i] - two;
  }
  volatile float de = 0.0f;
  float best = INFINITY;
  int64_t flips = 0, tests = 0;
  for (int k = 0; k < x->L; k++) {
    const int p = k % P;
    const uint32_t n = (uint32_t)(k / P);
    const float A = 4.0f * x->T[k];
    const float ck = (x->policy == 1 && x->c) ? x->c[k] : 0.0f;
    int8_t* sp = s + p * D;
    if (x->policy == 0) {
      int64_t tt = 1;
      for (int j = 0; j < D; j++) {
        uint32_t u = philox_word(n >> 2, (uint32_t)(p * D + j), r, inst, x->k0, x->k1, (int)(n & 3));
        float thr = orc_thr(u, A);
        float g = G[j * D + j];
        volatile float a = (float)sp[j] * w[j];
        volatile float bb = a + 2.0f * g;
        volatile float z = bb + x->q;
        if (z < thr) {
          int so = sp[j];
          volatile float e1 = (float)(4 * so) * w[j];
          volatile float e2 = e1 + 8.0f * g;
          de = de + e2;
          for (int i = 0; i < D; i++) {
            volatile float inc = (float)(4 * so) * G[i * D + j];
            w[i] = w[i] + inc;
          }
          sp[j] = (int8_t)(-so);
          flips++;
          if (j < D - 1) tt++;
        }
      }
      tests += tt;
    } else {
      for (int j = 0; j < D; j++) {
        uint32_t u = philox_word(n >> 2, (uint32_t)(p * D + j), r, inst, x->k0, x->k1, (int)(n & 3));
        float thr = orc_thr(u, A);
        float g = G[j * D + j];
        volatile float qk = x->q - ck * (pf[p * D + j] ? -1.0f : 1.0f);
        volatile float a = (float)sp[j] * w[j];
        volatile float bb = a + 2.0f * g;
        volatile float z = bb + qk;
        F[j] = z < thr;
      }
      memset(pf, 0, (size_t)P * D);
      for (int j = 0; j < D; j++) {
        if (!F[j]) continue;
        int so = sp[j];
        float g = G[j * D + j];
        volatile float e1 = (float)(4 * so) * w[j];
        volatile float e2 = e1 + 8.0f * g;
        de = de + e2;
        for (int i = 0; i < D; i++) {
          volatile float inc = (float)(4 * so) * G[i * D + j];
          w[i] = w[i] + inc;
        }
        sp[j] = (int8_t)(-so);
        pf[p * D + j] = 1;
        flips++;
      }
      tests += 1;
    }
    if (de < best) {
      best = de;
      memcpy(bs, s, (size_t)P * D);
    }
  }
  memcpy(x->out_s + (size_t)t * P * D, bs, (size_t)P * D);
  x->out_de[t] = best;
  x->out_st[2 * t] = flips;
  x->out_st[2 * t + 1] = tests;
}

int orc_anneal_dd_f32(const float* G, const float* h, int B, int D, int P, int R, const float* T, const float* c,
                      int L, float q, const uint32_t* inst, uint32_t k0, uint32_t k1, int start, int policy,
                      int8_t* out_s, float* out_de, int64_t* out_st, int nthreads) {
  if (D < 1 || D > 128 || !(P == 2 || P == 4 || P == 6 || (P == 1 && start == 0)) || L < 1 || R < 1 || B < 0)
    return 1;
  f32_ctx x = {G, h, T, c, B, D, P, R, L, q, inst, k0, k1, start, policy, out_s, out_de, out_st};
  orc_run(f32_job, &x, (long)B * R, nthreads);
  return 0;
}

/* ------------------------------------------------------------------ FP32 fields, full coupling J (N x N)
 * The float first-accept / Chord rules of arpeggio/sim/arpx55.py:28-99 (arpeggio_seq, rule (2)) on a generic
 * problem (the RI map of mimo.ising, mimo.py:132-149): N spins in P banks of D = N/P lanes, pass k tests bank
 * k % P; fields u = h + 2 J s (J symmetric, zero diagonal), one IEEE rounding per operation:
 *   u_i  = h_i + 2 (sum_j J_ij s_j)        sum in j order
 *   rr   = (x >> 8) 2^-24, thr = (rr - 1/2) (4 T_k)
 *   flip iff (s_i u_i + q) < thr           (Chord: q - c_k)
 *   de  += 2 s_g u_g                       (exact product, one rounding)
 *   u_i += (-4 s_g) J_ig                   (exact product, one rounding)
 * Start: 'rand' (Philox word 0 of (2^32-1, i, r, inst) >= 2^31) or given spins s0 (B, N).  Best: lowest de after
 * each pass. */
typedef struct {
  const float *J, *h, *T, *c;
  const int8_t* s0;
  int B, N, P, R, L;
  float q;
  const uint32_t* inst;
  uint32_t k0, k1;
  int policy;
  int8_t* out_s;
  float* out_de;
  int64_t* out_st;
} full_ctx;

static void full_job(void* vctx, long t) {
  const full_ctx* x = (const full_ctx*)vctx;
  const int N = x->N, P = x->P, R = x->R, D = N / P;
  const long b = t / R;
  const uint32_t r = (uint32_t)(t % R), inst = x->inst[b];
  const float* J = x->J + (size_t)b * N * N;
  const float* h = x->h + (size_t)b * N;
  int8_t s[256], bs[256];
  uint8_t F[256];
  float u[256];
  for (int i = 0; i < N; i++)
    s[i] = x->s0 ? x->s0[(size_t)b * N + i]
                 : (philox_word(0xFFFFFFFFu, (uint32_t)i, r, inst, x->k0, x->k1, 0) >= 0x80000000u ? 1 : -1);
  memcpy(bs, s, (size_t)N);
  for (int i = 0; i < N; i++) {
    volatile float acc = 0.0f;
    for (int j = 0; j < N; j++) {
      volatile float pj = J[i * N + j] * (float)s[j];
      acc = acc + pj;
    }
    volatile float two = 2.0f * acc;
    u[i] = h[i] + two;
  }
  volatile float de = 0.0f;
  float best = INFINITY;
  int64_t flips = 0, tests = 0;
  for (int k = 0; k < x->L; k++) {
    const int p = k % P;
    const uint32_t n = (uint32_t)(k / P);
    const float A = 4.0f * x->T[k];
    const float qk = (x->policy == 1 && x->c) ? x->q - x->c[k] : x->q;
    int64_t tt = 1;
    if (x->policy == 1) memset(F, 0, sizeof F);
    for (int jj = 0; jj < D; jj++) {
      const int g = p * D + jj;
      uint32_t w = philox_word(n >> 2, (uint32_t)g, r, inst, x->k0, x->k1, (int)(n & 3));
      float thr = orc_thr(w, A);
      volatile float su = (float)s[g] * u[g];
      volatile float z = su + qk;
      if (!(z < thr)) continue;
      if (x->policy == 1) {
        F[g] = 1;
        continue;
      }
      int so = s[g];
      volatile float e1 = (float)(2 * so) * u[g];
      de = de + e1;
      for (int i = 0; i < N; i++) {
        volatile float inc = (float)(-4 * so) * J[i * N + g];
        u[i] = u[i] + inc;
      }
      s[g] = (int8_t)(-so);
      flips++;
      if (jj < D - 1) tt++;
    }
    if (x->policy == 1) {
      for (int jj = 0; jj < D; jj++) {
        const int g = p * D + jj;
        if (!F[g]) continue;
        int so = s[g];
        volatile float e1 = (float)(2 * so) * u[g];
        de = de + e1;
        for (int i = 0; i < N; i++) {
          volatile float inc = (float)(-4 * so) * J[i * N + g];
          u[i] = u[i] + inc;
        }
        s[g] = (int8_t)(-so);
        flips++;
      }
      tt = 1;
    }
    tests += tt;
    if (de < best) {
      best = de;
      memcpy(bs, s, (size_t)N);
    }
  }
  memcpy(x->out_s + (size_t)t * N, bs, (size_t)N);
  x->out_de[t] = best;
  x->out_st[2 * t] = flips;
  x->out_st[2 * t + 1] = tests;
}

int orc_anneal_full_f32(const float* J, const float* h, const int8_t* s0, int B, int N, int P, int R, const float* T,
                        const float* c, int L, float q, const uint32_t* inst, uint32_t k0, uint32_t k1, int policy,
                        int8_t* out_s, float* out_de, int64_t* out_st, int nthreads) {
  if (N < 1 || N > 256 || P < 1 || N % P || L < 1 || R < 1 || B < 0) return 1;
  full_ctx x = {J, h, T, c, s0, B, N, P, R, L, q, inst, k0, k1, policy, out_s, out_de, out_st};
  orc_run(full_job, &x, (long)B * R, nthreads);
  return 0;
}

/* ------------------------------------------------------------------ trajectory soft output (RI map) */
/* The sampler of mimo.chord_soft (arpeggio/mimo/mimo.py:332-394) with this project's Philox draws, restated as the
 * device kernel computes it (one IEEE single operation per line): per chain, u = hf + 2 (sum_j J_ji s_j in j order),
 * E0 = -sum over lanes (in the warp's butterfly order) of the lane partials -sum_t s_i (h0_i + (u_i - hf_i)/2); per
 * step every spin tests z = s u + q < thr = (x/2^32 - 1/2) 4T (x: word k&3 of block (k>>2, i, r, inst)), the flips
 * commit in index order (E0 += (+-2) ((h0_j - hf_j) + u_j), u_i += (-+4) J_ji), and after a step that flips (and step
 * 0) d = scale E0 + c0 updates the per-bit minima and the chain's best (first minimum).  Chains are independent; the
 * problem keeps the minima over its chains and the best state by (d, step, chain). */
typedef struct {
  const float *J, *hf, *h0, *scale, *c0, *T;
  const int8_t* s0;
  float q;
  int S, R, N, D, M, B;
  const uint32_t* inst;
  uint32_t k0, k1;
  float *cm0, *cm1, *cbest; /* per (b, r): minima (nbits each) and best d */
  int *cstep;
  int8_t* cbs;              /* per (b, r): best spins (N) */
} soft_ctx;

static float f_add(float a, float b) { volatile float r = a + b; return r; }
static float f_sub(float a, float b) { volatile float r = a - b; return r; }
static float f_mul(float a, float b) { volatile float r = a * b; return r; }

static void soft_job(void* vctx, long t) {
  const soft_ctx* x = (const soft_ctx*)vctx;
  const int N = x->N, D = x->D, S = x->S, R = x->R, nb = x->M == 16 ? 2 : 1, nbits = D * nb;
  const long b = t / R;
  const uint32_t r = (uint32_t)(t % R), inst = x->inst[b];
  const float* J = x->J + (size_t)b * N * N;
  const float* hf = x->hf + (size_t)b * N;
  const float* h0 = x->h0 + (size_t)b * N;
  const float* Tb = x->T + (size_t)b * S;
  int8_t s[128], cb[128];
  float u[128], part[32];
  for (int i = 0; i < N; i++) {
    if (x->s0) s[i] = x->s0[(size_t)b * N + i] > 0 ? 1 : -1;
    else s[i] = philox_word(0xFFFFFFFFu, (uint32_t)i, r, inst, x->k0, x->k1, 0) >= 0x80000000u ? 1 : -1;
  }
  for (int i = 0; i < N; i++) {
    float acc = 0.0f;
    for (int j = 0; j < N; j++) acc = f_add(acc, f_mul(J[(size_t)j * N + i], s[j] > 0 ? 1.0f : -1.0f));
    u[i] = f_add(hf[i], f_mul(2.0f, acc));
  }
  for (int l = 0; l < 32; l++) {
    float e = 0.0f;
    for (int tt = 0; 32 * tt + l < N; tt++) {
      const int i = 32 * tt + l;
      const float si = s[i] > 0 ? 1.0f : -1.0f;
      e = f_sub(e, f_mul(si, f_add(h0[i], f_mul(0.5f, f_sub(u[i], hf[i])))));
    }
    part[l] = e;
  }
  for (int o = 1; o < 32; o <<= 1) {
    float nx[32];
    for (int l = 0; l < 32; l++) nx[l] = f_add(part[l], part[l ^ o]);
    memcpy(part, nx, sizeof nx);
  }
  float E = part[0];
  float* m0 = x->cm0 + (size_t)t * nbits;
  float* m1 = x->cm1 + (size_t)t * nbits;
  for (int k = 0; k < nbits; k++) m0[k] = m1[k] = INFINITY;
  float best = INFINITY;
  int bstep = INT32_MAX;
  memcpy(cb, s, (size_t)N);
  uint8_t F[128];
  for (int k = 0; k < S; k++) {
    const float A = f_mul(4.0f, Tb[k]);
    int any = 0;
    for (int i = 0; i < N; i++) {
      const uint32_t w = philox_word((uint32_t)(k >> 2), (uint32_t)i, r, inst, x->k0, x->k1, k & 3);
      const float thr = orc_thr(w, A);
      const float su = s[i] > 0 ? u[i] : -u[i];
      F[i] = f_add(su, x->q) < thr;
      any |= F[i];
    }
    for (int j = 0; j < N; j++) {
      if (!F[j]) continue;
      const int up = s[j] > 0;
      E = f_add(E, f_mul(up ? 2.0f : -2.0f, f_add(f_sub(h0[j], hf[j]), u[j])));
      const float cf = up ? -4.0f : 4.0f;
      for (int i = 0; i < N; i++) u[i] = f_add(u[i], f_mul(cf, J[(size_t)j * N + i]));
    }
    for (int j = 0; j < N; j++)
      if (F[j]) s[j] = (int8_t)(-s[j]);
    if (any || k == 0) {
      const float d = f_add(f_mul(x->scale[b], E), x->c0[b]);
      for (int j = 0; j < D; j++) {
        const int s1 = s[j] > 0;
        if (nb == 2) {
          const int b2 = s1 != (s[D + j] > 0);
          if (s1) { if (d < m1[2 * j]) m1[2 * j] = d; } else { if (d < m0[2 * j]) m0[2 * j] = d; }
          if (b2) { if (d < m1[2 * j + 1]) m1[2 * j + 1] = d; } else { if (d < m0[2 * j + 1]) m0[2 * j + 1] = d; }
        } else {
          if (s1) { if (d < m1[j]) m1[j] = d; } else { if (d < m0[j]) m0[j] = d; }
        }
      }
      if (d < best) {
        best = d;
        bstep = k;
        memcpy(cb, s, (size_t)N);
      }
    }
  }
  x->cbest[t] = best;
  x->cstep[t] = bstep;
  memcpy(x->cbs + (size_t)t * N, cb, (size_t)N);
}

/* J (B, N, N), hf, h0 (B, N), scale, c0 (B), T (B, S), s0 (B, N) or NULL; N = 2 D (M = 16) or D (M = 4).  Outputs
 * m0, m1 (B, D nb), best_d (B), best_l (B, D). */
int orc_soft_trajectory(const float* J, const float* hf, const float* h0, const float* scale, const float* c0,
                        const float* T, const int8_t* s0, float q, int S, int R, int D, int M, int B,
                        const uint32_t* inst, uint32_t k0, uint32_t k1, float* m0, float* m1, float* best_d,
                        int8_t* best_l, int nthreads) {
  if (!(M == 4 || M == 16)) return 1;
  const int N = M == 16 ? 2 * D : D, nb = M == 16 ? 2 : 1, nbits = D * nb;
  if (N < 1 || N > 128 || R < 1 || S < 1 || B < 0) return 1;
  const long BR = (long)B * R;
  float* cm0 = (float*)malloc(sizeof(float) * (size_t)BR * nbits);
  float* cm1 = (float*)malloc(sizeof(float) * (size_t)BR * nbits);
  float* cbest = (float*)malloc(sizeof(float) * (size_t)BR);
  int* cstep = (int*)malloc(sizeof(int) * (size_t)BR);
  int8_t* cbs = (int8_t*)malloc((size_t)BR * N);
  soft_ctx x = {J, hf, h0, scale, c0, T, s0, q, S, R, N, D, M, B, inst, k0, k1, cm0, cm1, cbest, cstep, cbs};
  orc_run(soft_job, &x, BR, nthreads);
  for (int b = 0; b < B; b++) {
    int br = 0;
    for (int k = 0; k < nbits; k++) {
      float v0 = INFINITY, v1 = INFINITY;
      for (int r = 0; r < R; r++) {
        const long t = (long)b * R + r;
        if (cm0[t * nbits + k] < v0) v0 = cm0[t * nbits + k];
        if (cm1[t * nbits + k] < v1) v1 = cm1[t * nbits + k];
      }
      m0[(size_t)b * nbits + k] = v0;
      m1[(size_t)b * nbits + k] = v1;
    }
    for (int r = 1; r < R; r++) {
      const long t = (long)b * R + r, tb = (long)b * R + br;
      if (cbest[t] < cbest[tb] || (cbest[t] == cbest[tb] && cstep[t] < cstep[tb])) br = r;
    }
    const long tb = (long)b * R + br;
    best_d[b] = cbest[tb];
    for (int j = 0; j < D; j++) {
      const int s1 = cbs[tb * N + j];
      best_l[(size_t)b * D + j] = (int8_t)(nb == 2 ? 2 * s1 + cbs[tb * N + D + j] : s1);
    }
  }
  free(cm0);
  free(cm1);
  free(cbest);
  free(cstep);
  free(cbs);
  return 0;
}
