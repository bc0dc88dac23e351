/*
 * arpeggio_b200 -- C ABI of the B200 (sm_100a) delta-encoded Ising MIMO detector path.
 *
 * Plain pointers and sizes; every array argument is DEVICE memory unless stated otherwise.  No entry
 * point of the detection path allocates memory; two training routines take stream-ordered workspaces
 * (cudaMallocAsync, freed on the same stream): arp_gemm_bf16 with split K and arp_colsum_bf16.  Every entry
 * point is stream-ordered on `stream` (a cudaStream_t, or NULL for the legacy default stream) and returns
 * without synchronising, except arp_serve_run, a host loop that returns when its requests are done.  Return value: ARP_OK or an
 * ARP_ERR_* code for errors found on the host (shapes, arguments, launch).  Errors that only the
 * device can see (coefficients beyond the exact 32-bit field range) are written to `status`
 * (one int32 in device memory, may be NULL; set to the first error code, never cleared here).
 *
 * Citations name the reference interface each entry point replaces (skethz/Arpeggio, path:line).
 */
#ifndef ARPEGGIO_B200_H
#define ARPEGGIO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum arp_status_code {
  ARP_OK = 0,
  ARP_ERR_SHAPE = 1,     /* unsupported D, P, N, R, B or L */
  ARP_ERR_RANGE = 2,     /* coefficients or schedule beyond the exact 32-bit field range */
  ARP_ERR_ARG = 3,       /* null pointer or bad enum value */
  ARP_ERR_LAUNCH = 4,    /* CUDA launch or configuration error */
  ARP_ERR_TIMEOUT = 5,   /* a bounded device-side wait gave up */
  ARP_ERR_WORKSPACE = 6  /* caller's workspace smaller than arp_*_workspace_bytes() */
};

/* Library version string and a message for a status code (host only). */
const char* arp_version(void);
const char* arp_status_string(int code);

/* The device address of page-locked host memory (cudaHostAlloc'd, mapped): kernels may write results straight
 * into it, so a captured one-frame detection needs no copy back.  ARP_ERR_ARG if host is not mapped memory.
 * Host only; no counterpart in the reference. */
int arp_host_device_pointer(const void* host, void** dev);

/* Philox4x32-10 known-answer check on the device: in (n x 6 words: counter c0..c3, key k0, k1),
 * out (n x 4 words).  Replaces chord_kernel.cu:26-32 `philox_kat` (launched by
 * arpeggio/mimo/chordfx.py:180-187). */
int arp_philox_kat(const uint32_t* in, uint32_t* out, int n, void* stream);

/* Integer-issue calibration: blocks x threads threads each run `iters` chained Philox4x32-10 blocks (the
 * anneal's dominant integer work).  `out` (one word) is written only by a one-in-2^32 coincidence.  No
 * reference counterpart: it measures the peak the benchmark's integer roofline divides by. */
int arp_philox_rate(uint32_t* out, int blocks, int threads, int iters, void* stream);

/* Fixed-point first-accept anneal (Arpeggio) on compressed dDI problems.
 * Replaces arpeggio/sim/arpeggio_fx.cu:35-37 `arpeggio_fx` as launched by arpeggio/sim/arpeggiofx.py:40-42,
 * same argument meaning: Gt (B, D, D) int32 transposed (Gt[b][j][i] = G[b][i][j]), h (B, D), T (L) one
 * temperature per pass (pass k tests copy k % P), q, P in {2, 4, 6}, R anneals per problem, D <= 128,
 * inst (B) instance numbers, Philox key (k0 = low, k1 = high word), start 0 = 'rand' / 1 = 'bal'.
 * Outputs: out_s (B, R, P*D) int8 best spins copy-major, out_de (B, R) best energy change,
 * out_st (B, R, 2) [flips, tests].  Bit-exact with the reference kernel and arpeggio_ref59.anneal. */
int arp_anneal_first_accept(const int32_t* Gt, const int32_t* h, const int32_t* T, int L, int q, int P, int R,
                            int D, int B, const uint32_t* inst, uint32_t k0, uint32_t k1, int start,
                            int8_t* out_s, int64_t* out_de, int64_t* out_st, int32_t* status, void* stream);

/* Fixed-point Chord round (snapshot test of the active copy, then in-order commits) on compressed dDI
 * problems, with the Onsager term c (L, may be NULL).  Same arguments and outputs as
 * arp_anneal_first_accept (tests = one per pass).  Replaces the compressed Chord of
 * arpeggio/sim/x3model/chord_ref.py:72-123 (rng='philox') and mode 'par' of
 * arpeggio/rtl/cycle_checks/rtl_a59/src/arpeggio_ref59.py:72-82; equals chordfx.chord_fx on the
 * expanded problem (its 2 E0 minus the start state's). */
int arp_anneal_chord_dd(const int32_t* Gt, const int32_t* h, const int32_t* T, const int32_t* c, int L, int q,
                        int P, int R, int D, int B, const uint32_t* inst, uint32_t k0, uint32_t k1, int start,
                        int8_t* out_s, int64_t* out_de, int64_t* out_st, int32_t* status, void* stream);

/* arp_anneal_chord_dd that also writes, per anneal, the rounds with at least one flip, out_n1 (B, R) int64: n1 of
 * the reference's oracle (arpeggio/rtl/cycle_checks/rtl_a59/src/arpeggio_ref59.py:74), the term that makes the
 * Chord engine's latency 3 L + F + n1 cycles per anneal (data/results/a59/A59.json, chord_lat_over_3LFn1 = 1). */
int arp_anneal_chord_dd_n1(const int32_t* Gt, const int32_t* h, const int32_t* T, const int32_t* c, int L, int q,
                           int P, int R, int D, int B, const uint32_t* inst, uint32_t k0, uint32_t k1, int start,
                           int8_t* out_s, int64_t* out_de, int64_t* out_st, int64_t* out_n1, int32_t* status,
                           void* stream);

/* The same Chord round with the random numbers of the reference's C++ engine model when it runs without Philox
 * (arpeggio/sim/x3model/engine_model.cpp, engine_solve_batch :336-379 with philox = 0, as its production
 * scripts arpeggio/sim/x3_prod.py:105-106 and run_a516.py:135-136 call it): per anneal a seed chain over
 * (k0 ^ inst, k1, r), one xorshift32 generator per coordinate whose bits are the start spins, advanced once per
 * step, 16-bit draws.  T and c (L) one entry per step, c may be NULL; key (k0 low, k1 high) = the engine's
 * 64-bit seed.  Outputs as arp_anneal_chord_dd (tests = one per step); best spins and best energy changes equal
 * the engine's, which starts its best at 2^35 - 1 (an anneal none of whose steps ends below that returns its
 * start spins here, where the engine keeps whatever its best-spin register last held).  No start argument: the
 * engine's start comes from its generators.  The engine runs only D that are a multiple of its lane-group width
 * (engine_model.cpp:145-183; width max(1, D / 32) as this project binds it: any D < 64, even D < 96, multiples of
 * 3 below 128, and 128); equality with the engine holds there.  Other D (up to 128) extend the same rule to
 * coordinates the engine cannot group and are pinned by the oracle's restatement only. */
int arp_anneal_chord_engine(const int32_t* Gt, const int32_t* h, const int32_t* T, const int32_t* c, int L, int q,
                            int P, int R, int D, int B, const uint32_t* inst, uint32_t k0, uint32_t k1,
                            int8_t* out_s, int64_t* out_de, int64_t* out_st, int32_t* status, void* stream);

/* FP32-field anneal on compressed dDI problems: policy 0 = first accept, 1 = Chord round.  Gt, h, T, c
 * (c may be NULL), q in float; out_de (B, R) float.  The float rule is the integer rule with the
 * decision z < thr, z = (s w_j + 2 G_jj) + q, thr = ((x >> 8) 2^-24 - 1/2) 4 T, one IEEE rounding per
 * operation.  The reference has no FP32 Philox kernel; the float semantics follow
 * arpeggio/sim/arpx55.py:28-99 (arpeggio_seq, rule (2)). */
int arp_anneal_dd_f32(int policy, const float* Gt, const float* h, const float* T, const float* c, int L, float q,
                      int P, int R, int D, int B, const uint32_t* inst, uint32_t k0, uint32_t k1, int start,
                      int8_t* out_s, float* out_de, int64_t* out_st, int32_t* status, void* stream);

/* Fixed-point Chord on a full int16 coupling J (B, N, N), h and h0 (B, N), Tq and Cq (S), with P phases.
 * Replaces arpeggio/mimo/chord_kernel.cu:177-184 `chord_m{1,2,3,4,6,8}` as launched by
 * arpeggio/mimo/chordfx.py:189-208 (Kernel.chord): N % 32 == 0, (N / P) % 32 == 0, N <= 256;
 * mode 0 ('chains'): out_e (B, R), out_s (B, R, N); mode 1 ('best'): out_e (B), out_s (B, N).
 * out_e is 2 E0 (int64).  stats (4 counters: flips, energy evaluations, Philox blocks, steps x anneals)
 * may be NULL; their totals equal the reference kernel's.  warps = anneals per block in flight: 1..16 as given
 * (8 at most for N = 256 with P = 1), <= 0 picks the width with the most resident warps per SM (16 at N = 256,
 * where the staged J leaves one block per SM).  The outputs do not depend on it.  J 16-byte aligned is staged
 * by bulk copies, otherwise by plain loads. */
int arp_anneal_chord(const int16_t* J, const int32_t* h, const int32_t* h0, const int32_t* Tq, const int32_t* Cq,
                     int q, int S, int P, int R, int N, int B, uint32_t k0, uint32_t k1, uint32_t inst0, int mode,
                     int warps, int64_t* out_e, int8_t* out_s, unsigned long long* stats, int32_t* status,
                     void* stream);

/* Gram / field formation with the MMSE guess, per channel use (one block each).  H (B, NR2, D) float32
 * real-lifted channels [[Re, -Im], [Im, Re]] scaled by the constellation factor, y (B, NR2), sigma2 (B)
 * the MMSE regulariser (N0/2)/E[l^2], M in {4, 16, 64} (64-QAM: levels -7..7, Gray-coded level index; no
 * reference counterpart, the reference's table stops at 16-QAM).  Outputs: G (B, D, D) = H^T H / scale (symmetric, so
 * also its own transpose Gt), h (B, D) = 2 H^T (y - H x_q) / scale, x_q (B, D) int8 hard MMSE guess,
 * scale (B).  quantize != 0: G and h are int32 round(x * 4096) (the integer problem); else float32.
 * Replaces the host chain mimo.mmse / mimo._mu / quantize_levels (arpeggio/mimo/mimo.py:86-109, 176-182),
 * mimo.ising_delta_at (mimo.py:506-523), chordfx.to_fixed (chordfx.py:60-76) and chord_ref.compress
 * (arpeggio/sim/x3model/chord_ref.py:47-59) as run_a513.detect calls them (run_a513.py:107-111). */
int arp_map_dd(const float* H, const float* y, const float* sigma2, int B, int NR2, int D, int M, int quantize,
               void* G, void* h, int8_t* xq, float* scale, int32_t* status, void* stream);

/* Readout: candidate levels clip(x_q + sum_p s_p) of each anneal's best spins (B, R, P*D), their distance
 * ||y - H x||^2, the first minimum over the R candidates and then the guess, Gray bits (MSB first per
 * dimension; M in {4, 16, 64}).  Outputs levels (B, D) int8, bits (B, D * log2(M)/2) int8, dist (B) float32, pick (B) int32
 * (index of the winner, R = the guess; may be NULL).  Replaces mimo.spins_to_levels_delta, mimo.dist,
 * mimo.select and mimo.levels_to_bits (arpeggio/mimo/mimo.py:185-190, 416-425, 45-51). */
int arp_readout_dd(const float* H, const float* y, const int8_t* xq, const int8_t* spins, int B, int NR2, int D,
                   int P, int R, int M, int8_t* levels, int8_t* bits, float* dist, int32_t* pick, void* stream);

/* The RI map (mimo.ising, arpeggio/mimo/mimo.py:132-149): each PAM coordinate as 2 s1 + s2 (T = [2I, I];
 * QPSK: s), N = 2D (16-QAM) or D spins: J (B, N, N) = -offdiag(T^T H^T H T) / scale, h0 (B, N) = 2 (HT)^T y / scale,
 * h = h0 + 2 r sP (B, N) with sP (B, N) the spins of the hard MMSE z (the MMSE initialisation), xq (B, D) the
 * bias-corrected hard MMSE decision (mimo.mmse_hard, mimo.py:91-95) for the selection, scale (B).  D <= 64. */
int arp_map_ri(const float* H, const float* y, const float* sigma2, int B, int NR2, int D, int M, float r, float* J,
               float* h0, float* h, int8_t* sP, int8_t* xq, float* scale, void* stream);

/* FP32-field anneal on a full symmetric J (B, N, N), N <= 128 spins in P banks of N/P lanes (a multiple of 32); pass
 * k tests bank k % P.  policy 0 = first accept, 1 = Chord round (Onsager c may be NULL); s0 (B, N) start spins
 * (the MMSE initialisation) or NULL for 'rand'.  Outputs spins (B, R, N), best energy change (B, R) (E0 units,
 * flipping s_g moves E0 by 2 s_g u_g), (flips, tests).  The float rule of arpeggio/sim/arpx55.py:28-99 (rule (2))
 * with Philox draws (counters as arp_anneal_first_accept's, spin index i = bank * N/P + lane). */
int arp_anneal_full_f32(int policy, const float* J, const float* h, const int8_t* s0, const float* T, const float* c,
                        int L, float q, int P, int R, int N, int B, const uint32_t* inst, uint32_t k0, uint32_t k1,
                        int8_t* out_s, float* out_de, int64_t* out_st, void* stream);

/* Readout of RI spins (B, R, 2D) or (B, R, D): candidate levels 2 s1 + s2 (mimo.spins_to_levels, mimo.py:39-42),
 * then the selection with the guess xq (mmse_hard) as arp_readout_dd (fxdetect.py:41-42). */
int arp_readout_ri(const float* H, const float* y, const int8_t* xq, const int8_t* spins, int B, int NR2, int D, int R,
                   int M, int8_t* levels, int8_t* bits, float* dist, int32_t* pick, void* stream);

/* Soft output: arp_readout_dd plus max-log LLRs (B, D * log2(M)/2) float32, positive = bit 1, over the candidate
 * list (the R candidates and the guess) and the single-bit-flip neighbours of the decision, divided by N0 (B)
 * and clipped to +-clip.  Replaces mimo.list_llr (arpeggio/mimo/mimo.py:434-462) as the reference's dDI soft
 * detector calls it (arpeggio/mimo/softlib.py:37-46, method 'aned'). */
int arp_readout_llr_dd(const float* H, const float* y, const int8_t* xq, const int8_t* spins, int B, int NR2, int D,
                       int P, int R, int M, const float* N0, float clip, int8_t* levels, int8_t* bits, float* dist,
                       int32_t* pick, float* llr, void* stream);

/* The detector call in one entry point: map (arp_map_dd) -> anneal (policy 0 = first accept, 1 = Chord round;
 * precision 0 = int32 fixed point with T, c int32 and q rounded to an integer, 1 = FP32 fields with T, c, q
 * float) -> readout (arp_readout_dd), stream-ordered, with the intermediates in the caller's workspace of at
 * least arp_detect_dd_workspace() bytes.  Instance numbers inst0 + b, Philox key (k0, k1), start 0 = 'rand',
 * 1 = 'bal', P = 2K copies, R anneals.  Outputs as arp_readout_dd.  This is the one-stage dDI detection of
 * arpeggio/mimo/fxdetect.py:24-43 (candidates of every anneal plus the MMSE guess, lowest ||y - Hx||^2) with
 * the sub-problem solve of arpeggio/sim/local_code_a513/run_a513.py:107-128. */
int arp_detect_dd(const float* H, const float* y, const float* sigma2, int B, int NR2, int D, int M, int policy,
                  int precision, int P, int R, const void* T, const void* c, int L, double q, uint32_t inst0,
                  uint32_t k0, uint32_t k1, int start, void* workspace, size_t workspace_bytes, int8_t* bits,
                  int8_t* levels, float* dist, int32_t* pick, int32_t* status, void* stream);

/* Workspace bytes arp_detect_dd needs; if offsets is not NULL it receives the 7 byte offsets of G, h, x_q,
 * scale, spins, best energy changes and (flips, tests) inside it (for inspection after a call). */
size_t arp_detect_dd_workspace(int B, int D, int P, int R, int precision, size_t* offsets);

/* Multi-stage delta-Ising detection (MDI-MIMO, arpeggio/mimo/mimo.py:553-602 and run_a513.mdi_logged,
 * arpeggio/sim/local_code_a513/run_a513.py:42-80): the host walks stages, guesses, K and groups exactly as the
 * reference does and calls these per group; the anneal is arp_anneal_first_accept / arp_anneal_chord_dd with
 * inst = the group's use indices.
 * arp_mdi_guesses: per use the hard MMSE guess (mimo.py:98-109, 176-182) and the ordered MMSE-SIC guess
 *   (mimo.py:466-503, per='real'), int8 levels (B, D) each.
 * arp_mdi_radius: per use and guess in cur (B, G, D): the search radius R (B, G) of mimo.mdi_radius
 *   (mimo.py:526-543, heuristic 'mean', capped at Rmax) and ||y - H x_g||^2 (B, G).
 * arp_mdi_map: the compressed dDI problem around guess gi of cur for the uses idx (n), as arp_map_dd
 *   (mimo.ising_delta_at + to_fixed + compress, mimo.py:506-523).
 * arp_mdi_update: the group's candidates (spins (n, R, P*D)) around guess gi; for each use the first closest
 *   candidate replaces next[idx, gi] and best_dist[idx, gi] if strictly closer (mimo.py:588-593).
 * arp_mdi_select: the first guess with the lowest distance (mimo.py:600-602), levels (B, D) and Gray bits. */
int arp_mdi_guesses(const float* H, const float* y, const float* sigma2, int B, int NR2, int D, int M, int8_t* xmmse,
                    int8_t* xsic, void* stream);
int arp_mdi_radius(const float* H, const float* y, const int8_t* cur, int B, int NR2, int D, int G, int M, int Rmax,
                   int32_t* R, float* dist, void* stream);
int arp_mdi_map(const float* H, const float* y, const int32_t* idx, int n, int NR2, int D, int M, const int8_t* cur,
                int G, int gi, int quantize, void* Gout, void* hout, int8_t* xq, float* scale, int32_t* status,
                void* stream);
int arp_mdi_update(const float* H, const float* y, const int32_t* idx, int n, int NR2, int D, int P, int R, int M,
                   const int8_t* cur, int G, int gi, const int8_t* spins, int8_t* next, float* best_dist, void* stream);
int arp_mdi_select(const int8_t* cur, const float* dist, int B, int D, int G, int M, int8_t* levels, int8_t* bits,
                   void* stream);

/* Trajectory soft output on the RI map (N = 2 D spins [s_MSB; s_LSB] for 16-QAM, N = D for QPSK; N <= 128):
 * Chord's synchronous rule as a sampler of the detection posterior, mimo.chord_soft (arpeggio/mimo/mimo.py:332-394),
 * with Philox draws of this library ((k >> 2, i, r, inst) word k & 3; start word 0 of (2^32 - 1, i, r, inst), or the
 * spins s0 (B, N) if non-NULL).  J (B, N, N) scaled with a zero diagonal, hf (B, N) the exploration field (h0, or
 * the RI field h), h0 (B, N), scale and c0 (B) with ||y - H x||^2 = scale E0(s) + c0, T (B, S) per-step temperatures,
 * q, R chains of S steps.  Outputs: per bit (B, D nb, dimension-major, MSB first) the smallest distance of a
 * visited state with the bit 0 (m0) and 1 (m1, +inf if none), the best distance (B) and its levels (B, D).  The LLRs
 * follow from mimo.trajectory_llr (arpeggio_b200.soft.trajectory_llr). */
int arp_soft_trajectory(const float* J, const float* hf, const float* h0, const float* scale, const float* c0,
                        const float* T, const int8_t* s0, float q, int S, int R, int D, int M, int B,
                        const uint32_t* inst, uint32_t k0, uint32_t k1, float* m0, float* m1, float* best_d,
                        int8_t* best_l, void* stream);

/* Autotuner hook (no reference counterpart): warps per block (1, 2, 4 or 8; 0 restores the occupancy heuristic)
 * of the compressed-problem anneal kernels for problems of D coordinates (by 32-wide slot count), P copies,
 * policy (0 first accept, 1 Chord round, 2 the warm-started first accept of arp_anneal_first_accept_warm*, P = 2
 * and int32 only) and precision (0 int32, 1 FP32 fields).  Process-wide; results do not depend on it (anneals are
 * independent of their block). */
int arp_anneal_tune(int D, int P, int policy, int precision, int warps);

/* One size class of a mixed batch for arp_anneal_first_accept_mixed: the arguments of arp_anneal_first_accept for
 * that class's B problems (integer fields, first accept, P = 2). */
typedef struct arp_mixed_class {
  const int32_t* Gt;
  const int32_t* h;
  const int32_t* T;
  int L, q, R, D, B;
  const uint32_t* inst;
  int start;
  int8_t* out_s;
  int64_t* out_de;
  int64_t* out_st;
} arp_mixed_class;

/* The first-accept anneals of every size class of a mixed batch (ncls <= 64 classes from host memory, one Philox
 * key k0/k1 for all) in persistent grids: one launch per 32-wide slot count (at most four, in this stream order),
 * each sized to the SMs' resident blocks, whose blocks take problems from a work counter in device memory
 * (counters: 4 ints, one per launch, zeroed here with cudaMemsetAsync before each launch) until the batch is done,
 * costly classes (L R D) first.  Every output equals that of arp_anneal_first_accept on the class alone; warps
 * (0, 1, 2, 4, 8) as arp_anneal_tune (0: the tuned or occupancy width).  Graph-capturable: the class table
 * travels in the kernel parameters.  Calls that share counters must not overlap on the GPU.  The per-class
 * launches of the reference's own scripts have no persistent counterpart (arpeggio/sim/arpeggiofx.py:22-44 is
 * one launch per call). */
int arp_anneal_first_accept_mixed(const arp_mixed_class* cls, int ncls, int P, uint32_t k0, uint32_t k1, int warps,
                                  int* counters, int32_t* status, void* stream);

/* ---- Learned warm start for first-accept annealing.  No counterpart in the reference, which has no learned
 * component: a per-coordinate MLP (16 features -> 256 -> 256 -> P+1 logits over the coordinate's spin sum
 * m_j = 2c - P, BF16 weights and activations, FP32 accumulate) emits the start state and the flip-test order.
 * bf16 arrays are passed as void* (2-byte IEEE bfloat16). */

/* arp_map_dd plus zs (B, D) float: the bias-corrected MMSE soft estimate z / mu behind x_q (a feature of the
 * warm start).  Same map as arp_map_dd (mimo.mmse, mimo._mu and mimo.ising_delta_at, arpeggio/mimo/mimo.py:98-109,
 * 176-182, 506-523). */
int arp_map_dd_soft(const float* H, const float* y, const float* sigma2, int B, int NR2, int D, int M, int quantize,
                    void* G, void* h, int8_t* xq, float* scale, float* zs, int32_t* status, void* stream);

/* C (M, N) = A B^T on the tensor cores (tcgen05.mma kind::f16, bf16 operands, fp32 accumulate in TMEM).
 * A is (M, K) row-major with row stride lda (a_mn_major = 0) or (K, M) row-major (a_mn_major = 1); B is (N, K)
 * (b_mn_major = 0) or (K, N) (b_mn_major = 1).  N and K multiples of 16, leading dimensions multiples of 8
 * elements, pointers 16-byte aligned.  epilogue: 0 C = acc (float), 1 C += acc (float; K is split over CTAs
 * whose partial products go to a stream-ordered workspace and are added in split order, so the result is the
 * same on every run), 2 C = bf16(max(acc + bias, 0)), 3 C = acc + bias (float), 4 C = bf16(acc if aux > 0 else
 * 0) with aux (M, N) bf16 of row stride ld_aux (the ReLU backward).  Products with M >= 128, N >= 64 and K >= 64
 * run on a persistent kernel fed by TMA tensor loads with warp-specialised producer, MMA and epilogue roles; the
 * rest on a cp.async-fed kernel.  Either way each shape gives the same result on every run. */
int arp_gemm_bf16(const void* A, int a_mn_major, int lda, const void* B, int b_mn_major, int ldb, int M, int N, int K,
                  int epilogue, const float* bias, const void* aux, int ld_aux, void* C, int ldc, int32_t* status,
                  void* stream);

/* Per-coordinate features X (B*D, 16) bf16 of mapped dDI problems G (B, D, D), h (B, D) (int32 when quantized,
 * else float), guesses xq (B, D), MMSE soft estimates zs (B, D) (may be NULL), snr_db (B) (may be NULL).  With
 * levels (B, D) given, labels (B*D) int8 receive the class (levels - xq)/2 + P/2 of each coordinate. */
int arp_warm_features(const void* G, const void* h, const int8_t* xq, const float* zs, const float* snr_db, int B,
                      int D, int M, int P, int quantized, void* X, const int8_t* levels, int8_t* labels, void* stream);

/* Softmax cross-entropy over the first `classes` logits of each row (row stride ldl), labels < 0 ignored:
 * dlogits (rows, ldd) bf16 = softmax - onehot (zero beyond `classes`); loss_sum and correct (may be NULL) are
 * incremented by the summed loss and the number of argmax hits. */
int arp_warm_loss(const float* logits, int ldl, const int8_t* labels, int rows, int classes, void* dlogits, int ldd,
                  float* loss_sum, int32_t* correct, void* stream);

/* out (cols) += column sums of X (rows, cols) bf16 with row stride ld (bias gradients), in a fixed order. */
int arp_colsum_bf16(const void* X, int rows, int cols, int ld, float* out, void* stream);

/* One Adam step on n FP32 master weights w with gradient grad * grad_scale, moments m and v, bias-corrected
 * for step `step` (1-based); w_bf16 (may be NULL) receives the rounded weights. */
int arp_adam(float* w, void* w_bf16, const float* grad, float* m, float* v, int n, float lr, float beta1, float beta2,
             float eps, int step, float grad_scale, void* stream);

/* W2 (256, 256) bf16 row-major -> W2p, the same 256 x 256 values in the order arp_mlp_forward keeps them in
 * shared memory (8 chunks of 256 rows x 32 k; within a chunk k-group of 8, then row, then element).  Once per
 * weight update. */
int arp_mlp_pack_w2(const void* W2, void* W2p, void* stream);

/* The network's forward pass in one persistent launch (no reference counterpart): logits (rows, 16) float =
 * relu(relu(X W1^T + b1) W2^T + b2) W3t + b3 with X (rows, 16), W1 (256, 16), W2 (256, 256) given packed as W2p
 * (arp_mlp_pack_w2), W3t (256, 16) bf16 and fp32 biases; the weights stay in shared memory for the whole launch
 * and per 128-row tile the hidden activations stay in TMEM and shared memory (bf16, the same roundings and
 * summation order as the three arp_gemm_bf16 calls of the training path). */
int arp_mlp_forward(const void* X, int rows, const void* W1, const float* b1, const void* W2p, const float* b2,
                    const void* W3t, const float* b3, float* logits, int32_t* status, void* stream);

/* Warm start from the logits (B*D, ldl): m0 (B, D) the start spin sum of each coordinate (argmax class, clamped
 * to the constellation), perm (B, D) the flip-test order (position j' tests coordinate perm[j'], by descending
 * 1 - p(m = 0)), e0 (B) the start's energy 2 (m^T G m - h^T m) relative to the guess, in the units of the
 * anneal's out_de (int64 when quantized, else float; may be NULL),
 * kept (B) 1 where the start is no worse than the guess (e0 <= 0); elsewhere m0 = 0 and perm is the index
 * order, i.e. the plain MMSE start. */
int arp_warm_start(const float* logits, int ldl, const void* G, const void* h, const int8_t* xq, int B, int D, int P,
                   int M, int quantized, int8_t* m0, uint8_t* perm, void* e0, int32_t* kept, void* stream);

/* arp_anneal_first_accept (P = 2) from a given start: coordinate perm[j'] is tested at scan position j' (its
 * Philox counters are those of position j'), and starts with spin sum m0 (m = 0: the 'bal' pattern of
 * position j''s draw; m = +-2: both copies +-1).  Outputs in coordinate order; out_de is relative to the start
 * (add e0 for the change from the guess).  perm entries outside 0..D-1 give ARP_ERR_RANGE in status. */
int arp_anneal_first_accept_warm(const int32_t* Gt, const int32_t* h, const int32_t* T, int L, int q, int P, int R,
                                 int D, int B, const uint32_t* inst, uint32_t k0, uint32_t k1, const int8_t* m0,
                                 const uint8_t* perm, int8_t* out_s, int64_t* out_de, int64_t* out_st, int32_t* status,
                                 void* stream);

/* arp_anneal_first_accept_warm where only anneals r < warm_r start from m0 and the others from the MMSE start
 * (m = 0, the 'bal' pattern), all in the given flip-test order: a mix of start diversity.  No counterpart in
 * the reference. */
int arp_anneal_first_accept_warm_mix(const int32_t* Gt, const int32_t* h, const int32_t* T, int L, int q, int P,
                                     int R, int D, int B, const uint32_t* inst, uint32_t k0, uint32_t k1,
                                     const int8_t* m0, const uint8_t* perm, int warm_r, int8_t* out_s,
                                     int64_t* out_de, int64_t* out_st, int32_t* status, void* stream);

/* arp_warm_start (P = 2) that also writes, per coordinate, the thresholds cdf (B, D, 2) uint32 of a draw from
 * softmax(tau z) over the classes whose spin sum keeps the level inside the constellation: with u a uniform
 * 32-bit word, class 0 (m = -2) if u < cdf[0], class 2 (m = +2) if u > cdf[1], else class 1 (m = 0).  Problems
 * that fall back to the plain start (kept = 0) get (0, 0xFFFFFFFF): always m = 0.  tau > 0 sharpens (> 1) or
 * flattens (< 1) the network's distribution.  With ra non-NULL it also writes per-problem anneal counts ra (B):
 * r_easy (1..R) where the start is kept and its confidence sum_j log max_c softmax(z_j)_c exceeds conf_min,
 * else R.  No counterpart in the reference. */
int arp_warm_start_sampled(const float* logits, int ldl, const void* G, const void* h, const int8_t* xq, int B, int D,
                           int P, int M, int quantized, int8_t* m0, uint8_t* perm, void* e0, int32_t* kept,
                           float tau, uint32_t* cdf, float conf_min, int r_easy, int R, int32_t* ra, void* stream);

/* arp_anneal_first_accept_warm_mix with sampled starts: anneal 0 starts from m0, each anneal 0 < r < warm_r
 * draws every coordinate's start spin sum from cdf (arp_warm_start_sampled) with word 1 of the Philox block
 * (0xFFFFFFFF, j', r, inst) of the coordinate's scan position j' (word 0 still picks the 'bal' pattern of m = 0),
 * anneals r >= warm_r start from the MMSE start; all in the given flip-test order.  With ra (B) non-NULL,
 * problem b runs only anneals r < ra[b] (clamped to 1..R; each exactly as in the full run, its counters being
 * its own) and the skipped anneals report all-zero spin sums (a candidate equal to the guess), out_de
 * INT64_MAX and zero statistics.  P = 2 only.  No counterpart in the reference. */
int arp_anneal_first_accept_warm_sampled(const int32_t* Gt, const int32_t* h, const int32_t* T, int L, int q, int P,
                                         int R, int D, int B, const uint32_t* inst, uint32_t k0, uint32_t k1,
                                         const int8_t* m0, const uint32_t* cdf, const uint8_t* perm, int warm_r,
                                         const int32_t* ra, int8_t* out_s, int64_t* out_de, int64_t* out_st,
                                         int32_t* status, void* stream);

/* Native serving loop (no counterpart in the reference; arpeggio_b200.serve.Server drives it).  A request
 * stream per size class: its requests' inputs in host memory (pinned, for the staging copies to overlap), their
 * arrival times in seconds on the loop's clock (ascending), and outputs.  h_elems / y_elems / bits_per are the
 * floats of one request's H and y and the bytes of its hard bits. */
typedef struct {
  const float* H;
  const float* y;
  const float* s2;          /* noise variance per real dimension */
  const float* snr;         /* SNR in dB (the warm start's feature) */
  const int32_t* rid;       /* instance numbers (a request's result depends on its id alone) */
  const double* t_arrival;  /* n, seconds, ascending */
  int n, h_elems, y_elems, bits_per;
  int8_t* bits;             /* n x bits_per */
  float* dist;              /* n */
  double* done;             /* n: completion time on the loop's clock */
} arp_serve_stream;

/* A lane: one detector of its class, the stream its work runs on, and captured CUDA graphs for ngraphs <= 32 batch
 * sizes (sizes ascending; graphs[i] detects the first sizes[i] slots of the lane's device buffers): inputs H, y,
 * noise variance, SNR and instance numbers, outputs bits and distances. */
typedef struct {
  int cls;
  void* stream;
  int ngraphs;
  int sizes[32];
  void* graphs[32]; /* cudaGraphExec_t */
  float *Hd, *yd, *s2d, *snrd;
  int32_t* instd;
  const int8_t* bitsd;
  const float* distd;
} arp_serve_lane;

/* Runs the continuous-batching loop on the calling thread until every request of every stream is done, polling
 * the clock (steady, seconds since the call): a lane whose last batch has completed records its requests'
 * completion time and becomes free; a free lane takes every request of its class that has arrived and is not
 * taken yet, up to its largest graph, copies their inputs from the stream's host arrays to its device buffers,
 * replays the graph of the smallest size that holds them (the padding slots are detected and discarded), copies bits and
 * distances straight into the stream's output rows and records an event -- all on the lane's stream, so the
 * batches of different lanes overlap on the GPU.  batches (nstreams, may be NULL) counts the batches per stream.
 * ARP_ERR_TIMEOUT if the requests are not all done within timeout_s (the batches in flight are waited for
 * first); ARP_ERR_LAUNCH on a CUDA error.  The host side of arpeggio_b200.serve's Python loop without the
 * interpreter in the polling path. */
int arp_serve_run(const arp_serve_stream* streams, int nstreams, const arp_serve_lane* lanes, int nlanes,
                  double timeout_s, int64_t* batches);

/* arp_detect_dd without a workspace argument, for callers that cannot allocate device memory: a receive
 * chain with a hard per-frame latency budget cannot call cudaMalloc on the frame path (it synchronises the
 * device and takes unbounded time), and a plugin inside a host program that owns all device memory may not
 * allocate at all.  Same arguments and outputs as arp_detect_dd minus (workspace, workspace_bytes); the
 * intermediates live in one 32 MiB array compiled into the library, which every GPU that loads the library
 * holds until the process exits.  A batch whose arp_detect_dd_workspace() exceeds 32 MiB is refused with
 * ARP_ERR_WORKSPACE before any launch.  All calls on a device share the array (it keeps the last call's
 * contents, and nothing in it needs to start at zero); calls whose work overlaps on the GPU race on it.  The
 * first call on each device looks up the array's address and should come before any stream capture.  The
 * address is kept for the life of the process: after a cudaDeviceReset (or any reset of the device's primary
 * context) it no longer names the array, so do not use this entry point on a device across such a reset.
 * No counterpart in the reference: it exists only for callers that cannot allocate. */
int arp_detect_dd_static(const float* H, const float* y, const float* sigma2, int B, int NR2, int D, int M,
                         int policy, int precision, int P, int R, const void* T, const void* c, int L, double q,
                         uint32_t inst0, uint32_t k0, uint32_t k1, int start, int8_t* bits, int8_t* levels,
                         float* dist, int32_t* pick, int32_t* status, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ARPEGGIO_B200_H */
