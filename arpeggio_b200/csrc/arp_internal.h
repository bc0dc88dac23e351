// Internal declarations shared by the kernel files (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace arp {

struct DDParams {
  const void* Gt;  // (B, D, D) int32 or float, Gt[b][j][i] = G[b][i][j]
  const void* h;   // (B, D)
  const void* T;   // (L)
  const void* c;   // (L) Onsager terms or null
  int L;
  int32_t qi;
  float qf;
  int R, D, B;
  const uint32_t* inst;  // (B) instance numbers, or null: inst0 + b
  uint32_t inst0;
  uint32_t k0, k1;
  int start;
  int8_t* out_s;
  void* out_de;
  int64_t* out_st;
  int32_t* status;
  uint32_t rk0[10], rk1[10];  // Philox round keys of (k0, k1), filled by anneal_dispatch
  int split;                  // blocks per problem (anneals r = s, s + split, ... in block s), set at launch
  // warm start (first accept, integer fields): start spin sums m0 (B, D) and the flip-test order perm (B, D)
  // (position j' of the scan tests coordinate perm[j']); null for the reference's starts and index order
  const int8_t* m0 = nullptr;
  const uint8_t* perm = nullptr;
  int warm_r = 1 << 30;  // anneals r < warm_r start from m0; the others from the MMSE start (m = 0), same order
  // per-coordinate sampling thresholds (B, D) x (t0, t1): anneals 0 < r < warm_r draw their start spin sum from
  // word 1 of their start Philox block u: class 0 if u < t0, 2 if u > t1, else 1 (m = 2 class - P); null: m0
  const uint32_t* cdf = nullptr;
  // per-problem anneal counts (B), or null: problem b runs anneals r < ra[b] (clamped to 1..R); the skipped
  // anneals report all-zero spin sums (the guess), best energy INT64_MAX and no tests or flips
  const int32_t* ra = nullptr;
  // Chord round (integer fields), or null: per anneal the rounds with at least one flip (B, R)
  int64_t* out_n1 = nullptr;
};

struct MapParams {
  const float* H;       // (B, NR2, D)
  const float* y;       // (B, NR2)
  const float* sigma2;  // (B) regulariser (N0/2)/E[l^2]
  int B, NR2, D, M;     // M: 4 (QPSK) or 16 (16-QAM)
  float qscale;         // 4096 for the integer problem, 0 for the float problem
  void* G;              // (B, D, D) int32 or float
  void* h;              // (B, D) int32 or float
  int8_t* xq;           // (B, D)
  float* scale;         // (B)
  int32_t* status;
  const int32_t* idx = nullptr;  // (B) rows of H, y (and of xg) for each problem, or null: b
  const int8_t* xg = nullptr;    // guesses to map around (row idx[b] with stride xg_stride), or null: MMSE guess
  int xg_stride = 0;
  // RI map (ri != 0; mimo.ising, mimo.py:132-149): N = D * log2(M)/2 spins, outputs J (B, N, N) float scaled,
  // h0 (B, N), h = h0 + 2 r sP (B, N), sP (B, N) int8 spins of the hard MMSE z; xq gets the biased-corrected
  // hard decision (mmse_hard) for the final selection; G/h above are not written.
  int ri = 0;
  float r_reg = 0.15f;
  float* Jri = nullptr;
  float* h0ri = nullptr;
  float* hri = nullptr;
  int8_t* sP = nullptr;
  float* zs = nullptr;  // (B, D) MMSE soft estimate z / mu (bias-corrected), or null
};

struct ReadParams {
  const float* H;       // (B, NR2, D)
  const float* y;       // (B, NR2)
  const int8_t* xq;     // (B, D)
  const int8_t* spins;  // (B, R, P*D)
  int B, NR2, D, P, R, M;
  int8_t* levels;       // (B, D)
  int8_t* bits;         // (B, D * nb)
  float* dist;          // (B)
  int32_t* pick;        // (B) winning candidate (R = the guess), may be null
  // MDI update mode (mdi != 0): problem b is use idx[b]; candidates are taken around xg[idx[b] * xg_stride];
  // the first best candidate replaces the use's current best bl[idx[b] * bl_stride * D] and
  // bd[idx[b] * bl_stride] only if it is strictly closer (mimo.py:590-593); levels/bits/dist/pick unused.
  const int32_t* idx = nullptr;
  const int8_t* xg = nullptr;
  int xg_stride = 0;
  int8_t* bl = nullptr;
  float* bd = nullptr;
  int bl_stride = 0;
  int mdi = 0;
  int ri = 0;  // candidates are RI spins (levels 2 s1 + s2, or s for QPSK) instead of dDI deltas
  // soft output (llr != null): max-log LLRs over the list and the single-bit-flip neighbours of the decision
  const float* N0 = nullptr;  // (B) noise density of each use
  float clip = 0.0f;
  float* llr = nullptr;       // (B, D * nb), positive = bit 1
};

// policy: 0 first accept, 1 Chord round; flt: FP32 fields.  Shapes already validated.
cudaError_t anneal_dispatch(int policy, bool flt, const DDParams& a, int P, int warps, cudaStream_t st);
cudaError_t map_dispatch(const MapParams& a, cudaStream_t st);
cudaError_t readout_dispatch(const ReadParams& a, cudaStream_t st);
int default_warps(int R);

}  // namespace arp
