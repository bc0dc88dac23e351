// Anneals on compressed dDI problems: first accept (Arpeggio) and the Chord round, integer or FP32 fields.
//
// Problem (arpeggio_ref59.py:41-85, chord_ref.py:72-123): the dDI coupling over N = P D spins is
// J = -offdiag(G (x) 1 1^T), so one lane field per coordinate, w_j = h_j - 2 (G m)_j with m = sum of the P
// copies, serves every copy: the field of spin (p, j) is w_j + 2 G_jj s_pj.
//
// Mapping (one warp = one anneal, lanes across threads): thread `lane` owns coordinates j = t*32 + lane for
// t < NS = ceil(D/32); its fields w[t] live in registers; spins are warp-uniform bit masks Sm[p][t]; G sits
// in shared memory transposed and zero-padded to NS*32 columns (Gs[j][i] = G[i][j]) so a flip of lane j
// streams one contiguous row.  A block holds one problem and W warps that take anneals r = w, w + W, ...
//
// First accept, exactly the reference's index-order scan: every remaining lane of the active copy tests
// against the current fields at once, a ballot + ffs picks the first accepted lane j, the flip commits
// (rank-1 update of every field from row j), and lanes after j re-test with the same draws.  Lanes that
// rejected before j stay rejected, as in the sequential scan, because their decision came before the flip.
// Chord: one snapshot test of the active copy, then the accepted lanes commit in index order.
//
// RNG: Philox4x32-10 with the reference's counters -- start (2^32-1, p*D+j, r, inst) word 0 ('rand') or
// (2^32-1, j, r, inst) ('bal'); pass k = n*P + p uses word n&3 of block (n>>2, p*D+j, r, inst).  One block
// serves four sweeps, so each quad of sweeps computes P*NS blocks per thread once (registers) instead of
// one block per test (the reference's arpeggio_fx.cu:75).
//
// Integer decision: u*4T > (s w + 2 G_jj + q + 2T) * 2^32 (arpeggio_fx.cu:76-79) is evaluated as
// s w < ceil(u*4T / 2^32) - 2 G_jj - q - 2T, a 32-bit compare; the entry points bound |G|, |h|, |T|, |q|
// so that every field and threshold fits 32 bits (ARP_ERR_RANGE otherwise).
#include <climits>
#include <cstring>
#include <mutex>
#include <type_traits>

#include "arp_common.cuh"
#include "arp_internal.h"

namespace arp {


constexpr int32_t kMaxG = 1 << 18, kMaxH = 1 << 28, kMaxT = 1 << 26;
constexpr int kMaxDevices = 64;

template <int NS, int P, bool CHORD, bool FLT, bool CACHE>
__global__ void __launch_bounds__(256) k_anneal_dd(const DDParams a) {
  using FT = typename std::conditional<FLT, float, int32_t>::type;
  using ET = typename std::conditional<FLT, float, long long>::type;
  constexpr int DP = NS * 32;
  extern __shared__ __align__(16) unsigned char smem[];
  FT* Gs = reinterpret_cast<FT*>(smem);
  __shared__ int s_bad;
  const int D = a.D, L = a.L, R = a.R;
  const int split = a.split, b = blockIdx.x / split, bs = blockIdx.x - b * split;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, W = blockDim.x >> 5;
  pdl_trigger();
  pdl_wait();
  if (threadIdx.x == 0) s_bad = 0;
  __syncthreads();
  {
    const FT* Gg = reinterpret_cast<const FT*>(a.Gt) + (size_t)b * D * D;
    bool bad = false;
    for (int x = threadIdx.x; x < D * DP; x += blockDim.x) {
      const int j = x / DP, i = x - j * DP;
      const FT v = i < D ? Gg[(size_t)j * D + i] : FT(0);
      if constexpr (!FLT) bad |= (v > kMaxG || v < -kMaxG);
      Gs[x] = v;
    }
    if constexpr (!FLT) {
      const int32_t* hg = reinterpret_cast<const int32_t*>(a.h) + (size_t)b * D;
      for (int x = threadIdx.x; x < D; x += blockDim.x) bad |= (hg[x] > kMaxH || hg[x] < -kMaxH);
      const int32_t* Tg = reinterpret_cast<const int32_t*>(a.T);
      const int32_t* cg = reinterpret_cast<const int32_t*>(a.c);
      for (int x = threadIdx.x; x < L; x += blockDim.x) {
        bad |= (Tg[x] > kMaxT || Tg[x] < -kMaxT);
        if (cg) bad |= (cg[x] > kMaxT || cg[x] < -kMaxT);
      }
      bad |= (a.qi > kMaxT || a.qi < -kMaxT);
    }
    if (bad) s_bad = 1;
  }
  __syncthreads();
  if (s_bad) {
    if (threadIdx.x == 0) set_status(a.status, ARP_ERR_RANGE);
    return;
  }
  const uint32_t inst = a.inst ? a.inst[b] : a.inst0 + (uint32_t)b;
  FT dg[NS], hv[NS];
  uint32_t vmask[NS];
#pragma unroll
  for (int t = 0; t < NS; ++t) {
    const int j = t * 32 + lane;
    const int nv = D - t * 32;
    vmask[t] = nv >= 32 ? ARP_FULL : (nv > 0 ? (1u << nv) - 1u : 0u);
    dg[t] = j < D ? Gs[j * DP + j] : FT(0);
    hv[t] = j < D ? reinterpret_cast<const FT*>(a.h)[(size_t)b * D + j] : FT(0);
  }
  const FT* Tg = reinterpret_cast<const FT*>(a.T);
  const FT* cg = reinterpret_cast<const FT*>(a.c);

  for (int r = bs + split * wid; r < R; r += split * W) {
    uint32_t Sm[P][NS], Bm[P][NS];
    // ---- start state (arpeggio_fx.cu:48-57)
    if (a.start == 0) {
#pragma unroll
      for (int p = 0; p < P; ++p)
#pragma unroll
        for (int t = 0; t < NS; ++t) {
          uint32_t c0 = 0xFFFFFFFFu, c1 = (uint32_t)(p * D + t * 32 + lane), c2 = (uint32_t)r, c3 = inst;
          philox10(c0, c1, c2, c3, a.k0, a.k1);
          Sm[p][t] = __ballot_sync(ARP_FULL, c0 >= 0x80000000u) & vmask[t];
        }
    } else {
#pragma unroll
      for (int t = 0; t < NS; ++t) {
        uint32_t c0 = 0xFFFFFFFFu, c1 = (uint32_t)(t * 32 + lane), c2 = (uint32_t)r, c3 = inst;
        philox10(c0, c1, c2, c3, a.k0, a.k1);
        const int pat = bal_pattern(P, (uint32_t)(((uint64_t)c0 * (uint64_t)bal_choose(P)) >> 32));
#pragma unroll
        for (int p = 0; p < P; ++p) Sm[p][t] = __ballot_sync(ARP_FULL, (pat >> p) & 1) & vmask[t];
      }
    }
    // ---- lane fields w = h - 2 G m (arpeggio_fx.cu:58-66); float: sum in j order, one rounding per op
    FT w[NS];
    FT acc[NS];
#pragma unroll
    for (int t = 0; t < NS; ++t) acc[t] = FT(0);
#pragma unroll
    for (int tj = 0; tj < NS; ++tj) {
      for (int l = 0; l < 32; ++l) {
        const int j = tj * 32 + l;
        if (j >= D) break;
        int m = 0;
#pragma unroll
        for (int p = 0; p < P; ++p) m += ((Sm[p][tj] >> l) & 1u) ? 1 : -1;
        if (m == 0) continue;
        const FT* gr = Gs + j * DP + lane;
#pragma unroll
        for (int t = 0; t < NS; ++t) {
          if constexpr (FLT)
            acc[t] = __fadd_rn(acc[t], __fmul_rn(gr[t * 32], (float)m));
          else
            acc[t] += gr[t * 32] * m;
        }
      }
    }
#pragma unroll
    for (int t = 0; t < NS; ++t) {
      if constexpr (FLT)
        w[t] = __fsub_rn(hv[t], __fmul_rn(2.0f, acc[t]));
      else
        w[t] = hv[t] - 2 * acc[t];
    }
#pragma unroll
    for (int p = 0; p < P; ++p)
#pragma unroll
      for (int t = 0; t < NS; ++t) Bm[p][t] = Sm[p][t];

    ET de = ET(0), best;
    if constexpr (FLT)
      best = __int_as_float(0x7f800000);
    else
      best = 1LL << 62;
    long long flips = 0, tests = 0;
    const int nquad = (L + 4 * P - 1) / (4 * P);
    for (int q4 = 0; q4 < nquad; ++q4) {
      uint32_t cw[CACHE ? P : 1][CACHE ? NS : 1][4];
      if constexpr (CACHE) {
#pragma unroll
        for (int p = 0; p < P; ++p)
#pragma unroll
          for (int t = 0; t < NS; ++t) {
            uint32_t c0 = (uint32_t)q4, c1 = (uint32_t)(p * D + t * 32 + lane), c2 = (uint32_t)r, c3 = inst;
            philox10(c0, c1, c2, c3, a.k0, a.k1);
            cw[p][t][0] = c0;
            cw[p][t][1] = c1;
            cw[p][t][2] = c2;
            cw[p][t][3] = c3;
          }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
#pragma unroll
        for (int p = 0; p < P; ++p) {
          const int k = (q4 * 4 + i) * P + p;
          if (k >= L) break;
          // ---- per-lane thresholds for this pass
          FT th[NS];
          FT qk;
          if constexpr (FLT) {
            const float A = __fmul_rn(4.0f, Tg[k]);
            qk = (CHORD && cg) ? __fsub_rn(a.qf, cg[k]) : a.qf;
#pragma unroll
            for (int t = 0; t < NS; ++t) {
              uint32_t u;
              if constexpr (CACHE) {
                u = cw[p][t][i];
              } else {
                uint32_t c0 = (uint32_t)q4, c1 = (uint32_t)(p * D + t * 32 + lane), c2 = (uint32_t)r, c3 = inst;
                philox10(c0, c1, c2, c3, a.k0, a.k1);
                u = i == 0 ? c0 : (i == 1 ? c1 : (i == 2 ? c2 : c3));
              }
              th[t] = __fmul_rn(__fsub_rn(unit24(u), 0.5f), A);
            }
          } else {
            const int32_t Tk = Tg[k];
            const long long A = 4LL * Tk;
            const int32_t Bk = a.qi + 2 * Tk - ((CHORD && cg) ? cg[k] : 0);
#pragma unroll
            for (int t = 0; t < NS; ++t) {
              uint32_t u;
              if constexpr (CACHE) {
                u = cw[p][t][i];
              } else {
                uint32_t c0 = (uint32_t)q4, c1 = (uint32_t)(p * D + t * 32 + lane), c2 = (uint32_t)r, c3 = inst;
                philox10(c0, c1, c2, c3, a.k0, a.k1);
                u = i == 0 ? c0 : (i == 1 ? c1 : (i == 2 ? c2 : c3));
              }
              th[t] = ((vmask[t] >> lane) & 1u) ? (int32_t)ceil_shift32(u, A) - 2 * dg[t] - Bk : INT_MIN;
            }
            qk = 0;
          }
          // ---- the test of one lane against the current fields
          auto accept = [&](int t) -> bool {
            const FT sw = ((Sm[p][t] >> lane) & 1u) ? w[t] : -w[t];
            if constexpr (FLT)
              return __fadd_rn(__fadd_rn(sw, __fmul_rn(2.0f, dg[t])), qk) < th[t];
            else
              return sw < th[t];
          };
          // ---- commit a flip of lane l of slot t (fields after earlier commits)
          auto commit = [&](FT wsel, FT dsel, uint32_t sbits, int j, int l) {
            const FT wj = __shfl_sync(ARP_FULL, wsel, l);
            const FT dj = __shfl_sync(ARP_FULL, dsel, l);
            const int so = ((sbits >> l) & 1u) ? 1 : -1;
            if constexpr (FLT)
              de = __fadd_rn(de, __fadd_rn(__fmul_rn((float)(4 * so), wj), __fmul_rn(8.0f, dj)));
            else
              de += 4LL * so * wj + 8LL * dj;
            const FT* gr = Gs + j * DP + lane;
#pragma unroll
            for (int t = 0; t < NS; ++t) {
              if constexpr (FLT)
                w[t] = __fadd_rn(w[t], __fmul_rn((float)(4 * so), gr[t * 32]));
              else
                w[t] += 4 * so * gr[t * 32];
            }
            ++flips;
          };
          if constexpr (!CHORD) {
            // the scan finishes slot t (positions 32 t .. 32 t + 31) before slot t + 1: a round accepts only after
            // the last flip, so a slot the scan has left has no candidate left this pass
            long long tt = 1;
#pragma unroll
            for (int t = 0; t < NS; ++t) {
              uint32_t rem = vmask[t];
              for (;;) {
                const uint32_t m = __ballot_sync(ARP_FULL, accept(t)) & rem;
                if (m == 0) break;
                const int l = __ffs(m) - 1;
                const int j = t * 32 + l;
                commit(w[t], dg[t], Sm[p][t], j, l);
                const uint32_t bit = 1u << l;
                Sm[p][t] ^= bit;
                rem &= ~((bit << 1) - 1u);
                if (j < D - 1) ++tt;
              }
            }
            tests += tt;
          } else {
            uint32_t am[NS];
#pragma unroll
            for (int t = 0; t < NS; ++t) am[t] = __ballot_sync(ARP_FULL, accept(t)) & vmask[t];
#pragma unroll
            for (int t = 0; t < NS; ++t) {
              uint32_t m = am[t];
              while (m) {
                const int l = __ffs(m) - 1;
                m &= m - 1u;
                commit(w[t], dg[t], Sm[p][t], t * 32 + l, l);
              }
              Sm[p][t] ^= am[t];
            }
            tests += 1;
          }
          if (de < best) {  // best state after each pass (arpeggio_fx.cu:90-93)
            best = de;
#pragma unroll
            for (int pp = 0; pp < P; ++pp)
#pragma unroll
              for (int t = 0; t < NS; ++t) Bm[pp][t] = Sm[pp][t];
          }
        }
      }
    }
    // ---- outputs (arpeggio_fx.cu:95-99)
    const size_t ar = (size_t)b * R + r;
    int8_t* os = a.out_s + ar * P * D;
#pragma unroll
    for (int p = 0; p < P; ++p)
#pragma unroll
      for (int t = 0; t < NS; ++t) {
        const int j = t * 32 + lane;
        if (j < D) os[p * D + j] = ((Bm[p][t] >> lane) & 1u) ? 1 : -1;
      }
    if (lane == 0) {
      reinterpret_cast<ET*>(a.out_de)[ar] = best;
      a.out_st[2 * ar] = flips;
      a.out_st[2 * ar + 1] = tests;
    }
  }
}

// Integer fields, margin form.  For the pass's copy p each lane keeps psi = s w + 2 G_jj, with s the lane's
// spin at the start of the pass, packed as psi2 = 2 psi + (s == +1).  Lane j accepts iff
// s w < theta = ceil(u 4T / 2^32) - 2 G_jj - q - 2T (the reference's decision as a 32-bit compare), i.e. iff
// psi < kappa = theta + 2 G_jj, i.e. iff psi2 < 2 kappa.  A flip of lane j (old spin so) adds 4 so G_ij to w_i,
// so psi2_i moves by 8 so s_i G_ij (one IMAD; bit 0 stays), and the energy moves by 4 so w_j + 8 G_jj = 4 psi_j:
// one shuffle of the owner's psi2 gives both the energy change and so.  Fields come back at the end of the pass
// as w = s (psi - 2 G_jj).  Spins are per-thread bits (bit p*NS + t = coordinate t*32 + lane of copy p is +1).
// First accept: a ballot over the lanes after the last commit finds the first acceptance; the pass ends on an
// empty ballot.  The reference's counters follow from the ballots: a pass with f flips takes 1 + f ballots here
// and reports tests = 1 + f - [its last flip was on lane D-1], flips = f.
// d = a b + c with a 32 x 32 -> 64-bit signed product (one multiply-add instead of a widened shift and add).
__device__ __forceinline__ long long mad_wide_s32(int32_t a, int32_t b, long long c) {
  long long d;
  asm("mad.wide.s32 %0, %1, %2, %3;" : "=l"(d) : "r"(a), "r"(b), "l"(c));
  return d;
}

// The random numbers of the reference's C++ engine model run without Philox (arpeggio/sim/x3model/engine_model.cpp,
// philox = 0): murmur-style mixing steps for the per-anneal seed chain and the lane seeds, xorshift32 per lane.
__device__ __forceinline__ uint32_t eng_mix_a(uint32_t v) { return (v ^ (v >> 16)) * 0x85EBCA6Bu; }
__device__ __forceinline__ uint32_t eng_mix_b(uint32_t v) { return (v ^ (v >> 13)) * 0xC2B2AE35u; }
__device__ __forceinline__ uint32_t eng_fin(uint32_t v) { return v ^ (v >> 16); }
__device__ __forceinline__ uint32_t eng_xs32(uint32_t x) {
  x ^= x << 13;
  x ^= x >> 17;
  x ^= x << 5;
  return x;
}

// Resident 256-thread blocks per SM that the integer anneal's registers are bounded for: four slots (D > 96) at two
// blocks (128 registers: four 4-warp blocks per SM instead of three, no spills; 64 users: 129 -> 120 ms per 32768
// uses); two slots at P = 2 at four blocks (64 registers, no spills; 32 users: anneal 32.7 -> 31.7 ms per 65536
// uses); the rest unbounded (64 registers would spill there, or, at one slot, made the 16-user MDI chain slower).
template <int NS, int P>
constexpr int anneal_min_blocks() {
  return NS >= 4 ? 2 : (NS == 2 && P == 2) ? 4 : 1;
}

// ENG (Chord only): the engine's own numbers instead of Philox -- lane j's xorshift32 state starts from the anneal's
// seed chain (engine_model.cpp:185-194, 170-184, 142-163), its bits 31, 30, ... give the start spins of copies
// 0, 1, ..., and every step advances it once and tests with its top 16 bits: u 4 T > z 2^16 (:229-257).
template <int NS, int P, bool CHORD, bool CACHE, bool WARM = false, bool ENG = false>
// One problem b of a block: its G staged in shared memory, anneals r = bs + split w, + split W, ... by the block's
// warps.  Called by the per-launch kernel below (one problem per block) and by the persistent mixed-size kernel
// (problems taken from a work counter, one after another).  Returns with every thread done reading shared memory.
__device__ __forceinline__ void anneal_int_problem(const DDParams& a, const PhiloxKeys& K, const int b, const int bs) {
  constexpr int DP = NS * 32;
  extern __shared__ __align__(16) unsigned char smem[];
  int32_t* Gs = reinterpret_cast<int32_t*>(smem);
  __shared__ int s_bad;
  __shared__ uint8_t s_perm[WARM ? 128 : 1];
  const int D = a.D, L = a.L, R = a.R;
  const int split = a.split;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, W = blockDim.x >> 5;
  if (threadIdx.x == 0) s_bad = 0;
  __syncthreads();
  const int32_t* hg = reinterpret_cast<const int32_t*>(a.h) + (size_t)b * D;
  const int32_t* Tg = reinterpret_cast<const int32_t*>(a.T);
  const int32_t* cg = reinterpret_cast<const int32_t*>(a.c);
  if constexpr (WARM) {
    // position j' of the scan holds coordinate perm[j']: G and h are gathered into that order
    for (int x = threadIdx.x; x < D; x += blockDim.x) {
      const uint8_t pv = a.perm[(size_t)b * D + x];
      if (pv >= D) s_bad = 1;  // not an order of 0..D-1: reported as ARP_ERR_RANGE, never dereferenced
      s_perm[x] = pv < D ? pv : 0;
    }
    __syncthreads();
  }
  {
    const int32_t* Gg = reinterpret_cast<const int32_t*>(a.Gt) + (size_t)b * D * D;
    bool bad = false;
    const int nG = D * DP, bt = blockDim.x;
    for (int x0 = threadIdx.x; x0 < nG; x0 += 8 * bt) {  // eight loads in flight per thread
      int32_t v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int x = x0 + u * bt, j = x / DP, i = x - j * DP;
        v[u] = 0;
        if (x < nG && i < D) {
          if constexpr (WARM)
            v[u] = Gg[(size_t)s_perm[j] * D + s_perm[i]];
          else
            v[u] = Gg[(size_t)j * D + i];
        }
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int x = x0 + u * bt;
        if (x < nG) {
          bad |= (v[u] > kMaxG || v[u] < -kMaxG);
          Gs[x] = v[u];
        }
      }
    }
    for (int x = threadIdx.x; x < D; x += blockDim.x) bad |= (hg[x] > kMaxH || hg[x] < -kMaxH);
    for (int x = threadIdx.x; x < L; x += blockDim.x) {
      bad |= (Tg[x] > kMaxT || Tg[x] < -kMaxT);
      if (cg) bad |= (cg[x] > kMaxT || cg[x] < -kMaxT);
    }
    bad |= (a.qi > kMaxT || a.qi < -kMaxT);
    if (bad) s_bad = 1;
  }
  __syncthreads();
  if (s_bad) {
    if (threadIdx.x == 0) set_status(a.status, ARP_ERR_RANGE);
    return;
  }
  const uint32_t inst = a.inst ? a.inst[b] : a.inst0 + (uint32_t)b;
  // 2 G_jj; a padding lane (j >= D: h_j = 0 and G's row and column j are zero, so w_j stays 0) gets 2^29, making
  // its margin psi2 = 2^30 + s at least every threshold kap2 = 2 (ceil(u 4 T / 2^32) - B) <= 2^30 (|4 T| <= 2^28,
  // |B| <= 2^28 by the range checks): it never accepts, with no per-pass validity select.
  int32_t dg2[NS];
#pragma unroll
  for (int t = 0; t < NS; ++t) {
    const int j = t * 32 + lane;
    dg2[t] = j < D ? 2 * Gs[j * DP + j] : (1 << 29);
  }

  int Rb = R;
  if constexpr (WARM) {
    if (a.ra) {  // a per-problem anneal count: the skipped anneals report the guess
      const int v = a.ra[b];
      Rb = v < 1 ? 1 : (v > R ? R : v);
      for (int r = Rb + bs; r < R; r += split) {
        const size_t ar = (size_t)b * R + r;
        for (int x = threadIdx.x; x < P * D; x += blockDim.x) a.out_s[ar * P * D + x] = 0;
        if (threadIdx.x == 0) {
          reinterpret_cast<long long*>(a.out_de)[ar] = LLONG_MAX;
          a.out_st[2 * ar] = 0;
          a.out_st[2 * ar + 1] = 0;
        }
      }
    }
  }
  for (int r = bs + split * wid; r < Rb; r += split * W) {
    // ---- start state (arpeggio_fx.cu:48-57), packed per thread
    uint32_t sp = 0;
    uint32_t es[ENG ? NS : 1];  // the engine's per-lane generator states
    if constexpr (ENG) {
      constexpr uint32_t PHI = 0x9E3779B9u;
      uint32_t f = eng_fin(eng_mix_b(eng_mix_a(a.k0 ^ inst)));
      f = eng_fin(eng_mix_b(eng_mix_a(f ^ a.k1)));
      f = eng_fin(eng_mix_b(eng_mix_a(f ^ (uint32_t)r)));
      const uint32_t seed = f + PHI;
#pragma unroll
      for (int t = 0; t < NS; ++t) {
        uint32_t v = eng_fin(eng_mix_b(eng_mix_a(seed + (uint32_t)(t * 32 + lane) * PHI)));
        es[t] = eng_xs32(v == 0 ? PHI : v);
#pragma unroll
        for (int p = 0; p < P; ++p)
          if ((es[t] >> (31 - p)) & 1u) sp |= 1u << (p * NS + t);
      }
    } else if constexpr (WARM) {
      // given spin sums: m = 0 takes the 'bal' pattern of the position's draw, m != 0 sets copies p < (m + P)/2
#pragma unroll
      for (int t = 0; t < NS; ++t) {
        const int j = t * 32 + lane;
        uint32_t c0 = 0xFFFFFFFFu, c1 = (uint32_t)j, c2 = (uint32_t)r, c3 = inst;
        philox10(c0, c1, c2, c3, K);
        int mv = 0;
        if (j < D && r < a.warm_r) {
          if (a.cdf && r > 0) {  // a sampled start: the position's own draw against the coordinate's thresholds
            const uint2 th = reinterpret_cast<const uint2*>(a.cdf)[(size_t)b * D + s_perm[j]];
            mv = c1 < th.x ? -2 : (c1 > th.y ? 2 : 0);
          } else {
            mv = a.m0[(size_t)b * D + s_perm[j]];
          }
        }
        mv = mv < -P ? -P : (mv > P ? P : mv);
        const int pat = mv == 0 ? bal_pattern(P, (uint32_t)(((uint64_t)c0 * (uint64_t)bal_choose(P)) >> 32))
                                : (1 << ((mv + P) >> 1)) - 1;
#pragma unroll
        for (int p = 0; p < P; ++p)
          if ((pat >> p) & 1) sp |= 1u << (p * NS + t);
      }
    } else if (a.start == 0) {
#pragma unroll
      for (int p = 0; p < P; ++p)
#pragma unroll
        for (int t = 0; t < NS; ++t) {
          uint32_t c0 = 0xFFFFFFFFu, c1 = (uint32_t)(p * D + t * 32 + lane), c2 = (uint32_t)r, c3 = inst;
          philox10(c0, c1, c2, c3, K);
          if (c0 >= 0x80000000u) sp |= 1u << (p * NS + t);
        }
    } else {
#pragma unroll
      for (int t = 0; t < NS; ++t) {
        uint32_t c0 = 0xFFFFFFFFu, c1 = (uint32_t)(t * 32 + lane), c2 = (uint32_t)r, c3 = inst;
        philox10(c0, c1, c2, c3, K);
        const int pat = bal_pattern(P, (uint32_t)(((uint64_t)c0 * (uint64_t)bal_choose(P)) >> 32));
#pragma unroll
        for (int p = 0; p < P; ++p)
          if ((pat >> p) & 1) sp |= 1u << (p * NS + t);
      }
    }
    // ---- fields w = h - 2 G m (arpeggio_fx.cu:58-66); m of coordinate j is broadcast from its owner lane
    int32_t w[NS], mloc[NS];
#pragma unroll
    for (int t = 0; t < NS; ++t) {
      const int j = t * 32 + lane;
      int m = 0;
#pragma unroll
      for (int p = 0; p < P; ++p) m += ((sp >> (p * NS + t)) & 1u) ? 1 : -1;
      mloc[t] = j < D ? m : 0;
      if constexpr (WARM)
        w[t] = j < D ? hg[s_perm[j]] : 0;
      else
        w[t] = j < D ? hg[j] : 0;
    }
#pragma unroll
    for (int tj = 0; tj < NS; ++tj) {
      uint32_t mm = __ballot_sync(ARP_FULL, mloc[tj] != 0);
      while (mm) {
        const int l = __ffs(mm) - 1;
        mm &= mm - 1u;
        const int m2 = 2 * __shfl_sync(ARP_FULL, mloc[tj], l);
        const int32_t* gr = Gs + (tj * 32 + l) * DP + lane;
#pragma unroll
        for (int t = 0; t < NS; ++t) w[t] -= m2 * gr[t * 32];
      }
    }
    long long de = 0, best = ENG ? (1LL << 35) - 1 : 1LL << 62;  // the engine's best register starts at 2^35 - 1
    uint32_t bsp = sp;
    int32_t flips = 0, lastflips = 0, n1 = 0;
    const int nquad = (L + 4 * P - 1) / (4 * P);
    for (int q4 = 0; q4 < nquad; ++q4) {
      uint32_t cw[CACHE ? P : 1][CACHE ? NS : 1][4];
      if constexpr (CACHE && !ENG) {
#pragma unroll
        for (int p = 0; p < P; ++p)
#pragma unroll
          for (int t = 0; t < NS; ++t) {
            uint32_t c0 = (uint32_t)q4, c1 = (uint32_t)(p * D + t * 32 + lane), c2 = (uint32_t)r, c3 = inst;
            philox10(c0, c1, c2, c3, K);
            cw[p][t][0] = c0;
            cw[p][t][1] = c1;
            cw[p][t][2] = c2;
            cw[p][t][3] = c3;
          }
      }
#pragma unroll(NS <= 2 ? 4 : 1)  // three and four slots: one copy of the pass body (code size)
      for (int i = 0; i < 4; ++i) {
#pragma unroll
        for (int p = 0; p < P; ++p) {
          const int k = (q4 * 4 + i) * P + p;
          if (k >= L) break;
          const int32_t Tk = Tg[k];
          // ceil(u 4 T / 2^32) as one unsigned multiply-add: with A = 4 T as a 32-bit pattern (|4 T| <= 2^28),
          // u A + 2^32 - 1 < 2^64, and for T < 0 the pattern adds u 2^32, taken back by subtracting u
          const uint32_t A32 = 4u * (uint32_t)Tk, Aneg = Tk < 0 ? 0xFFFFFFFFu : 0u;
          const int32_t Bk = a.qi + 2 * Tk - ((CHORD && cg) ? cg[k] : 0);
          int32_t psi2[NS], kap2[NS], cp[NS];
#pragma unroll
          for (int t = 0; t < NS; ++t) {
            uint32_t u;
            if constexpr (ENG) {
              es[t] = eng_xs32(es[t]);
              u = es[t] >> 16;
            } else if constexpr (CACHE) {
              // word i of the cached block, by selects (a runtime i must not index the register array)
              u = i == 0 ? cw[p][t][0] : (i == 1 ? cw[p][t][1] : (i == 2 ? cw[p][t][2] : cw[p][t][3]));
            } else {
              uint32_t c0 = (uint32_t)q4, c1 = (uint32_t)(p * D + t * 32 + lane), c2 = (uint32_t)r, c3 = inst;
              philox10(c0, c1, c2, c3, K);
              u = i == 0 ? c0 : (i == 1 ? c1 : (i == 2 ? c2 : c3));
            }
            const int32_t upb = (int32_t)((sp >> (p * NS + t)) & 1u), sg = 2 * upb - 1;
            psi2[t] = 2 * (sg * w[t] + dg2[t]) + upb;
            int32_t thr;
            if constexpr (ENG) {  // ceil(u 4 T / 2^16), u < 2^16: |thr| <= |4 T| <= 2^28
              thr = (int32_t)(((long long)u * (4LL * Tk) + 0xFFFFLL) >> 16);
            } else {
              const uint32_t hi = (uint32_t)(((uint64_t)u * A32 + 0xFFFFFFFFull) >> 32);
              thr = (int32_t)(hi - (u & Aneg));
            }
            kap2[t] = 2 * (thr - Bk);
            cp[t] = 8 * sg;
          }
          int jl = -1;
          // commit the flip of lane l of slot ts: energy, margins, spin bit
          auto commit = [&](int ts, int l, int32_t vsel) {
            const int32_t packed = __shfl_sync(ARP_FULL, vsel, l);
            de = mad_wide_s32(packed >> 1, 4, de);
            ++flips;
            const int32_t so = 2 * (packed & 1) - 1;  // the flipped coordinate's old spin
            const int32_t* gr = Gs + (ts * 32 + l) * DP + lane;
#pragma unroll
            for (int t = 0; t < NS; ++t) psi2[t] += (so * cp[t]) * gr[t * 32];
            if (lane == l) sp ^= 1u << (p * NS + ts);
            jl = ts * 32 + l;
          };
          if constexpr (!CHORD) {
            // A round accepts the first position after the last flip whose test passes, so once the scan has
            // left slot t (positions 32 t .. 32 t + 31) no later round of this pass can accept there: finish slot
            // t, then slot t + 1 -- one ballot of one slot per round, the same flips in the same order.  (Measured
            // 19 % faster at two slots than a joint scan of every slot's ballot per round.)
#pragma unroll
            for (int t = 0; t < NS; ++t) {
              for (;;) {
                const uint32_t m = __ballot_sync(ARP_FULL, psi2[t] < kap2[t] && t * 32 + lane > jl);
                if (m == 0) break;
                commit(t, __ffs(m) - 1, psi2[t]);
              }
            }
          } else {
            uint32_t am[NS], anyf = 0;
#pragma unroll
            for (int t = 0; t < NS; ++t) {
              am[t] = __ballot_sync(ARP_FULL, psi2[t] < kap2[t]);
              anyf |= am[t];
            }
            n1 += anyf != 0u;
#pragma unroll
            for (int t = 0; t < NS; ++t) {
              uint32_t m = am[t];
              while (m) {
                const int l = __ffs(m) - 1;
                m &= m - 1u;
                commit(t, l, psi2[t]);
              }
            }
          }
          if (jl == D - 1) ++lastflips;
          // fields back: w = s (psi - 2 G_jj) with the pass-start spin
#pragma unroll
          for (int t = 0; t < NS; ++t) {
            w[t] = (cp[t] >> 3) * ((psi2[t] >> 1) - dg2[t]);
          }
          if (de < best) {  // best state after each pass (arpeggio_fx.cu:90-93)
            best = de;
            bsp = sp;
          }
        }
      }
    }
    const size_t ar = (size_t)b * R + r;
    int8_t* os = a.out_s + ar * P * D;
#pragma unroll
    for (int p = 0; p < P; ++p)
#pragma unroll
      for (int t = 0; t < NS; ++t) {
        const int j = t * 32 + lane;
        if (j < D) os[p * D + (WARM ? (int)s_perm[j] : j)] = ((bsp >> (p * NS + t)) & 1u) ? 1 : -1;
      }
    if (lane == 0) {
      // every anneal runs all L passes; first accept takes flips + 1 ballots per pass
      reinterpret_cast<long long*>(a.out_de)[ar] = best;
      a.out_st[2 * ar] = flips;
      a.out_st[2 * ar + 1] = CHORD ? L : L + flips - lastflips;
      if (CHORD && a.out_n1) a.out_n1[ar] = n1;
    }
  }
}

template <int NS, int P, bool CHORD, bool CACHE, bool WARM = false, bool ENG = false>
__global__ void __launch_bounds__(256, anneal_min_blocks<NS, P>()) k_anneal_int(const DDParams a) {
  const int split = a.split, b = blockIdx.x / split, bs = blockIdx.x - b * split;
  pdl_trigger();
  pdl_wait();
  anneal_int_problem<NS, P, CHORD, CACHE, WARM, ENG>(a, *reinterpret_cast<const PhiloxKeys*>(a.rk0), b, bs);
}

// The same anneal without the register bound, for batches too small to fill the GPU (a frame's chain): no other
// block waits for the SM there, and with its registers unbounded each anneal runs faster (one 32-user frame:
// 91.5 -> 85.2 us p50 against the bounded kernel).  The explicit minimum of one block matters: with the thread
// bound alone ptxas settles on fewer registers and spills.
template <int NS, int P, bool CHORD, bool CACHE, bool WARM = false, bool ENG = false>
__global__ void __launch_bounds__(256, 1) k_anneal_int_lat(const DDParams a) {
  const int split = a.split, b = blockIdx.x / split, bs = blockIdx.x - b * split;
  pdl_trigger();
  pdl_wait();
  anneal_int_problem<NS, P, CHORD, CACHE, WARM, ENG>(a, *reinterpret_cast<const PhiloxKeys*>(a.rk0), b, bs);
}

using AnnealKernel = void (*)(const DDParams);

template <int NS, int P, bool CHORD, bool FLT, bool WARM, bool ENG, bool LAT>
static AnnealKernel anneal_kernel() {
  constexpr bool CACHE = P * NS <= 8;
  if constexpr (FLT)
    return k_anneal_dd<NS, P, CHORD, true, CACHE>;
  else if constexpr (LAT)
    return k_anneal_int_lat<NS, P, CHORD, CACHE, WARM, ENG>;
  else
    return k_anneal_int<NS, P, CHORD, CACHE, WARM, ENG>;
}

// Warps per block: a block holds one problem and its warps share the anneals, so fewer warps per block let
// more blocks (problems) share an SM.  Pick the width with the most resident warps per SM for this kernel's
// registers and shared memory (ties go to the wider block, which loads G fewer times per anneal).
template <typename K>
static int pick_warps(K kern, size_t smem, int R) {
  int best_w = 1, best_res = -1;
  for (int w = 1; w <= 8; w *= 2) {
    if (w > R && w > 1) break;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 32 * w, smem) != cudaSuccess) return R < 8 ? R : 8;
    const int res = nb * w;
    if (res >= best_res) {
      best_res = res;
      best_w = w;
    }
  }
  return best_w;
}

// Warps per block chosen by a caller's autotuner per (slots NS, copies P, policy: first accept, Chord round, warm
// first accept, FP32 fields); 0 = occupancy heuristic.  Process-wide, set through arp_anneal_tune.
static int g_tuned_warps[5][7][3][2];

template <int NS, int P, bool CHORD, bool FLT, bool WARM = false, bool ENG = false, bool LAT = false>
static cudaError_t launch_ns_p(const DDParams& a, int warps, cudaStream_t st) {
  if constexpr (!FLT && !LAT && anneal_min_blocks<NS, P>() > 1) {
    if (a.B <= kPdlMaxB) return launch_ns_p<NS, P, CHORD, FLT, WARM, ENG, true>(a, warps, st);
  }
  const AnnealKernel kern = anneal_kernel<NS, P, CHORD, FLT, WARM, ENG, LAT>();
  const size_t smem = (size_t)a.D * NS * 32 * 4;
  // Launch settings per device (the shared-memory limit raised by cudaFuncSetAttribute applies to the current
  // device only; occupancy and SM count are per device too), behind one lock per instantiation.
  struct Slot {
    size_t attr_smem = 48 * 1024, cached_smem = 0;
    int cached_w = 0, cached_nb = 0, sms = 0;
  };
  static Slot slots_by_dev[kMaxDevices];
  static std::mutex mu;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  int per_sm = 1, sms = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    Slot& sl = slots_by_dev[dev];
    if (smem > sl.attr_smem) {
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      sl.attr_smem = smem;
    }
    if (warps <= 0 && (sl.cached_w == 0 || sl.cached_smem != smem)) {
      sl.cached_w = pick_warps(kern, smem, 8);
      sl.cached_smem = smem;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sl.cached_nb, kern, 32 * sl.cached_w, smem) != cudaSuccess)
        sl.cached_nb = 1;
      cudaDeviceGetAttribute(&sl.sms, cudaDevAttrMultiProcessorCount, dev);
    }
    per_sm = sl.cached_nb > 0 ? sl.cached_nb : 1;
    sms = sl.sms;
    if (warps <= 0) {
      warps = sl.cached_w;
      const int tw = g_tuned_warps[NS][P][WARM ? 2 : (CHORD ? 1 : 0)][FLT ? 1 : 0];
      if (tw > 0 && tw != warps) {  // same resident warps per SM, another width
        per_sm = sl.cached_nb * sl.cached_w / tw > 0 ? sl.cached_nb * sl.cached_w / tw : 1;
        warps = tw;
      }
      while (warps > 1 && warps > a.R) warps >>= 1;
    }
  }
  // Small batches: split each problem's anneals over several blocks so the batch still fills the GPU.
  DDParams b = a;
  b.split = 1;
  const long long slots = (long long)per_sm * (sms > 0 ? sms : 148);
  if ((long long)a.B < slots) {
    const int most = (a.R + warps - 1) / warps;
    long long sp = (slots + a.B - 1) / a.B;
    b.split = (int)(sp < most ? sp : most);
    if (b.split < 1) b.split = 1;
  }
  // small integer batches (a frame's chain) launch with programmatic serialization: the kernel waits for its
  // predecessor before any read
  return launch_ex(kern, dim3((unsigned)((long long)a.B * b.split)), dim3(warps * 32), smem, st,
                   !FLT && a.B <= kPdlMaxB, b);
}

template <bool CHORD, bool FLT>
static cudaError_t launch_dd(const DDParams& a, int P, int warps, cudaStream_t st) {
  const int NS = (a.D + 31) / 32;
#define ARP_CASE(ns, pp) \
  if (NS == ns && P == pp) return launch_ns_p<ns, pp, CHORD, FLT>(a, warps, st);
  ARP_CASE(1, 2) ARP_CASE(1, 4) ARP_CASE(1, 6)
  ARP_CASE(2, 2) ARP_CASE(2, 4) ARP_CASE(2, 6)
  ARP_CASE(3, 2) ARP_CASE(3, 4) ARP_CASE(3, 6)
  ARP_CASE(4, 2) ARP_CASE(4, 4) ARP_CASE(4, 6)
#undef ARP_CASE
  return cudaErrorInvalidValue;
}

static int check_dd(const void* Gt, const void* h, const void* T, int L, int P, int R, int D, int B,
                    const uint32_t* inst, int start, const int8_t* out_s, const void* out_de, const int64_t* out_st) {
  if (B < 0 || R < 1 || D < 1 || D > 128 || L < 1 || !(P == 2 || P == 4 || P == 6)) return ARP_ERR_SHAPE;
  if (start != 0 && start != 1) return ARP_ERR_ARG;
  if (B > 0 && (!Gt || !h || !T || !inst || !out_s || !out_de || !out_st)) return ARP_ERR_ARG;
  return ARP_OK;
}

int default_warps(int R) { return 0; }  // 0: chosen per kernel by occupancy (pick_warps)

// Warm-started first accept (integer fields, P = 2).
static cudaError_t launch_warm(const DDParams& a0, cudaStream_t st) {
  DDParams a = a0;
  const PhiloxKeys K = philox_keys(a.k0, a.k1);
  for (int i = 0; i < 10; ++i) {
    a.rk0[i] = K.k0[i];
    a.rk1[i] = K.k1[i];
  }
  switch ((a.D + 31) / 32) {
    case 1: return launch_ns_p<1, 2, false, false, true>(a, 0, st);
    case 2: return launch_ns_p<2, 2, false, false, true>(a, 0, st);
    case 3: return launch_ns_p<3, 2, false, false, true>(a, 0, st);
    case 4: return launch_ns_p<4, 2, false, false, true>(a, 0, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t anneal_dispatch(int policy, bool flt, const DDParams& a0, int P, int warps, cudaStream_t st) {
  DDParams a = a0;
  const PhiloxKeys K = philox_keys(a.k0, a.k1);
  for (int i = 0; i < 10; ++i) {
    a.rk0[i] = K.k0[i];
    a.rk1[i] = K.k1[i];
  }
  if (flt) return policy == 0 ? launch_dd<false, true>(a, P, warps, st) : launch_dd<true, true>(a, P, warps, st);
  return policy == 0 ? launch_dd<false, false>(a, P, warps, st) : launch_dd<true, false>(a, P, warps, st);
}

// Chord with the engine's own numbers (integer fields; no Philox keys needed).
static cudaError_t launch_engine(const DDParams& a, int P, cudaStream_t st) {
  const int NS = (a.D + 31) / 32;
#define ARP_CASE(ns, pp) \
  if (NS == ns && P == pp) return launch_ns_p<ns, pp, true, false, false, true>(a, 0, st);
  ARP_CASE(1, 2) ARP_CASE(1, 4) ARP_CASE(1, 6)
  ARP_CASE(2, 2) ARP_CASE(2, 4) ARP_CASE(2, 6)
  ARP_CASE(3, 2) ARP_CASE(3, 4) ARP_CASE(3, 6)
  ARP_CASE(4, 2) ARP_CASE(4, 4) ARP_CASE(4, 6)
#undef ARP_CASE
  return cudaErrorInvalidValue;
}

}  // namespace arp

using namespace arp;

extern "C" int arp_anneal_chord_engine(const int32_t* Gt, const int32_t* h, const int32_t* T, const int32_t* c,
                                       int L, int q, int P, int R, int D, int B, const uint32_t* inst, uint32_t k0,
                                       uint32_t k1, int8_t* out_s, int64_t* out_de, int64_t* out_st,
                                       int32_t* status, void* stream) {
  int rc = check_dd(Gt, h, T, L, P, R, D, B, inst, 0, out_s, out_de, out_st);
  if (rc || B == 0) return rc;
  DDParams a{Gt, h, T, c, L, q, 0.0f, R, D, B, inst, 0u, k0, k1, 0, out_s, out_de, out_st, status};
  return launch_engine(a, P, (cudaStream_t)stream) == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_anneal_first_accept(const int32_t* Gt, const int32_t* h, const int32_t* T, int L, int q, int P,
                                       int R, int D, int B, const uint32_t* inst, uint32_t k0, uint32_t k1,
                                       int start, int8_t* out_s, int64_t* out_de, int64_t* out_st,
                                       int32_t* status, void* stream) {
  int rc = check_dd(Gt, h, T, L, P, R, D, B, inst, start, out_s, out_de, out_st);
  if (rc || B == 0) return rc;
  DDParams a{Gt, h, T, nullptr, L, q, 0.0f, R, D, B, inst, 0u, k0, k1, start, out_s, out_de, out_st, status};
  return anneal_dispatch(0, false, a, P, default_warps(R), (cudaStream_t)stream) == cudaSuccess ? ARP_OK
                                                                                                : ARP_ERR_LAUNCH;
}

extern "C" int arp_anneal_chord_dd(const int32_t* Gt, const int32_t* h, const int32_t* T, const int32_t* c, int L,
                                   int q, int P, int R, int D, int B, const uint32_t* inst, uint32_t k0, uint32_t k1,
                                   int start, int8_t* out_s, int64_t* out_de, int64_t* out_st, int32_t* status,
                                   void* stream) {
  int rc = check_dd(Gt, h, T, L, P, R, D, B, inst, start, out_s, out_de, out_st);
  if (rc || B == 0) return rc;
  DDParams a{Gt, h, T, c, L, q, 0.0f, R, D, B, inst, 0u, k0, k1, start, out_s, out_de, out_st, status};
  return anneal_dispatch(1, false, a, P, default_warps(R), (cudaStream_t)stream) == cudaSuccess ? ARP_OK
                                                                                                : ARP_ERR_LAUNCH;
}

extern "C" int arp_anneal_chord_dd_n1(const int32_t* Gt, const int32_t* h, const int32_t* T, const int32_t* c, int L,
                                      int q, int P, int R, int D, int B, const uint32_t* inst, uint32_t k0,
                                      uint32_t k1, int start, int8_t* out_s, int64_t* out_de, int64_t* out_st,
                                      int64_t* out_n1, int32_t* status, void* stream) {
  int rc = check_dd(Gt, h, T, L, P, R, D, B, inst, start, out_s, out_de, out_st);
  if (rc || B == 0) return rc;
  if (!out_n1) return ARP_ERR_ARG;
  DDParams a{Gt, h, T, c, L, q, 0.0f, R, D, B, inst, 0u, k0, k1, start, out_s, out_de, out_st, status};
  a.out_n1 = out_n1;
  return anneal_dispatch(1, false, a, P, default_warps(R), (cudaStream_t)stream) == cudaSuccess ? ARP_OK
                                                                                                : ARP_ERR_LAUNCH;
}

extern "C" int arp_anneal_dd_f32(int policy, const float* Gt, const float* h, const float* T, const float* c, int L,
                                 float q, int P, int R, int D, int B, const uint32_t* inst, uint32_t k0, uint32_t k1,
                                 int start, int8_t* out_s, float* out_de, int64_t* out_st, int32_t* status,
                                 void* stream) {
  if (policy != 0 && policy != 1) return ARP_ERR_ARG;
  int rc = check_dd(Gt, h, T, L, P, R, D, B, inst, start, out_s, out_de, out_st);
  if (rc || B == 0) return rc;
  DDParams a{Gt, h, T, c, L, 0, q, R, D, B, inst, 0u, k0, k1, start, out_s, out_de, out_st, status};
  cudaError_t e = anneal_dispatch(policy, true, a, P, default_warps(R), (cudaStream_t)stream);
  return e == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_anneal_first_accept_warm_sampled(const int32_t* Gt, const int32_t* h, const int32_t* T, int L,
                                                    int q, int P, int R, int D, int B, const uint32_t* inst,
                                                    uint32_t k0, uint32_t k1, const int8_t* m0, const uint32_t* cdf,
                                                    const uint8_t* perm, int warm_r, const int32_t* ra,
                                                    int8_t* out_s, int64_t* out_de, int64_t* out_st,
                                                    int32_t* status, void* stream) {
  int rc = check_dd(Gt, h, T, L, P, R, D, B, inst, 1, out_s, out_de, out_st);
  if (rc || B == 0) return rc;
  if (P != 2) return ARP_ERR_SHAPE;
  if (!m0 || !perm || !cdf || warm_r < 0) return ARP_ERR_ARG;
  DDParams a{Gt, h, T, nullptr, L, q, 0.0f, R, D, B, inst, 0u, k0, k1, 1, out_s, out_de, out_st, status};
  a.m0 = m0;
  a.perm = perm;
  a.warm_r = warm_r;
  a.cdf = cdf;
  a.ra = ra;
  return launch_warm(a, (cudaStream_t)stream) == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_anneal_first_accept_warm_mix(const int32_t* Gt, const int32_t* h, const int32_t* T, int L, int q,
                                                int P, int R, int D, int B, const uint32_t* inst, uint32_t k0,
                                                uint32_t k1, const int8_t* m0, const uint8_t* perm, int warm_r,
                                                int8_t* out_s, int64_t* out_de, int64_t* out_st, int32_t* status,
                                                void* stream) {
  int rc = check_dd(Gt, h, T, L, P, R, D, B, inst, 1, out_s, out_de, out_st);
  if (rc || B == 0) return rc;
  if (P != 2) return ARP_ERR_SHAPE;
  if (!m0 || !perm || warm_r < 0) return ARP_ERR_ARG;
  DDParams a{Gt, h, T, nullptr, L, q, 0.0f, R, D, B, inst, 0u, k0, k1, 1, out_s, out_de, out_st, status};
  a.m0 = m0;
  a.perm = perm;
  a.warm_r = warm_r;
  return launch_warm(a, (cudaStream_t)stream) == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_anneal_first_accept_warm(const int32_t* Gt, const int32_t* h, const int32_t* T, int L, int q, int P,
                                            int R, int D, int B, const uint32_t* inst, uint32_t k0, uint32_t k1,
                                            const int8_t* m0, const uint8_t* perm, int8_t* out_s, int64_t* out_de,
                                            int64_t* out_st, int32_t* status, void* stream) {
  int rc = check_dd(Gt, h, T, L, P, R, D, B, inst, 1, out_s, out_de, out_st);
  if (rc || B == 0) return rc;
  if (P != 2) return ARP_ERR_SHAPE;
  if (!m0 || !perm) return ARP_ERR_ARG;
  DDParams a{Gt, h, T, nullptr, L, q, 0.0f, R, D, B, inst, 0u, k0, k1, 1, out_s, out_de, out_st, status};
  a.m0 = m0;
  a.perm = perm;
  return launch_warm(a, (cudaStream_t)stream) == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

// ---------------------------------------------------------------- persistent mixed-size first accept
// Every problem of every size class of a mixed batch in one grid per coordinate-slot count NS (at most four
// launches): the grid is sized to the SMs' resident blocks, and each block takes problems from a work counter in
// global memory (one atomicAdd per problem, no waiting on other blocks) until the batch is done, running the
// per-size body compiled for its NS.  Problems are numbered class by class, the classes in decreasing cost per
// problem (L R D), so the costly problems start first and the short ones fill the tail.  Each problem's anneals are
// exactly those of the per-class launch (same body, same counters), so the outputs do not depend on the schedule.
constexpr int kMaxMixed = 64;

struct MixedArgs {
  PhiloxKeys K;  // one key for the whole batch (kernel parameter: the rounds read it as constant operands)
  int total;
  int* counter;
  int first[kMaxMixed + 1];  // problems of class c: first[c] .. first[c + 1] - 1
  DDParams cls[kMaxMixed];
};

// Bounds as the per-class anneal's, but two slots unbounded: with the work loop around it, 64 registers spill there.
template <int NS>
__global__ void __launch_bounds__(256, NS == 2 ? 1 : anneal_min_blocks<NS, 2>()) k_anneal_mixed(const __grid_constant__ MixedArgs g) {
  __shared__ int s_item;
  for (;;) {
    __syncthreads();  // the previous problem's shared memory is no longer read
    if (threadIdx.x == 0) s_item = atomicAdd(g.counter, 1);
    __syncthreads();
    const int i = s_item;
    if (i >= g.total) break;
    int c = 0;
    while (c + 1 < kMaxMixed && g.first[c + 1] <= i) ++c;
    anneal_int_problem<NS, 2, false, (2 * NS <= 8)>(g.cls[c], g.K, i - g.first[c], 0);
  }
}

template <int NS>
static cudaError_t launch_mixed(MixedArgs& g, int Dmax, int warps, int* counter, cudaStream_t st) {
  auto kern = k_anneal_mixed<NS>;
  const size_t smem = (size_t)Dmax * NS * 32 * 4;
  struct Slot {
    size_t attr_smem = 48 * 1024;
    int sms = 0;
  };
  static Slot slots_by_dev[kMaxDevices];
  static std::mutex mu;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  int sms = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    Slot& sl = slots_by_dev[dev];
    if (smem > sl.attr_smem) {
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      sl.attr_smem = smem;
    }
    if (sl.sms == 0) cudaDeviceGetAttribute(&sl.sms, cudaDevAttrMultiProcessorCount, dev);
    sms = sl.sms;
  }
  int W = warps;
  if (W <= 0) W = g_tuned_warps[NS][2][0][0];
  if (W <= 0) W = pick_warps(kern, smem, 8);
  int nb = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 32 * W, smem);
  if (e != cudaSuccess) return e;
  if (nb < 1) return cudaErrorInvalidConfiguration;
  long long grid = (long long)nb * (sms > 0 ? sms : 148);
  if (grid > g.total) grid = g.total;
  g.counter = counter;
  e = cudaMemsetAsync(counter, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  kern<<<(unsigned)grid, 32 * W, smem, st>>>(g);
  return cudaGetLastError();
}

extern "C" int arp_anneal_tune(int D, int P, int policy, int precision, int warps) {
  if (D < 1 || D > 128 || !(P == 2 || P == 4 || P == 6) || policy < 0 || policy > 2 ||
      (precision != 0 && precision != 1) || (policy == 2 && (P != 2 || precision != 0)))
    return ARP_ERR_SHAPE;
  if (!(warps == 0 || warps == 1 || warps == 2 || warps == 4 || warps == 8)) return ARP_ERR_ARG;
  g_tuned_warps[(D + 31) / 32][P][policy][precision] = warps;
  return ARP_OK;
}

/* Persistent mixed-size first accept: see the header.  Classes are grouped by slot count and ordered by cost. */
extern "C" int arp_anneal_first_accept_mixed(const arp_mixed_class* cls, int ncls, int P, uint32_t k0, uint32_t k1,
                                             int warps, int* counters, int32_t* status, void* stream) {
  if (ncls < 0 || ncls > kMaxMixed || P != 2) return ARP_ERR_SHAPE;
  if (ncls == 0) return ARP_OK;
  if (!cls || !counters) return ARP_ERR_ARG;
  if (!(warps == 0 || warps == 1 || warps == 2 || warps == 4 || warps == 8)) return ARP_ERR_ARG;
  for (int c = 0; c < ncls; ++c) {
    const arp_mixed_class& m = cls[c];
    const int rc = check_dd(m.Gt, m.h, m.T, m.L, 2, m.R, m.D, m.B, m.inst, m.start, m.out_s, m.out_de, m.out_st);
    if (rc != ARP_OK) return rc;
  }
  const PhiloxKeys K = philox_keys(k0, k1);
  cudaStream_t st = (cudaStream_t)stream;
  for (int ns = 4; ns >= 1; --ns) {
    // this group's classes, in decreasing cost per problem
    int idx[kMaxMixed], n = 0, Dmax = 0;
    for (int c = 0; c < ncls; ++c)
      if ((cls[c].D + 31) / 32 == ns && cls[c].B > 0) idx[n++] = c;
    if (n == 0) continue;
    auto cost = [&](int c) { return (double)cls[c].L * cls[c].R * cls[c].D; };
    for (int i = 1; i < n; ++i)
      for (int j = i; j > 0 && cost(idx[j]) > cost(idx[j - 1]); --j) {
        const int t = idx[j];
        idx[j] = idx[j - 1];
        idx[j - 1] = t;
      }
    MixedArgs g;
    memset(&g, 0, sizeof(g));
    g.K = K;
    int total = 0;
    for (int i = 0; i < n; ++i) {
      const arp_mixed_class& m = cls[idx[i]];
      DDParams& a = g.cls[i];
      a.Gt = m.Gt;
      a.h = m.h;
      a.T = m.T;
      a.c = nullptr;
      a.L = m.L;
      a.qi = m.q;
      a.R = m.R;
      a.D = m.D;
      a.B = m.B;
      a.inst = m.inst;
      a.start = m.start;
      a.out_s = m.out_s;
      a.out_de = m.out_de;
      a.out_st = m.out_st;
      a.status = status;
      a.split = 1;
      a.m0 = nullptr;
      a.perm = nullptr;
      a.warm_r = 1 << 30;
      a.cdf = nullptr;
      a.ra = nullptr;
      g.first[i] = total;
      total += m.B;
      if (m.D > Dmax) Dmax = m.D;
    }
    for (int i = n; i <= kMaxMixed; ++i) g.first[i] = total;
    g.total = total;
    cudaError_t e;
    switch (ns) {
      case 1: e = launch_mixed<1>(g, Dmax, warps, counters + 0, st); break;
      case 2: e = launch_mixed<2>(g, Dmax, warps, counters + 1, st); break;
      case 3: e = launch_mixed<3>(g, Dmax, warps, counters + 2, st); break;
      default: e = launch_mixed<4>(g, Dmax, warps, counters + 3, st); break;
    }
    if (e != cudaSuccess) return ARP_ERR_LAUNCH;
  }
  return ARP_OK;
}
