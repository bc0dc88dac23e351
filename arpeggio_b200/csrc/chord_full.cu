// Chord on a full int16 coupling J (N = 32 MPL <= 256 spins, P phases): the contract of the reference's
// chord_m{MPL} launch (arpeggio/mimo/chord_kernel.cu:177-184, as chordfx.Kernel.chord calls it, chordfx.py:189-208)
// and the bit-exact definition chordfx.chord_fx (chordfx.py:80-118).
//
// Design (this file's own):
// - One block per problem.  Its J (N x N int16, 128 KB at N = 256) is staged once into shared memory by bulk
//   copies (cp.async.bulk, one thread, completion on an mbarrier with a bounded wait) while the other threads
//   check the coefficient ranges; the block's warps then share it, one anneal per warp at a time.  At N = 256 the
//   staged J leaves room for one block per SM, so the launcher fills that block with up to 16 warps (the
//   reference's blocks hold at most 8).
// - Spins are warp-uniform bit masks Sm[t] (slot t = spins 32 t .. 32 t + 31; lane l owns spin 32 t + l and its
//   field u in a register).  Phases are compile-time: at step k = n P + p only the slots p TPC .. (p+1) TPC - 1 are
//   tested, so a step's body names its registers directly (no per-step slot checks, no selects of cached words).
// - Random numbers: the reference's Philox counters (start (2^32-1, i, r, inst) word 0; step k uses word n&3 of
//   block (n>>2, i, r, inst), n = k / P).  At the start of each quad of sweeps every slot's block is computed once
//   and its four words serve the quad's four sweeps.
// - Decision as one 32-bit compare: s u < ceil(x 4T / 2^32) - 2T - q + c_k sgn, sgn = -1 for a spin flipped at
//   the previous step (only possible at P = 1), else +1 -- the reference's x 4T > (z + 2T) 2^32 with
//   z = s u + q - c_k sgn, exactly.
// - Commits in index order against the step's snapshot: the flipped spin's old sign comes from the uniform mask,
//   row j of J moves every field (u_i -= 4 s_j J_ji).  The energy change of the flip, 4 s_j (u_j - h_j + h0_j) -
//   8 J_jj with u_j after the earlier commits of the step, is added by the owner lane alone into a per-lane
//   accumulator; one warp reduction (two redux.sync) per step with flips brings it into the warp's energy.
// - Start fields u = h + 2 J^T s from the column sums c_i = sum_j J_ji (once per block): u = h - 2c + 4 sum over
//   the up spins of row j, or h + 2c - 4 sum over the down spins, whichever set is smaller.
// - Best state: first minimum over the steps that flip (and step 0); mode 1 keeps per warp the first minimum over
//   its anneals, then the block takes the lowest (energy, anneal).
// Rows of J serve both the start fields and the updates, like the reference's kernel; for the symmetric J that
// to_fixed produces that is J's columns too, as chord_fx reads them.
#include <atomic>
#include <climits>

#include "arp_common.cuh"
#include "arp_internal.h"
#include "umma.cuh"

namespace arp {
namespace chordj {

constexpr int32_t kMaxH = 1 << 28, kMaxT = 1 << 26;
constexpr int kMaxWarps = 16;

// Warps per block at most: 16 (one block per SM holds the 128 KB J at N = 256), 8 for the one instantiation whose
// registers need more than 128 per thread (N = 256 in one phase, where every slot is tested at every step).
template <int MPL, int P>
constexpr int max_warps() {
  return (MPL == 8 && P == 1) ? 8 : kMaxWarps;
}

struct Args {
  const int16_t* J;  // (B, N, N)
  const int32_t *h, *h0, *T, *C;
  int q, S, R, B;
  uint32_t inst0;
  int mode;  // 0: every anneal's best (chains), 1: the problem's best anneal
  int bulk;  // J and its per-problem blocks are 16-byte aligned: staged by cp.async.bulk
  long long* out_e;
  int8_t* out_s;
  unsigned long long* stats;
  int32_t* status;
  PhiloxKeys K;
};

// Sum over the warp of per-lane 64-bit values below 2^40 in magnitude: the low 20 bits and the rest reduced
// separately by redux.sync (each partial sum fits 32 bits).
__device__ __forceinline__ long long warp_sum64(long long v) {
  const unsigned lo = (unsigned)v & 0xFFFFFu;
  const int hi = (int)(v >> 20);
  const unsigned slo = __reduce_add_sync(ARP_FULL, lo);
  const int shi = __reduce_add_sync(ARP_FULL, hi);
  return ((long long)shi << 20) + (long long)slo;
}

__device__ __forceinline__ long long mad_wide(int32_t a, int32_t b, long long c) {
  long long d;
  asm("mad.wide.s32 %0, %1, %2, %3;" : "=l"(d) : "r"(a), "r"(b), "l"(c));
  return d;
}

// Philox blocks the reference's kernel draws per anneal (its statistic 2): slot t (phase t / TPC) draws a block at
// every fourth of its steps, counted over the 32 lanes.
template <int MPL, int P>
__device__ __forceinline__ unsigned long long rng_blocks(int S) {
  constexpr int TPC = MPL / P;
  unsigned long long n = 0;
#pragma unroll
  for (int t = 0; t < MPL; ++t) {
    const int p = t / TPC;
    const int steps = S > p ? (S - p - 1) / P + 1 : 0;
    n += (unsigned long long)((steps + 3) >> 2);
  }
  return 32ull * n;
}

template <int MPL, int P>
__global__ void __launch_bounds__(32 * max_warps<MPL, P>(), 1) k_chord_j(const Args a) {
  constexpr int N = 32 * MPL, TPC = MPL / P;
  extern __shared__ __align__(128) unsigned char smem[];
  int16_t* Js = reinterpret_cast<int16_t*>(smem);
  int32_t* csum = reinterpret_cast<int32_t*>(smem + (size_t)N * N * 2);  // column sums of J
  int32_t* hs = csum + N;
  long long* red_e = reinterpret_cast<long long*>(hs + N);
  int* red_r = reinterpret_cast<int*>(red_e + kMaxWarps);
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_bad;
  const int b = blockIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, W = blockDim.x >> 5;
  const int16_t* Jg = a.J + (size_t)b * N * N;
  if (threadIdx.x == 0) {
    s_bad = 0;
    if (a.bulk) {
      umma::mbar_init(&bar, 1);
      umma::fence_mbar_init();
    }
  }
  __syncthreads();
  if (a.bulk) {
    if (threadIdx.x == 0) {
      constexpr uint32_t bytes = (uint32_t)N * N * 2, chunk = bytes < 32768u ? bytes : 32768u;
      umma::expect_tx(&bar, bytes);
      for (uint32_t o = 0; o < bytes; o += chunk)
        umma::bulk_g2s(umma::su32(smem) + o, reinterpret_cast<const unsigned char*>(Jg) + o,
                       bytes - o < chunk ? bytes - o : chunk, &bar);
    }
  } else {
    for (int x = threadIdx.x; x < N * N; x += blockDim.x) Js[x] = Jg[x];
  }
  {  // coefficient ranges (every field and threshold stays inside int32), while J arrives
    bool bad = false;
    for (int x = threadIdx.x; x < N; x += blockDim.x) {
      const int32_t hv = a.h[(size_t)b * N + x], h0v = a.h0[(size_t)b * N + x];
      hs[x] = hv;
      bad |= hv > kMaxH || hv < -kMaxH || h0v > kMaxH || h0v < -kMaxH;
    }
    for (int x = threadIdx.x; x < a.S; x += blockDim.x)
      bad |= a.T[x] > kMaxT || a.T[x] < -kMaxT || a.C[x] > kMaxT || a.C[x] < -kMaxT;
    bad |= a.q > kMaxT || a.q < -kMaxT;
    if (bad) s_bad = 1;
  }
  if (a.bulk && !umma::mbar_wait(&bar, 0)) s_bad = 2;
  __syncthreads();
  if (s_bad) {
    if (threadIdx.x == 0) {
      set_status(a.status, s_bad == 2 ? ARP_ERR_TIMEOUT : ARP_ERR_RANGE);
      if (a.bulk && s_bad == 2) umma::mbar_wait(&bar, 0);  // the copy in flight, once more with a bound
    }
    return;
  }
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    int32_t c = 0;
    for (int j = 0; j < N; ++j) c += Js[j * N + i];
    csum[i] = c;
  }
  __syncthreads();

  const uint32_t inst = a.inst0 + (uint32_t)b;
  // per lane and slot: h - h0 and 8 J_jj (the owner's energy terms)
  int32_t hm[MPL], jd8[MPL];
#pragma unroll
  for (int t = 0; t < MPL; ++t) {
    const int i = t * 32 + lane;
    hm[t] = hs[i] - a.h0[(size_t)b * N + i];
    jd8[t] = 8 * (int32_t)Js[i * N + i];
  }
  const int S = a.S, R = a.R;
  const int32_t qv = a.q;
  long long wbest_e = LLONG_MAX;
  int wbest_r = INT_MAX;
  uint32_t Wm[MPL];
  unsigned long long n_flip = 0, n_eval = 0;
  int n_anneals = 0;
  for (int r = wid; r < R; r += W) {
    ++n_anneals;
    uint32_t Sm[MPL];
    int nup = 0;
#pragma unroll
    for (int t = 0; t < MPL; ++t) {
      uint32_t c0 = 0xFFFFFFFFu, c1 = (uint32_t)(t * 32 + lane), c2 = (uint32_t)r, c3 = inst;
      philox10(c0, c1, c2, c3, a.K);
      Sm[t] = __ballot_sync(ARP_FULL, c0 >= 0x80000000u);
      nup += __popc(Sm[t]);
    }
    // start fields from the smaller of the up and down sets
    const bool by_up = 2 * nup <= N;
    int32_t u[MPL];
#pragma unroll
    for (int t = 0; t < MPL; ++t) {
      const int i = t * 32 + lane;
      u[t] = by_up ? hs[i] - 2 * csum[i] : hs[i] + 2 * csum[i];
    }
    const int32_t f4 = by_up ? 4 : -4;
#pragma unroll
    for (int tj = 0; tj < MPL; ++tj) {
      uint32_t m = by_up ? Sm[tj] : ~Sm[tj];
      while (m) {
        const int l = __ffs(m) - 1;
        m &= m - 1u;
        const int16_t* row = Js + (tj * 32 + l) * N + lane;
#pragma unroll
        for (int t = 0; t < MPL; ++t) u[t] += f4 * (int32_t)row[t * 32];
      }
    }
    // 2 E0 = sum_i s_i (h_i - 2 h0_i - u_i)
    long long e;
    {
      long long el = 0;
#pragma unroll
      for (int t = 0; t < MPL; ++t) {
        const long long v = 2LL * hm[t] - hs[t * 32 + lane] - u[t];
        el += ((Sm[t] >> lane) & 1u) ? v : -v;
      }
      e = warp_sum64(el);
    }
    long long best = 1LL << 62, acc = 0;
    uint32_t Bm[MPL];
#pragma unroll
    for (int t = 0; t < MPL; ++t) Bm[t] = Sm[t];
    uint32_t pf[P == 1 ? MPL : 1];
#pragma unroll
    for (int t = 0; t < (P == 1 ? MPL : 1); ++t) pf[t] = 0;
    const int nquad = (S + 4 * P - 1) / (4 * P);
    for (int q4 = 0; q4 < nquad; ++q4) {
      uint32_t cw[MPL][4];
#pragma unroll
      for (int t = 0; t < MPL; ++t) {
        uint32_t c0 = (uint32_t)q4, c1 = (uint32_t)(t * 32 + lane), c2 = (uint32_t)r, c3 = inst;
        philox10(c0, c1, c2, c3, a.K);
        cw[t][0] = c0;
        cw[t][1] = c1;
        cw[t][2] = c2;
        cw[t][3] = c3;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
#pragma unroll
        for (int p = 0; p < P; ++p) {
          const int k = (q4 * 4 + i) * P + p;
          if (k >= S) break;
          const int32_t Tk = __ldg(a.T + k), ck = __ldg(a.C + k);
          // ceil(x 4T / 2^32) by one unsigned multiply-add (4T as a 32-bit pattern, x taken back for T < 0)
          const uint32_t A32 = 4u * (uint32_t)Tk, Aneg = Tk < 0 ? 0xFFFFFFFFu : 0u;
          const int32_t base = ck - 2 * Tk - qv;
          uint32_t fl[TPC];
#pragma unroll
          for (int s = 0; s < TPC; ++s) {
            const int t = p * TPC + s;
            const uint32_t x = cw[t][i];
            const uint32_t hi = (uint32_t)(((uint64_t)x * A32 + 0xFFFFFFFFull) >> 32);
            int32_t thr = (int32_t)(hi - (x & Aneg)) + base;
            if constexpr (P == 1) thr -= ((pf[t] >> lane) & 1u) ? 2 * ck : 0;
            const int32_t su = ((Sm[t] >> lane) & 1u) ? u[t] : -u[t];
            fl[s] = __ballot_sync(ARP_FULL, su < thr);
          }
          bool any = false;
#pragma unroll
          for (int s = 0; s < TPC; ++s) {
            const int t = p * TPC + s;
            uint32_t m = fl[s];
            any |= m != 0u;
            while (m) {
              const int l = __ffs(m) - 1;
              m &= m - 1u;
              const int32_t so4 = ((Sm[t] >> l) & 1u) ? 4 : -4;
              if (lane == l) acc = mad_wide(so4, u[t] - hm[t], acc) - jd8[t];
              const int16_t* row = Js + (t * 32 + l) * N + lane;
#pragma unroll
              for (int t2 = 0; t2 < MPL; ++t2) u[t2] -= so4 * (int32_t)row[t2 * 32];
              ++n_flip;
            }
            Sm[t] ^= fl[s];
            if constexpr (P == 1) pf[t] = fl[s];
          }
          if (any || k == 0) {
            ++n_eval;
            if (any) {
              e += warp_sum64(acc);
              acc = 0;
            }
            if (e < best) {
              best = e;
#pragma unroll
              for (int t = 0; t < MPL; ++t) Bm[t] = Sm[t];
            }
          }
        }
      }
    }
    if (a.mode == 0) {
      const size_t ar = (size_t)b * R + r;
      if (lane == 0) a.out_e[ar] = best;
#pragma unroll
      for (int t = 0; t < MPL; ++t) a.out_s[ar * N + t * 32 + lane] = ((Bm[t] >> lane) & 1u) ? 1 : -1;
    } else if (best < wbest_e) {
      wbest_e = best;
      wbest_r = r;
#pragma unroll
      for (int t = 0; t < MPL; ++t) Wm[t] = Bm[t];
    }
  }
  if (a.stats && lane == 0) {
    atomicAdd(&a.stats[0], n_flip);
    atomicAdd(&a.stats[1], n_eval);
    atomicAdd(&a.stats[2], rng_blocks<MPL, P>(S) * (unsigned long long)n_anneals);
    atomicAdd(&a.stats[3], (unsigned long long)S * (unsigned long long)n_anneals);
  }
  if (a.mode == 1) {
    if (lane == 0) {
      red_e[wid] = wbest_e;
      red_r[wid] = wbest_r;
    }
    __syncthreads();
    long long be = LLONG_MAX;
    int br = INT_MAX;
    for (int v = 0; v < W; ++v)
      if (red_e[v] < be || (red_e[v] == be && red_r[v] < br)) {
        be = red_e[v];
        br = red_r[v];
      }
    if (wbest_r == br) {
      if (lane == 0) a.out_e[b] = be;
#pragma unroll
      for (int t = 0; t < MPL; ++t) a.out_s[(size_t)b * N + t * 32 + lane] = ((Wm[t] >> lane) & 1u) ? 1 : -1;
    }
  }
}

constexpr int kMaxDev = 64;

template <int MPL, int P>
static cudaError_t launch(const Args& a, int warps, cudaStream_t st) {
  constexpr int N = 32 * MPL;
  auto kern = k_chord_j<MPL, P>;
  const size_t smem = (size_t)N * N * 2 + (size_t)2 * N * 4 + (size_t)kMaxWarps * 12;
  // per device: the raised shared-memory limit and the width with the most resident warps per SM
  static std::atomic<int> ready[kMaxDev];
  static std::atomic<int> auto_w[kMaxDev];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const bool cached = dev >= 0 && dev < kMaxDev && ready[dev].load(std::memory_order_acquire);
  int W = cached ? auto_w[dev].load(std::memory_order_relaxed) : 0;
  if (!cached) {
    if (smem > 48 * 1024) {
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
    }
    int best_res = -1;
    for (int w = 1; w <= max_warps<MPL, P>(); w *= 2) {
      int nb = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 32 * w, smem);
      if (e != cudaSuccess) return e;
      if (nb * w >= best_res && nb > 0) {
        best_res = nb * w;
        W = w;
      }
    }
    if (W < 1) return cudaErrorInvalidConfiguration;
    if (dev >= 0 && dev < kMaxDev) {
      auto_w[dev].store(W, std::memory_order_relaxed);
      ready[dev].store(1, std::memory_order_release);
    }
  }
  if (warps > 0) W = warps < max_warps<MPL, P>() ? warps : max_warps<MPL, P>();
  if (W > a.R) W = a.R;
  kern<<<a.B, 32 * W, smem, st>>>(a);
  return cudaGetLastError();
}

template <int MPL>
static cudaError_t launch_p(const Args& a, int P, int warps, cudaStream_t st) {
  switch (P) {
    case 1: return launch<MPL, 1>(a, warps, st);
    case 2: if constexpr (MPL % 2 == 0) return launch<MPL, 2>(a, warps, st); break;
    case 3: if constexpr (MPL % 3 == 0) return launch<MPL, 3>(a, warps, st); break;
    case 4: if constexpr (MPL % 4 == 0) return launch<MPL, 4>(a, warps, st); break;
    case 6: if constexpr (MPL % 6 == 0) return launch<MPL, 6>(a, warps, st); break;
    case 8: if constexpr (MPL % 8 == 0) return launch<MPL, 8>(a, warps, st); break;
    default: break;
  }
  return cudaErrorInvalidValue;
}

}  // namespace chordj
}  // namespace arp

using namespace arp;

extern "C" int arp_anneal_chord(const int16_t* J, const int32_t* h, const int32_t* h0, const int32_t* Tq,
                                const int32_t* Cq, int q, int S, int P, int R, int N, int B, uint32_t k0, uint32_t k1,
                                uint32_t inst0, int mode, int warps, int64_t* out_e, int8_t* out_s,
                                unsigned long long* stats, int32_t* status, void* stream) {
  if (B < 0 || R < 1 || S < 1 || P < 1 || N < 32 || N > 256 || N % 32 || N % P || (N / P) % 32) return ARP_ERR_SHAPE;
  const int mpl = N / 32;
  if (!(mpl == 1 || mpl == 2 || mpl == 3 || mpl == 4 || mpl == 6 || mpl == 8)) return ARP_ERR_SHAPE;
  if (mode != 0 && mode != 1) return ARP_ERR_ARG;
  if (B == 0) return ARP_OK;
  if (!J || !h || !h0 || !Tq || !Cq || !out_e || !out_s) return ARP_ERR_ARG;
  chordj::Args a{};
  a.J = J;
  a.h = h;
  a.h0 = h0;
  a.T = Tq;
  a.C = Cq;
  a.q = q;
  a.S = S;
  a.R = R;
  a.B = B;
  a.inst0 = inst0;
  a.mode = mode;
  a.bulk = (reinterpret_cast<uintptr_t>(J) & 15u) == 0;  // each problem's block of N^2 int16 is a multiple of 2 KB
  a.out_e = reinterpret_cast<long long*>(out_e);
  a.out_s = out_s;
  a.stats = stats;
  a.status = status;
  a.K = philox_keys(k0, k1);
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  switch (mpl) {
    case 1: e = chordj::launch_p<1>(a, P, warps, st); break;
    case 2: e = chordj::launch_p<2>(a, P, warps, st); break;
    case 3: e = chordj::launch_p<3>(a, P, warps, st); break;
    case 4: e = chordj::launch_p<4>(a, P, warps, st); break;
    case 6: e = chordj::launch_p<6>(a, P, warps, st); break;
    default: e = chordj::launch_p<8>(a, P, warps, st); break;
  }
  return e == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}
