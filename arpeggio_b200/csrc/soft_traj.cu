// Trajectory soft output: Chord's synchronous rule as a sampler of the detection posterior on the RI map, with per-bit
// minima of ||y - H x||^2 over every visited state of every chain (the reference's mimo.chord_soft,
// arpeggio/mimo/mimo.py:332-394; the LLRs themselves are formed by arpeggio_b200.soft.trajectory_llr, mimo.py:397-413).
//
// Problem: N = nb D spins s = [s_MSB; s_LSB] (16-QAM, levels 2 s1 + s2) or N = D (QPSK), scaled J (B, N, N) with a
// zero diagonal, exploration field hf (the unregularised h0, or the RI field h), h0, scale and the distance constant
// c0 of ||y - H x||^2 = scale E0(s) + c0, E0(s) = -h0.s - s^T J s (mimo.energy0).
// Step k (temperature T[b][k], shared q): every spin tests the snapshot, z = s u + q against thr = (x/2^32 - 1/2) 4T
// with x the Philox word k & 3 of block (k >> 2, i, r, inst) (24-bit uniform, as the FP32 anneals), flips where
// z < thr; the flips commit in index order (u_i += -4 s_j J_ij, u_j after the earlier commits), E0 moving by
// 2 s_j (h0_j + u_j - hf_j) per flip.  After every step that flips (and step 0) the chain's distance
// d = scale E0 + c0 updates the minima m1 (bit = 1) and m0 (bit = 0) of each bit of the current levels (Gray bits:
// b1 = l > 0, b2 = |l| == 1, i.e. s1 > 0 and s1 != s2; QPSK b = s > 0) and the best state (lowest d; the earliest
// step, then the lowest chain, on ties).  One block per problem, one warp per chain (chains r = w, w + W, ...), J in
// shared memory, fields in registers, spins as warp-uniform masks; the block reduces the minima over its chains.
// The reference draws its chains' start and tests from torch.rand; this sampler draws them from Philox counters of
// its own (start: word 0 of (2^32 - 1, i, r, inst), spin +1 iff >= 2^31), so its trajectories are its own while the
// rule, the visited-state bookkeeping and the LLR formation are the reference's.
#include <cfloat>

#include "arp_common.cuh"
#include "arp_internal.h"

namespace arp {

struct SoftParams {
  const float *J, *hf, *h0, *scale, *c0, *T;  // T: (B, S) per-problem temperatures
  const int8_t* s0;                             // (B, N) start spins, or null: Philox
  float q;
  int S, R, N, D, M, B;
  const uint32_t* inst;
  float* m0;       // (B, D nb)
  float* m1;       // (B, D nb)
  float* best_d;   // (B)
  int8_t* best_l;  // (B, D)
  PhiloxKeys K;
};

constexpr int kSoftWarps = 8;

template <int MPL>
__global__ void __launch_bounds__(32 * kSoftWarps) k_traj_soft(const SoftParams a) {
  constexpr int TD = MPL;  // coordinates per lane (D <= N <= 32 MPL)
  extern __shared__ __align__(16) float sms[];
  const int N = a.N, D = a.D, S = a.S, R = a.R;
  const bool qam = a.M == 16;
  const int nb = qam ? 2 : 1;
  float* Js = sms;                       // N x N
  float* redm = Js + N * N;              // W x (2 D nb): m0 then m1 per warp
  float* redb = redm + kSoftWarps * 2 * D * nb;  // W x 3: best d, step, chain
  uint32_t* redS = reinterpret_cast<uint32_t*>(redb + kSoftWarps * 3);  // W x MPL: best spin masks
  const int b = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5, W = blockDim.x >> 5;
  {
    const float4* src = reinterpret_cast<const float4*>(a.J + (size_t)b * N * N);
    float4* dst = reinterpret_cast<float4*>(Js);
    for (int x = threadIdx.x; x < N * N / 4; x += blockDim.x) dst[x] = src[x];
  }
  __syncthreads();
  const uint32_t inst = a.inst[b];
  const float scale = a.scale[b], c0 = a.c0[b];
  const float* Tb = a.T + (size_t)b * S;
  float hfv[MPL], h0v[MPL];
#pragma unroll
  for (int t = 0; t < MPL; ++t) {
    const int i = t * 32 + lane;
    hfv[t] = i < N ? a.hf[(size_t)b * N + i] : 0.0f;
    h0v[t] = i < N ? a.h0[(size_t)b * N + i] : 0.0f;
  }
  const float inf = __int_as_float(0x7f800000);
  float mn0[2 * TD], mn1[2 * TD];
#pragma unroll
  for (int c = 0; c < 2 * TD; ++c) {
    mn0[c] = inf;
    mn1[c] = inf;
  }
  float wbest = inf;
  int wstep = INT_MAX, wchain = INT_MAX;
  uint32_t Wm[MPL];
#pragma unroll
  for (int t = 0; t < MPL; ++t) Wm[t] = 0u;
  const uint32_t vmask_last = (N % 32) ? ((1u << (N % 32)) - 1u) : ARP_FULL;
  for (int r = wid; r < R; r += W) {
    uint32_t Sm[MPL];
#pragma unroll
    for (int t = 0; t < MPL; ++t) {
      const int i = t * 32 + lane;
      bool up = false;
      if (i < N) {
        if (a.s0) {
          up = a.s0[(size_t)b * N + i] > 0;
        } else {
          uint32_t x0 = 0xFFFFFFFFu, x1 = (uint32_t)i, x2 = (uint32_t)r, x3 = inst;
          philox10(x0, x1, x2, x3, a.K);
          up = x0 >= 0x80000000u;
        }
      }
      Sm[t] = __ballot_sync(ARP_FULL, up);
    }
    // u = hf + 2 J s (sum in j order)
    float u[MPL];
#pragma unroll
    for (int t = 0; t < MPL; ++t) u[t] = 0.0f;
    for (int j = 0; j < N; ++j) {
      const float sj = ((Sm[j >> 5] >> (j & 31)) & 1u) ? 1.0f : -1.0f;
      const float* Jr = Js + j * N + lane;
#pragma unroll
      for (int t = 0; t < MPL; ++t)
        if (t * 32 + lane < N) u[t] = __fadd_rn(u[t], __fmul_rn(Jr[t * 32], sj));
    }
#pragma unroll
    for (int t = 0; t < MPL; ++t) u[t] = __fadd_rn(hfv[t], __fmul_rn(2.0f, u[t]));
    // E0 = -sum_i s_i (h0_i + (u_i - hf_i) / 2): lane partial sums, then the warp's in lane order
    float E;
    {
      float e = 0.0f;
#pragma unroll
      for (int t = 0; t < MPL; ++t) {
        if (t * 32 + lane < N) {
          const float si = ((Sm[t] >> lane) & 1u) ? 1.0f : -1.0f;
          e = __fsub_rn(e, __fmul_rn(si, __fadd_rn(h0v[t], __fmul_rn(0.5f, __fsub_rn(u[t], hfv[t])))));
        }
      }
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) e = __fadd_rn(e, __shfl_xor_sync(ARP_FULL, e, o));
      E = e;
    }
    float cbest = inf;
    int cstep = INT_MAX;
    uint32_t Cm[MPL];
#pragma unroll
    for (int t = 0; t < MPL; ++t) Cm[t] = Sm[t];
    uint32_t cw[MPL][4];
    for (int k = 0; k < S; ++k) {
      if ((k & 3) == 0) {
#pragma unroll
        for (int t = 0; t < MPL; ++t) {
          uint32_t x0 = (uint32_t)(k >> 2), x1 = (uint32_t)(t * 32 + lane), x2 = (uint32_t)r, x3 = inst;
          philox10(x0, x1, x2, x3, a.K);
          cw[t][0] = x0;
          cw[t][1] = x1;
          cw[t][2] = x2;
          cw[t][3] = x3;
        }
      }
      const int km = k & 3;
      const float A = __fmul_rn(4.0f, Tb[k]);
      uint32_t fl[MPL];
#pragma unroll
      for (int t = 0; t < MPL; ++t) {
        const uint32_t x = km == 0 ? cw[t][0] : km == 1 ? cw[t][1] : km == 2 ? cw[t][2] : cw[t][3];
        const float thr = __fmul_rn(__fsub_rn(unit24(x), 0.5f), A);
        const float su = ((Sm[t] >> lane) & 1u) ? u[t] : -u[t];
        fl[t] = __ballot_sync(ARP_FULL, __fadd_rn(su, a.q) < thr) & (t == MPL - 1 ? vmask_last : ARP_FULL);
      }
      bool any = false;
#pragma unroll
      for (int t = 0; t < MPL; ++t) {
        uint32_t m = fl[t];
        any |= m != 0u;
        while (m) {
          const int l = __ffs(m) - 1;
          m &= m - 1u;
          const int g = t * 32 + l;
          const bool so_up = (Sm[t] >> l) & 1u;
          const float ug = __shfl_sync(ARP_FULL, u[t], l);
          const float hg = __shfl_sync(ARP_FULL, __fsub_rn(h0v[t], hfv[t]), l);
          // dE0 = 2 s_j (h0_j + u_j - hf_j)
          E = __fadd_rn(E, __fmul_rn(so_up ? 2.0f : -2.0f, __fadd_rn(hg, ug)));
          const float* Jg = Js + g * N + lane;
          const float cf = so_up ? -4.0f : 4.0f;
#pragma unroll
          for (int t2 = 0; t2 < MPL; ++t2)
            if (t2 * 32 + lane < N) u[t2] = __fadd_rn(u[t2], __fmul_rn(cf, Jg[t2 * 32]));
        }
        Sm[t] ^= fl[t];
      }
      if (any || k == 0) {
        const float d = __fadd_rn(__fmul_rn(scale, E), c0);
        // this lane's coordinates j = tc * 32 + lane and their bits
#pragma unroll
        for (int tc = 0; tc < TD; ++tc) {
          const int j = tc * 32 + lane;
          if (j < D) {
            const bool s1 = (Sm[j >> 5] >> (j & 31)) & 1u;
            if (qam) {
              const int j2 = D + j;
              const bool s2 = (Sm[j2 >> 5] >> (j2 & 31)) & 1u;
              const bool b2 = s1 != s2;
              if (s1) mn1[2 * tc] = fminf(mn1[2 * tc], d); else mn0[2 * tc] = fminf(mn0[2 * tc], d);
              if (b2) mn1[2 * tc + 1] = fminf(mn1[2 * tc + 1], d); else mn0[2 * tc + 1] = fminf(mn0[2 * tc + 1], d);
            } else {
              if (s1) mn1[2 * tc] = fminf(mn1[2 * tc], d); else mn0[2 * tc] = fminf(mn0[2 * tc], d);
            }
          }
        }
        if (d < cbest) {
          cbest = d;
          cstep = k;
#pragma unroll
          for (int t = 0; t < MPL; ++t) Cm[t] = Sm[t];
        }
      }
    }
    // this chain's best against the warp's: lowest d, then earliest step, then lowest chain
    if (cbest < wbest || (cbest == wbest && (cstep < wstep || (cstep == wstep && r < wchain)))) {
      wbest = cbest;
      wstep = cstep;
      wchain = r;
#pragma unroll
      for (int t = 0; t < MPL; ++t) Wm[t] = Cm[t];
    }
  }
  // ---- the block's minima over its warps
  const int nbits = D * nb;
#pragma unroll
  for (int tc = 0; tc < TD; ++tc) {
    const int j = tc * 32 + lane;
    if (j < D) {
      for (int c = 0; c < nb; ++c) {
        redm[(wid * 2 + 0) * nbits + j * nb + c] = mn0[2 * tc + c];
        redm[(wid * 2 + 1) * nbits + j * nb + c] = mn1[2 * tc + c];
      }
    }
  }
  if (lane == 0) {
    redb[wid * 3] = wbest;
    redb[wid * 3 + 1] = __int_as_float(wstep);
    redb[wid * 3 + 2] = __int_as_float(wchain);
  }
  if (lane == 0) {
#pragma unroll
    for (int t = 0; t < MPL; ++t) redS[wid * MPL + t] = Wm[t];
  }
  __syncthreads();
  for (int x = threadIdx.x; x < nbits; x += blockDim.x) {
    float v0 = inf, v1 = inf;
    for (int w = 0; w < W; ++w) {
      v0 = fminf(v0, redm[(w * 2) * nbits + x]);
      v1 = fminf(v1, redm[(w * 2 + 1) * nbits + x]);
    }
    a.m0[(size_t)b * nbits + x] = v0;
    a.m1[(size_t)b * nbits + x] = v1;
  }
  if (threadIdx.x < 32) {
    int bw = 0;
    for (int w = 1; w < W; ++w) {
      const float dw = redb[w * 3], db = redb[bw * 3];
      const int sw = __float_as_int(redb[w * 3 + 1]), sb = __float_as_int(redb[bw * 3 + 1]);
      const int cw2 = __float_as_int(redb[w * 3 + 2]), cb = __float_as_int(redb[bw * 3 + 2]);
      if (dw < db || (dw == db && (sw < sb || (sw == sb && cw2 < cb)))) bw = w;
    }
    if (threadIdx.x == 0) a.best_d[b] = redb[bw * 3];
    for (int j = lane; j < D; j += 32) {
      const bool s1 = (redS[bw * MPL + (j >> 5)] >> (j & 31)) & 1u;
      int l = s1 ? 1 : -1;
      if (qam) {
        const int j2 = D + j;
        const bool s2 = (redS[bw * MPL + (j2 >> 5)] >> (j2 & 31)) & 1u;
        l = 2 * l + (s2 ? 1 : -1);
      }
      a.best_l[(size_t)b * D + j] = (int8_t)l;
    }
  }
}

template <int MPL>
static cudaError_t launch_soft(const SoftParams& a, cudaStream_t st) {
  const int nb = a.M == 16 ? 2 : 1;
  const size_t smem = sizeof(float) * ((size_t)a.N * a.N + (size_t)kSoftWarps * 2 * a.D * nb + kSoftWarps * 3) +
                      sizeof(uint32_t) * kSoftWarps * MPL;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_traj_soft<MPL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  const int W = a.R < kSoftWarps ? a.R : kSoftWarps;
  k_traj_soft<MPL><<<a.B, 32 * W, smem, st>>>(a);
  return cudaGetLastError();
}

}  // namespace arp

using namespace arp;

extern "C" int arp_soft_trajectory(const float* J, const float* hf, const float* h0, const float* scale,
                                   const float* c0, const float* T, const int8_t* s0, float q, int S, int R, int D,
                                   int M, int B, const uint32_t* inst, uint32_t k0, uint32_t k1, float* m0, float* m1,
                                   float* best_d, int8_t* best_l, void* stream) {
  if (!(M == 4 || M == 16)) return ARP_ERR_SHAPE;
  const int N = M == 16 ? 2 * D : D;
  if (B < 0 || R < 1 || S < 1 || D < 1 || N > 128 || (N % 4)) return ARP_ERR_SHAPE;
  if (B == 0) return ARP_OK;
  if (!J || !hf || !h0 || !scale || !c0 || !T || !inst || !m0 || !m1 || !best_d || !best_l) return ARP_ERR_ARG;
  SoftParams a{J, hf, h0, scale, c0, T, s0, q, S, R, N, D, M, B, inst, m0, m1, best_d, best_l, philox_keys(k0, k1)};
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  switch ((N + 31) / 32) {
    case 1: e = launch_soft<1>(a, st); break;
    case 2: e = launch_soft<2>(a, st); break;
    case 3: e = launch_soft<3>(a, st); break;
    default: e = launch_soft<4>(a, st); break;
  }
  return e == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}
