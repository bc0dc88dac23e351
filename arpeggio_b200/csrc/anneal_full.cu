// FP32-field anneals on a full symmetric coupling J (N <= 128 spins): first accept and the Chord round, for
// problems without the dDI structure (the RI map of mimo.ising, mimo.py:132-149, "each PAM-4 coordinate as
// 2 s1 + s2").  The float rule is arpx55.arpeggio_seq's (arpeggio/sim/arpx55.py:28-99, rule (2)) with Philox draws:
//   u = h + 2 J s (sum in j order), thr = ((x >> 8) 2^-24 - 1/2) 4T, flip iff (s u + q) < thr,
//   de += 2 s_g u_g, u_i += (-4 s_g) J_ig, one IEEE rounding per operation.
// N spins in P banks of D = N/P lanes (D a multiple of 32); pass k tests bank k % P.  One warp per anneal, lane i of
// slot t is spin t*32 + lane; J in shared memory (row j = column j by symmetry, so every access is lane-contiguous);
// spins are warp-uniform masks; Philox counters (n>>2, i, r, inst), word n&3, as the integer kernels.
#include <cfloat>
#include <climits>

#include "arp_common.cuh"
#include "arp_internal.h"

namespace arp {

struct FullParams {
  const float *J, *h, *T, *c;
  const int8_t* s0;  // (B, N) start spins, or null: 'rand'
  int L;
  float q;
  int P, R, N, B;
  const uint32_t* inst;
  int8_t* out_s;     // (B, R, N)
  float* out_de;     // (B, R)
  int64_t* out_st;   // (B, R, 2)
  PhiloxKeys K;
};

template <int MPL, bool CHORD>
__global__ void __launch_bounds__(256) k_anneal_full_f32(const FullParams a) {
  extern __shared__ __align__(16) float smf[];
  const int N = a.N, P = a.P, R = a.R, L = a.L, D = N / P, tpc = D / 32;
  float* Js = smf;
  float* sh = Js + N * N;
  const int b = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5, W = blockDim.x >> 5;
  {
    const float4* src = reinterpret_cast<const float4*>(a.J + (size_t)b * N * N);
    float4* dst = reinterpret_cast<float4*>(Js);
    for (int x = threadIdx.x; x < N * N / 4; x += blockDim.x) dst[x] = src[x];
    for (int x = threadIdx.x; x < N; x += blockDim.x) sh[x] = a.h[(size_t)b * N + x];
  }
  __syncthreads();
  const uint32_t inst = a.inst[b];
  for (int r = wid; r < R; r += W) {
    uint32_t Sm[MPL], Bm[MPL];
#pragma unroll
    for (int t = 0; t < MPL; ++t) {
      const int i = t * 32 + lane;
      bool up;
      if (a.s0) {
        up = a.s0[(size_t)b * N + i] > 0;
      } else {
        uint32_t c0 = 0xFFFFFFFFu, c1 = (uint32_t)i, c2 = (uint32_t)r, c3 = inst;
        philox10(c0, c1, c2, c3, a.K);
        up = c0 >= 0x80000000u;
      }
      Sm[t] = __ballot_sync(ARP_FULL, up);
      Bm[t] = Sm[t];
    }
    float u[MPL];
#pragma unroll
    for (int t = 0; t < MPL; ++t) u[t] = 0.0f;
#pragma unroll
    for (int tj = 0; tj < MPL; ++tj)
      for (int l = 0; l < 32; ++l) {
        const float sj = ((Sm[tj] >> l) & 1u) ? 1.0f : -1.0f;
        const float* Jr = Js + (tj * 32 + l) * N + lane;
#pragma unroll
        for (int t = 0; t < MPL; ++t) u[t] = __fadd_rn(u[t], __fmul_rn(Jr[t * 32], sj));
      }
#pragma unroll
    for (int t = 0; t < MPL; ++t) u[t] = __fadd_rn(sh[t * 32 + lane], __fmul_rn(2.0f, u[t]));
    float de = 0.0f, best = __int_as_float(0x7f800000);
    int32_t ballots = 0, lastflips = 0, passes = 0;
    uint32_t cw[MPL][4];
    for (int k = 0; k < L; ++k) {
      const int p = k % P, n = k / P;
      if ((k % (4 * P)) == 0) {  // a new quad of sweeps: one Philox block per spin serves four sweeps
#pragma unroll
        for (int t = 0; t < MPL; ++t) {
          uint32_t c0 = (uint32_t)(n >> 2), c1 = (uint32_t)(t * 32 + lane), c2 = (uint32_t)r, c3 = inst;
          philox10(c0, c1, c2, c3, a.K);
          cw[t][0] = c0;
          cw[t][1] = c1;
          cw[t][2] = c2;
          cw[t][3] = c3;
        }
      }
      ++passes;
      const int nm = n & 3;
      const float A = __fmul_rn(4.0f, a.T[k]);
      const float qk = (CHORD && a.c) ? __fsub_rn(a.q, a.c[k]) : a.q;
      float thr[MPL];
#pragma unroll
      for (int t = 0; t < MPL; ++t) {
        const uint32_t x = nm == 0 ? cw[t][0] : nm == 1 ? cw[t][1] : nm == 2 ? cw[t][2] : cw[t][3];
        thr[t] = __fmul_rn(__fsub_rn(unit24(x), 0.5f), A);
      }
      auto accept = [&](int t) -> bool {
        const float su = ((Sm[t] >> lane) & 1u) ? u[t] : -u[t];
        return __fadd_rn(su, qk) < thr[t];
      };
      auto commit = [&](int ts, int l) {
        const int g = ts * 32 + l;
        const bool so_up = (Sm[ts] >> l) & 1u;
        float ug = u[0];
#pragma unroll
        for (int t = 1; t < MPL; ++t)
          if (t == ts) ug = u[t];
        ug = __shfl_sync(ARP_FULL, ug, l);
        de = __fadd_rn(de, __fmul_rn(so_up ? 2.0f : -2.0f, ug));
        const float* Jg = Js + g * N + lane;
        const float cf = so_up ? -4.0f : 4.0f;
#pragma unroll
        for (int t = 0; t < MPL; ++t) u[t] = __fadd_rn(u[t], __fmul_rn(cf, Jg[t * 32]));
#pragma unroll
        for (int t = 0; t < MPL; ++t)
          if (t == ts) Sm[t] ^= 1u << l;
      };
      if constexpr (!CHORD) {
        // the scan finishes slot t before slot t + 1 (a round accepts only after the last flip, so a slot the
        // scan has left has no candidate left this pass): one ballot of one slot per round, the same flips
        int jl = -1;
        ++ballots;  // the round that finds no further flip (ballots = flips + 1 per pass)
#pragma unroll
        for (int t = 0; t < MPL; ++t) {
          if (t / tpc != p) continue;
          for (;;) {
            const uint32_t m = __ballot_sync(ARP_FULL, accept(t) && t * 32 + lane > jl);
            if (m == 0) break;
            ++ballots;
            const int l = __ffs(m) - 1;
            commit(t, l);
            jl = t * 32 + l;
          }
        }
        if (jl == (p + 1) * D - 1) ++lastflips;
      } else {
        uint32_t am[MPL];
#pragma unroll
        for (int t = 0; t < MPL; ++t) am[t] = (t / tpc == p) ? __ballot_sync(ARP_FULL, accept(t)) : 0u;
        ++ballots;
#pragma unroll
        for (int t = 0; t < MPL; ++t) {
          uint32_t m = am[t];
          while (m) {
            const int l = __ffs(m) - 1;
            m &= m - 1u;
            // Chord commits against the snapshot decisions; Sm[t] bit l is still the old spin here
            commit(t, l);
            ++ballots;
          }
        }
      }
      if (de < best) {
        best = de;
#pragma unroll
        for (int t = 0; t < MPL; ++t) Bm[t] = Sm[t];
      }
    }
    const size_t ar = (size_t)b * R + r;
#pragma unroll
    for (int t = 0; t < MPL; ++t) a.out_s[ar * N + t * 32 + lane] = ((Bm[t] >> lane) & 1u) ? 1 : -1;
    if (lane == 0) {
      a.out_de[ar] = best;
      a.out_st[2 * ar] = ballots - passes;
      a.out_st[2 * ar + 1] = CHORD ? passes : ballots - lastflips;
    }
  }
}

template <int MPL>
static cudaError_t launch_full(const FullParams& a, int policy, cudaStream_t st) {
  const size_t smem = sizeof(float) * ((size_t)a.N * a.N + a.N);
  auto kern = policy == 0 ? k_anneal_full_f32<MPL, false> : k_anneal_full_f32<MPL, true>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  const int W = a.R < 8 ? a.R : 8;
  kern<<<a.B, 32 * W, smem, st>>>(a);
  return cudaGetLastError();
}

}  // namespace arp

using namespace arp;

extern "C" int arp_anneal_full_f32(int policy, const float* J, const float* h, const int8_t* s0, const float* T,
                                   const float* c, int L, float q, int P, int R, int N, int B, const uint32_t* inst,
                                   uint32_t k0, uint32_t k1, int8_t* out_s, float* out_de, int64_t* out_st,
                                   void* stream) {
  if (B < 0 || R < 1 || L < 1 || P < 1 || N < 32 || N > 128 || N % 32 || N % P || (N / P) % 32) return ARP_ERR_SHAPE;
  if (policy != 0 && policy != 1) return ARP_ERR_ARG;
  if (B == 0) return ARP_OK;
  if (!J || !h || !T || !inst || !out_s || !out_de || !out_st) return ARP_ERR_ARG;
  FullParams a{J, h, T, c, s0, L, q, P, R, N, B, inst, out_s, out_de, out_st, philox_keys(k0, k1)};
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  switch (N / 32) {
    case 1: e = launch_full<1>(a, policy, st); break;
    case 2: e = launch_full<2>(a, policy, st); break;
    case 3: e = launch_full<3>(a, policy, st); break;
    default: e = launch_full<4>(a, policy, st); break;
  }
  return e == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}
