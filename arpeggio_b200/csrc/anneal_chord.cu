// Fixed-point Chord on a full int16 coupling (N <= 256 spins): the contract of chord_kernel.cu:177-184 and
// the bit-exact definition chordfx.chord_fx (chordfx.py:80-118).
//
// One block per problem, one warp per anneal (warps take r = w, w + W, ...).  Thread `lane` owns spins
// a = t*32 + lane (t < MPL = N/32) with their fields u[t] in registers; J sits in shared memory as given
// (row-major int16).  J is symmetric (chordfx.to_fixed symmetrises it before rounding), so row j serves both
// the field start u = h + 2 J s (loop over j, contiguous reads) and the rank-1 update after a flip of j.
//
// Step k tests only copy p = k % P (spins [p N/P, (p+1) N/P)): z = s u + q - c_k (flipped at k-1 ? -1 : 1),
// flip iff x 4T > (z + 2T) 2^32, evaluated as the 32-bit compare s u < ceil(x 4T / 2^32) - 2T - q + c_k sgn.
// All accepted spins of the step commit in index order against the snapshot decisions; the energy
// 2 E0 = sum s (h - 2 h0 - u) moves by 4 s_j (u_j - h_j + h0_j) - 8 J_jj per flip (u_j after earlier
// commits), which equals chord_fx's recomputation for symmetric J.  Best state: first minimum over steps.
#include <climits>

#include "arp_common.cuh"

namespace arp {

struct ChordParams {
  const int16_t* J;
  const int32_t *h, *h0, *T, *C;
  int q, S, P, R, N, B;
  uint32_t k0, k1, inst0;
  int mode;
  long long* out_e;
  int8_t* out_s;
  unsigned long long* stats;
  int32_t* status;
};

template <int MPL>
__global__ void __launch_bounds__(256) k_chord_full(const ChordParams a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int N = a.N;
  int16_t* Js = reinterpret_cast<int16_t*>(smem);
  int32_t* sh = reinterpret_cast<int32_t*>(smem + ((N * N * 2 + 15) & ~15));
  int32_t* sh0 = sh + N;
  long long* red_e = reinterpret_cast<long long*>(sh0 + N);  // 8 warps
  int* red_r = reinterpret_cast<int*>(red_e + 8);
  __shared__ int s_bad;
  const int b = blockIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, W = blockDim.x >> 5;
  if (threadIdx.x == 0) s_bad = 0;
  __syncthreads();
  {
    const int4* src = reinterpret_cast<const int4*>(a.J + (size_t)b * N * N);
    int4* dst = reinterpret_cast<int4*>(Js);
    for (int x = threadIdx.x; x < N * N / 8; x += blockDim.x) dst[x] = src[x];
    bool bad = false;
    for (int x = threadIdx.x; x < N; x += blockDim.x) {
      const int32_t hv = a.h[(size_t)b * N + x], h0v = a.h0[(size_t)b * N + x];
      sh[x] = hv;
      sh0[x] = h0v;
      bad |= hv > (1 << 28) || hv < -(1 << 28) || h0v > (1 << 28) || h0v < -(1 << 28);
    }
    for (int x = threadIdx.x; x < a.S; x += blockDim.x)
      bad |= a.T[x] > (1 << 26) || a.T[x] < -(1 << 26) || a.C[x] > (1 << 26) || a.C[x] < -(1 << 26);
    bad |= a.q > (1 << 26) || a.q < -(1 << 26);
    if (bad) s_bad = 1;
  }
  __syncthreads();
  if (s_bad) {
    if (threadIdx.x == 0) set_status(a.status, ARP_ERR_RANGE);
    return;
  }
  const uint32_t inst = a.inst0 + (uint32_t)b;
  const int P = a.P, S = a.S, R = a.R;
  const int tpc = (N / P) >> 5;
  int32_t hv[MPL], hd[MPL];
  int cp[MPL];
#pragma unroll
  for (int t = 0; t < MPL; ++t) {
    const int i = t * 32 + lane;
    hv[t] = sh[i];
    hd[t] = sh[i] - 2 * sh0[i];
    cp[t] = t / tpc;
  }
  long long wbest_e = LLONG_MAX;
  int wbest_r = INT_MAX;
  uint32_t wbest_bits = 0;
  unsigned long long n_flip = 0, n_eval = 0, n_rng = 0;
  for (int r = wid; r < R; r += W) {
    uint32_t Sm[MPL];
#pragma unroll
    for (int t = 0; t < MPL; ++t) {
      uint32_t c0 = 0xFFFFFFFFu, c1 = (uint32_t)(t * 32 + lane), c2 = (uint32_t)r, c3 = inst;
      philox10(c0, c1, c2, c3, a.k0, a.k1);
      Sm[t] = __ballot_sync(ARP_FULL, c0 >= 0x80000000u);
    }
    int32_t u[MPL];
#pragma unroll
    for (int t = 0; t < MPL; ++t) u[t] = 0;
#pragma unroll
    for (int tj = 0; tj < MPL; ++tj) {
      for (int l = 0; l < 32; ++l) {
        const int16_t* Jj = Js + (tj * 32 + l) * N + lane;
        const bool up = (Sm[tj] >> l) & 1u;
#pragma unroll
        for (int t = 0; t < MPL; ++t) u[t] += up ? (int32_t)Jj[t * 32] : -(int32_t)Jj[t * 32];
      }
    }
    long long e = 0;
#pragma unroll
    for (int t = 0; t < MPL; ++t) {
      u[t] = hv[t] + 2 * u[t];
      e += (long long)(((Sm[t] >> lane) & 1u) ? 1 : -1) * (hd[t] - u[t]);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) e += __shfl_xor_sync(ARP_FULL, e, o);
    uint32_t rw[MPL][4];
    uint32_t pf[MPL];
#pragma unroll
    for (int t = 0; t < MPL; ++t) pf[t] = 0;
    long long best_e = 1LL << 62;
    uint32_t best_bits = 0;
    int p = 0, n = 0;
    for (int k = 0; k < S; ++k) {
      const int nm = n & 3;
      const int32_t Tk = a.T[k], ck = a.C[k];
      const long long A = 4LL * Tk;
      uint32_t fl[MPL];
#pragma unroll
      for (int t = 0; t < MPL; ++t) {
        fl[t] = 0;
        if (cp[t] != p) continue;
        if (nm == 0) {
          uint32_t c0 = (uint32_t)(n >> 2), c1 = (uint32_t)(t * 32 + lane), c2 = (uint32_t)r, c3 = inst;
          philox10(c0, c1, c2, c3, a.k0, a.k1);
          rw[t][0] = c0;
          rw[t][1] = c1;
          rw[t][2] = c2;
          rw[t][3] = c3;
          if (a.stats) ++n_rng;
        }
        const uint32_t x = nm == 0 ? rw[t][0] : nm == 1 ? rw[t][1] : nm == 2 ? rw[t][2] : rw[t][3];
        const bool up = (Sm[t] >> lane) & 1u;
        const int32_t su = up ? u[t] : -u[t];
        const int32_t thr = (int32_t)ceil_shift32(x, A) - 2 * Tk - a.q + (((pf[t] >> lane) & 1u) ? -ck : ck);
        fl[t] = __ballot_sync(ARP_FULL, su < thr);
      }
      bool any = false;
#pragma unroll
      for (int t = 0; t < MPL; ++t) {
        uint32_t m = fl[t];
        if (m) {
          any = true;
          while (m) {
            const int l = __ffs(m) - 1;
            m &= m - 1u;
            const int j = t * 32 + l;
            const int32_t so4 = ((Sm[t] >> l) & 1u) ? 4 : -4;
            const int32_t uj = __shfl_sync(ARP_FULL, u[t], l);
            const int16_t* Jj = Js + j * N + lane;
            e += (long long)so4 * (uj - sh[j] + sh0[j]) - 8LL * Js[j * N + j];
#pragma unroll
            for (int tt = 0; tt < MPL; ++tt) u[tt] -= so4 * (int32_t)Jj[tt * 32];
            if (a.stats) ++n_flip;
          }
          Sm[t] ^= fl[t];
        }
        pf[t] = fl[t];
      }
      if (++p == P) {
        p = 0;
        ++n;
      }
      if (any || k == 0) {
        if (a.stats) ++n_eval;
        if (e < best_e) {
          best_e = e;
          best_bits = 0;
#pragma unroll
          for (int t = 0; t < MPL; ++t) best_bits |= ((Sm[t] >> lane) & 1u) << t;
        }
      }
    }
    if (a.mode == 0) {
      if (lane == 0) a.out_e[(size_t)b * R + r] = best_e;
#pragma unroll
      for (int t = 0; t < MPL; ++t)
        a.out_s[((size_t)b * R + r) * N + t * 32 + lane] = ((best_bits >> t) & 1u) ? 1 : -1;
    } else if (best_e < wbest_e) {
      wbest_e = best_e;
      wbest_r = r;
      wbest_bits = best_bits;
    }
  }
  if (a.stats) {
    unsigned long long v = n_rng;
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(ARP_FULL, v, o);
    if (lane == 0) {
      atomicAdd(&a.stats[0], n_flip);
      atomicAdd(&a.stats[1], n_eval);
      atomicAdd(&a.stats[2], v);
      atomicAdd(&a.stats[3], (unsigned long long)S * (unsigned long long)((R - wid + W - 1) / W));
    }
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
      for (int t = 0; t < MPL; ++t) a.out_s[(size_t)b * N + t * 32 + lane] = ((wbest_bits >> t) & 1u) ? 1 : -1;
    }
  }
}

template <int MPL>
static cudaError_t launch_chord(const ChordParams& a, int W, cudaStream_t st) {
  const size_t smem = (size_t)((a.N * a.N * 2 + 15) & ~15) + 4 * 2 * a.N + 8 * 8 + 4 * 8;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_chord_full<MPL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_chord_full<MPL><<<a.B, 32 * W, smem, st>>>(a);
  return cudaGetLastError();
}

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
  int W = warps < 1 ? 1 : (warps > 8 ? 8 : warps);
  if (W > R) W = R;
  ChordParams a{J, h, h0, Tq, Cq, q, S, P, R, N, B, k0, k1, inst0, mode, reinterpret_cast<long long*>(out_e), out_s,
                stats, status};
  cudaError_t e;
  cudaStream_t st = (cudaStream_t)stream;
  switch (mpl) {
    case 1: e = launch_chord<1>(a, W, st); break;
    case 2: e = launch_chord<2>(a, W, st); break;
    case 3: e = launch_chord<3>(a, W, st); break;
    case 4: e = launch_chord<4>(a, W, st); break;
    case 6: e = launch_chord<6>(a, W, st); break;
    default: e = launch_chord<8>(a, W, st); break;
  }
  return e == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}
