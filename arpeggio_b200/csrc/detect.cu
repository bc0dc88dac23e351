// Detector stages around the anneal: Gram/field formation with the MMSE guess (map) and the readout.
//
// map (one block per channel use; mimo.py:98-109 mmse, :176-182 _mu, :86-88 quantize_levels,
// :506-523 ising_delta_at, chordfx.py:60-76 to_fixed, chord_ref.py:47-59 compress):
//   Q = H^T H and g = H^T y, streamed over 32-row chunks of H (every Q_ij and Q_ji is the same ordered
//   sum, so Q is exactly symmetric, as the symmetrised J of to_fixed);
//   A = Q + sigma2 I inverted in shared memory (Gauss-Jordan; A is SPD), z = A^-1 g, mu = diag(A^-1 Q),
//   x_q = nearest level of z / mu (first level on ties);
//   h = 2 (g - Q x_q) = 2 H^T (y - H x_q);  scale = max(|h|_inf, |Q|_inf) clamped at 1e-12;
//   integer problem: G = round(Q / scale * 4096), h = round(h / scale * 4096) (half to even, torch.round);
//   float problem: G = Q / scale, h = h / scale.  G is symmetric, so it is also its own transpose Gt.
// readout (mimo.py:185-190 spins_to_levels_delta, :416-425 dist/select, :45-51 levels_to_bits):
//   candidate r: x = clip(x_q + sum_p s_p) to the constellation; dist = ||y - H x||^2; the first
//   minimum over the R candidates then the guess x_q; Gray bits per dimension, MSB first.
#include <cfloat>

#include "arp_common.cuh"

namespace arp {

constexpr int kMapThreads = 256;
constexpr int kChunk = 32;
constexpr int kMaxE = 64;  // Gram entries per thread: D^2 / 256 for D <= 128

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
};

__device__ __forceinline__ float nearest_level(float v, int M) {
  if (M == 4) return fabsf(v - 1.0f) < fabsf(v + 1.0f) ? 1.0f : -1.0f;  // ties -> the first level, -1
  float best = -3.0f, bd = fabsf(v + 3.0f);
#pragma unroll
  for (int i = 1; i < 4; ++i) {
    const float lv = -3.0f + 2.0f * i;
    const float d = fabsf(v - lv);
    if (d < bd) {
      bd = d;
      best = lv;
    }
  }
  return best;
}

__global__ void __launch_bounds__(kMapThreads) k_map_dd(const MapParams a) {
  extern __shared__ __align__(16) float sm[];
  const int D = a.D, NR2 = a.NR2, DP = D + 1;
  float* Hc = sm;                 // kChunk x D
  float* Qs = Hc + kChunk * D;    // D x DP
  float* Ai = Qs + D * DP;        // D x DP
  float* gv = Ai + D * DP;        // D
  float* xv = gv + D;             // D
  float* rk = xv + D;             // D
  float* ck = rk + D;             // D
  float* red = ck + D;            // 32
  const int tid = threadIdx.x, b = blockIdx.x;
  const float* Hb = a.H + (size_t)b * NR2 * D;
  const float* yb = a.y + (size_t)b * NR2;
  float acc[kMaxE];
#pragma unroll
  for (int m = 0; m < kMaxE; ++m) acc[m] = 0.0f;
  float gacc = 0.0f;
  for (int r0 = 0; r0 < NR2; r0 += kChunk) {
    const int nr = min(kChunk, NR2 - r0);
    __syncthreads();
    for (int x = tid; x < nr * D; x += kMapThreads) Hc[x] = Hb[(size_t)r0 * D + x];
    __syncthreads();
#pragma unroll
    for (int m = 0; m < kMaxE; ++m) {
      const int e = tid + m * kMapThreads;
      if (e < D * D) {
        const int i = e / D, j = e - (e / D) * D;
        float s = acc[m];
        for (int r = 0; r < nr; ++r) s = __fmaf_rn(Hc[r * D + i], Hc[r * D + j], s);
        acc[m] = s;
      }
    }
    if (tid < D)
      for (int r = 0; r < nr; ++r) gacc = __fmaf_rn(Hc[r * D + tid], yb[r0 + r], gacc);
  }
  float qmax = 0.0f;
#pragma unroll
  for (int m = 0; m < kMaxE; ++m) {
    const int e = tid + m * kMapThreads;
    if (e < D * D) {
      const int i = e / D, j = e - (e / D) * D;
      Qs[i * DP + j] = acc[m];
      Ai[i * DP + j] = i == j ? __fadd_rn(acc[m], a.sigma2[b]) : acc[m];
      qmax = fmaxf(qmax, fabsf(acc[m]));
    }
  }
  if (tid < D) gv[tid] = gacc;
  // ---- in-place Gauss-Jordan inverse of A (SPD, no pivoting)
  for (int k = 0; k < D; ++k) {
    __syncthreads();
    if (tid < D) {
      rk[tid] = Ai[k * DP + tid];
      ck[tid] = Ai[tid * DP + k];
    }
    __syncthreads();
    const float inv = __frcp_rn(rk[k]);
    for (int e = tid; e < D * D; e += kMapThreads) {
      const int i = e / D, j = e - (e / D) * D;
      float v;
      if (i == k)
        v = j == k ? inv : __fmul_rn(rk[j], inv);
      else if (j == k)
        v = -__fmul_rn(ck[i], inv);
      else
        v = __fmaf_rn(-__fmul_rn(ck[i], inv), rk[j], Ai[i * DP + j]);
      Ai[i * DP + j] = v;
    }
  }
  __syncthreads();
  // ---- z = A^-1 g, mu = diag(A^-1 Q), x_q
  if (tid < D) {
    float z = 0.0f, mu = 0.0f;
    for (int j = 0; j < D; ++j) {
      z = __fmaf_rn(Ai[tid * DP + j], gv[j], z);
      mu = __fmaf_rn(Ai[tid * DP + j], Qs[j * DP + tid], mu);
    }
    const float lv = nearest_level(__fdiv_rn(z, mu), a.M);
    xv[tid] = lv;
    a.xq[(size_t)b * D + tid] = (int8_t)lv;
  }
  __syncthreads();
  // ---- h = 2 (g - Q x_q), scale
  float hval = 0.0f;
  if (tid < D) {
    float s = 0.0f;
    for (int j = 0; j < D; ++j) s = __fmaf_rn(Qs[tid * DP + j], xv[j], s);
    hval = __fmul_rn(2.0f, __fsub_rn(gv[tid], s));
    qmax = fmaxf(qmax, fabsf(hval));
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) qmax = fmaxf(qmax, __shfl_xor_sync(ARP_FULL, qmax, o));
  if ((tid & 31) == 0) red[tid >> 5] = qmax;
  __syncthreads();
  float sc = 0.0f;
  for (int w = 0; w < kMapThreads / 32; ++w) sc = fmaxf(sc, red[w]);
  sc = fmaxf(sc, 1e-12f);
  if (tid == 0) a.scale[b] = sc;
  // ---- outputs
  if (a.qscale > 0.0f) {
    int32_t* Go = reinterpret_cast<int32_t*>(a.G) + (size_t)b * D * D;
    for (int e = tid; e < D * D; e += kMapThreads) {
      const int i = e / D, j = e - (e / D) * D;
      Go[e] = (int32_t)rintf(__fmul_rn(__fdiv_rn(Qs[i * DP + j], sc), a.qscale));
    }
    if (tid < D)
      reinterpret_cast<int32_t*>(a.h)[(size_t)b * D + tid] = (int32_t)rintf(__fmul_rn(__fdiv_rn(hval, sc), a.qscale));
  } else {
    float* Go = reinterpret_cast<float*>(a.G) + (size_t)b * D * D;
    for (int e = tid; e < D * D; e += kMapThreads) {
      const int i = e / D, j = e - (e / D) * D;
      Go[e] = __fdiv_rn(Qs[i * DP + j], sc);
    }
    if (tid < D) reinterpret_cast<float*>(a.h)[(size_t)b * D + tid] = __fdiv_rn(hval, sc);
  }
}

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
};

constexpr int kReadThreads = 256;

__global__ void __launch_bounds__(kReadThreads) k_readout_dd(const ReadParams a) {
  extern __shared__ __align__(16) float sm[];
  const int D = a.D, NR2 = a.NR2, P = a.P, R = a.R, b = blockIdx.x;
  float* Hs = sm;                   // NR2 x D
  float* ys = Hs + NR2 * D;         // NR2
  float* xs = ys + NR2;             // 8 warps x D candidate levels
  float* bd = xs + 8 * D;           // 8
  int* br = reinterpret_cast<int*>(bd + 8);
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, W = kReadThreads / 32;
  const float lo = a.M == 4 ? -1.0f : -3.0f, hi = -lo;
  for (int x = tid; x < NR2 * D; x += kReadThreads) Hs[x] = a.H[(size_t)b * NR2 * D + x];
  for (int x = tid; x < NR2; x += kReadThreads) ys[x] = a.y[(size_t)b * NR2 + x];
  __syncthreads();
  float best = FLT_MAX;
  int bi = INT_MAX;
  float* xw = xs + wid * D;
  for (int c = wid; c <= R; c += W) {
    for (int j = lane; j < D; j += 32) {
      float v = (float)a.xq[(size_t)b * D + j];
      if (c < R) {
        const int8_t* s = a.spins + ((size_t)b * R + c) * P * D;
        int d = 0;
        for (int p = 0; p < P; ++p) d += s[p * D + j];
        v = fminf(fmaxf(v + (float)d, lo), hi);
      }
      xw[j] = v;
    }
    __syncwarp();
    float acc = 0.0f;
    for (int i = lane; i < NR2; i += 32) {
      float r = ys[i];
      for (int j = 0; j < D; ++j) r = __fmaf_rn(-Hs[i * D + j], xw[j], r);
      acc = __fmaf_rn(r, r, acc);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(ARP_FULL, acc, o);
    if (acc < best) {
      best = acc;
      bi = c;
    }
    __syncwarp();
  }
  if (lane == 0) {
    bd[wid] = best;
    br[wid] = bi;
  }
  __syncthreads();
  float gb = FLT_MAX;
  int gi = INT_MAX;
  for (int w = 0; w < W; ++w)
    if (bd[w] < gb || (bd[w] == gb && br[w] < gi)) {
      gb = bd[w];
      gi = br[w];
    }
  const int nb = a.M == 4 ? 1 : 2;
  for (int j = tid; j < D; j += kReadThreads) {
    int v = a.xq[(size_t)b * D + j];
    if (gi < R) {
      const int8_t* s = a.spins + ((size_t)b * R + gi) * P * D;
      int d = 0;
      for (int p = 0; p < P; ++p) d += s[p * D + j];
      v = min(max(v + d, (int)lo), (int)hi);
    }
    a.levels[(size_t)b * D + j] = (int8_t)v;
    if (nb == 1) {
      a.bits[(size_t)b * D + j] = v > 0;
    } else {
      a.bits[(size_t)b * D * 2 + 2 * j] = v > 0;
      a.bits[(size_t)b * D * 2 + 2 * j + 1] = (v == 1 || v == -1);
    }
  }
  if (tid == 0) {
    a.dist[b] = gb;
    if (a.pick) a.pick[b] = gi;
  }
}

}  // namespace arp

using namespace arp;

extern "C" int arp_map_dd(const float* H, const float* y, const float* sigma2, int B, int NR2, int D, int M,
                          int quantize, void* G, void* h, int8_t* xq, float* scale, int32_t* status, void* stream) {
  if (B < 0 || D < 1 || D > 128 || NR2 < 1 || NR2 > 1024 || !(M == 4 || M == 16)) return ARP_ERR_SHAPE;
  if (B == 0) return ARP_OK;
  if (!H || !y || !sigma2 || !G || !h || !xq || !scale) return ARP_ERR_ARG;
  MapParams a{H, y, sigma2, B, NR2, D, M, quantize ? 4096.0f : 0.0f, G, h, xq, scale, status};
  const size_t smem = sizeof(float) * ((size_t)kChunk * D + 2 * (size_t)D * (D + 1) + 4 * (size_t)D + 32);
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(k_map_dd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return ARP_ERR_LAUNCH;
  k_map_dd<<<B, kMapThreads, smem, (cudaStream_t)stream>>>(a);
  return cudaGetLastError() == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_readout_dd(const float* H, const float* y, const int8_t* xq, const int8_t* spins, int B, int NR2,
                              int D, int P, int R, int M, int8_t* levels, int8_t* bits, float* dist, int32_t* pick,
                              void* stream) {
  if (B < 0 || D < 1 || D > 128 || NR2 < 1 || P < 1 || P > 6 || R < 0 || !(M == 4 || M == 16)) return ARP_ERR_SHAPE;
  if (B == 0) return ARP_OK;
  if (!H || !y || !xq || (R > 0 && !spins) || !levels || !bits || !dist) return ARP_ERR_ARG;
  const size_t smem = sizeof(float) * ((size_t)NR2 * D + NR2 + 8 * (size_t)D + 8) + 8 * sizeof(int);
  if (smem > 227 * 1024) return ARP_ERR_SHAPE;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(k_readout_dd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return ARP_ERR_LAUNCH;
  ReadParams a{H, y, xq, spins, B, NR2, D, P, R, M, levels, bits, dist, pick};
  k_readout_dd<<<B, kReadThreads, smem, (cudaStream_t)stream>>>(a);
  return cudaGetLastError() == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}
