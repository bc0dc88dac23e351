// Kernels of the multi-stage delta-Ising detector (MDI-MIMO) around the anneal: the MMSE and ordered
// MMSE-SIC guesses, the search radius per stage and guess, and the final choice between the guesses.
//
// guesses (one block per use; mimo.py:98-109 mmse, :176-182 _mu, :466-503 mmse_sic per='real'):
//   Q = H^T H, g = H^T y, P = (Q + sigma2 I)^-1 by Gauss-Jordan in shared memory;
//   MMSE guess: nearest level of z_i / mu_i, z = P g, mu = diag(P Q);
//   SIC: D stages; each picks the active stream with the smallest diag(P) (first on ties), decides it from
//   z_j = (P g)_j and mu_j = (P Q)_jj over the active set, cancels it (g -= Q[:, j] x_j) and removes it from
//   the active set.  Removing stream j from the regularised inverse is the Schur complement
//   P <- P - P[:, j] P[j, :] / P_jj with row and column j cleared, which equals the reference's fresh
//   inverse of the masked Gram plus sigma2 I (its inactive streams decouple) up to rounding.
// radius (mimo.py:526-543, heuristic 'mean'): Gamma = 2 ||H^T (y - H x_g)|| / mean(diag(H^T H)); R = omega
//   if 2 omega <= Gamma else floor(Gamma / 2), clamped to [0, Rmax]; with ||y - H x_g||^2 for the selection.
// select (mimo.py:600-602): the first guess with the lowest ||y - H x||^2; Gray bits (mimo.py:45-51).
#include <cfloat>

#include "arp_common.cuh"
#include "arp_internal.h"

namespace arp {

constexpr int kGThreads = 256;

__device__ __forceinline__ float nearest_level_m(float v, int M) {
  if (M == 4) return fabsf(v - 1.0f) < fabsf(v + 1.0f) ? 1.0f : -1.0f;
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

// Block-wide argmin (first index on ties) of v over threads; returns the index in every thread.
__device__ __forceinline__ int block_argmin(float v, int i, float* rv, int* ri) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    const float ov = __shfl_xor_sync(ARP_FULL, v, o);
    const int oi = __shfl_xor_sync(ARP_FULL, i, o);
    if (ov < v || (ov == v && oi < i)) {
      v = ov;
      i = oi;
    }
  }
  if (lane == 0) {
    rv[w] = v;
    ri[w] = i;
  }
  __syncthreads();
  float bv = rv[0];
  int bi = ri[0];
  for (int k = 1; k < kGThreads / 32; ++k)
    if (rv[k] < bv || (rv[k] == bv && ri[k] < bi)) {
      bv = rv[k];
      bi = ri[k];
    }
  __syncthreads();
  return bi;
}

struct GuessParams {
  const float *H, *y, *sigma2;
  int B, NR2, D, M;
  int8_t* xmmse;  // (B, D)
  int8_t* xsic;   // (B, D)
};

__global__ void __launch_bounds__(kGThreads) k_mdi_guess(const GuessParams a) {
  extern __shared__ __align__(16) float sm[];
  const int D = a.D, NR2 = a.NR2, DP = D + 1, b = blockIdx.x, tid = threadIdx.x;
  float* Qs = sm;              // D x DP
  float* Ps = Qs + D * DP;     // D x DP (A, then its inverse)
  float* gv = Ps + D * DP;     // D
  float* rk = gv + D;          // D
  float* ck = rk + D;          // D
  float* rv = ck + D;          // 8
  int* ri = reinterpret_cast<int*>(rv + 8);  // 8
  int* act = ri + 8;           // D
  const float* Hb = a.H + (size_t)b * NR2 * D;
  const float* yb = a.y + (size_t)b * NR2;
  const float s2 = a.sigma2[b];
  // Q and g straight from global memory (each Q_ij and Q_ji the same ordered chain)
  for (int e = tid; e < D * D; e += kGThreads) {
    const int i = e / D, j = e - i * D;
    float s = 0.0f;
    for (int r = 0; r < NR2; ++r) s = __fmaf_rn(Hb[(size_t)r * D + i], Hb[(size_t)r * D + j], s);
    Qs[i * DP + j] = s;
    Ps[i * DP + j] = i == j ? __fadd_rn(s, s2) : s;
  }
  for (int i = tid; i < D; i += kGThreads) {
    float s = 0.0f;
    for (int r = 0; r < NR2; ++r) s = __fmaf_rn(Hb[(size_t)r * D + i], yb[r], s);
    gv[i] = s;
    act[i] = 1;
  }
  // Gauss-Jordan inverse in place
  for (int k = 0; k < D; ++k) {
    __syncthreads();
    for (int x = tid; x < D; x += kGThreads) {
      rk[x] = Ps[k * DP + x];
      ck[x] = Ps[x * DP + k];
    }
    __syncthreads();
    const float inv = __frcp_rn(rk[k]);
    for (int e = tid; e < D * D; e += kGThreads) {
      const int i = e / D, j = e - i * D;
      float v;
      if (i == k)
        v = j == k ? inv : __fmul_rn(rk[j], inv);
      else if (j == k)
        v = -__fmul_rn(ck[i], inv);
      else
        v = __fmaf_rn(-__fmul_rn(ck[i], inv), rk[j], Ps[i * DP + j]);
      Ps[i * DP + j] = v;
    }
  }
  __syncthreads();
  // MMSE guess
  for (int i = tid; i < D; i += kGThreads) {
    float z = 0.0f, mu = 0.0f;
    for (int j = 0; j < D; ++j) {
      z = __fmaf_rn(Ps[i * DP + j], gv[j], z);
      mu = __fmaf_rn(Ps[i * DP + j], Qs[j * DP + i], mu);
    }
    a.xmmse[(size_t)b * D + i] = (int8_t)nearest_level_m(__fdiv_rn(z, mu), a.M);
  }
  // ordered SIC on the downdated inverse
  for (int st = 0; st < D; ++st) {
    __syncthreads();
    float v = FLT_MAX;
    int vi = INT_MAX;
    for (int i = tid; i < D; i += kGThreads)
      if (act[i] && (Ps[i * DP + i] < v || (Ps[i * DP + i] == v && i < vi))) {
        v = Ps[i * DP + i];
        vi = i;
      }
    const int j = block_argmin(v, vi, rv, ri);
    // z_j, mu_j over the active set (inactive couplings of P are zero)
    if (tid < 32) {
      float z = 0.0f, mu = 0.0f;
      for (int k = tid; k < D; k += 32) {
        const float p = Ps[j * DP + k];
        z = __fmaf_rn(p, gv[k], z);
        mu = __fmaf_rn(p, act[k] ? Qs[k * DP + j] : 0.0f, mu);
      }
#pragma unroll
      for (int o = 16; o; o >>= 1) {
        z += __shfl_xor_sync(ARP_FULL, z, o);
        mu += __shfl_xor_sync(ARP_FULL, mu, o);
      }
      if (tid == 0) rv[0] = nearest_level_m(__fdiv_rn(z, mu), a.M);
    }
    for (int x = tid; x < D; x += kGThreads) {
      rk[x] = Ps[j * DP + x];
      ck[x] = Ps[x * DP + j];
    }
    __syncthreads();
    const float xj = rv[0];
    const float pinv = __frcp_rn(rk[j]);
    if (tid == 0) {
      a.xsic[(size_t)b * D + j] = (int8_t)xj;
      act[j] = 0;
    }
    for (int e = tid; e < D * D; e += kGThreads) {
      const int i = e / D, k = e - i * D;
      float p;
      if (i == j || k == j)
        p = 0.0f;
      else
        p = __fmaf_rn(-__fmul_rn(ck[i], pinv), rk[k], Ps[i * DP + k]);
      Ps[i * DP + k] = p;
    }
    for (int i = tid; i < D; i += kGThreads) gv[i] = __fmaf_rn(-Qs[i * DP + j], xj, gv[i]);
  }
}

struct RadiusParams {
  const float *H, *y;
  const int8_t* cur;  // (B, G, D) guesses
  int B, NR2, D, G, Rmax, omega;
  int32_t* R;         // (B, G)
  float* dist;        // (B, G)
};

// One warp per (use, guess): residual ybar = y - H x_g (lanes over rows), c = H^T ybar (lanes over columns).
__global__ void __launch_bounds__(256) k_mdi_radius(const RadiusParams a) {
  const int wg = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (wg >= a.B * a.G) return;
  const int b = wg / a.G;
  const int D = a.D, NR2 = a.NR2;
  const float* Hb = a.H + (size_t)b * NR2 * D;
  const int8_t* x = a.cur + (size_t)wg * D;
  extern __shared__ float sm[];
  float* yb = sm + (threadIdx.x >> 5) * NR2;
  float d2 = 0.0f;
  for (int i = lane; i < NR2; i += 32) {
    float r = a.y[(size_t)b * NR2 + i];
    for (int j = 0; j < D; ++j) r = __fmaf_rn(-Hb[(size_t)i * D + j], (float)x[j], r);
    yb[i] = r;
    d2 = __fmaf_rn(r, r, d2);
  }
  __syncwarp();
  float c2 = 0.0f, tr = 0.0f;
  for (int j = lane; j < D; j += 32) {
    float c = 0.0f, q = 0.0f;
    for (int i = 0; i < NR2; ++i) {
      const float h = Hb[(size_t)i * D + j];
      c = __fmaf_rn(h, yb[i], c);
      q = __fmaf_rn(h, h, q);
    }
    c2 = __fmaf_rn(c, c, c2);
    tr += q;
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    d2 += __shfl_xor_sync(ARP_FULL, d2, o);
    c2 += __shfl_xor_sync(ARP_FULL, c2, o);
    tr += __shfl_xor_sync(ARP_FULL, tr, o);
  }
  if (lane == 0) {
    const float lam = tr / (float)D;
    const float gam = 2.0f * sqrtf(c2) / lam;
    int R = (2.0f * a.omega <= gam) ? a.omega : (int)floorf(gam / 2.0f);
    R = R < 0 ? 0 : (R > a.Rmax ? a.Rmax : R);
    a.R[wg] = R;
    a.dist[wg] = d2;
  }
}

// The first guess with the lowest distance; levels and Gray bits.
__global__ void k_mdi_select(const int8_t* cur, const float* dist, int B, int D, int G, int M, int8_t* levels,
                             int8_t* bits) {
  const int b = blockIdx.x;
  int gi = 0;
  for (int g = 1; g < G; ++g)
    if (dist[(size_t)b * G + g] < dist[(size_t)b * G + gi]) gi = g;
  for (int j = threadIdx.x; j < D; j += blockDim.x) {
    const int v = cur[((size_t)b * G + gi) * D + j];
    levels[(size_t)b * D + j] = (int8_t)v;
    if (M == 4) {
      bits[(size_t)b * D + j] = v > 0;
    } else {
      bits[(size_t)b * D * 2 + 2 * j] = v > 0;
      bits[(size_t)b * D * 2 + 2 * j + 1] = (v == 1 || v == -1);
    }
  }
}

}  // namespace arp

using namespace arp;

extern "C" int arp_mdi_guesses(const float* H, const float* y, const float* sigma2, int B, int NR2, int D, int M,
                               int8_t* xmmse, int8_t* xsic, void* stream) {
  if (B < 0 || D < 1 || D > 128 || NR2 < 1 || !(M == 4 || M == 16)) return ARP_ERR_SHAPE;
  if (B == 0) return ARP_OK;
  if (!H || !y || !sigma2 || !xmmse || !xsic) return ARP_ERR_ARG;
  const size_t smem = sizeof(float) * (2 * (size_t)D * (D + 1) + 3 * (size_t)D + 8) + sizeof(int) * (8 + (size_t)D);
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(k_mdi_guess, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return ARP_ERR_LAUNCH;
  GuessParams a{H, y, sigma2, B, NR2, D, M, xmmse, xsic};
  k_mdi_guess<<<B, kGThreads, smem, (cudaStream_t)stream>>>(a);
  return cudaGetLastError() == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_mdi_radius(const float* H, const float* y, const int8_t* cur, int B, int NR2, int D, int G, int M,
                              int Rmax, int32_t* R, float* dist, void* stream) {
  if (B < 0 || D < 1 || D > 128 || NR2 < 1 || NR2 > 1024 || G < 1 || Rmax < 0 || !(M == 4 || M == 16))
    return ARP_ERR_SHAPE;
  if (B == 0) return ARP_OK;
  if (!H || !y || !cur || !R || !dist) return ARP_ERR_ARG;
  RadiusParams a{H, y, cur, B, NR2, D, G, Rmax, M == 4 ? 1 : 3, R, dist};
  const int warps = B * G;
  k_mdi_radius<<<(warps + 7) / 8, 256, sizeof(float) * 8 * NR2, (cudaStream_t)stream>>>(a);
  return cudaGetLastError() == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_mdi_select(const int8_t* cur, const float* dist, int B, int D, int G, int M, int8_t* levels,
                              int8_t* bits, void* stream) {
  if (B < 0 || D < 1 || G < 1 || !(M == 4 || M == 16)) return ARP_ERR_SHAPE;
  if (B == 0) return ARP_OK;
  if (!cur || !dist || !levels || !bits) return ARP_ERR_ARG;
  k_mdi_select<<<B, 128, 0, (cudaStream_t)stream>>>(cur, dist, B, D, G, M, levels, bits);
  return cudaGetLastError() == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_mdi_map(const float* H, const float* y, const int32_t* idx, int n, int NR2, int D, int M,
                           const int8_t* cur, int G, int gi, int quantize, void* Gout, void* hout, int8_t* xq,
                           float* scale, int32_t* status, void* stream) {
  if (n < 0 || D < 1 || D > 128 || NR2 < 1 || NR2 > 1024 || G < 1 || gi < 0 || gi >= G || !(M == 4 || M == 16))
    return ARP_ERR_SHAPE;
  if (n == 0) return ARP_OK;
  if (!H || !y || !idx || !cur || !Gout || !hout || !xq || !scale) return ARP_ERR_ARG;
  MapParams a{H, y, nullptr, n, NR2, D, M, quantize ? 4096.0f : 0.0f, Gout, hout, xq, scale, status};
  a.idx = idx;
  a.xg = cur + (size_t)gi * D;
  a.xg_stride = G * D;
  return map_dispatch(a, (cudaStream_t)stream) == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_mdi_update(const float* H, const float* y, const int32_t* idx, int n, int NR2, int D, int P, int R,
                              int M, const int8_t* cur, int G, int gi, const int8_t* spins, int8_t* next,
                              float* best_dist, void* stream) {
  if (n < 0 || D < 1 || D > 128 || NR2 < 1 || NR2 > 256 || P < 1 || P > 6 || R < 1 || G < 1 || gi < 0 || gi >= G ||
      !(M == 4 || M == 16))
    return ARP_ERR_SHAPE;
  if (n == 0) return ARP_OK;
  if (!H || !y || !idx || !cur || !spins || !next || !best_dist) return ARP_ERR_ARG;
  ReadParams a{H, y, nullptr, spins, n, NR2, D, P, R, M, nullptr, nullptr, nullptr, nullptr};
  a.idx = idx;
  a.xg = cur + (size_t)gi * D;
  a.xg_stride = G * D;
  a.bl = next + (size_t)gi * D;
  a.bd = best_dist + gi;
  a.bl_stride = G;
  a.mdi = 1;
  return readout_dispatch(a, (cudaStream_t)stream) == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}
