// Learned warm start for first-accept annealing: a per-coordinate MLP (features -> 512 -> 512 -> P+1 logits,
// BF16 weights and activations, FP32 accumulate) trained and run by this file's kernels.
//
//   k_gemm_bf16   C = A B^T on the 5th-generation tensor cores: a 128 x BN output tile per CTA accumulates in
//                 TMEM (tcgen05.mma kind::f16, one issuing thread), operands staged by cp.async into the
//                 canonical no-swizzle shared-memory layouts (K-major or MN-major per operand, so forward and
//                 both backward products use the same kernel), a 4-slot ring whose slots are released by
//                 tcgen05.commit on per-slot mbarriers; fused epilogues (bias + ReLU to bf16, bias to f32,
//                 ReLU-mask to bf16, f32 store, f32 accumulate for split K) read TMEM with tcgen05.ld.  It serves
//                 the small products (M < 128, N < 64 or K < 64); the large ones go to the TMA-fed,
//                 warp-specialised kernel of gemm_tma.cu, which shares the epilogues (gemm.cuh).
//   k_warm_features  per-coordinate features of a mapped dDI problem (and training labels).
//   k_warm_loss      softmax cross-entropy over the P+1 classes of the spin sum, its gradient in bf16.
//   k_colsum_bf16    bias gradients.
//   k_adam           Adam on FP32 master weights, writing the BF16 copies.
//   k_warm_start     logits -> per-coordinate start (spin sum m_j), flip-test order, start energy, fallback.
//
// The reference has no learned component; nothing here has a reference counterpart.
#include <cuda_bf16.h>

#include "../../include/arpeggio_b200.h"
#include "arp_common.cuh"
#include "gemm.cuh"
#include "umma.cuh"

namespace arp {

constexpr int kStages = 4;

// Stages one operand tile (R rows along M or N, 64 along K) into the canonical layout; zero fill outside.
template <bool MN, int R>
__device__ __forceinline__ void load_tile(uint32_t sbase, const bf16* g, int ld, int mn0, int mnlim, int k0, int K,
                                          int tid) {
  constexpr int CH = R * 8;
#pragma unroll
  for (int c = tid; c < CH; c += 128) {
    int mn, k;
    uint32_t off;
    const bf16* src;
    if constexpr (!MN) {
      const int row = c >> 3, kc = c & 7;
      mn = mn0 + row;
      k = k0 + kc * 8;
      off = (uint32_t)((row >> 3) * 1024 + kc * 128 + (row & 7) * 16);
      src = g + (size_t)mn * ld + k;
    } else {
      const int kr = c / (R / 8), mc = c - kr * (R / 8);
      k = k0 + kr;
      mn = mn0 + mc * 8;
      off = (uint32_t)((kr >> 3) * (R * 16) + mc * 128 + (kr & 7) * 16);
      src = g + (size_t)k * ld + mn;
    }
    const bool valid = mn < mnlim && k < K;
    umma::cp16(sbase + off, valid ? (const void*)src : (const void*)g, valid);
  }
}

template <int BN, bool AMN, bool BMN>
__global__ void __launch_bounds__(128) k_gemm_bf16(const GemmParams p) {
  constexpr int S = kStages;
  constexpr uint32_t ABYTES = 128 * 128, BBYTES = BN * 128, SBYTES = ABYTES + BBYTES;
  constexpr uint32_t NCOL = BN < 32 ? 32 : BN;
  constexpr int CW = BN < 32 ? BN : 32;
  constexpr uint32_t IDESC = umma::idesc_bf16(BN, AMN, BMN);
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ __align__(8) uint64_t bars[S];
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * 128, n0 = blockIdx.y * BN;
  const int nkt = (p.K + 63) / 64;
  const int kt0 = blockIdx.z * p.kt_per;
  const int kt1 = min(nkt, kt0 + p.kt_per);
  const int nk = kt1 - kt0;
  if (nk <= 0) return;
  const uint32_t sbase = umma::su32(smem);
  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < S; ++s) umma::mbar_init(&bars[s], 1);
    umma::fence_mbar_init();
    s_abort = 0;
  }
  if (warp == 0) umma::tmem_alloc(&s_tmem, NCOL);
  umma::tc_before_sync();
  __syncthreads();
  umma::tc_after_sync();
  const uint32_t tmem = s_tmem;

  auto load = [&](int t, int slot) {
    const uint32_t sa = sbase + (uint32_t)slot * SBYTES;
    const int k0 = (kt0 + t) * 64;
    load_tile<AMN, 128>(sa, p.A, p.lda, m0, p.M, k0, p.K, tid);
    load_tile<BMN, BN>(sa + ABYTES, p.B, p.ldb, n0, p.N, k0, p.K, tid);
  };
#pragma unroll
  for (int i = 0; i < S - 2; ++i) {
    if (i < nk) load(i, i);
    umma::cp_commit();
  }
  bool ok = true;
  for (int t = 0; t < nk; ++t) {
    const int tl = t + S - 2;
    if (tl < nk) {
      // slot tl % S was last read by the MMAs of tile t - 2
      if (t >= 2 && !umma::mbar_wait(&bars[(t - 2) % S], ((t - 2) / S) & 1)) s_abort = 1;
      load(tl, tl % S);
    }
    umma::cp_commit();
    umma::cp_wait<S - 2>();
    umma::fence_async_smem();
    __syncthreads();
    if (s_abort) {
      ok = false;
      break;
    }
    if (tid == 0) {
      umma::tc_after_sync();
      const int slot = t % S;
      const uint32_t sa = sbase + (uint32_t)slot * SBYTES, sb = sa + ABYTES;
      const int krem = p.K - (kt0 + t) * 64;
      const int nmma = krem >= 64 ? 4 : (krem + 15) / 16;
      for (int kk = 0; kk < nmma; ++kk) {
        const uint64_t ad = AMN ? umma::sdesc(sa + kk * 2 * (128 * 16), 128 * 16, 128)
                                : umma::sdesc(sa + kk * 256, 128, 1024);
        const uint64_t bd = BMN ? umma::sdesc(sb + kk * 2 * (BN * 16), BN * 16, 128)
                                : umma::sdesc(sb + kk * 256, 128, 1024);
        umma::mma(tmem, ad, bd, IDESC, (t > 0 || kk > 0) ? 1u : 0u);
      }
      umma::commit(&bars[slot]);
    }
  }
  if (ok && !umma::mbar_wait(&bars[(nk - 1) % S], ((nk - 1) / S) & 1)) s_abort = 1;
  umma::cp_wait<0>();
  __syncthreads();
  umma::tc_after_sync();
  if (!s_abort) {
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c = 0; c < BN; c += CW) {
      if (n0 + c >= p.N) break;
      uint32_t v[32];
      const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c;
      if constexpr (CW == 32)
        umma::tmem_ld32(ta, v);
      else
        umma::tmem_ld16(ta, v);
      if (row < p.M) epilogue<CW>(p, row, n0 + c, v, blockIdx.z);
    }
  } else if (tid == 0) {
    set_status(p.status, ARP_ERR_TIMEOUT);
  }
  umma::tc_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tmem, NCOL);
}

// C (M x N, leading dimension ldc) += sum over s = 0..splits-1 of part[s] (M x N, dense), summed in s order.
__global__ void __launch_bounds__(256) k_sum_splits(const float* __restrict__ part, int splits, int M, int N,
                                                    float* __restrict__ C, int ldc) {
  const size_t mn = (size_t)M * N;
  for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < mn; x += (size_t)gridDim.x * blockDim.x) {
    float acc = 0.0f;
    int z = 0;
    for (; z + 8 <= splits; z += 8) {  // eight loads in flight, added in split order
      float v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = part[(size_t)(z + u) * mn + x];
#pragma unroll
      for (int u = 0; u < 8; ++u) acc += v[u];
    }
    for (; z < splits; ++z) acc += part[(size_t)z * mn + x];
    const size_t i = x / N, j = x - i * N;
    C[i * ldc + j] += acc;
  }
}

cudaError_t sum_splits(const float* ws, int splits, int M, int N, float* C, int ldc, cudaStream_t st) {
  const size_t mn = (size_t)M * N;
  const int th = 256;
  const int nb = (int)((mn + th - 1) / th);
  k_sum_splits<<<nb < 4096 ? nb : 4096, th, 0, st>>>(ws, splits, M, N, C, ldc);
  return cudaGetLastError();
}

template <int BN, bool AMN, bool BMN>
static cudaError_t launch_gemm(GemmParams p, cudaStream_t st) {
  constexpr size_t smem = (size_t)kStages * (128 * 128 + BN * 128);
  static DeviceAttr attr;
  if (cudaError_t e = smem_attr(attr, k_gemm_bf16<BN, AMN, BMN>, smem); e != cudaSuccess) return e;
  const int gx = (p.M + 127) / 128, gy = (p.N + BN - 1) / BN, nkt = (p.K + 63) / 64;
  int split = 1;
  if (p.epi == EPI_F32_ACC) {
    const int want = (2 * 148 + gx * gy - 1) / (gx * gy);
    split = want < nkt ? want : nkt;
    if (split < 1) split = 1;
  }
  p.kt_per = (nkt + split - 1) / split;
  split = (nkt + p.kt_per - 1) / p.kt_per;
  dim3 grid(gx, gy, split);
  if (split == 1) {  // one CTA per output tile: its single add into C is already deterministic
    k_gemm_bf16<BN, AMN, BMN><<<grid, 128, smem, st>>>(p);
    return cudaGetLastError();
  }
  // split K: each split's partial tile to a stream-ordered workspace, then C += the partials in split order, so
  // the result does not depend on which split finishes first
  float* ws = nullptr;
  const size_t mn = (size_t)p.M * p.N;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&ws), mn * split * sizeof(float), st);
  if (e != cudaSuccess) return e;
  GemmParams q = p;
  q.epi = EPI_F32_PART;
  q.C = ws;
  q.ldc = p.N;
  k_gemm_bf16<BN, AMN, BMN><<<grid, 128, smem, st>>>(q);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = sum_splits(ws, split, p.M, p.N, reinterpret_cast<float*>(p.C), p.ldc, st);
  const cudaError_t ef = cudaFreeAsync(ws, st);
  return e != cudaSuccess ? e : ef;
}

template <int BN>
static cudaError_t gemm_bn(const GemmParams& p, bool amn, bool bmn, cudaStream_t st) {
  if (!amn && !bmn) return launch_gemm<BN, false, false>(p, st);
  if (!amn && bmn) return launch_gemm<BN, false, true>(p, st);
  if (amn && !bmn) return launch_gemm<BN, true, false>(p, st);
  return launch_gemm<BN, true, true>(p, st);
}

// ------------------------------------------------------------------------------------------------ features
constexpr int kFeat = 16;

// One coordinate's feature row (bf16, kFeat wide) and, with labels, its training label: the same arithmetic for
// the warp-per-problem and block-per-problem kernels.
template <typename GT>
__device__ __forceinline__ void feature_row(const GT* __restrict__ h, const int8_t* __restrict__ xq,
                                            const float* __restrict__ zs, size_t row, int Lmax, int P, float dg,
                                            float ss, float mdg, float snr, float u1, float u2, bf16* __restrict__ X,
                                            const int8_t* __restrict__ levels, int8_t* __restrict__ labels) {
  const int x = xq[row];
  float f[kFeat];
#pragma unroll
  for (int i = 0; i < kFeat; ++i) f[i] = 0.0f;
  const float hj = (float)h[row];
  f[0] = dg > 0.0f ? hj / (4.0f * dg) : 0.0f;  // best single-coordinate move, in level steps
  f[1] = mdg > 0.0f ? dg / mdg : 0.0f;
  f[2] = dg > 0.0f ? sqrtf(ss) / dg : 0.0f;  // coupling of this coordinate to the others
  f[3] = snr;
  f[4] = (float)x / (float)Lmax;
  f[5] = x == Lmax ? 1.0f : 0.0f;
  f[6] = x == -Lmax ? 1.0f : 0.0f;
  f[7] = zs ? fminf(fmaxf(0.5f * (zs[row] - (float)x), -4.0f), 4.0f) : 0.0f;  // MMSE soft residual
  f[8] = 1.0f;
  f[0] = fminf(fmaxf(f[0], -8.0f), 8.0f);
  f[2] = fminf(f[2], 64.0f);
  f[9] = u1;
  f[10] = u2;
  uint32_t pk[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const __nv_bfloat162 h2 = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
    pk[i] = *reinterpret_cast<const uint32_t*>(&h2);
  }
  uint4* o = reinterpret_cast<uint4*>(X + row * kFeat);
  o[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
  o[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
  if (labels) {
    int c = (levels[row] - x) / 2 + P / 2;
    labels[row] = (int8_t)(c < 0 ? 0 : (c > P ? P : c));
  }
}

// The greedy move of the Jacobi refinements: 2 clamp(rint(u), -1, 1), kept inside the constellation.
__device__ __forceinline__ int jacobi_move(float u, int x, int Lmax) {
  int m = 2 * (int)fminf(fmaxf(rintf(u), -1.0f), 1.0f);
  if (x + m > Lmax) m = Lmax - x;
  if (x + m < -Lmax) m = -Lmax - x;
  return m;
}

template <typename GT>
__global__ void __launch_bounds__(128) k_warm_features(const GT* __restrict__ G, const GT* __restrict__ h,
                                                       const int8_t* __restrict__ xq, const float* __restrict__ zs,
                                                       const float* __restrict__ snr_db, int B, int D, int M, int P,
                                                       bf16* __restrict__ X, const int8_t* __restrict__ levels,
                                                       int8_t* __restrict__ labels) {
  const int b = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (b >= B) return;
  const GT* Gb = G + (size_t)b * D * D;
  float dg[4] = {0, 0, 0, 0}, ss[4] = {0, 0, 0, 0};
  // the row loops carry no load dependence: unrolled so one warp keeps several rows of G in flight
#pragma unroll 8
  for (int i = 0; i < D; ++i) {
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int j = t * 32 + lane;
      if (j < D) {
        const float g = (float)Gb[(size_t)i * D + j];
        if (i == j)
          dg[t] = g;
        else
          ss[t] = fmaf(g, g, ss[t]);
      }
    }
  }
  float sdg = dg[0] + dg[1] + dg[2] + dg[3];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sdg += __shfl_xor_sync(0xffffffffu, sdg, o);
  const float mdg = sdg / (float)D;
  const int Lmax = M == 4 ? 1 : (M == 16 ? 3 : 7);
  // Two Jacobi refinements of the single-coordinate move: u_j = (h_j - 2 sum_{i != j} G_ij m_i) / 4 G_jj (level
  // steps) with every other coordinate at its previous greedy move m_i = 2 clamp(rint(u_i), -1, 1), kept inside
  // the constellation.  They see the coupling G m, which the per-coordinate network cannot.
  float u1[4], u2[4];
  {
    float hv[4];
    int mq[4], xv[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int j = t * 32 + lane;
      hv[t] = j < D ? (float)h[(size_t)b * D + j] : 0.0f;
      xv[t] = j < D ? xq[(size_t)b * D + j] : 0;
    }
    auto quant = [&](float u, int x) { return jacobi_move(u, x, Lmax); };
#pragma unroll
    for (int t = 0; t < 4; ++t) mq[t] = dg[t] > 0.0f ? quant(hv[t] / (4.0f * dg[t]), xv[t]) : 0;
#pragma unroll
    for (int pass = 0; pass < 2; ++pass) {
      float acc[4] = {0, 0, 0, 0};
#pragma unroll
      for (int ti = 0; ti < 4; ++ti) {  // rows i = 32 ti + l with m_i != 0, in order, four loads in flight
        if (ti * 32 >= D) break;
        const int src = mq[ti];
        uint32_t mk = __ballot_sync(0xffffffffu, src != 0);
        while (mk) {
          int li[4];
          float g[4][4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            li[u] = mk ? __ffs(mk) - 1 : -1;
            if (mk) mk &= mk - 1u;
          }
#pragma unroll
          for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int t = 0; t < 4; ++t) {
              const int j = t * 32 + lane;
              g[u][t] = (li[u] >= 0 && j < D) ? (float)Gb[(size_t)(ti * 32 + li[u]) * D + j] : 0.0f;
            }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (li[u] < 0) break;
            const int i = ti * 32 + li[u];
            const float mi = (float)__shfl_sync(0xffffffffu, src, li[u]);
#pragma unroll
            for (int t = 0; t < 4; ++t)
              if (t * 32 + lane < D && t * 32 + lane != i) acc[t] = fmaf(g[u][t], mi, acc[t]);
          }
        }
      }
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const float v = dg[t] > 0.0f ? (hv[t] - 2.0f * acc[t]) / (4.0f * dg[t]) : 0.0f;
        const float uc = fminf(fmaxf(v, -8.0f), 8.0f);
        if (pass == 0)
          u1[t] = uc;
        else
          u2[t] = uc;
        mq[t] = (t * 32 + lane) < D && dg[t] > 0.0f ? quant(uc, xv[t]) : 0;
      }
    }
  }
  const float snr = snr_db ? snr_db[b] * 0.05f : 0.0f;
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int j = t * 32 + lane;
    if (j < D)
      feature_row(h, xq, zs, (size_t)b * D + j, Lmax, P, dg[t], ss[t], mdg, snr, u1[t], u2[t], X, levels, labels);
  }
}

// ------------------------------------------------------------------------------------------------ loss
__global__ void __launch_bounds__(256) k_warm_loss(const float* __restrict__ logits, int ldl,
                                                   const int8_t* __restrict__ labels, int rows, int C,
                                                   bf16* __restrict__ dl, int ldd, float* loss_sum, int* correct) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.0f;
  int ok = 0;
  if (row < rows) {
    const float* z = logits + (size_t)row * ldl;
    float zm = -INFINITY;
    int am = 0;
    for (int c = 0; c < C; ++c)
      if (z[c] > zm) {
        zm = z[c];
        am = c;
      }
    float se = 0.0f;
    for (int c = 0; c < C; ++c) se += __expf(z[c] - zm);
    const int lab = labels[row];
    if (lab >= 0) {
      l = __logf(se) + zm - z[lab];
      ok = am == lab;
    }
    bf16* g = dl + (size_t)row * ldd;
    for (int c = 0; c < ldd; ++c) {
      float v = 0.0f;
      if (c < C && lab >= 0) v = __expf(z[c] - zm) / se - (c == lab ? 1.0f : 0.0f);
      g[c] = __float2bfloat16_rn(v);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    l += __shfl_xor_sync(0xffffffffu, l, o);
    ok += __shfl_xor_sync(0xffffffffu, ok, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (loss_sum) atomicAdd(loss_sum, l);
    if (correct) atomicAdd(correct, ok);
  }
}

// ------------------------------------------------------------------------------------------------ bias grads
__global__ void __launch_bounds__(256) k_colsum_bf16(const bf16* __restrict__ X, int rows, int cols, int ld,
                                                     float* __restrict__ out) {
  __shared__ float part[8][33];
  const int c = blockIdx.x * 32 + (threadIdx.x & 31), ty = threadIdx.x >> 5;
  float acc = 0.0f;
  if (c < cols)
    for (int r = blockIdx.y * 8 + ty; r < rows; r += gridDim.y * 8) acc += __bfloat162float(X[(size_t)r * ld + c]);
  part[ty][threadIdx.x & 31] = acc;
  __syncthreads();
  if (ty == 0 && c < cols) {
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += part[i][threadIdx.x & 31];
    if (gridDim.y == 1)
      out[c] += s;
    else
      out[(size_t)blockIdx.y * cols + c] = s;  // a row band's partial, summed by k_colsum_reduce
  }
}

// out[c] += sum over the gy row bands' partials, in band order.
__global__ void __launch_bounds__(256) k_colsum_reduce(const float* __restrict__ part, int gy, int cols,
                                                       float* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.0f;
  for (int y = 0; y < gy; ++y) s += part[(size_t)y * cols + c];
  out[c] += s;
}

// ------------------------------------------------------------------------------------------------ Adam
__global__ void __launch_bounds__(256) k_adam(float* __restrict__ w, bf16* __restrict__ wb,
                                              const float* __restrict__ g, float* __restrict__ m,
                                              float* __restrict__ v, int n, float lr, float b1, float b2, float eps,
                                              float bc1, float bc2, float gscale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i] * gscale;
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16_rn(wi);
}

// ------------------------------------------------------------------------------------------------ warm start
// One warp per problem.  Class c of coordinate j means the spin sum m_j = 2c - P (the move away from the guess in
// level units), clamped so the level stays in the constellation.  Flip-test order: coordinates by descending
// 1 - p(m_j = 0), ties by index.  The start is kept only when its energy e0 = 2 (m^T G m - h^T m) (the dDI energy
// change from the guess, in the units of the anneal's out_de) is no worse than the guess's (0); otherwise the
// problem falls back to the plain MMSE start (m = 0) in index order.
// One coordinate of the warm start from its logits z (C = P + 1 classes): the argmax spin sum clamped to the
// constellation (returned), the order score 1 - p(m = 0), with_cdf: the sampling thresholds of softmax(tau z)
// over the classes that stay in the constellation, and log sum_c exp(z_c - max z) (minus the log-probability of
// the argmax class).  Shared by the warp-per-problem and block-per-problem kernels.
__device__ __forceinline__ int start_coord(const float* __restrict__ z, int C, int P, int x, int Lmax, float tau,
                                           bool with_cdf, float& sc, uint2& th, float& lg) {
  float zm = z[0];
  int am = 0;
  for (int c = 1; c < C; ++c)
    if (z[c] > zm) {
      zm = z[c];
      am = c;
    }
  float se = 0.0f;
  for (int c = 0; c < C; ++c) se += __expf(z[c] - zm);
  sc = 1.0f - __expf(z[P / 2] - zm) / se;
  lg = __logf(se);
  int m = 2 * am - P;
  if (with_cdf && P == 2) {
    const bool ok0 = x - 2 >= -Lmax, ok2 = x + 2 <= Lmax;
    const float q0 = ok0 ? __expf(tau * (z[0] - zm)) : 0.0f, q1 = __expf(tau * (z[1] - zm));
    const float q2 = ok2 ? __expf(tau * (z[2] - zm)) : 0.0f, qs = q0 + q1 + q2;
    th.x = ok0 ? __float2uint_rz(q0 / qs * 4294967296.0f) : 0u;
    th.y = ok2 ? __float2uint_rz((q0 + q1) / qs * 4294967296.0f) : 0xFFFFFFFFu;
  }
  if (x + m > Lmax) m = Lmax - x;
  if (x + m < -Lmax) m = -Lmax - x;
  return m;
}

template <typename GT, typename ET>
__global__ void __launch_bounds__(128) k_warm_start(const float* __restrict__ logits, int ldl,
                                                    const GT* __restrict__ G, const GT* __restrict__ h,
                                                    const int8_t* __restrict__ xq, int B, int D, int P, int M,
                                                    int8_t* __restrict__ m0, uint8_t* __restrict__ perm,
                                                    ET* __restrict__ e0, int32_t* __restrict__ kept, float tau,
                                                    uint2* __restrict__ cdf, float conf_min, int r_easy, int R,
                                                    int32_t* __restrict__ ra) {
  const int b = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (b >= B) return;
  const int C = P + 1, Lmax = M == 4 ? 1 : (M == 16 ? 3 : 7);
  int mv[4];
  float sc[4];
  uint2 th[4];
  float lse = 0.0f;  // sum over coordinates of -log max_c p_c: minus the log-probability of the argmax start
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int j = t * 32 + lane;
    mv[t] = 0;
    sc[t] = -1.0f;
    if (j >= D) continue;
    float lg;
    mv[t] = start_coord(logits + ((size_t)b * D + j) * ldl, C, P, xq[(size_t)b * D + j], Lmax, tau, cdf != nullptr,
                        sc[t], th[t], lg);
    lse += lg;
  }
  // start energy m^T G m - h^T m
  ET e = ET(0);
  const GT* Gb = G + (size_t)b * D * D;
#pragma unroll
  for (int ti = 0; ti < 4; ++ti) {  // rows with m_i != 0 only, four loads in flight
    if (ti * 32 >= D) break;
    const int src = mv[ti];
    uint32_t mk = __ballot_sync(0xffffffffu, src != 0);
    while (mk) {
      int li[4];
      GT g[4][4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        li[u] = mk ? __ffs(mk) - 1 : -1;
        if (mk) mk &= mk - 1u;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const int j = t * 32 + lane;
          g[u][t] = (li[u] >= 0 && j < D) ? Gb[(size_t)(ti * 32 + li[u]) * D + j] : GT(0);
        }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (li[u] < 0) break;
        const int mi = __shfl_sync(0xffffffffu, src, li[u]);
#pragma unroll
        for (int t = 0; t < 4; ++t)
          if (t * 32 + lane < D) e += (ET)g[u][t] * (ET)(mi * mv[t]);
      }
    }
  }
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int j = t * 32 + lane;
    if (j < D) e -= (ET)h[(size_t)b * D + j] * (ET)mv[t];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  e = e + e;  // the anneal's energy units: a flip moves out_de by 4 s w_j + 8 G_jj = 2 x the change of this form
  const bool keep = e <= ET(0);
  // ranks by descending score
  int rk[4] = {0, 0, 0, 0};
#pragma unroll
  for (int ti = 0; ti < 4; ++ti) {
    if (ti * 32 >= D) break;
    const float src = sc[ti];
    const int nl = min(32, D - ti * 32);
#pragma unroll 8
    for (int l = 0; l < nl; ++l) {
      const int i = ti * 32 + l;
      const float si = __shfl_sync(0xffffffffu, src, l);
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int j = t * 32 + lane;
        if (si > sc[t] || (si == sc[t] && i < j)) ++rk[t];
      }
    }
  }
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int j = t * 32 + lane;
    if (j >= D) continue;
    m0[(size_t)b * D + j] = (int8_t)(keep ? mv[t] : 0);
    perm[(size_t)b * D + (keep ? rk[t] : j)] = (uint8_t)j;
    if (cdf) cdf[(size_t)b * D + j] = keep ? th[t] : make_uint2(0u, 0xFFFFFFFFu);  // fallback: always m = 0
  }
  if (ra) {  // confident kept starts get r_easy anneals, the others R
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lse += __shfl_xor_sync(0xffffffffu, lse, o);
    if (lane == 0) ra[b] = (keep && -lse > conf_min) ? r_easy : R;
  }
  if (lane == 0) {
    if (e0) e0[b] = keep ? e : ET(0);
    if (kept) kept[b] = keep ? 1 : 0;
  }
}


// ------------------------------------------------------------------------ small batches: a block per problem
// A one-frame (or few-frame) batch leaves a warp per problem waiting on one G row after another.  These kernels
// give each problem a block of 128 threads, stage its G (int32, D x D) into shared memory with every 16-byte
// copy in flight at once, and give each coordinate a thread that runs the warp kernel's loops in the same order,
// so every output is bit-identical to the warp kernel's; the warp reductions are replayed in their lane order.
constexpr int kBlkThreads = 128;

__device__ __forceinline__ void stage_g(int32_t* Gs, const int32_t* __restrict__ Gb, int D) {
  const int n = D * D;
  if (((n & 3) == 0) && ((reinterpret_cast<uintptr_t>(Gb) & 15u) == 0)) {
    const uint32_t base = umma::su32(Gs);
    for (int x = threadIdx.x; x < n / 4; x += blockDim.x) umma::cp16(base + 16u * x, Gb + 4 * x, true);
    umma::cp_commit();
    umma::cp_wait<0>();
  } else {
    for (int x = threadIdx.x; x < n; x += blockDim.x) Gs[x] = Gb[x];
  }
}

// The warp kernels' butterfly sum of per-lane partials, lane l holding coordinates l, 32 + l, 64 + l, 96 + l
// summed in that order (absent coordinates contribute nothing): warp 0 of the block computes it from v (128
// entries in shared memory) and returns it in every lane of warp 0.
template <typename T>
__device__ __forceinline__ T lane_order_sum(const T* v, int D) {
  const int lane = threadIdx.x & 31;
  T a = T(0);
#pragma unroll
  for (int t = 0; t < 4; ++t)
    if (t * 32 + lane < D) a += v[t * 32 + lane];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  return a;
}

__global__ void __launch_bounds__(kBlkThreads) k_warm_features_blk(const int32_t* __restrict__ G,
                                                                   const int32_t* __restrict__ h,
                                                                   const int8_t* __restrict__ xq,
                                                                   const float* __restrict__ zs,
                                                                   const float* __restrict__ snr_db, int D, int M,
                                                                   int P, bf16* __restrict__ X,
                                                                   const int8_t* __restrict__ levels,
                                                                   int8_t* __restrict__ labels) {
  extern __shared__ __align__(16) int32_t Gs[];
  __shared__ float s_dg[128];
  __shared__ int s_mq[128];
  __shared__ float s_mdg;
  const int b = blockIdx.x, j = threadIdx.x;
  pdl_trigger();
  pdl_wait();
  stage_g(Gs, G + (size_t)b * D * D, D);
  __syncthreads();
  float dg = 0.0f, ss = 0.0f;
  if (j < D)
    for (int i = 0; i < D; ++i) {
      const float g = (float)Gs[i * D + j];
      if (i == j)
        dg = g;
      else
        ss = fmaf(g, g, ss);
    }
  s_dg[j] = dg;
  __syncthreads();
  if (j < 32) {
    const float sdg = lane_order_sum(s_dg, 128);  // the warp kernel adds the zero dg of absent coordinates too
    if (j == 0) s_mdg = sdg / (float)D;
  }
  const int Lmax = M == 4 ? 1 : (M == 16 ? 3 : 7);
  const float hv = j < D ? (float)h[(size_t)b * D + j] : 0.0f;
  const int xv = j < D ? xq[(size_t)b * D + j] : 0;
  int mq = dg > 0.0f ? jacobi_move(hv / (4.0f * dg), xv, Lmax) : 0;
  s_mq[j] = mq;
  __syncthreads();
  float u1 = 0.0f, u2 = 0.0f;
  for (int pass = 0; pass < 2; ++pass) {
    float acc = 0.0f;
    if (j < D)
      for (int i = 0; i < D; ++i) {
        const int mi = s_mq[i];
        if (mi != 0 && i != j) acc = fmaf((float)Gs[i * D + j], (float)mi, acc);
      }
    const float v = dg > 0.0f ? (hv - 2.0f * acc) / (4.0f * dg) : 0.0f;
    const float uc = fminf(fmaxf(v, -8.0f), 8.0f);
    if (pass == 0)
      u1 = uc;
    else
      u2 = uc;
    mq = j < D && dg > 0.0f ? jacobi_move(uc, xv, Lmax) : 0;
    __syncthreads();
    s_mq[j] = mq;
    __syncthreads();
  }
  const float snr = snr_db ? snr_db[b] * 0.05f : 0.0f;
  if (j < D)
    feature_row(h, xq, zs, (size_t)b * D + j, Lmax, P, dg, ss, s_mdg, snr, u1, u2, X, levels, labels);
}

__global__ void __launch_bounds__(kBlkThreads) k_warm_start_blk(const float* __restrict__ logits, int ldl,
                                                                const int32_t* __restrict__ G,
                                                                const int32_t* __restrict__ h,
                                                                const int8_t* __restrict__ xq, int D, int P, int M,
                                                                int8_t* __restrict__ m0, uint8_t* __restrict__ perm,
                                                                long long* __restrict__ e0,
                                                                int32_t* __restrict__ kept, float tau,
                                                                uint2* __restrict__ cdf, float conf_min, int r_easy,
                                                                int R, int32_t* __restrict__ ra) {
  extern __shared__ __align__(16) int32_t Gs[];
  __shared__ float s_sc[128], s_lg[128];
  __shared__ int s_m[128];
  __shared__ long long s_e[kBlkThreads / 32];
  __shared__ int s_keep;
  __shared__ float s_lse;
  const int b = blockIdx.x, j = threadIdx.x, lane = j & 31, w = j >> 5;
  pdl_trigger();
  pdl_wait();
  const int32_t* Gb = G + (size_t)b * D * D;
  // the copies of G fly while the logits are read
  const int n = D * D;
  const bool vec = ((n & 3) == 0) && ((reinterpret_cast<uintptr_t>(Gb) & 15u) == 0);
  if (vec) {
    const uint32_t base = umma::su32(Gs);
    for (int x = j; x < n / 4; x += blockDim.x) umma::cp16(base + 16u * x, Gb + 4 * x, true);
    umma::cp_commit();
  } else {
    for (int x = j; x < n; x += blockDim.x) Gs[x] = Gb[x];
  }
  const int C = P + 1, Lmax = M == 4 ? 1 : (M == 16 ? 3 : 7);
  int mv = 0;
  float sc = -1.0f, lg = 0.0f;
  uint2 th = make_uint2(0u, 0xFFFFFFFFu);
  if (j < D)
    mv = start_coord(logits + ((size_t)b * D + j) * ldl, C, P, xq[(size_t)b * D + j], Lmax, tau, cdf != nullptr,
                     sc, th, lg);
  s_m[j] = mv;
  s_sc[j] = sc;
  s_lg[j] = lg;
  if (vec) umma::cp_wait<0>();
  __syncthreads();
  // start energy m^T G m - h^T m, exact in 64-bit integers (any order)
  long long e = 0;
  if (j < D && mv != 0) {
    for (int i = 0; i < D; ++i) {
      const int mi = s_m[i];
      if (mi != 0) e += (long long)Gs[i * D + j] * (long long)(mi * mv);
    }
  }
  if (j < D) e -= (long long)h[(size_t)b * D + j] * (long long)mv;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  if (lane == 0) s_e[w] = e;
  // rank by descending score (ties by index)
  int rk = 0;
  if (j < D)
    for (int i = 0; i < D; ++i) {
      const float si = s_sc[i];
      if (si > sc || (si == sc && i < j)) ++rk;
    }
  __syncthreads();
  if (j == 0) {
    long long et = 0;
    for (int q = 0; q < kBlkThreads / 32; ++q) et += s_e[q];
    et = et + et;  // the anneal's energy units
    s_keep = et <= 0 ? 1 : 0;
    if (e0) e0[b] = et <= 0 ? et : 0;
    if (kept) kept[b] = et <= 0 ? 1 : 0;
  }
  if (ra && j < 32) {
    const float lse = lane_order_sum(s_lg, D);
    if (j == 0) s_lse = lse;
  }
  __syncthreads();
  const bool keep = s_keep != 0;
  if (j < D) {
    m0[(size_t)b * D + j] = (int8_t)(keep ? mv : 0);
    perm[(size_t)b * D + (keep ? rk : j)] = (uint8_t)j;
    if (cdf) cdf[(size_t)b * D + j] = keep ? th : make_uint2(0u, 0xFFFFFFFFu);
  }
  if (ra && j == 0) ra[b] = (keep && -s_lse > conf_min) ? r_easy : R;
}
}  // namespace arp

using namespace arp;

static bool al16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// Batches of at most this many problems (integer fields) use the block-per-problem features and start kernels.
constexpr int kSmallBatch = 2048;

// Opts a block-per-problem kernel into D x D int32 of dynamic shared memory (64 KB at D = 128).
template <typename K>
static cudaError_t blk_smem_attr(K kern, int D) {
  const int bytes = D * D * 4;
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

extern "C" int arp_gemm_bf16(const void* A, int a_mn_major, int lda, const void* B, int b_mn_major, int ldb, int M,
                             int N, int K, int epilogue, const float* bias, const void* aux, int ld_aux, void* C,
                             int ldc, int32_t* status, void* stream) {
  if (M < 0 || N < 0 || K < 0) return ARP_ERR_SHAPE;
  if (M == 0 || N == 0) return ARP_OK;
  if (K == 0 || N % 16 || K % 16 || lda % 8 || ldb % 8 || ldc % 8) return ARP_ERR_SHAPE;
  if (a_mn_major && M % 8) return ARP_ERR_SHAPE;
  if (epilogue < EPI_F32 || epilogue > EPI_MASK_BF16) return ARP_ERR_ARG;
  if (!A || !B || !C || !al16(A) || !al16(B) || !al16(C)) return ARP_ERR_ARG;
  if ((epilogue == EPI_BIAS_RELU_BF16 || epilogue == EPI_BIAS_F32) && !bias) return ARP_ERR_ARG;
  if (epilogue == EPI_MASK_BF16 && (!aux || !al16(aux) || ld_aux % 8)) return ARP_ERR_ARG;
  GemmParams p{(const bf16*)A, (const bf16*)B, lda, ldb, M, N, K, epilogue, bias, (const bf16*)aux, ld_aux, C, ldc, 0,
               status};
  const bool amn = a_mn_major != 0, bmn = b_mn_major != 0;
  cudaStream_t st = (cudaStream_t)stream;
  // the large products: TMA-fed, warp-specialised; the rest (or no tensor-map encoder): the cp.async kernel
  cudaError_t e = gemm_tma_fits(p) ? gemm_tma(p, amn, bmn, st) : cudaErrorNotSupported;
  if (e == cudaErrorNotSupported) {
    if (N <= 16)
      e = gemm_bn<16>(p, amn, bmn, st);
    else if (N <= 64)
      e = gemm_bn<64>(p, amn, bmn, st);
    else if (N <= 128)
      e = gemm_bn<128>(p, amn, bmn, st);
    else
      e = gemm_bn<256>(p, amn, bmn, st);
  }
  return e == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_warm_features(const void* G, const void* h, const int8_t* xq, const float* zs, const float* snr_db,
                                 int B, int D, int M, int P, int quantized, void* X, const int8_t* levels,
                                 int8_t* labels, void* stream) {
  if (B < 0 || D < 1 || D > 128 || !(M == 4 || M == 16 || M == 64) || P < 1 || P > 6) return ARP_ERR_SHAPE;
  if (B == 0) return ARP_OK;
  if (!G || !h || !xq || !X || !al16(X) || (labels && !levels)) return ARP_ERR_ARG;
  const int th = 128, nb = (int)(((size_t)B * 32 + th - 1) / th);
  cudaStream_t st = (cudaStream_t)stream;
  if (quantized && B <= kSmallBatch) {
    if (blk_smem_attr(k_warm_features_blk, D) != cudaSuccess) return ARP_ERR_LAUNCH;
    if (launch_ex(k_warm_features_blk, dim3(B), dim3(kBlkThreads), (size_t)D * D * 4, st, B <= kPdlMaxB,
                  (const int32_t*)G, (const int32_t*)h, xq, zs, snr_db, D, M, P, (bf16*)X, levels, labels) !=
        cudaSuccess)
      return ARP_ERR_LAUNCH;
  } else if (quantized)
    k_warm_features<int32_t><<<nb, th, 0, st>>>((const int32_t*)G, (const int32_t*)h, xq, zs, snr_db, B, D, M, P,
                                                (bf16*)X, levels, labels);
  else
    k_warm_features<float><<<nb, th, 0, st>>>((const float*)G, (const float*)h, xq, zs, snr_db, B, D, M, P, (bf16*)X,
                                              levels, labels);
  return cudaGetLastError() == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_warm_loss(const float* logits, int ldl, const int8_t* labels, int rows, int classes, void* dlogits,
                             int ldd, float* loss_sum, int32_t* correct, void* stream) {
  if (rows < 0 || classes < 2 || classes > ldl || classes > ldd || classes > 8) return ARP_ERR_SHAPE;
  if (rows == 0) return ARP_OK;
  if (!logits || !labels || !dlogits) return ARP_ERR_ARG;
  k_warm_loss<<<(rows + 255) / 256, 256, 0, (cudaStream_t)stream>>>(logits, ldl, labels, rows, classes, (bf16*)dlogits,
                                                                    ldd, loss_sum, correct);
  return cudaGetLastError() == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_colsum_bf16(const void* X, int rows, int cols, int ld, float* out, void* stream) {
  if (rows < 0 || cols < 0 || ld < cols) return ARP_ERR_SHAPE;
  if (rows == 0 || cols == 0) return ARP_OK;
  if (!X || !out) return ARP_ERR_ARG;
  int gy = (rows + 8 * 64 - 1) / (8 * 64);
  if (gy > 256) gy = 256;
  dim3 grid((cols + 31) / 32, gy);
  cudaStream_t st = (cudaStream_t)stream;
  if (gy == 1) {
    k_colsum_bf16<<<grid, 256, 0, st>>>((const bf16*)X, rows, cols, ld, out);
    return cudaGetLastError() == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
  }
  // row bands' partials to a stream-ordered workspace, then summed in band order (no float atomics: the
  // gradients, and so the trained network, are the same on every run)
  float* ws = nullptr;
  if (cudaMallocAsync(reinterpret_cast<void**>(&ws), (size_t)gy * cols * sizeof(float), st) != cudaSuccess)
    return ARP_ERR_LAUNCH;
  k_colsum_bf16<<<grid, 256, 0, st>>>((const bf16*)X, rows, cols, ld, ws);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    k_colsum_reduce<<<(cols + 255) / 256, 256, 0, st>>>(ws, gy, cols, out);
    e = cudaGetLastError();
  }
  const cudaError_t ef = cudaFreeAsync(ws, st);
  return e == cudaSuccess && ef == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_adam(float* w, void* w_bf16, const float* grad, float* m, float* v, int n, float lr, float beta1,
                        float beta2, float eps, int step, float grad_scale, void* stream) {
  if (n < 0 || step < 1) return ARP_ERR_SHAPE;
  if (n == 0) return ARP_OK;
  if (!w || !grad || !m || !v) return ARP_ERR_ARG;
  const float bc1 = 1.0f - powf(beta1, (float)step), bc2 = 1.0f - powf(beta2, (float)step);
  k_adam<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(w, (bf16*)w_bf16, grad, m, v, n, lr, beta1, beta2, eps,
                                                            bc1, bc2, grad_scale);
  return cudaGetLastError() == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_warm_start_sampled(const float* logits, int ldl, const void* G, const void* h, const int8_t* xq,
                                      int B, int D, int P, int M, int quantized, int8_t* m0, uint8_t* perm, void* e0,
                                      int32_t* kept, float tau, uint32_t* cdf, float conf_min, int r_easy, int R,
                                      int32_t* ra, void* stream) {
  if (B < 0 || D < 1 || D > 128 || P != 2 || ldl < P + 1 || !(M == 4 || M == 16 || M == 64)) return ARP_ERR_SHAPE;
  if (B == 0) return ARP_OK;
  if (!logits || !G || !h || !xq || !m0 || !perm || !cdf || !(tau > 0.0f)) return ARP_ERR_ARG;
  if (ra && (R < 1 || r_easy < 1 || r_easy > R)) return ARP_ERR_ARG;
  const int th = 128, nb = (int)(((size_t)B * 32 + th - 1) / th);
  cudaStream_t st = (cudaStream_t)stream;
  if (quantized && B <= kSmallBatch) {
    if (blk_smem_attr(k_warm_start_blk, D) != cudaSuccess) return ARP_ERR_LAUNCH;
    if (launch_ex(k_warm_start_blk, dim3(B), dim3(kBlkThreads), (size_t)D * D * 4, st, B <= kPdlMaxB, logits, ldl,
                  (const int32_t*)G, (const int32_t*)h, xq, D, P, M, m0, perm, (long long*)e0, kept, tau,
                  (uint2*)cdf, conf_min, r_easy, R, ra) != cudaSuccess)
      return ARP_ERR_LAUNCH;
  } else if (quantized)
    k_warm_start<int32_t, long long><<<nb, th, 0, st>>>(logits, ldl, (const int32_t*)G, (const int32_t*)h, xq, B, D,
                                                        P, M, m0, perm, (long long*)e0, kept, tau, (uint2*)cdf,
                                                        conf_min, r_easy, R, ra);
  else
    k_warm_start<float, float><<<nb, th, 0, st>>>(logits, ldl, (const float*)G, (const float*)h, xq, B, D, P, M, m0,
                                                  perm, (float*)e0, kept, tau, (uint2*)cdf, conf_min, r_easy, R,
                                                  ra);
  return cudaGetLastError() == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_warm_start(const float* logits, int ldl, const void* G, const void* h, const int8_t* xq, int B,
                              int D, int P, int M, int quantized, int8_t* m0, uint8_t* perm, void* e0,
                              int32_t* kept, void* stream) {
  if (B < 0 || D < 1 || D > 128 || P < 1 || P > 6 || ldl < P + 1 || !(M == 4 || M == 16 || M == 64))
    return ARP_ERR_SHAPE;
  if (B == 0) return ARP_OK;
  if (!logits || !G || !h || !xq || !m0 || !perm) return ARP_ERR_ARG;
  const int th = 128, nb = (int)(((size_t)B * 32 + th - 1) / th);
  cudaStream_t st = (cudaStream_t)stream;
  if (quantized && B <= kSmallBatch) {
    if (blk_smem_attr(k_warm_start_blk, D) != cudaSuccess) return ARP_ERR_LAUNCH;
    if (launch_ex(k_warm_start_blk, dim3(B), dim3(kBlkThreads), (size_t)D * D * 4, st, B <= kPdlMaxB, logits, ldl,
                  (const int32_t*)G, (const int32_t*)h, xq, D, P, M, m0, perm, (long long*)e0, kept, 1.0f,
                  (uint2*)nullptr, 0.0f, 1, 1, (int32_t*)nullptr) != cudaSuccess)
      return ARP_ERR_LAUNCH;
  } else if (quantized)
    k_warm_start<int32_t, long long><<<nb, th, 0, st>>>(logits, ldl, (const int32_t*)G, (const int32_t*)h, xq, B, D,
                                                        P, M, m0, perm, (long long*)e0, kept, 1.0f, nullptr, 0.0f, 1, 1,
                                                        nullptr);
  else
    k_warm_start<float, float><<<nb, th, 0, st>>>(logits, ldl, (const float*)G, (const float*)h, xq, B, D, P, M, m0,
                                                  perm, (float*)e0, kept, 1.0f, nullptr, 0.0f, 1, 1, nullptr);
  return cudaGetLastError() == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

// ------------------------------------------------------------------------------------------------ fused inference
// The whole network for a 128-row tile in one CTA (persistent over tiles, one CTA per SM; eight epilogue warps and
// one MMA warp), every weight resident in shared memory for the whole launch:
//   L1: acc1 = X W1^T              (X tile 128 x 16; one N = 256 MMA into TMEM columns 256..511)
//   epilogue 1: acc1 -> bias + ReLU -> bf16 -> H tile (128 x 256, K-major canonical layout), 32 columns at a time,
//               each chunk announced on its mbarrier
//   L2: acc2 = H1 W2^T             (TMEM columns 0..255; the two MMAs of k-chunk t issued as soon as chunk t of H1
//                                   is in place, so layer 2 runs behind epilogue 1)
//   epilogue 2: acc2 -> bias + ReLU -> bf16 -> the same H tile (every L2 MMA has completed), chunk by chunk
//   L3: acc1[0:16) = H2 W3         (W3t (256 x 16) MN-major; its MMAs behind epilogue 2)
//   epilogue 3: acc1[0:16) + b3 -> logits (rows, 16) float in global memory
// Only X and the logits touch HBM.  Shared memory: W2 128 KB + H 64 KB + X 4 KB + W1 and W3t 8 KB each.
// W2's order in shared memory (K-major, no swizzle): byte(n, k) = (k / 32) 16384 + ((k % 32) / 8) 4096 + n 16 +
// (k % 8) 2; arp_mlp_pack_w2 writes W2 in this order once per weight update, so it arrives by eight contiguous
// 16 KB bulk copies (whole L2 sectors, no gather).
namespace arp {

constexpr int kNH = 256;  // hidden width of the warm-start network
constexpr int kMlpEpiWarps = 8;                       // epilogue warps (TMEM lane quarter w % 4, column half w / 4)
constexpr int kMlpThreads = 32 * (kMlpEpiWarps + 1);  // and one MMA warp
constexpr uint32_t kMlpCols = 2 * kNH;                // two accumulators: layer 2, and layers 1 and 3
// Shared memory of the fused forward: W2 resident for the whole launch (8 chunks of 256 rows x 32 k, 128 KB),
// the H tile (128 rows x 256, H1 then H2), the X tile, W1 and W3t resident (8 KB each).
constexpr uint32_t kW2Bytes = kNH * kNH * 2, kHsBytes = 128 * kNH * 2, kXsBytes = 128 * 16 * 2;
constexpr uint32_t kW1Bytes = kNH * 16 * 2, kW3Bytes = kNH * 16 * 2, kChunkBytes = kNH * 32 * 2;
constexpr uint32_t kMlpSmem = kW2Bytes + kHsBytes + kXsBytes + kW1Bytes + kW3Bytes;

struct MlpParams {
  const bf16* X;
  const bf16 *W1, *W2p, *W3t;
  const float *b1, *b2, *b3;
  float* logits;
  int rows;
  int32_t* status;
  int bias16;  // b1 and b2 16-byte aligned: staged with cp.async
};

// W2 (256 x 256, row-major: output n, input k) -> the fused kernel's shared-memory order: chunk t = k
// [32 t, +32) of all 256 rows, within a chunk k-group b (8 wide) then row n then element: W2p[t][b][n][e] (the
// canonical K-major layout of a 256 x 32 B operand, k-groups 4096 B apart, 8-row groups 128 B apart).
__global__ void __launch_bounds__(256) k_pack_w2(const bf16* __restrict__ W2, bf16* __restrict__ W2p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // one 16-byte group of 8 elements
  if (i >= kNH * kNH / 8) return;
  const int t = i >> 10, b = (i >> 8) & 3, n = i & 255;  // 1024 groups per chunk, 256 per k-group
  const int k = t * 32 + b * 8;
  reinterpret_cast<uint4*>(W2p)[i] = *reinterpret_cast<const uint4*>(W2 + (size_t)n * kNH + k);
}

// One 32-column chunk t of a hidden layer: TMEM (the accumulator's columns 32 t ..) -> bias (shared memory) + ReLU
// -> bf16 -> the H tile (K-major, 8-row groups 4096 B apart).  Warp w (of the eight epilogue warps) takes rows
// 32 (w % 4) .. + 31 and 16 of the chunk's columns (half w / 4), so the eight warps finish chunk t together and
// the next layer's MMAs over k-chunk t can start right behind them.
__device__ __forceinline__ void mlp_epi_chunk(uint32_t acc, uint32_t hs, const float* bias, int t, int warp,
                                              int lane) {
  const int m = (warp & 3) * 32 + lane, c0 = t * 32 + (warp >> 2) * 16;
  uint32_t v[32];
  umma::tmem_ld16(acc + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)c0, v);
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const float4 bl = *reinterpret_cast<const float4*>(bias + c0 + q * 8);
    const float4 bh = *reinterpret_cast<const float4*>(bias + c0 + q * 8 + 4);
    const float bb[8] = {bl.x, bl.y, bl.z, bl.w, bh.x, bh.y, bh.z, bh.w};
    uint32_t pk[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int j = q * 8 + 2 * i;
      const float a = fmaxf(__uint_as_float(v[j]) + bb[2 * i], 0.0f);
      const float b = fmaxf(__uint_as_float(v[j + 1]) + bb[2 * i + 1], 0.0f);
      const __nv_bfloat162 h2 = __floats2bfloat162_rn(a, b);
      pk[i] = *reinterpret_cast<const uint32_t*>(&h2);
    }
    const uint32_t addr = hs + (uint32_t)((m >> 3) * 4096 + ((c0 >> 3) + q) * 128 + (m & 7) * 16);
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(pk[0]), "r"(pk[1]), "r"(pk[2]),
                 "r"(pk[3])
                 : "memory");
  }
}

// The whole network per 128-row tile, one persistent CTA per SM: the weights are loaded once per launch (W2 by
// eight bulk copies on one mbarrier, W1, W3t and the biases by cp.async) and stay in shared memory.  Per tile:
// layer 1 (one MMA, N = 256) into the accumulator at TMEM columns 256..511; the eight epilogue warps drain it chunk
// by chunk (32 hidden units) into the H tile, arriving on the chunk's mbarrier, while the MMA warp issues layer 2's
// two MMAs of each k-chunk as soon as that chunk is in place (accumulator at columns 0..255); the epilogue warps
// then drain layer 2 chunk by chunk over H1 (every layer-2 MMA has completed) while the MMA warp issues layer 3's
// MMAs (N = 16, accumulator at columns 256..271) behind them; logits + b3 to global.  The next tile's X is fetched
// as soon as layer 1 has read the current one.  Same roundings and summation order as the layer-by-layer GEMMs.
__global__ void __launch_bounds__(kMlpThreads, 1) k_mlp_fused(const MlpParams p) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ __align__(8) uint64_t bar_w, bar_l1, bar_l2, bar_l3, bar_done, bar_h1[kNH / 32], bar_h2[kNH / 32];
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  __shared__ __align__(16) float s_b1[kNH], s_b2[kNH];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool mma_warp = warp == kMlpEpiWarps;
  const int ntiles = (p.rows + 127) / 128;
  if ((int)blockIdx.x >= ntiles) return;
  pdl_trigger();
  const uint32_t w2s = umma::su32(smem), hs = w2s + kW2Bytes, xs = hs + kHsBytes, w1s = xs + kXsBytes,
                 w3s = w1s + kW1Bytes;
  constexpr uint32_t ID_HID = umma::idesc_bf16(kNH, false, false), ID_OUT = umma::idesc_bf16(16, false, true);
  if (tid == 0) {
    umma::mbar_init(&bar_w, 1);
    umma::mbar_init(&bar_l1, 1);
    umma::mbar_init(&bar_l2, 1);
    umma::mbar_init(&bar_l3, 1);
    umma::mbar_init(&bar_done, 1);
    for (int t = 0; t < kNH / 32; ++t) {
      umma::mbar_init(&bar_h1[t], kMlpEpiWarps);
      umma::mbar_init(&bar_h2[t], kMlpEpiWarps);
    }
    umma::fence_mbar_init();
    s_abort = 0;
  }
  if (warp == 0) umma::tmem_alloc(&s_tmem, kMlpCols);
  umma::tc_before_sync();
  __syncthreads();
  umma::tc_after_sync();
  const uint32_t acc2 = s_tmem, acc1 = s_tmem + kNH;  // layer 2 at columns 0..255; layers 1 and 3 at 256..
  pdl_wait();  // everything above touches no global memory

  auto load_x = [&](int tile) {  // 128 x 16: one 16-byte chunk per epilogue thread
    const int row = tid >> 1, kc = tid & 1, m = tile * 128 + row;
    const bool ok = m < p.rows;
    umma::cp16(xs + (uint32_t)((row >> 3) * 256 + kc * 128 + (row & 7) * 16),
               ok ? (const void*)(p.X + (size_t)m * 16 + kc * 8) : (const void*)p.X, ok);
  };
  // weights, once: W2 by bulk copies (thread 0), W1 (256 x 16, K-major, SBO 256) and W3t (256 k x 16 n,
  // MN-major: LBO 256 between k-groups, SBO 128) and the biases by cp.async
  constexpr int E = kMlpEpiWarps * 32;  // epilogue threads
  if (tid == 0) {
    umma::expect_tx(&bar_w, kW2Bytes);
    for (int t = 0; t < kNH / 32; ++t)
      umma::bulk_g2s(w2s + (uint32_t)t * kChunkBytes, p.W2p + (size_t)t * (kChunkBytes / 2), kChunkBytes, &bar_w);
  }
  if (tid < E) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int c = tid + i * E, r = c >> 1, h = c & 1;
      umma::cp16(w1s + (uint32_t)((r >> 3) * 256 + h * 128 + (r & 7) * 16), p.W1 + (size_t)r * 16 + h * 8, true);
      umma::cp16(w3s + (uint32_t)((r >> 3) * 256 + h * 128 + (r & 7) * 16), p.W3t + (size_t)r * 16 + h * 8, true);
    }
  }
  if (p.bias16) {
    if (tid < 2 * kNH / 4)
      umma::cp16(umma::su32(tid < kNH / 4 ? s_b1 + 4 * tid : s_b2 + 4 * (tid - kNH / 4)),
                 tid < kNH / 4 ? p.b1 + 4 * tid : p.b2 + 4 * (tid - kNH / 4), true);
  } else {
    for (int i = tid; i < kNH; i += kMlpThreads) {
      s_b1[i] = p.b1[i];
      s_b2[i] = p.b2[i];
    }
  }
  if (tid < E) load_x(blockIdx.x);
  umma::cp_commit();
  bool w2_ready = false;
  int it = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
    const uint32_t ph = (uint32_t)(it & 1);
    // ---- layer 1 (X landed; the previous tile's TMEM reads and layer-3 MMAs are done)
    umma::cp_wait<0>();
    umma::fence_async_smem();
    umma::tc_before_sync();
    __syncthreads();
    if (s_abort) break;
    if (mma_warp) {
      if (lane == 0) {
        umma::tc_after_sync();
        umma::mma(acc1, umma::sdesc(xs, 128, 256), umma::sdesc(w1s, 128, 256), ID_HID, 0u);
        umma::commit(&bar_l1);
        // ---- layer 2, k-chunk by k-chunk behind epilogue 1: A = H1 (K-major, SBO 4096), B = the resident W2
        bool ok = w2_ready || umma::mbar_wait(&bar_w, 0);
        for (int t = 0; t < kNH / 32 && ok; ++t) {
          if (!umma::mbar_wait(&bar_h1[t], ph)) {
            ok = false;
            break;
          }
          umma::tc_after_sync();
#pragma unroll
          for (int kk = 0; kk < 2; ++kk)
            umma::mma(acc2, umma::sdesc(hs + (uint32_t)((t * 4 + kk * 2) * 128), 128, 4096),
                      umma::sdesc(w2s + (uint32_t)t * kChunkBytes + (uint32_t)(kk * 8192), 4096, 128), ID_HID,
                      (t > 0 || kk > 0) ? 1u : 0u);
        }
        umma::commit(&bar_l2);  // also when nothing was issued: it completes at once, nobody waits out the bound
        // ---- layer 3, behind epilogue 2: A = H2, B = W3t (MN-major), accumulator over layer 1's columns
        for (int t = 0; t < kNH / 32 && ok; ++t) {
          if (!umma::mbar_wait(&bar_h2[t], ph)) {
            ok = false;
            break;
          }
          umma::tc_after_sync();
#pragma unroll
          for (int k2 = 0; k2 < 2; ++k2) {
            const int kk = 2 * t + k2;
            umma::mma(acc1, umma::sdesc(hs + (uint32_t)(kk * 256), 128, 4096),
                      umma::sdesc(w3s + (uint32_t)(kk * 512), 256, 128), ID_OUT, kk > 0 ? 1u : 0u);
          }
        }
        umma::commit(&bar_l3);
        if (!ok) s_abort = 1;
      }
      w2_ready = true;
      __syncwarp();
    } else {
      if (!umma::mbar_wait(&bar_l1, ph)) s_abort = 1;
      if (tile + (int)gridDim.x < ntiles) load_x(tile + gridDim.x);  // layer 1 has read X
      umma::cp_commit();
      umma::tc_after_sync();
      for (int t = 0; t < kNH / 32; ++t) {  // epilogue 1, chunk by chunk
        mlp_epi_chunk(acc1, hs, s_b1, t, warp, lane);
        umma::fence_async_smem();
        umma::tc_before_sync();
        __syncwarp();
        if (lane == 0) umma::mbar_arrive(&bar_h1[t]);
      }
      if (!umma::mbar_wait(&bar_l2, ph)) s_abort = 1;
      umma::tc_after_sync();
      for (int t = 0; t < kNH / 32; ++t) {  // epilogue 2 over H1, chunk by chunk
        mlp_epi_chunk(acc2, hs, s_b2, t, warp, lane);
        umma::fence_async_smem();
        umma::tc_before_sync();
        __syncwarp();
        if (lane == 0) umma::mbar_arrive(&bar_h2[t]);
      }
      if (warp < 4) {
        if (!umma::mbar_wait(&bar_l3, ph)) s_abort = 1;
        umma::tc_after_sync();
        uint32_t v[32];
        umma::tmem_ld16(acc1 + ((uint32_t)(warp * 32) << 16), v);
        const int row = tile * 128 + warp * 32 + lane;
        if (row < p.rows && !s_abort) {
          float4* o = reinterpret_cast<float4*>(p.logits + (size_t)row * 16);
#pragma unroll
          for (int i = 0; i < 4; ++i)
            o[i] = make_float4(__uint_as_float(v[4 * i]) + __ldg(p.b3 + 4 * i),
                               __uint_as_float(v[4 * i + 1]) + __ldg(p.b3 + 4 * i + 1),
                               __uint_as_float(v[4 * i + 2]) + __ldg(p.b3 + 4 * i + 2),
                               __uint_as_float(v[4 * i + 3]) + __ldg(p.b3 + 4 * i + 3));
        }
      }
    }
  }
  if (mma_warp && lane == 0) {  // every MMA issued has completed before TMEM is released (bounded)
    umma::commit(&bar_done);
    if (!umma::mbar_wait(&bar_done, 0)) s_abort = 1;
  }
  umma::cp_wait<0>();
  umma::tc_before_sync();
  __syncthreads();
  if (s_abort && tid == 0) set_status(p.status, ARP_ERR_TIMEOUT);
  if (warp == 0) umma::tmem_free(s_tmem, kMlpCols);
}

}  // namespace arp

extern "C" int arp_mlp_forward(const void* X, int rows, const void* W1, const float* b1, const void* W2p,
                               const float* b2, const void* W3t, const float* b3, float* logits, int32_t* status,
                               void* stream) {
  if (rows < 0) return ARP_ERR_SHAPE;
  if (rows == 0) return ARP_OK;
  if (!X || !W1 || !b1 || !W2p || !b2 || !W3t || !b3 || !logits) return ARP_ERR_ARG;
  if (!al16(X) || !al16(W1) || !al16(W2p) || !al16(W3t) || !al16(logits)) return ARP_ERR_ARG;
  static DeviceAttr attr;
  if (smem_attr(attr, k_mlp_fused, kMlpSmem) != cudaSuccess) return ARP_ERR_LAUNCH;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ntiles = (rows + 127) / 128;
  MlpParams p{(const bf16*)X, (const bf16*)W1, (const bf16*)W2p, (const bf16*)W3t, b1, b2, b3, logits, rows, status,
              al16(b1) && al16(b2) ? 1 : 0};
  const bool pdl = rows <= kPdlMaxB * 128;
  return launch_ex(k_mlp_fused, dim3(ntiles < sms ? ntiles : sms), dim3(kMlpThreads), kMlpSmem, (cudaStream_t)stream,
                   pdl, p) == cudaSuccess
             ? ARP_OK
             : ARP_ERR_LAUNCH;
}

extern "C" int arp_mlp_pack_w2(const void* W2, void* W2p, void* stream) {
  if (!W2 || !W2p || !al16(W2) || !al16(W2p)) return ARP_ERR_ARG;
  k_pack_w2<<<(kNH * kNH / 8 + 255) / 256, 256, 0, (cudaStream_t)stream>>>((const bf16*)W2, (bf16*)W2p);
  return cudaGetLastError() == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}
