// The bf16 GEMM's parameter block and fused epilogues, shared by the cp.async-fed kernel (warm.cu) and the
// TMA-fed, warp-specialised kernel (gemm_tma.cu): C = A B^T with A (M x K) and B (N x K), each stored K-major
// (rows of K) or MN-major (rows of M or N), bf16 operands, fp32 accumulation in TMEM.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace arp {

using bf16 = __nv_bfloat16;

struct GemmParams {
  const bf16* A;
  const bf16* B;
  int lda, ldb;
  int M, N, K;
  int epi;
  const float* bias;
  const bf16* aux;
  int ldaux;
  void* C;
  int ldc;
  int kt_per;  // k tiles (of 64) per split
  int32_t* status;
};

enum { EPI_F32 = 0, EPI_F32_ACC = 1, EPI_BIAS_RELU_BF16 = 2, EPI_BIAS_F32 = 3, EPI_MASK_BF16 = 4 };
// Internal: split z of a split-K product stores its partial tile at C + z M ldc (summed afterwards in split order).
constexpr int EPI_F32_PART = 5;

template <int CW>
__device__ __forceinline__ void epilogue(const GemmParams& p, int row, int n, const uint32_t (&v)[32], int z) {
#pragma unroll
  for (int g = 0; g < CW; g += 16) {
    const int nn = n + g;
    if (nn >= p.N) break;
    float f[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) f[i] = __uint_as_float(v[g + i]);
    if (p.epi == EPI_F32 || p.epi == EPI_BIAS_F32 || p.epi == EPI_F32_PART) {
      if (p.epi == EPI_BIAS_F32)
#pragma unroll
        for (int i = 0; i < 16; ++i) f[i] += p.bias[nn + i];
      float* base = reinterpret_cast<float*>(p.C);
      if (p.epi == EPI_F32_PART) base += (size_t)z * p.M * p.ldc;
      float4* o = reinterpret_cast<float4*>(base + (size_t)row * p.ldc + nn);
#pragma unroll
      for (int i = 0; i < 4; ++i) o[i] = make_float4(f[4 * i], f[4 * i + 1], f[4 * i + 2], f[4 * i + 3]);
    } else if (p.epi == EPI_F32_ACC) {
      float* o = reinterpret_cast<float*>(p.C) + (size_t)row * p.ldc + nn;
#pragma unroll
      for (int i = 0; i < 16; ++i) atomicAdd(o + i, f[i]);
    } else {
      if (p.epi == EPI_BIAS_RELU_BF16) {
#pragma unroll
        for (int i = 0; i < 16; ++i) f[i] = fmaxf(f[i] + p.bias[nn + i], 0.0f);
      } else {  // EPI_MASK_BF16: ReLU backward through the stored activation
        const uint4* ax = reinterpret_cast<const uint4*>(p.aux + (size_t)row * p.ldaux + nn);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const uint4 u = ax[q];
          const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const __nv_bfloat162 h2 = *reinterpret_cast<const __nv_bfloat162*>(&w[i]);
            if (!(__low2float(h2) > 0.0f)) f[8 * q + 2 * i] = 0.0f;
            if (!(__high2float(h2) > 0.0f)) f[8 * q + 2 * i + 1] = 0.0f;
          }
        }
      }
      uint32_t pk[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const __nv_bfloat162 h2 = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
        pk[i] = *reinterpret_cast<const uint32_t*>(&h2);
      }
      uint4* o = reinterpret_cast<uint4*>(reinterpret_cast<bf16*>(p.C) + (size_t)row * p.ldc + nn);
      o[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
      o[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
    }
  }
}

// C (M x N, leading dimension ldc) += the split-K partials ws[0 .. splits-1] (dense M x N each), summed in split
// order on the stream (warm.cu).
cudaError_t sum_splits(const float* ws, int splits, int M, int N, float* C, int ldc, cudaStream_t st);

// The TMA-fed, warp-specialised kernel (gemm_tma.cu) for products with M >= 128, N >= 64 and K >= 64;
// cudaErrorNotSupported when the driver's tensor-map encoder is unavailable or refuses the operands.
bool gemm_tma_fits(const GemmParams& p);
cudaError_t gemm_tma(const GemmParams& p, bool a_mn, bool b_mn, cudaStream_t st);

}  // namespace arp
