// Shared device helpers: Philox4x32-10, warp masks, status reporting.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "../../include/arpeggio_b200.h"

#define ARP_FULL 0xffffffffu

namespace arp {

// Programmatic dependent launch along a small batch's kernel chain.  Every kernel of the chain triggers its
// dependents on entry; a dependent launched with programmatic serialization (launch_ex, pdl = true) may start
// as soon as every block of its predecessor has triggered, runs only work that reads nothing the chain
// produces (weights, the host inputs the chain's first kernel was ordered after), and calls pdl_wait() before
// its first read of a predecessor's output: that returns once the predecessor grid has completed and its
// writes are visible (so, transitively, every earlier kernel of the chain).  Without the launch attribute
// both instructions do nothing.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Batches of at most this many problems launch their dependent kernels with programmatic serialization.
constexpr int kPdlMaxB = 64;

template <typename... KArgs, typename... Args>
inline cudaError_t launch_ex(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, bool pdl,
                             Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = pdl ? at : nullptr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

// A kernel's dynamic shared-memory limit (a size fixed per kernel) raised once per device: cudaFuncSetAttribute
// applies to the current device only.  Each launcher keeps one DeviceAttr per kernel; its lock guards the flags.
struct DeviceAttr {
  std::mutex mu;
  bool done[64] = {};
};
template <typename K>
inline cudaError_t smem_attr(DeviceAttr& st, K kern, size_t bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(st.mu);
  if (!st.done[dev]) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    st.done[dev] = true;
  }
  return cudaSuccess;
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): ten rounds of two 32x32->64 multiplies,
// Weyl key increments 0x9E3779B9 / 0xBB67AE85.  Counter (c0..c3) in place, key (k0, k1).
// The counter layout each caller uses is the reference's (arpeggio_fx.cu:51,75; chord_kernel.cu:74,107).
__device__ __forceinline__ void philox10(uint32_t& c0, uint32_t& c1, uint32_t& c2, uint32_t& c3, uint32_t k0,
                                         uint32_t k1) {
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    c0 = n0;
    c1 = (uint32_t)p1;
    c2 = n2;
    c3 = (uint32_t)p0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// The ten round keys of a key.  Filled on the host and passed inside a kernel's parameter block, so the
// rounds read them as constant-bank operands (no registers, no per-block key additions).
struct PhiloxKeys {
  uint32_t k0[10], k1[10];
};

__host__ __device__ inline PhiloxKeys philox_keys(uint32_t a, uint32_t b) {
  PhiloxKeys K;
  for (int i = 0; i < 10; ++i) {
    K.k0[i] = a;
    K.k1[i] = b;
    a += 0x9E3779B9u;
    b += 0xBB67AE85u;
  }
  return K;
}

__device__ __forceinline__ void philox10(uint32_t& c0, uint32_t& c1, uint32_t& c2, uint32_t& c3,
                                         const PhiloxKeys& K) {
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ K.k0[i], n2 = (uint32_t)(p0 >> 32) ^ c3 ^ K.k1[i];
    c0 = n0;
    c1 = (uint32_t)p1;
    c2 = n2;
    c3 = (uint32_t)p0;
  }
}

// ceil(u * A / 2^32) for u < 2^32 and |A| < 2^31, as a signed 64-bit floor shift.  For an integer z,
// u * A > z * 2^32  <=>  z < ceil(u * A / 2^32): the reference's exact int64/bignum decision
// (arpeggio_fx.cu:76-79, arpeggio_ref59.py:62) becomes one 32-bit compare once the threshold is known.
__device__ __forceinline__ int64_t ceil_shift32(uint32_t u, int64_t A) {
  return ((int64_t)u * A + 0xFFFFFFFFLL) >> 32;
}

// Uniform float in [0, 1) with 24 exact bits: (x >> 8) * 2^-24.
__device__ __forceinline__ float unit24(uint32_t x) { return __fmul_rn((float)(x >> 8), 5.9604644775390625e-08f); }

__device__ __forceinline__ void set_status(int32_t* status, int code) {
  if (status) atomicCAS(status, 0, code);
}

// Index (within [0, C(P, P/2))) -> the P-bit pattern with P/2 ones, in increasing order
// (arpeggio_ref59.py:31-38).  Tables for P = 2, 4, 6.
__device__ __forceinline__ int bal_pattern(int P, uint32_t i) {
  int n = 0;
  for (int v = 0; v < (1 << P); ++v)
    if (__popc(v) == P / 2) {
      if (n == (int)i) return v;
      ++n;
    }
  return 0;
}

__host__ __device__ __forceinline__ int bal_choose(int P) { return P == 2 ? 2 : (P == 4 ? 6 : 20); }

// Square QAM per real dimension: L = sqrt(M) odd levels -(L-1) .. L-1, log2(L) Gray bits (binary-reflected code
// of the level index, MSB first; for QPSK and 16-QAM this is the reference's table, mimo.py:21-22).
__host__ __device__ __forceinline__ int pam_size(int M) { return M == 4 ? 2 : (M == 16 ? 4 : 8); }
__host__ __device__ __forceinline__ int pam_bits(int M) { return M == 4 ? 1 : (M == 16 ? 2 : 3); }
__device__ __forceinline__ int gray_bit(int l, int k, int M) {
  const int L = pam_size(M), nb = pam_bits(M);
  const int i = (l + L - 1) >> 1;
  const int g = i ^ (i >> 1);
  return (g >> (nb - 1 - k)) & 1;
}

}  // namespace arp
