// Test infrastructure, not product code: a host launcher for the reference's own Chord kernel
// (arpeggio/mimo/chord_kernel.cu, chord_m{1,2,3,4,6,8}: one block per problem, one warp per anneal in flight),
// compiled from the reference's source where it lies -- the Makefile passes its path as REF_CHORD_KERNEL -- into
// oracle/_ref/libref_chord.so.  Launch shape and shared memory are the reference wrapper's
// (arpeggio/mimo/chordfx.py:189-208).  The GPU parity test runs it beside this project's arp_anneal_chord.
#include <cuda_runtime.h>

#include REF_CHORD_KERNEL

typedef void (*ChordEntry)(const int16_t*, const int32_t*, const int32_t*, const int32_t*, const int32_t*, int, int,
                           int, int, int, uint32_t, uint32_t, int, int, int32_t*, int8_t*, unsigned long long*);

extern "C" int ref_chord(const int16_t* J, const int32_t* h, const int32_t* h0, const int32_t* Tq, const int32_t* Cq,
                         int q, int S, int P, int R, int N, int B, uint32_t k0, uint32_t k1, int inst0, int mode,
                         int warps, int32_t* out_e, int8_t* out_s, unsigned long long* stats, void* stream) {
  if (B < 1 || R < 1 || P < 1 || N % 32 || (N / P) % 32 || warps < 1) return 1;
  ChordEntry k = nullptr;
  switch (N / 32) {
    case 1: k = chord_m1; break;
    case 2: k = chord_m2; break;
    case 3: k = chord_m3; break;
    case 4: k = chord_m4; break;
    case 6: k = chord_m6; break;
    case 8: k = chord_m8; break;
    default: return 1;
  }
  const int W = warps < R ? (warps < 8 ? warps : 8) : (R < 8 ? R : 8);
  const size_t smem = (((size_t)N * N * 2 + 15) / 16) * 16 + 4 * (2 * (size_t)N + 64);
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return 2;
  k<<<B, 32 * W, smem, (cudaStream_t)stream>>>(J, h, h0, Tq, Cq, q, S, P, R, N, k0, k1, inst0, mode, out_e, out_s,
                                                stats);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
