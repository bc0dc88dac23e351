// Test infrastructure, not product code: a host launcher for the reference's own first-accept kernel
// (arpeggio/sim/arpeggio_fx.cu, one thread per anneal), compiled from the reference's source where it lies --
// the Makefile passes its path as REF_ARPEGGIO_FX -- into oracle/_ref/libref_arpeggio.so.  The GPU parity test
// runs it beside this project's kernel on the same inputs (bit-exact outputs, both timed).  The launch shape is
// the reference wrapper's (arpeggio/sim/arpeggiofx.py:39-42: 128 threads, one per anneal).
#include <cuda_runtime.h>

#include REF_ARPEGGIO_FX

extern "C" int ref_arpeggio_fx(const int32_t* Gt, const int32_t* h, const int32_t* T, int L, int q, int P, int R,
                               int D, int B, const uint32_t* inst, uint32_t k0, uint32_t k1, int start,
                               int8_t* out_s, long long* out_de, long long* out_st, void* stream) {
  if (B < 1 || R < 1 || D < 1 || D > DMAX || !(P == 2 || P == 4 || P == 6) || L < 1) return 1;
  const int n = B * R;
  arpeggio_fx<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(Gt, h, T, L, q, P, R, D, B, inst, k0, k1, start,
                                                                   out_s, out_de, out_st);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
