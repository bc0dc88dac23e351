// Small C-ABI entry points: version, status strings, the device Philox known-answer kernel.
#include "arp_common.cuh"

namespace arp {

// chord_kernel.cu:26-32 (`philox_kat`): one thread per (counter, key) row.
__global__ void k_philox_kat(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  uint32_t c0 = in[6 * t], c1 = in[6 * t + 1], c2 = in[6 * t + 2], c3 = in[6 * t + 3];
  philox10(c0, c1, c2, c3, in[6 * t + 4], in[6 * t + 5]);
  out[4 * t] = c0;
  out[4 * t + 1] = c1;
  out[4 * t + 2] = c2;
  out[4 * t + 3] = c3;
}

// Calibration: `iters` chained Philox4x32-10 blocks per thread (the anneal's dominant integer work, with the
// round keys in the parameter block exactly as the anneal kernels take them), for the measured integer-issue
// peak the benchmark divides by.
__global__ void k_philox_rate(uint32_t* out, int iters, const PhiloxKeys K) {
  uint32_t c0 = blockIdx.x, c1 = threadIdx.x, c2 = 0, c3 = 0;
  for (int i = 0; i < iters; ++i) {
    philox10(c0, c1, c2, c3, K);
    c2 += (uint32_t)i;
  }
  if ((c0 ^ c1 ^ c2 ^ c3) == 0x9E3779B9u) out[0] = c0;  // keeps the work live; almost never stores
}

}  // namespace arp

extern "C" int arp_philox_rate(uint32_t* out, int blocks, int threads, int iters, void* stream) {
  if (blocks < 1 || threads < 32 || threads > 1024 || iters < 1) return ARP_ERR_SHAPE;
  if (!out) return ARP_ERR_ARG;
  arp::k_philox_rate<<<blocks, threads, 0, (cudaStream_t)stream>>>(out, iters, arp::philox_keys(0x12345678u, 0x9abcdef0u));
  return cudaGetLastError() == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" const char* arp_version(void) { return "arpeggio_b200 0.1 (sm_100a)"; }

extern "C" int arp_host_device_pointer(const void* host, void** dev) {
  if (!host || !dev) return ARP_ERR_ARG;
  *dev = nullptr;
  void* d = nullptr;
  if (cudaHostGetDevicePointer(&d, const_cast<void*>(host), 0) != cudaSuccess || !d) {
    cudaGetLastError();  // reset the runtime's last error after the failed query
    return ARP_ERR_ARG;
  }
  *dev = d;
  return ARP_OK;
}

extern "C" const char* arp_status_string(int code) {
  switch (code) {
    case ARP_OK: return "ok";
    case ARP_ERR_SHAPE: return "unsupported shape";
    case ARP_ERR_RANGE: return "coefficients or schedule beyond the exact 32-bit field range";
    case ARP_ERR_ARG: return "null pointer or bad argument";
    case ARP_ERR_LAUNCH: return "CUDA launch or configuration error";
    case ARP_ERR_TIMEOUT: return "bounded device wait gave up";
    case ARP_ERR_WORKSPACE: return "workspace too small";
    default: return "unknown status";
  }
}

extern "C" int arp_philox_kat(const uint32_t* in, uint32_t* out, int n, void* stream) {
  if (n < 0) return ARP_ERR_SHAPE;
  if (n == 0) return ARP_OK;
  if (!in || !out) return ARP_ERR_ARG;
  arp::k_philox_kat<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(in, out, n);
  return cudaGetLastError() == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}
