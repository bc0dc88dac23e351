// arp_detect_dd_static: the detector call for callers that cannot allocate device memory.
//
// Who needs it: a receive chain that detects every frame under a hard latency budget cannot call cudaMalloc
// on the frame path (it synchronises the device and its latency is unbounded), and a plugin loaded into a
// host program whose allocator owns all device memory may not allocate at all.  Such callers still pass
// their own inputs and outputs, but the intermediates that arp_detect_dd keeps in a caller workspace (G, h,
// the MMSE guess, scale, spins, energies, counters) live here in one fixed array compiled into the library.
//
// Limits and sharing:
//  * the array holds kStaticScratchBytes (32 MiB); a batch whose arp_detect_dd_workspace() is larger is
//    refused with ARP_ERR_WORKSPACE before anything is launched (about 1500 uses of 32 users x 32 antennas
//    with 32 anneals, about 5900 uses of 16 x 16 with 16 anneals);
//  * every GPU that loads the library holds the 32 MiB until the process exits;
//  * all calls on a device share the one array and it keeps the last call's contents; nothing in it has to
//    start at zero because each stage writes its part before the next stage reads it, but two calls whose
//    work overlaps on the GPU (different streams, or different host threads without ordering) race on it;
//  * the first call on each device looks up the array's device address (cudaGetSymbolAddress, with that
//    device current) and caches it; make that first call before any stream capture.  The cached address
//    outlives a cudaDeviceReset (or any reset of the primary context), after which it no longer names the
//    array: the entry point is not for use on a device across such a reset.
#include <mutex>

#include "arp_common.cuh"
#include "arp_internal.h"

namespace arp {

constexpr size_t kStaticScratchBytes = (size_t)32 << 20;
constexpr int kMaxDevices = 128;

// The scratch itself.  In host code this name is only a stand-in for the symbol, never a device address.
static __device__ __align__(256) unsigned char g_detect_scratch[kStaticScratchBytes];

static std::mutex g_scratch_mu;
static void* g_scratch_addr[kMaxDevices];

// Device address of the scratch on the current device, looked up once per device.
static int static_scratch(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return ARP_ERR_LAUNCH;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_detect_scratch) != cudaSuccess || p == nullptr) return ARP_ERR_LAUNCH;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return ARP_OK;
}

}  // namespace arp

extern "C" int arp_detect_dd_static(const float* H, const float* y, const float* sigma2, int B, int NR2, int D,
                                    int M, int policy, int precision, int P, int R, const void* T, const void* c,
                                    int L, double q, uint32_t inst0, uint32_t k0, uint32_t k1, int start,
                                    int8_t* bits, int8_t* levels, float* dist, int32_t* pick, int32_t* status,
                                    void* stream) {
  if (B < 0 || D < 1 || D > 128 || !(P == 2 || P == 4 || P == 6) || R < 1) return ARP_ERR_SHAPE;
  if (precision != 0 && precision != 1) return ARP_ERR_ARG;
  if (B == 0) return ARP_OK;
  const size_t need = arp_detect_dd_workspace(B, D, P, R, precision, nullptr);
  if (need == 0 || need > arp::kStaticScratchBytes) return ARP_ERR_WORKSPACE;
  void* scratch = nullptr;
  const int rc = arp::static_scratch(&scratch);
  if (rc != ARP_OK) return rc;
  return arp_detect_dd(H, y, sigma2, B, NR2, D, M, policy, precision, P, R, T, c, L, q, inst0, k0, k1, start,
                       scratch, arp::kStaticScratchBytes, bits, levels, dist, pick, status, stream);
}
