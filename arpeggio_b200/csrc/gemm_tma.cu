// C = A B^T for the warm-start network's large training products (bf16 operands, fp32 accumulation in TMEM): a
// persistent, warp-specialised tcgen05 kernel fed by TMA.
//
// Roles (320 threads, one CTA per SM):
//   warp 0     producer: one lane issues 2D tiled TMA loads (128-byte swizzle) of the A tile (128 rows) and the
//              B tile (BN rows) of each 64-wide k step into an S-slot shared-memory ring; a slot completes on its
//              `full` mbarrier by the loads' byte count;
//   warp 1     allocates TMEM for two BN-column accumulators; one lane issues the MMAs (M = 128, N = BN, K = 16,
//              four per k step) and commits them twice: to the slot's `empty` mbarrier (the slot may be refilled
//              once its MMAs have read it) and, after a work item's last k step, to the accumulator's `tfull`;
//   warps 2-9  epilogue: warp w reads TMEM lane quarter w % 4 (rows 32 (w % 4) ..), half (w - 2) / 4 of the
//              columns, of the finished accumulator with tcgen05.ld, applies the fused epilogue (gemm.cuh), stores
//              to global memory and releases the accumulator (`tempty`), so the MMAs of the next work item run
//              while this one drains.
// Work items (128-row tile, BN-column tile, K split) are dealt round-robin to the persistent CTAs.
// Every wait is bounded (ARP_ERR_TIMEOUT).  After a timeout every role stops issuing; before TMEM is released the
// producer waits (bounded) for the loads it has in flight and the MMA lane for the MMAs it has issued.
//
// Shared-memory layouts (every load fills this CTA's own shared memory only): a K-major operand box {64 k, R rows} lands as R rows of 128 bytes
// (SBO 1024); an MN-major operand is loaded as boxes {64 of M or N, 64 k}, 64 rows of 128 bytes each (SBO 1024
// between 8-k groups, LBO 8192 between the 64-element blocks).
#include <cuda.h>

#include <mutex>

#include "../../include/arpeggio_b200.h"
#include "arp_common.cuh"
#include "gemm.cuh"
#include "umma.cuh"

namespace arp {
namespace tmagemm {

constexpr int kThreads = 320;  // producer warp, MMA warp, eight epilogue warps
constexpr uint32_t kABytes = 128 * 128;  // 128 rows x 64 k x 2 bytes

template <int BN>
__host__ __device__ constexpr int stages() {
  return (192 * 1024) / (int)(kABytes + BN * 128) > 8 ? 8 : (192 * 1024) / (int)(kABytes + BN * 128);
}
template <int BN>
__host__ __device__ constexpr size_t smem_bytes() {
  return (size_t)stages<BN>() * (kABytes + BN * 128) + 1024;  // + room to align the ring to 1024 bytes
}

struct Work {
  int items, gx, gy, nkt, kt_per;
};

__device__ __forceinline__ void decode(const Work& w, int item, int& m0, int& n0, int& z, int& kt0, int& kt1, int BN) {
  // column tiles fastest: CTAs running at the same time share their A tile through L2
  const int nt = item % w.gy, rest = item / w.gy;
  n0 = nt * BN;
  m0 = (rest % w.gx) * 128;
  z = rest / w.gx;
  kt0 = z * w.kt_per;
  kt1 = min(w.nkt, kt0 + w.kt_per);
}

template <int BN, bool AMN, bool BMN>
__global__ void __launch_bounds__(kThreads, 1)
    k_gemm_tma(const __grid_constant__ CUtensorMap tma_a, const __grid_constant__ CUtensorMap tma_b,
               const GemmParams p, const Work wk) {
  constexpr int S = stages<BN>();
  constexpr uint32_t BBYTES = BN * 128, SBYTES = kABytes + BBYTES;
  constexpr uint32_t NCOL = 2 * BN < 32 ? 32 : 2 * BN;  // two accumulators
  constexpr uint32_t IDESC = umma::idesc_bf16(BN, AMN, BMN);
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ __align__(8) uint64_t full[S], empty[S], tfull[2], tempty[2], done;
  __shared__ uint32_t s_tmem;
  __shared__ volatile int s_abort;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t ring = (umma::su32(smem) + 1023u) & ~1023u;
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      umma::mbar_init(&full[s], 1);
      umma::mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      umma::mbar_init(&tfull[a], 1);
      umma::mbar_init(&tempty[a], 8);
    }
    umma::mbar_init(&done, 1);
    umma::fence_mbar_init();
    s_abort = 0;
    umma::tma_prefetch(&tma_a);
    umma::tma_prefetch(&tma_b);
  }
  if (warp == 1) umma::tmem_alloc(&s_tmem, NCOL);
  umma::tc_before_sync();
  __syncthreads();
  umma::tc_after_sync();
  const uint32_t tmem = s_tmem;

  if (warp == 0) {
    if (lane == 0) {
      // ---- producer
      int slot = 0, armed[S];
      uint32_t ph = 0;
      for (int s = 0; s < S; ++s) armed[s] = 0;
      for (int item = blockIdx.x; item < wk.items && !s_abort; item += gridDim.x) {
        int m0, n0, z, kt0, kt1;
        decode(wk, item, m0, n0, z, kt0, kt1, BN);
        for (int kt = kt0; kt < kt1; ++kt) {
          if (s_abort) break;
          if (!umma::mbar_wait(&empty[slot], ph ^ 1u)) {
            s_abort = 1;
            break;
          }
          const uint32_t sa = ring + (uint32_t)slot * SBYTES, sb = sa + kABytes;
          const int k0 = kt * 64;
          umma::expect_tx(&full[slot], SBYTES);
          if constexpr (AMN) {
            umma::tma_load_2d(sa, &tma_a, m0, k0, &full[slot]);
            umma::tma_load_2d(sa + 8192, &tma_a, m0 + 64, k0, &full[slot]);
          } else {
            umma::tma_load_2d(sa, &tma_a, k0, m0, &full[slot]);
          }
          if constexpr (BMN) {
#pragma unroll
            for (int c = 0; c < BN / 64; ++c) umma::tma_load_2d(sb + (uint32_t)c * 8192, &tma_b, n0 + 64 * c, k0, &full[slot]);
          } else {
            umma::tma_load_2d(sb, &tma_b, k0, n0, &full[slot]);
          }
          ++armed[slot];
          if (++slot == S) {
            slot = 0;
            ph ^= 1u;
          }
        }
      }
      // every load issued has landed before the CTA may leave (bounded)
      for (int s = 0; s < S; ++s)
        if (armed[s] > 0 && !umma::mbar_wait(&full[s], (uint32_t)((armed[s] - 1) & 1))) s_abort = 1;
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      // ---- MMA issue
      int slot = 0, it = 0;
      uint32_t ph = 0;
      for (int item = blockIdx.x; item < wk.items && !s_abort; item += gridDim.x, ++it) {
        int m0, n0, z, kt0, kt1;
        decode(wk, item, m0, n0, z, kt0, kt1, BN);
        const int ab = it & 1;
        const uint32_t aph = (uint32_t)((it >> 1) & 1);
        if (!umma::mbar_wait(&tempty[ab], aph ^ 1u)) {
          s_abort = 1;
          break;
        }
        umma::tc_after_sync();
        const uint32_t acc = tmem + (uint32_t)(ab * BN);
        bool ok = true;
        for (int kt = kt0; kt < kt1; ++kt) {
          if (!umma::mbar_wait(&full[slot], ph)) {
            ok = false;
            break;
          }
          umma::tc_after_sync();
          const uint32_t sa = ring + (uint32_t)slot * SBYTES, sb = sa + kABytes;
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            const uint64_t ad = AMN ? umma::sdesc_sw128(sa + kk * 2048, 8192, 1024) : umma::sdesc_sw128(sa + kk * 32, 16, 1024);
            const uint64_t bd = BMN ? umma::sdesc_sw128(sb + kk * 2048, 8192, 1024) : umma::sdesc_sw128(sb + kk * 32, 16, 1024);
            umma::mma(acc, ad, bd, IDESC, (kt > kt0 || kk > 0) ? 1u : 0u);
          }
          umma::commit(&empty[slot]);
          if (++slot == S) {
            slot = 0;
            ph ^= 1u;
          }
        }
        umma::commit(&tfull[ab]);  // arrives even on a timeout, so the epilogue is not left waiting
        if (!ok) {
          s_abort = 1;
          break;
        }
      }
      // every MMA issued has completed before TMEM is released (bounded)
      umma::commit(&done);
      if (!umma::mbar_wait(&done, 0)) s_abort = 1;
    }
    __syncwarp();
  } else {
    // ---- epilogue: warp w drains TMEM lane quarter w % 4, column half (w - 2) / 4
    const int q = warp & 3, c_lo = ((warp - 2) >> 2) * (BN / 2);
    int it = 0;
    for (int item = blockIdx.x; item < wk.items && !s_abort; item += gridDim.x, ++it) {
      int m0, n0, z, kt0, kt1;
      decode(wk, item, m0, n0, z, kt0, kt1, BN);
      const int ab = it & 1;
      const bool ok = umma::mbar_wait(&tfull[ab], (uint32_t)((it >> 1) & 1));
      umma::tc_after_sync();
      if (ok && !s_abort) {
        const int row = m0 + q * 32 + lane;
#pragma unroll 1
        for (int c = c_lo; c < c_lo + BN / 2; c += 32) {
          if (n0 + c >= p.N) break;
          uint32_t v[32];
          umma::tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * BN + c), v);
          if (row < p.M) epilogue<32>(p, row, n0 + c, v, z);
        }
      } else {
        s_abort = 1;
      }
      umma::tc_before_sync();
      __syncwarp();
      if (lane == 0) umma::mbar_arrive(&tempty[ab]);
      if (!ok) break;
    }
  }
  umma::tc_before_sync();
  __syncthreads();
  if (tid == 0 && s_abort) set_status(p.status, ARP_ERR_TIMEOUT);
  if (warp == 1) umma::tmem_free(tmem, NCOL);
}

}  // namespace tmagemm
}  // namespace arp

namespace arp {
namespace tmagemm {

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The driver's tensor-map encoder, looked up once through the runtime (no link against the driver library).
static EncodeTiled encoder() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(f);
  });
  return fn;
}

// A 2D bf16 tensor (inner x outer elements, rows ld elements apart) tiled in boxes of box_inner x box_outer with
// 128-byte swizzle; elements outside the tensor read as zero.
static bool tensor_map(CUtensorMap* m, const bf16* base, int inner, int outer, int ld, int box_inner, int box_outer) {
  const EncodeTiled enc = encoder();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)box_inner, (cuuint32_t)box_outer};
  const cuuint32_t es[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(base), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

constexpr int kMaxDevices = 64;

template <int BN, bool AMN, bool BMN>
static cudaError_t launch(const GemmParams& p, const Work& w, cudaStream_t st) {
  CUtensorMap ta, tb;
  // A: 128 rows x 64 k per step (K-major: one box; MN-major: two boxes of 64 rows); B: BN rows x 64 k
  const bool ok_a = AMN ? tensor_map(&ta, p.A, p.M, p.K, p.lda, 64, 64) : tensor_map(&ta, p.A, p.K, p.M, p.lda, 64, 128);
  const bool ok_b = BMN ? tensor_map(&tb, p.B, p.N, p.K, p.ldb, 64, 64) : tensor_map(&tb, p.B, p.K, p.N, p.ldb, 64, BN);
  if (!ok_a || !ok_b) return cudaErrorNotSupported;
  constexpr size_t smem = smem_bytes<BN>();
  static bool attr[kMaxDevices];
  static int sms[kMaxDevices];
  static std::mutex mu;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  {
    std::lock_guard<std::mutex> lock(mu);
    if (!attr[dev]) {
      e = cudaFuncSetAttribute(k_gemm_tma<BN, AMN, BMN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      e = cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return e;
      attr[dev] = true;
    }
  }
  const int grid = w.items < sms[dev] ? w.items : sms[dev];
  k_gemm_tma<BN, AMN, BMN><<<grid, kThreads, smem, st>>>(ta, tb, p, w);
  return cudaGetLastError();
}

template <int BN>
static cudaError_t launch_bn(const GemmParams& p, const Work& w, bool amn, bool bmn, cudaStream_t st) {
  if (!amn && !bmn) return launch<BN, false, false>(p, w, st);
  if (!amn && bmn) return launch<BN, false, true>(p, w, st);
  if (amn && !bmn) return launch<BN, true, false>(p, w, st);
  return launch<BN, true, true>(p, w, st);
}

}  // namespace tmagemm

bool gemm_tma_fits(const GemmParams& p) { return p.M >= 128 && p.N >= 64 && p.K >= 64; }

// Column tile width and K split from a small cost model: the operand bytes the tiles pull through L2
// (tiles x k steps x (A tile + B tile)) over the SMs that work at once (items per wave, at ~60 GB/s each), plus,
// for a split-K product, its partial tiles written and summed through HBM (~6 TB/s).  Wider tiles read A fewer
// times; narrower ones cover more SMs in short products and need fewer splits in long ones.
static int plan(const GemmParams& p, int sms, tmagemm::Work& out) {
  using namespace tmagemm;
  double best = 1e30;
  int best_bn = 64;
  for (int BN = 256; BN >= 64; BN >>= 1) {
    if (BN > 64 && BN > p.N) continue;
    Work w;
    w.gx = (p.M + 127) / 128;
    w.gy = (p.N + BN - 1) / BN;
    w.nkt = (p.K + 63) / 64;
    int split = 1;
    if (p.epi == EPI_F32_ACC) {  // split K until the work items fill the SMs once
      const int want = sms / (w.gx * w.gy);
      split = want < w.nkt ? want : w.nkt;
      if (split < 1) split = 1;
    }
    w.kt_per = (w.nkt + split - 1) / split;
    split = (w.nkt + w.kt_per - 1) / w.kt_per;
    w.items = w.gx * w.gy * split;
    const double waves = (double)((w.items + sms - 1) / sms);
    const double busy = w.items / waves;  // CTAs at work per wave, on average
    const double bytes = (double)w.gx * w.gy * w.nkt * (kABytes + BN * 128.0);
    double t = bytes / (busy * 60e9);
    if (split > 1) t += (double)split * p.M * p.N * 8.0 / 6e12;
    if (t < best) {
      best = t;
      best_bn = BN;
      out = w;
    }
  }
  return best_bn;
}

cudaError_t gemm_tma(const GemmParams& p0, bool amn, bool bmn, cudaStream_t st) {
  using namespace tmagemm;
  GemmParams p = p0;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    sms = 148;
  Work w;
  const int BN = plan(p, sms, w);
  const int split = w.items / (w.gx * w.gy);
  auto run = [&](const GemmParams& q) {
    return BN == 256 ? launch_bn<256>(q, w, amn, bmn, st)
                     : (BN == 128 ? launch_bn<128>(q, w, amn, bmn, st) : launch_bn<64>(q, w, amn, bmn, st));
  };
  if (split == 1) return run(p);
  // split K: each split's partial tile to a stream-ordered workspace, then C += the partials in split order
  float* ws = nullptr;
  const size_t mn = (size_t)p.M * p.N;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&ws), mn * split * sizeof(float), st);
  if (e != cudaSuccess) return e;
  GemmParams q = p;
  q.epi = EPI_F32_PART;
  q.C = ws;
  q.ldc = p.N;
  e = run(q);
  if (e == cudaSuccess) e = sum_splits(ws, split, p.M, p.N, reinterpret_cast<float*>(p.C), p.ldc, st);
  const cudaError_t ef = cudaFreeAsync(ws, st);
  return e != cudaSuccess ? e : ef;
}

}  // namespace arp
