// Detector stages around the anneal: Gram/field formation with the MMSE guess (map) and the readout.
//
// map (one block per channel use; mimo.py:98-109 mmse, :176-182 _mu, :86-88 quantize_levels,
// :506-523 ising_delta_at, chordfx.py:60-76 to_fixed, chord_ref.py:47-59 compress):
//   Q = H^T H on the tensor cores, exactly: per use H is scaled by a power of two so that its largest entry
//   is just below 2^30, rounded to integers x and split into four signed 8-bit digits (x = sum_a 2^(8a) d_a);
//   tcgen05.mma kind::i8 forms the digit products d_a^T d_b with exact s32 accumulation in TMEM, grouped by
//   weight a + b (classes 6, 5, 4, 3; the dropped lower classes move an entry by ~2^-26 of the largest |Q|, well
//   below the FP32 rounding of the reference's own product), and the epilogue
//   sums the classes exactly as a 64-bit integer and rounds once to float.  Q is exactly symmetric (an exact integer
//   sum), as the symmetrised J of to_fixed.  g = H^T y as an ordered fma chain per coordinate;
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
#include "arp_internal.h"
#include "umma.cuh"

namespace arp {

// Rows of H staged per chunk (Dp = padded width): all of a 64 x 64 problem at once; 32-row chunks at 128.
template <int Dp>
__host__ __device__ constexpr int kChunkRows() { return Dp <= 64 ? 64 : 32; }

__device__ __forceinline__ float nearest_level(float v, int M) {
  if (M == 4) return fabsf(v - 1.0f) < fabsf(v + 1.0f) ? 1.0f : -1.0f;  // ties -> the first level, -1
  if (M == 64) {  // nearest odd level in [-7, 7], the lower one on ties
    const float l = 2.0f * ceilf(0.5f * v) - 1.0f;
    return fminf(fmaxf(l, -7.0f), 7.0f);
  }
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

// Half-warp sum (the 16 threads that share a tile row).
__device__ __forceinline__ float hsum16(float v) {
#pragma unroll
  for (int o = 8; o; o >>= 1) v += __shfl_xor_sync(ARP_FULL, v, o);
  return v;
}

// TB consecutive floats of shared memory in one access (16-byte aligned when TB % 4 == 0, 8-byte when TB == 2).
template <int TB>
__device__ __forceinline__ void lds_vec(const float* p, float (&v)[TB]) {
  if constexpr (TB % 4 == 0) {
#pragma unroll
    for (int q = 0; q < TB / 4; ++q) {
      const float4 t = reinterpret_cast<const float4*>(p)[q];
      v[4 * q] = t.x;
      v[4 * q + 1] = t.y;
      v[4 * q + 2] = t.z;
      v[4 * q + 3] = t.w;
    }
  } else if constexpr (TB == 2) {
    const float2 t = *reinterpret_cast<const float2*>(p);
    v[0] = t.x;
    v[1] = t.y;
  } else {
#pragma unroll
    for (int i = 0; i < TB; ++i) v[i] = p[i];
  }
}
template <int TB>
__device__ __forceinline__ void sts_vec(float* p, const float (&v)[TB]) {
  if constexpr (TB % 4 == 0) {
#pragma unroll
    for (int q = 0; q < TB / 4; ++q)
      reinterpret_cast<float4*>(p)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  } else if constexpr (TB == 2) {
    *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
  } else {
#pragma unroll
    for (int i = 0; i < TB; ++i) p[i] = v[i];
  }
}

// A row's dot product sum_j x_j y_j: the thread's TB columns as one fma chain (from 0), then the butterfly over
// the 16 threads of the row.
template <int TB>
__device__ __forceinline__ float row_dot(const float (&x)[TB], const float (&y)[TB]) {
  float v = 0.0f;
#pragma unroll
  for (int j = 0; j < TB; ++j) v = __fmaf_rn(x[j], y[j], v);
  return hsum16(v);
}

// The D x D work is tiled over a GS x GS (16 x 16) thread grid: thread (ty, tx) owns rows ty*TB .. ty*TB+TB-1
// and columns tx*TB .. tx*TB+TB-1 of Q and of the inverse, in registers.  Dp = GS TB >= D; padded rows and
// columns of H are zero and the padded diagonal of A is 1, so the inverse's D x D block is unchanged.  (A 32 x 32
// grid of 2 x 2 tiles was measured for one frame and is slower: the 64 elimination steps are latency-bound and
// a 1024-thread barrier per step costs more than the smaller tiles save.)
// Gram on the tensor cores: digit planes of one row chunk (CH rows of H) in the canonical K-major no-swizzle
// layout of 8-bit operands -- core matrices of 8 rows (coordinates) x 16 bytes (rows of H), LBO = 128 B between
// neighbours along K, SBO = (CH / 16) 128 B between 8-coordinate groups; one MMA consumes K = 32 (two core
// matrices).  MP = the MMA's M: 64 for Dp <= 64 (rows Dp .. 63 zero), else 128.
template <int Dp>
__host__ __device__ constexpr int kMmaM() { return Dp <= 64 ? 64 : 128; }
template <int Dp>
__host__ __device__ constexpr int kPlaneBytes() { return kMmaM<Dp>() * kChunkRows<Dp>(); }
template <int Dp>
__host__ __device__ constexpr int kTmemCols() {  // four class accumulators of Dp columns, a power of two >= 32
  return 4 * Dp <= 32 ? 32 : (4 * Dp <= 64 ? 64 : (4 * Dp <= 128 ? 128 : (4 * Dp <= 256 ? 256 : 512)));
}

// The digit pairs (a, b) of each class a + b = 6, 5, 4, 3, in issue order.
__constant__ int8_t kPairA[10] = {3, 3, 2, 3, 1, 2, 3, 0, 2, 1};
__constant__ int8_t kPairB[10] = {3, 2, 3, 1, 3, 2, 0, 3, 1, 2};
__constant__ int8_t kPairC[10] = {0, 1, 1, 2, 2, 2, 3, 3, 3, 3};  // accumulator: class 6 - c

// Register bounds for more resident blocks (the Gauss-Jordan steps are barrier-latency bound, so blocks overlap):
// four per SM at 32 users (64 registers, a few spilled: 3.95 -> 3.73 ms per 65536 uses), two per SM at 64 users
// (126 registers: 28.8 -> 19.3 ms per 65536 uses); the same outputs bit for bit.
template <int TB, int GS>
__global__ void __launch_bounds__(GS * GS, TB == 8 ? 2 : (TB == 4 ? 4 : 1)) k_map_dd(const MapParams a) {
  constexpr int Dp = GS * TB, QP = Dp + 4, NT = GS * GS;
  constexpr int CH = kChunkRows<Dp>(), MP = kMmaM<Dp>(), KG = CH / 16, PB = kPlaneBytes<Dp>();
  constexpr uint32_t NCOL = kTmemCols<Dp>();
  extern __shared__ __align__(128) float smap[];
  uint8_t* planes = reinterpret_cast<uint8_t*>(smap);  // 4 digit planes, PB bytes each (aliases Qs below)
  float* Hc = smap + (PB * 4 > Dp * QP * 4 ? PB : Dp * QP);  // CH x Dp
  float* Qs = smap;                            // Dp x QP, written once the Gram's MMAs have completed
  float* rk = Hc + CH * Dp;       // 2 x Dp (double-buffered row k)
  float* ck = rk + 2 * Dp;        // 2 x Dp (double-buffered column k)
  float* gv = ck + 2 * Dp;        // Dp
  float* xv = gv + Dp;            // Dp
  float* red = xv + Dp;           // NT / 32
  float* yc = red + NT / 32;      // CH: the chunk's rows of y
  __shared__ __align__(8) uint64_t mma_bar;
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort, s_exp;
  const int D = a.D, NR2 = a.NR2, b = blockIdx.x;
  const int tid = threadIdx.x, tx = tid % GS, ty = tid / GS, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    umma::mbar_init(&mma_bar, 1);
    umma::fence_mbar_init();
    s_abort = 0;
  }
  const int u = a.idx ? a.idx[b] : b;
  const float* Hb = a.H + (size_t)u * NR2 * D;
  const float* yb = a.y + (size_t)u * NR2;
  // ---- the use's power-of-two scale (largest |H| just below 2^30 after scaling): from the staged rows when they
  //      fit one chunk, else from a pass over H first
  const bool one_chunk = NR2 <= CH;
  auto set_scale = [&](float mx) {  // mx: this thread's part; every thread leaves with s_exp set
#pragma unroll
    for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(ARP_FULL, mx, o));
    if (lane == 0) red[warp] = mx;
    __syncthreads();
    if (tid == 0) {
      float m = 0.0f;
      for (int w = 0; w < NT / 32; ++w) m = fmaxf(m, red[w]);
      int e = 0;
      if (m > 0.0f) frexpf(m, &e);  // m in [2^(e-1), 2^e)
      s_exp = m > 0.0f ? 30 - e : 0;
    }
    __syncthreads();
  };
  if (!one_chunk) {
    float mx = 0.0f;
    for (int x = tid; x < NR2 * D; x += NT) mx = fmaxf(mx, fabsf(Hb[x]));
    set_scale(mx);
  }
  float gacc = 0.0f;
  constexpr uint32_t IDESC = umma::idesc_s8(MP, Dp);
  const uint32_t pbase = umma::su32(planes);
  int nchunk = 0;
  for (int r0 = 0; r0 < NR2; r0 += CH, ++nchunk) {
    const int nr = min(CH, NR2 - r0);
    __syncthreads();  // the previous chunk's digits were read by MMAs that have completed (waited below)
    if (s_abort) break;
    for (int x = tid; x < nr; x += NT) yc[x] = yb[r0 + x];
    float mx = 0.0f;
    if (D == Dp && (D & 3) == 0) {
      const float4* src = reinterpret_cast<const float4*>(Hb + (size_t)r0 * D);
      float4* dst = reinterpret_cast<float4*>(Hc);
      for (int x = tid; x < nr * Dp / 4; x += NT) {
        const float4 v = src[x];
        dst[x] = v;
        mx = fmaxf(fmaxf(mx, fmaxf(fabsf(v.x), fabsf(v.y))), fmaxf(fabsf(v.z), fabsf(v.w)));
      }
    } else {
      for (int x = tid; x < nr * Dp; x += NT) {
        const int r = x / Dp, j = x - r * Dp;
        const float v = j < D ? Hb[(size_t)(r0 + r) * D + j] : 0.0f;
        Hc[x] = v;
        mx = fmaxf(mx, fabsf(v));
      }
    }
    if (one_chunk)
      set_scale(mx);  // its barriers also publish the staged rows
    else
      __syncthreads();
    const int sx = s_exp;
    if (tid < Dp)
      for (int r = 0; r < nr; ++r) gacc = __fmaf_rn(Hc[r * Dp + tid], yc[r], gacc);
    // digit planes: a warp writes one core matrix (8 coordinates x 16 rows) at a time, lane = coordinate m % 8
    // + 8 (row quad), one 32-bit word of four rows per plane (conflict-free); rows >= nr and coordinates >= Dp
    // are zero.  The signed digits of x (|x| < 2^30) are the bytes of (x + 0x808080) ^ 0x808080: adding 128 at each
    // of the three low digit positions makes every low byte u_a = d_a + 128 with the borrow carried up, and the
    // XOR turns u_a into d_a's two's-complement byte; the top byte is d3.  A 4 x 4 byte transpose (eight byte
    // permutes) turns four rows' digit words into one word per plane.
    const int ksteps = (nr + 31) >> 5;
    const bool fast_scale = sx >= -126 && sx <= 127;
    const float fs = fast_scale ? __int_as_float((sx + 127) << 23) : 1.0f;
    for (int cm = warp; cm < (MP / 8) * KG; cm += NT / 32) {
      const int mg = cm / KG, kg = cm - mg * KG;
      const int m = mg * 8 + (lane & 7), k0 = kg * 16 + (lane >> 3) * 4;
      uint32_t z[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int k = k0 + i;
        const float v = (m < Dp && k < nr) ? Hc[k * Dp + m] : 0.0f;
        const int32_t x = __float2int_rn(fast_scale ? __fmul_rn(v, fs) : ldexpf(v, sx));
        z[i] = ((uint32_t)x + 0x808080u) ^ 0x808080u;
      }
      const uint32_t t0 = __byte_perm(z[0], z[1], 0x5140), t1 = __byte_perm(z[2], z[3], 0x5140);
      const uint32_t t2 = __byte_perm(z[0], z[1], 0x7362), t3 = __byte_perm(z[2], z[3], 0x7362);
      const uint32_t wd[4] = {__byte_perm(t0, t1, 0x5410), __byte_perm(t0, t1, 0x7632), __byte_perm(t2, t3, 0x5410),
                              __byte_perm(t2, t3, 0x7632)};
      const uint32_t off = (uint32_t)(mg * KG * 128 + kg * 128 + (lane & 7) * 16 + (lane >> 3) * 4);
#pragma unroll
      for (int p = 0; p < 4; ++p) *reinterpret_cast<uint32_t*>(planes + p * PB + off) = wd[p];
    }
    umma::fence_async_smem();
    // TMEM is held only from the first MMA to the end of the epilogue; this grid lets dependent kernels launch
    // (pdl_trigger) only after its blocks have released it, so a dependent that holds TMEM while it waits for
    // this grid can never take the columns a block of this grid still needs
    if (nchunk == 0 && warp == 0) umma::tmem_alloc(&s_tmem, NCOL);
    umma::tc_before_sync();
    __syncthreads();
    umma::tc_after_sync();
    if (tid == 0) {
      const uint32_t tmem = s_tmem;
      for (int ks = 0; ks < ksteps; ++ks) {
#pragma unroll
        for (int q = 0; q < 10; ++q) {
          const uint64_t ad = umma::sdesc(pbase + kPairA[q] * PB + ks * 256, 128, KG * 128);
          const uint64_t bd = umma::sdesc(pbase + kPairB[q] * PB + ks * 256, 128, KG * 128);
          // the first product of each class in the first chunk starts its accumulator
          const bool first = nchunk == 0 && ks == 0 && (q == 0 || q == 1 || q == 3 || q == 6);
          umma::mma_s8(tmem + (uint32_t)(kPairC[q] * Dp), ad, bd, IDESC, first ? 0u : 1u);
        }
      }
      umma::commit(&mma_bar);
    }
    if (!umma::mbar_wait(&mma_bar, (uint32_t)(nchunk & 1))) s_abort = 1;
  }
  __syncthreads();
  umma::tc_after_sync();
  const uint32_t tmem = s_tmem;
  if (s_abort) {  // an MMA never completed: report, wait once more for it, free TMEM, leave
    if (tid == 0) {
      set_status(a.status, ARP_ERR_TIMEOUT);
      umma::mbar_wait(&mma_bar, (uint32_t)((nchunk - 1) & 1));
    }
    __syncthreads();
    if (warp == 0) umma::tmem_free(tmem, NCOL);
    return;
  }
  // ---- epilogue: each entry of Q from the four class accumulators, summed exactly as an integer
  //      P = ((c6 2^8 + c5) 2^8 + c4) 2^8 + c3 (|P| < 2^50), converted once with rounding to nearest and scaled by
  //      2^(24 - 2s) (exact).  TMEM lane of row m: m (M = 128), or m % 16 + 32 (m / 16) (M = 64); warps w and w + 4
  //      read lanes 32 (w % 4) .. + 31, the first and the second half of the columns.
  {
    const int wq = warp & 3, half = warp >> 2;
    const int m = MP == 128 ? wq * 32 + lane : wq * 16 + lane;
    const bool valid = (MP == 128 || lane < 16) && m < Dp;
    const int e2 = 24 - 2 * s_exp;
    // scaling by 2^e2 as one multiply where 2^e2 is a normal float (the same correctly rounded product as ldexpf)
    const bool fast_e2 = e2 >= -126 && e2 <= 127;
    const float f2 = fast_e2 ? __int_as_float((e2 + 127) << 23) : 1.0f;
    constexpr int CW = Dp >= 16 ? Dp / 2 : Dp;
#pragma unroll 1
    for (int c0 = half * CW; c0 < (half + 1) * CW && c0 < Dp; c0 += 8) {
      uint32_t v6[8], v5[8], v4[8], v3[8];
      const uint32_t ta = tmem + ((uint32_t)(wq * 32) << 16) + (uint32_t)c0;
      umma::tmem_ld8_nowait(ta, v6);
      umma::tmem_ld8_nowait(ta + Dp, v5);
      umma::tmem_ld8_nowait(ta + 2 * Dp, v4);
      umma::tmem_ld8_nowait(ta + 3 * Dp, v3);
      umma::tmem_wait_ld();
      if (valid) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const long long q = ((((long long)(int32_t)v6[j] * 256 + (int32_t)v5[j]) * 256 + (int32_t)v4[j]) * 256) +
                              (int32_t)v3[j];
          const float qf = __ll2float_rn(q);
          Qs[m * QP + c0 + j] = fast_e2 ? __fmul_rn(qf, f2) : ldexpf(qf, e2);
        }
      }
    }
  }
  umma::tc_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tmem, NCOL);
  pdl_trigger();  // the chain's next kernel may launch and set up; it waits for this grid before reading
  float A[TB][TB];
  float qmax = 0.0f;
  const float s2 = a.xg ? 0.0f : a.sigma2[b];  // only the MMSE solve reads sigma2 (null for a given guess)
#pragma unroll
  for (int i = 0; i < TB; ++i) lds_vec<TB>(Qs + (ty * TB + i) * QP + tx * TB, A[i]);  // TB floats per access
#pragma unroll
  for (int i = 0; i < TB; ++i)
#pragma unroll
    for (int j = 0; j < TB; ++j) {
      const int gi = ty * TB + i, gj = tx * TB + j;
      qmax = fmaxf(qmax, fabsf(A[i][j]));
      if (gi == gj) A[i][j] = gi < D ? __fadd_rn(A[i][j], s2) : 1.0f;
    }
  if (tid < Dp) gv[tid] = gacc;
  if (a.xg) {
    // the guess is given (MDI stages): map around it, no MMSE solve
    if (tid < Dp) {
      const float lv = tid < D ? (float)a.xg[(size_t)u * a.xg_stride + tid] : 0.0f;
      xv[tid] = lv;
      if (tid < D) a.xq[(size_t)b * D + tid] = (int8_t)lv;
    }
    __syncthreads();
  } else {
    // ---- in-place Gauss-Jordan inverse of A = Q + sigma2 I (SPD, no pivoting), one barrier per step;
    //      k = kt*TB + kr with kr unrolled so the register tile is always indexed at compile time
    for (int kt = 0; kt < GS; ++kt) {
#pragma unroll
      for (int kr = 0; kr < TB; ++kr) {
        const int k = kt * TB + kr, buf = (k & 1) * Dp;
        if (ty == kt) {
          float rw[TB];
#pragma unroll
          for (int j = 0; j < TB; ++j) rw[j] = A[kr][j];
          sts_vec<TB>(rk + buf + tx * TB, rw);
        }
        if (tx == kt) {
          float cw[TB];
#pragma unroll
          for (int i = 0; i < TB; ++i) cw[i] = A[i][kr];
          sts_vec<TB>(ck + buf + ty * TB, cw);
        }
        __syncthreads();
        const float inv = __frcp_rn(rk[buf + k]);
        float f[TB], rj[TB];
        lds_vec<TB>(ck + buf + ty * TB, f);
        lds_vec<TB>(rk + buf + tx * TB, rj);
#pragma unroll
        for (int i = 0; i < TB; ++i) f[i] = __fmul_rn(f[i], inv);
#pragma unroll
        for (int i = 0; i < TB; ++i)
#pragma unroll
          for (int j = 0; j < TB; ++j) A[i][j] = __fmaf_rn(-f[i], rj[j], A[i][j]);
        if (ty == kt) {
#pragma unroll
          for (int j = 0; j < TB; ++j) A[kr][j] = __fmul_rn(rj[j], inv);
        }
        if (tx == kt) {
#pragma unroll
          for (int i = 0; i < TB; ++i) A[i][kr] = -f[i];
          if (ty == kt) A[kr][kr] = inv;
        }
      }
    }
    // ---- z = A^-1 g, mu = diag(A^-1 Q) (Q symmetric: sum_j Ainv_ij Q_ij), x_q
    float zp[TB], mp[TB], gj[TB];
    lds_vec<TB>(gv + tx * TB, gj);
#pragma unroll
    for (int i = 0; i < TB; ++i) {
      float ar[TB], qj[TB];
      lds_vec<TB>(Qs + (ty * TB + i) * QP + tx * TB, qj);
#pragma unroll
      for (int j = 0; j < TB; ++j) ar[j] = A[i][j];
      zp[i] = row_dot<TB>(ar, gj);
      mp[i] = row_dot<TB>(ar, qj);
    }
    if (tx == 0) {
#pragma unroll
      for (int i = 0; i < TB; ++i) {
        const int gi = ty * TB + i;
        const float zu = gi < D ? __fdiv_rn(zp[i], mp[i]) : 0.0f;
        const float lv = gi < D ? nearest_level(zu, a.M) : 0.0f;
        xv[gi] = lv;
        if (gi < D) a.xq[(size_t)b * D + gi] = (int8_t)lv;
        if (a.zs && gi < D) a.zs[(size_t)b * D + gi] = zu;
        ck[gi] = gi < D ? nearest_level(zp[i], a.M) : 0.0f;  // RI map: spins of the unbiased z (mimo.py:148)
      }
    }
    __syncthreads();
  }
  if (a.ri) {
    // ---- RI map: T = [2I, I] (16-QAM) or I (QPSK); h = 2 (HT)^T y, J = -offdiag(T^T Q T), scale by max
    const bool qam = a.M == 16;
    const int N = qam ? 2 * D : D;
    float off = 0.0f, dgm = 0.0f, gm = 0.0f;
#pragma unroll
    for (int i = 0; i < TB; ++i)
#pragma unroll
      for (int j = 0; j < TB; ++j) {
        const int gi = ty * TB + i, gj = tx * TB + j;
        if (gi < D && gj < D) {
          const float v = fabsf(Qs[gi * QP + gj]);
          if (gi == gj)
            dgm = fmaxf(dgm, v);
          else
            off = fmaxf(off, v);
        }
      }
    if (tid < D) gm = fabsf(gv[tid]);
    float sc = qam ? fmaxf(fmaxf(4.0f * off, 2.0f * dgm), 4.0f * gm) : fmaxf(off, 2.0f * gm);
#pragma unroll
    for (int o = 16; o; o >>= 1) sc = fmaxf(sc, __shfl_xor_sync(ARP_FULL, sc, o));
    if (lane == 0) red[tid >> 5] = sc;
    __syncthreads();
    sc = 0.0f;
#pragma unroll
    for (int w = 0; w < NT / 32; ++w) sc = fmaxf(sc, red[w]);
    sc = fmaxf(sc, 1e-12f);
    if (tid == 0) a.scale[b] = sc;
    float* Jo = a.Jri + (size_t)b * N * N;
#pragma unroll
    for (int i = 0; i < TB; ++i)
#pragma unroll
      for (int j = 0; j < TB; ++j) {
        const int gi = ty * TB + i, gj = tx * TB + j;
        if (gi >= D || gj >= D) continue;
        const float q = Qs[gi * QP + gj];
        if (qam) {
          Jo[(size_t)gi * N + gj] = gi == gj ? 0.0f : __fdiv_rn(-4.0f * q, sc);
          Jo[(size_t)gi * N + D + gj] = __fdiv_rn(-2.0f * q, sc);
          Jo[(size_t)(D + gi) * N + gj] = __fdiv_rn(-2.0f * q, sc);
          Jo[(size_t)(D + gi) * N + D + gj] = gi == gj ? 0.0f : __fdiv_rn(-q, sc);
        } else {
          Jo[(size_t)gi * N + gj] = gi == gj ? 0.0f : __fdiv_rn(-q, sc);
        }
      }
    const float r2 = __fmul_rn(2.0f, a.r_reg);
    for (int i = tid; i < D; i += NT) {
      const float lv = ck[i];
      const float hv[2] = {qam ? __fmul_rn(4.0f, gv[i]) : __fmul_rn(2.0f, gv[i]), __fmul_rn(2.0f, gv[i])};
      const float sp[2] = {qam ? (lv > 0.0f ? 1.0f : -1.0f) : lv, (lv == 3.0f || lv == -1.0f) ? 1.0f : -1.0f};
      for (int c = 0; c < (qam ? 2 : 1); ++c) {
        const int k = c * D + i;
        const float h0 = __fdiv_rn(hv[c], sc);
        a.h0ri[(size_t)b * N + k] = h0;
        a.hri[(size_t)b * N + k] = __fadd_rn(h0, __fmul_rn(r2, sp[c]));
        a.sP[(size_t)b * N + k] = (int8_t)sp[c];
      }
    }
    return;
  }
  // ---- h = 2 (g - Q x_q), scale = max(|h|, |Q|)
  float hp[TB], xj[TB];
  lds_vec<TB>(xv + tx * TB, xj);
#pragma unroll
  for (int i = 0; i < TB; ++i) {
    float qj[TB];
    lds_vec<TB>(Qs + (ty * TB + i) * QP + tx * TB, qj);
    hp[i] = row_dot<TB>(qj, xj);
    hp[i] = __fmul_rn(2.0f, __fsub_rn(gv[ty * TB + i], hp[i]));
    if (ty * TB + i < D) qmax = fmaxf(qmax, fabsf(hp[i]));
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) qmax = fmaxf(qmax, __shfl_xor_sync(ARP_FULL, qmax, o));
  if (lane == 0) red[tid >> 5] = qmax;
  __syncthreads();
  float sc = 0.0f;
#pragma unroll
  for (int w = 0; w < NT / 32; ++w) sc = fmaxf(sc, red[w]);
  sc = fmaxf(sc, 1e-12f);
  if (tid == 0) a.scale[b] = sc;
  // ---- outputs: G = Q / scale (x 4096, rounded half to even), h likewise
  const bool quant = a.qscale > 0.0f;
#pragma unroll
  for (int i = 0; i < TB; ++i) {
    const int gi = ty * TB + i;
    if (gi >= D) continue;
#pragma unroll
    for (int j = 0; j < TB; ++j) {
      const int gj = tx * TB + j;
      if (gj >= D) continue;
      const float v = __fdiv_rn(Qs[gi * QP + gj], sc);
      if (quant)
        reinterpret_cast<int32_t*>(a.G)[((size_t)b * D + gi) * D + gj] = (int32_t)rintf(__fmul_rn(v, a.qscale));
      else
        reinterpret_cast<float*>(a.G)[((size_t)b * D + gi) * D + gj] = v;
    }
    if (tx == 0) {
      const float v = __fdiv_rn(hp[i], sc);
      if (quant)
        reinterpret_cast<int32_t*>(a.h)[(size_t)b * D + gi] = (int32_t)rintf(__fmul_rn(v, a.qscale));
      else
        reinterpret_cast<float*>(a.h)[(size_t)b * D + gi] = v;
    }
  }
}

template <int TB, int GS>
static size_t map_smem() {
  constexpr int Dp = GS * TB, PB = kPlaneBytes<Dp>();
  constexpr size_t front = PB * 4 > Dp * (Dp + 4) * 4 ? (size_t)PB : (size_t)Dp * (Dp + 4);  // planes | Qs, floats
  return sizeof(float) * (front + (size_t)kChunkRows<Dp>() * (Dp + 1) + 6 * (size_t)Dp + GS * GS / 32);
}

template <int TB, int GS = 16>
static cudaError_t launch_map(const MapParams& a, cudaStream_t st) {
  const size_t smem = map_smem<TB, GS>();
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_map_dd<TB, GS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_map_dd<TB, GS><<<a.B, GS * GS, smem, st>>>(a);
  return cudaGetLastError();
}


constexpr int kReadThreads = 256;

// One block per channel use.  H is staged transposed with a padded stride (Hs[j][i], NR2 + 1) so that the
// 32 lanes of a warp, which own rows i = lane + 32 m, read consecutive words.  r0 = y - H x_q is formed once;
// candidate c's residual is r0 - sum_j H[:, j] e_j over the few coordinates where its clipped level differs
// from the guess (e = x - x_q), and its distance is ||r||^2.
// MR: rows of H per lane (NR2 <= 32 MR); rows beyond NR2 add exact zeros, so every MR gives the same sums.
template <int MR>
__global__ void __launch_bounds__(kReadThreads) k_readout_dd(const ReadParams a) {
  extern __shared__ __align__(16) float sm[];
  const int D = a.D, NR2 = a.NR2, P = a.P, R = a.R, b = blockIdx.x;
  const int HS = NR2 + 1;
  pdl_wait();
  float* Hs = sm;                   // D x HS (transposed)
  float* r0 = Hs + D * HS;          // NR2
  float* bd = r0 + NR2;             // 8
  int* br = reinterpret_cast<int*>(bd + 8);  // 8
  int8_t* ek = reinterpret_cast<int8_t*>(br + 8);  // (R + 1) x D: candidate level minus guess; row R = x_q
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, W = kReadThreads / 32;
  const int lo = 1 - pam_size(a.M), hi = -lo;
  const int u = a.idx ? a.idx[b] : b;
  const float* Hb = a.H + (size_t)u * NR2 * D;
  if ((D & 3) == 0 && (reinterpret_cast<uintptr_t>(Hb) & 15u) == 0) {  // 16-byte loads, four columns of a row
    const float4* H4 = reinterpret_cast<const float4*>(Hb);
    for (int x = tid; x < NR2 * D / 4; x += kReadThreads) {
      const float4 v = H4[x];
      const int i = (4 * x) / D, j = 4 * x - i * D;
      Hs[j * HS + i] = v.x;
      Hs[(j + 1) * HS + i] = v.y;
      Hs[(j + 2) * HS + i] = v.z;
      Hs[(j + 3) * HS + i] = v.w;
    }
  } else {
    for (int x = tid; x < NR2 * D; x += kReadThreads) {
      const int i = x / D, j = x - i * D;
      Hs[j * HS + i] = Hb[x];
    }
  }
  int8_t* xq8 = ek + R * D;
  for (int j = tid; j < D; j += kReadThreads)
    xq8[j] = a.mdi ? a.xg[(size_t)u * a.xg_stride + j] : a.xq[(size_t)b * D + j];
  __syncthreads();
  // every candidate's clipped delta from the guess, from one coalesced pass over its spins
  const int8_t* sb = a.spins + (size_t)b * R * P * D;  // spins are per problem b (group-local)
  if (!a.ri && (D & 15) == 0 && P <= 6 && (reinterpret_cast<uintptr_t>(sb) & 15u) == 0) {
    // 16 coordinates of one candidate per thread: its P 16-byte spin loads are all in flight at once
    const int ng = D >> 4;
    for (int x = tid; x < R * ng; x += kReadThreads) {
      const int c = x / ng, j0 = (x - c * ng) << 4;
      int4 sv[6];
#pragma unroll
      for (int p = 0; p < 6; ++p)
        if (p < P) sv[p] = *reinterpret_cast<const int4*>(sb + (size_t)c * P * D + p * D + j0);
      int8_t* ec = ek + c * D + j0;
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        int d = 0;
#pragma unroll
        for (int p = 0; p < 6; ++p)
          if (p < P) d += reinterpret_cast<const int8_t*>(&sv[p])[q];
        const int xv = min(max((int)xq8[j0 + q] + d, lo), hi);
        ec[q] = (int8_t)(xv - xq8[j0 + q]);
      }
    }
  } else {
    for (int x = tid; x < R * D; x += kReadThreads) {
      const int c = x / D, j = x - c * D;
      int xv;
      if (a.ri) {  // RI spins: l = 2 s1 + s2 (16-QAM) or s (QPSK), mimo.spins_to_levels (mimo.py:39-42)
        xv = P == 1 ? sb[(size_t)c * D + j] : 2 * sb[(size_t)c * 2 * D + j] + sb[(size_t)c * 2 * D + D + j];
      } else {
        int d = 0;
        for (int p = 0; p < P; ++p) d += sb[(size_t)c * P * D + p * D + j];
        xv = min(max((int)xq8[j] + d, lo), hi);
      }
      ek[x] = (int8_t)(xv - xq8[j]);
    }
  }
  for (int i = tid; i < NR2; i += kReadThreads) {
    float r = a.y[(size_t)u * NR2 + i];
    for (int j = 0; j < D; ++j) r = __fmaf_rn(-Hs[j * HS + i], (float)xq8[j], r);
    r0[i] = r;
  }
  __syncthreads();
  float best = FLT_MAX;
  int bi = INT_MAX;
  const int last = a.mdi ? R - 1 : R;  // MDI stages compare the candidates with the use's current best instead
  const int nbl = a.M == 4 ? 1 : 2, nbits = D * nbl;
  const bool soft = a.llr != nullptr;
  float mb0[8], mb1[8];  // per-warp minima of the distance over list entries with bit k = 0 / 1, k = lane + 32 m
#pragma unroll
  for (int m = 0; m < 8; ++m) mb0[m] = mb1[m] = FLT_MAX;
  for (int c = wid; c <= last; c += W) {
    float acc = 0.0f;
    if (c == R) {
      for (int i = lane; i < NR2; i += 32) acc = __fmaf_rn(r0[i], r0[i], acc);
    } else {
      const int8_t* e = ek + c * D;
      uint32_t nzm[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int j = t * 32 + lane;
        nzm[t] = __ballot_sync(ARP_FULL, j < D && e[j] != 0);
      }
      constexpr int U = MR <= 2 ? 4 : (MR == 4 ? 2 : 1);  // coordinates in flight, within the registers of MR rows
      float rr[MR];
#pragma unroll
      for (int m = 0; m < MR; ++m) rr[m] = (lane + 32 * m < NR2) ? r0[lane + 32 * m] : 0.0f;
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        uint32_t mm = nzm[t];
        while (mm) {  // U differing coordinates at a time, in ascending order, their column loads in flight
          int jj[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            jj[u] = mm ? t * 32 + __ffs(mm) - 1 : -1;
            if (mm) mm &= mm - 1u;
          }
          float ev[U], hv[U][MR];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            ev[u] = jj[u] >= 0 ? (float)e[jj[u]] : 0.0f;
#pragma unroll
            for (int m = 0; m < MR; ++m)
              hv[u][m] = (jj[u] >= 0 && lane + 32 * m < NR2) ? Hs[jj[u] * HS + lane + 32 * m] : 0.0f;
          }
#pragma unroll
          for (int u = 0; u < U; ++u) {
            if (jj[u] < 0) break;
#pragma unroll
            for (int m = 0; m < MR; ++m)
              if (lane + 32 * m < NR2) rr[m] = __fmaf_rn(-hv[u][m], ev[u], rr[m]);
          }
        }
      }
#pragma unroll
      for (int m = 0; m < MR; ++m) acc = __fmaf_rn(rr[m], rr[m], acc);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(ARP_FULL, acc, o);
    if (acc < best) {
      best = acc;
      bi = c;
    }
    if (soft) {
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        const int k = lane + 32 * m;
        if (k < nbits) {
          const int j = k / nbl;
          const int v = xq8[j] + (c < R ? ek[c * D + j] : 0);
          const bool bit = (k - j * nbl) == 0 ? v > 0 : (v == 1 || v == -1);
          if (bit)
            mb1[m] = fminf(mb1[m], acc);
          else
            mb0[m] = fminf(mb0[m], acc);
        }
      }
    }
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
  if (soft) {
    // ---- max-log LLRs over the list and the single-bit-flip neighbours of the decision (mimo.py:434-462)
    unsigned char* base = reinterpret_cast<unsigned char*>(ek) + (size_t)(R + 1) * D;
    base += (16 - (reinterpret_cast<uintptr_t>(base) & 15)) & 15;
    int* s0 = reinterpret_cast<int*>(base);  // list minima, bit 0 (non-negative floats order as their patterns)
    int* s1 = s0 + nbits;                    // list minima, bit 1
    float* rh = reinterpret_cast<float*>(s1 + nbits);  // residual of the decision, NR2
    float* cj = rh + NR2;                    // H_j^T rh
    float* nj = cj + D;                      // ||H_j||^2
    float* dn = nj + D;                      // neighbour distances, nbits
    float* rv = dn + nbits;                  // 8 warps x (min1, min2)
    int* ri = reinterpret_cast<int*>(rv + 16);
    for (int k = tid; k < nbits; k += kReadThreads) s0[k] = s1[k] = __float_as_int(FLT_MAX);
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int k = lane + 32 * m;
      if (k < nbits) {
        atomicMin(&s0[k], __float_as_int(mb0[m]));
        atomicMin(&s1[k], __float_as_int(mb1[m]));
      }
    }
    for (int i = tid; i < NR2; i += kReadThreads) {
      float r = r0[i];
      if (gi < R)
        for (int j = 0; j < D; ++j)
          if (ek[gi * D + j]) r = __fmaf_rn(-Hs[j * HS + i], (float)ek[gi * D + j], r);
      rh[i] = r;
    }
    __syncthreads();
    for (int j = tid; j < D; j += kReadThreads) {
      float c = 0.0f, n = 0.0f;
      for (int i = 0; i < NR2; ++i) {
        const float hv = Hs[j * HS + i];
        c = __fmaf_rn(hv, rh[i], c);
        n = __fmaf_rn(hv, hv, n);
      }
      cj[j] = c;
      nj[j] = n;
    }
    __syncthreads();
    float n1 = FLT_MAX, n2 = FLT_MAX;
    int i1 = INT_MAX;
    for (int k = tid; k < nbits; k += kReadThreads) {
      const int j = k / nbl;
      const int lv = xq8[j] + (gi < R ? ek[gi * D + j] : 0);
      // Gray neighbour: the MSB flips the sign; the LSB swaps +-1 and +-3 (16-QAM)
      const int nl = (k - j * nbl) == 0 ? -lv : (lv > 0 ? 4 - lv : -4 - lv);
      const float del = (float)(nl - lv);
      const float d = __fmaf_rn(del * del, nj[j], __fmaf_rn(-2.0f * del, cj[j], gb));
      dn[k] = d;
      if (d < n1) {
        n2 = n1;
        n1 = d;
        i1 = k;
      } else if (d < n2) {
        n2 = d;
      }
    }
    // block-wide smallest and second smallest neighbour distance
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      const float o1 = __shfl_xor_sync(ARP_FULL, n1, o), o2 = __shfl_xor_sync(ARP_FULL, n2, o);
      const int oi = __shfl_xor_sync(ARP_FULL, i1, o);
      if (o1 < n1 || (o1 == n1 && oi < i1)) {
        n2 = fminf(n1, o2);
        n1 = o1;
        i1 = oi;
      } else {
        n2 = fminf(n2, o1);
      }
    }
    if (lane == 0) {
      rv[2 * wid] = n1;
      rv[2 * wid + 1] = n2;
      ri[wid] = i1;
    }
    __syncthreads();
    n1 = FLT_MAX;
    n2 = FLT_MAX;
    i1 = INT_MAX;
    for (int w = 0; w < W; ++w) {
      const float o1 = rv[2 * w], o2 = rv[2 * w + 1];
      const int oi = ri[w];
      if (o1 < n1 || (o1 == n1 && oi < i1)) {
        n2 = fminf(n1, o2);
        n1 = o1;
        i1 = oi;
      } else {
        n2 = fminf(n2, o1);
      }
    }
    const float inv_n0 = 1.0f / a.N0[u];
    for (int k = tid; k < nbits; k += kReadThreads) {
      const int j = k / nbl;
      const int lv = xq8[j] + (gi < R ? ek[gi * D + j] : 0);
      const bool bh = (k - j * nbl) == 0 ? lv > 0 : (lv == 1 || lv == -1);
      const float same = k == i1 ? n2 : n1;  // nearest neighbour that keeps bit k
      float m0 = __int_as_float(s0[k]), m1 = __int_as_float(s1[k]);
      if (bh) {
        m1 = fminf(m1, same);
        m0 = fminf(m0, dn[k]);
      } else {
        m0 = fminf(m0, same);
        m1 = fminf(m1, dn[k]);
      }
      const float l = (m0 - m1) * inv_n0;
      a.llr[(size_t)b * nbits + k] = fminf(fmaxf(l, -a.clip), a.clip);
    }
  }
  if (a.mdi) {
    const float cur = a.bd[(size_t)u * a.bl_stride];
    __syncthreads();
    if (gb < cur) {
      for (int j = tid; j < D; j += kReadThreads) a.bl[(size_t)u * a.bl_stride * D + j] = (int8_t)(xq8[j] + ek[gi * D + j]);
      if (tid == 0) a.bd[(size_t)u * a.bl_stride] = gb;
    }
    return;
  }
  const int nb = pam_bits(a.M);
  for (int j = tid; j < D; j += kReadThreads) {
    const int v = xq8[j] + (gi < R ? ek[gi * D + j] : 0);
    a.levels[(size_t)b * D + j] = (int8_t)v;
    if (nb == 1) {
      a.bits[(size_t)b * D + j] = v > 0;
    } else if (nb == 2) {
      a.bits[(size_t)b * D * 2 + 2 * j] = v > 0;
      a.bits[(size_t)b * D * 2 + 2 * j + 1] = (v == 1 || v == -1);
    } else {
      for (int k = 0; k < nb; ++k) a.bits[((size_t)b * D + j) * nb + k] = (int8_t)gray_bit(v, k, a.M);
    }
  }
  if (tid == 0) {
    a.dist[b] = gb;
    if (a.pick) a.pick[b] = gi;
  }
}

}  // namespace arp

namespace arp {

cudaError_t map_dispatch(const MapParams& a, cudaStream_t st) {
  const int D = a.D;
  return D <= 16 ? launch_map<1>(a, st) : D <= 32 ? launch_map<2>(a, st) : D <= 64 ? launch_map<4>(a, st)
                                                                          : launch_map<8>(a, st);
}

static size_t readout_smem(int D, int NR2, int R, bool soft = false) {
  size_t s = sizeof(float) * ((size_t)D * (NR2 + 1) + NR2 + 8) + 8 * sizeof(int) + (size_t)(R + 1) * D + 16;
  if (soft) s += 16 + sizeof(float) * (3 * (size_t)D * 2 + NR2 + 2 * (size_t)D + 24);  // s0, s1, dn, rh, cj, nj, rv, ri
  return s;
}

cudaError_t readout_dispatch(const ReadParams& a, cudaStream_t st) {
  const size_t smem = readout_smem(a.D, a.NR2, a.R, a.llr != nullptr);
  if (smem > 48 * 1024) {
    for (auto k : {k_readout_dd<1>, k_readout_dd<2>, k_readout_dd<4>, k_readout_dd<8>}) {
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
    }
  }
  const bool pdl = a.B <= kPdlMaxB;
  const dim3 g(a.B), t(kReadThreads);
  if (a.NR2 <= 32) return launch_ex(k_readout_dd<1>, g, t, smem, st, pdl, a);
  if (a.NR2 <= 64) return launch_ex(k_readout_dd<2>, g, t, smem, st, pdl, a);
  if (a.NR2 <= 128) return launch_ex(k_readout_dd<4>, g, t, smem, st, pdl, a);
  return launch_ex(k_readout_dd<8>, g, t, smem, st, pdl, a);
}

// Workspace of the fused detector call: G, h, x_q, scale, spins, de, (flips, tests), 256-byte aligned.
static size_t det_layout(int B, int D, int P, int R, int flt, size_t* off) {
  const size_t sz[7] = {(size_t)B * D * D * 4, (size_t)B * D * 4, (size_t)B * D, (size_t)B * 4,
                        (size_t)B * R * P * D, (size_t)B * R * (flt ? 4 : 8), (size_t)B * R * 16};
  size_t o = 0;
  for (int i = 0; i < 7; ++i) {
    if (off) off[i] = o;
    o = (o + sz[i] + 255) & ~(size_t)255;
  }
  return o;
}

}  // namespace arp

using namespace arp;

extern "C" size_t arp_detect_dd_workspace(int B, int D, int P, int R, int precision, size_t* offsets) {
  if (B < 0 || D < 1 || P < 1 || R < 1) return 0;
  return det_layout(B, D, P, R, precision == 1, offsets);
}

extern "C" int arp_detect_dd(const float* H, const float* y, const float* sigma2, int B, int NR2, int D, int M,
                             int policy, int precision, int P, int R, const void* T, const void* c, int L, double q,
                             uint32_t inst0, uint32_t k0, uint32_t k1, int start, void* workspace,
                             size_t workspace_bytes, int8_t* bits, int8_t* levels, float* dist, int32_t* pick,
                             int32_t* status, void* stream) {
  if (B < 0 || D < 1 || D > 128 || NR2 < 1 || NR2 > 256 || !(P == 2 || P == 4 || P == 6) || R < 1 || L < 1 ||
      !(M == 4 || M == 16 || M == 64))
    return ARP_ERR_SHAPE;
  if ((policy != 0 && policy != 1) || (precision != 0 && precision != 1) || (start != 0 && start != 1))
    return ARP_ERR_ARG;
  if (B == 0) return ARP_OK;
  if (!H || !y || !sigma2 || !T || !workspace || !bits || !levels || !dist) return ARP_ERR_ARG;
  const bool flt = precision == 1;
  size_t off[7];
  if (workspace_bytes < det_layout(B, D, P, R, flt, off)) return ARP_ERR_WORKSPACE;
  unsigned char* w = static_cast<unsigned char*>(workspace);
  void* G = w + off[0];
  void* h = w + off[1];
  int8_t* xq = reinterpret_cast<int8_t*>(w + off[2]);
  float* scale = reinterpret_cast<float*>(w + off[3]);
  int8_t* spins = reinterpret_cast<int8_t*>(w + off[4]);
  cudaStream_t st = (cudaStream_t)stream;
  MapParams m{H, y, sigma2, B, NR2, D, M, flt ? 0.0f : 4096.0f, G, h, xq, scale, status};
  if (map_dispatch(m, st) != cudaSuccess) return ARP_ERR_LAUNCH;
  DDParams a{G, h, T, c, L, flt ? 0 : (int32_t)q, (float)q, R, D, B, nullptr, inst0, k0, k1, start, spins,
             w + off[5], reinterpret_cast<int64_t*>(w + off[6]), status};
  if (anneal_dispatch(policy, flt, a, P, default_warps(R), st) != cudaSuccess) return ARP_ERR_LAUNCH;
  ReadParams rp{H, y, xq, spins, B, NR2, D, P, R, M, levels, bits, dist, pick};
  if (readout_dispatch(rp, st) != cudaSuccess) return ARP_ERR_LAUNCH;
  return ARP_OK;
}

extern "C" int arp_map_dd(const float* H, const float* y, const float* sigma2, int B, int NR2, int D, int M,
                          int quantize, void* G, void* h, int8_t* xq, float* scale, int32_t* status, void* stream) {
  if (B < 0 || D < 1 || D > 128 || NR2 < 1 || NR2 > 1024 || !(M == 4 || M == 16 || M == 64)) return ARP_ERR_SHAPE;
  if (B == 0) return ARP_OK;
  if (!H || !y || !sigma2 || !G || !h || !xq || !scale) return ARP_ERR_ARG;
  MapParams a{H, y, sigma2, B, NR2, D, M, quantize ? 4096.0f : 0.0f, G, h, xq, scale, status};
  return map_dispatch(a, (cudaStream_t)stream) == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_map_dd_soft(const float* H, const float* y, const float* sigma2, int B, int NR2, int D, int M,
                               int quantize, void* G, void* h, int8_t* xq, float* scale, float* zs, int32_t* status,
                               void* stream) {
  if (B < 0 || D < 1 || D > 128 || NR2 < 1 || NR2 > 1024 || !(M == 4 || M == 16 || M == 64)) return ARP_ERR_SHAPE;
  if (B == 0) return ARP_OK;
  if (!H || !y || !sigma2 || !G || !h || !xq || !scale || !zs) return ARP_ERR_ARG;
  MapParams a{H, y, sigma2, B, NR2, D, M, quantize ? 4096.0f : 0.0f, G, h, xq, scale, status};
  a.zs = zs;
  return map_dispatch(a, (cudaStream_t)stream) == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_readout_dd(const float* H, const float* y, const int8_t* xq, const int8_t* spins, int B, int NR2,
                              int D, int P, int R, int M, int8_t* levels, int8_t* bits, float* dist, int32_t* pick,
                              void* stream) {
  if (B < 0 || D < 1 || D > 128 || NR2 < 1 || NR2 > 256 || P < 1 || P > 6 || R < 0 || !(M == 4 || M == 16 || M == 64))
    return ARP_ERR_SHAPE;
  if (B == 0) return ARP_OK;
  if (!H || !y || !xq || (R > 0 && !spins) || !levels || !bits || !dist) return ARP_ERR_ARG;
  if (readout_smem(D, NR2, R) > 227 * 1024) return ARP_ERR_SHAPE;
  ReadParams a{H, y, xq, spins, B, NR2, D, P, R, M, levels, bits, dist, pick};
  return readout_dispatch(a, (cudaStream_t)stream) == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_readout_llr_dd(const float* H, const float* y, const int8_t* xq, const int8_t* spins, int B, int NR2,
                                  int D, int P, int R, int M, const float* N0, float clip, int8_t* levels,
                                  int8_t* bits, float* dist, int32_t* pick, float* llr, void* stream) {
  if (B < 0 || D < 1 || D > 128 || NR2 < 1 || NR2 > 256 || P < 1 || P > 6 || R < 0 || !(M == 4 || M == 16))
    return ARP_ERR_SHAPE;
  if (B == 0) return ARP_OK;
  if (!H || !y || !xq || (R > 0 && !spins) || !levels || !bits || !dist || !N0 || !llr) return ARP_ERR_ARG;
  if (readout_smem(D, NR2, R, true) > 227 * 1024) return ARP_ERR_SHAPE;
  ReadParams a{H, y, xq, spins, B, NR2, D, P, R, M, levels, bits, dist, pick};
  a.N0 = N0;
  a.clip = clip;
  a.llr = llr;
  return readout_dispatch(a, (cudaStream_t)stream) == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_map_ri(const float* H, const float* y, const float* sigma2, int B, int NR2, int D, int M, float r,
                          float* J, float* h0, float* h, int8_t* sP, int8_t* xq, float* scale, void* stream) {
  if (B < 0 || D < 1 || D > 64 || NR2 < 1 || NR2 > 1024 || !(M == 4 || M == 16)) return ARP_ERR_SHAPE;
  if (B == 0) return ARP_OK;
  if (!H || !y || !sigma2 || !J || !h0 || !h || !sP || !xq || !scale) return ARP_ERR_ARG;
  MapParams a{H, y, sigma2, B, NR2, D, M, 0.0f, nullptr, nullptr, xq, scale, nullptr};
  a.ri = 1;
  a.r_reg = r;
  a.Jri = J;
  a.h0ri = h0;
  a.hri = h;
  a.sP = sP;
  return map_dispatch(a, (cudaStream_t)stream) == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}

extern "C" int arp_readout_ri(const float* H, const float* y, const int8_t* xq, const int8_t* spins, int B, int NR2,
                              int D, int R, int M, int8_t* levels, int8_t* bits, float* dist, int32_t* pick,
                              void* stream) {
  if (B < 0 || D < 1 || D > 128 || NR2 < 1 || NR2 > 256 || R < 0 || !(M == 4 || M == 16)) return ARP_ERR_SHAPE;
  if (B == 0) return ARP_OK;
  if (!H || !y || !xq || (R > 0 && !spins) || !levels || !bits || !dist) return ARP_ERR_ARG;
  if (readout_smem(D, NR2, R) > 227 * 1024) return ARP_ERR_SHAPE;
  ReadParams a{H, y, xq, spins, B, NR2, D, M == 16 ? 2 : 1, R, M, levels, bits, dist, pick};
  a.ri = 1;
  return readout_dispatch(a, (cudaStream_t)stream) == cudaSuccess ? ARP_OK : ARP_ERR_LAUNCH;
}
