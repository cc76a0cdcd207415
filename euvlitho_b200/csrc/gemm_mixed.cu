// Mixed-precision complex GEMM on the 5th-generation tensor cores (tcgen05).
//
// C = alpha*scale[b] * A B + beta C + diag*I for complex FP64 A (MxK), B (KxN),
// C (MxN), column-major and batched (the beta term may read a separate Cin of
// C's shape), computed as TF32x3: every FP64 real
// operand is split into two TF32 values x = hi + lo (hi = x rounded to TF32,
// lo = x - hi), and each real product is hi*hi + hi*lo + lo*hi with FP32
// accumulation in tensor memory.  The complex product uses four real products:
//   Re = ArBr - AiBi,  Im = ArBi + AiBr   (the minus sign through the MMA's
//   negate-A bit): twelve real TF32 products per K=8 step, issued as nine
//   tcgen05.mma (the three Ar products as N = 256 against [Br | Bi], writing
//   the adjacent Re and Im accumulators at once).  The FP32 accumulation error grows with the K it spans, so
//   the two halves of K have their own Re/Im accumulators (four in all),
//   summed in FP64 by the epilogue.
// Error per product ~1e-6 relative: the bulk products of the slab matrix
// functions tolerate it (intensity error < 1e-4, see the tests); the interface
// solves stay FP64.
//
// The FP64 operands are read straight from global memory by eight converter
// warps, which split them in registers and store the four fp32 planes of a
// K-block (Re_hi, Re_lo, Im_hi, Im_lo) into the shared-memory stage in the
// 64-byte-swizzled K-major layout the UMMA descriptors read -- no operand
// copies in HBM.  Per CTA (one 128x128 complex tile of C):
//   warp 0     : TMEM allocation (512 columns: four 128-column accumulators of
//                the tile) and the single-thread MMA issue loop;
//   warps 1..8 : converters (ring of 3 stages of 4x(128x16) A + 4x(128x16) B
//                fp32 = 64 KB), then the epilogue: tcgen05.ld of their TMEM
//                lane quarter (= 32 rows) over half of the columns, complex
//                FP64 result written column by column (coalesced).
// C must not overlap A or B (the host checks): other CTAs still read A and B
// while a tile of C is written.
// All waits are bounded (about 2 s); a timeout ORs EUV_STATUS_TIMEOUT into the
// status word, stops the other roles, drains the MMAs in flight, frees TMEM
// and returns.
#include "tcgen05.cuh"

namespace euv {

int zgemm(int m, int n, int k, cplx alpha, const double* scale, const double2* a, long long lda,
          long long sa, const double2* b, long long ldb, long long sb, cplx beta, double2* c,
          long long ldc, long long sc, cplx diag, int batch, const int* steps, int step,
          cudaStream_t stream);

constexpr int MX_BM = 128;
constexpr int MX_BN = 128;
constexpr int MX_BK = 16;  // fp32 elements: 64-byte rows, one 64B swizzle span
constexpr int MX_STAGES = 3;
constexpr int MX_PLANES = 4;
constexpr int MX_A_TILE = MX_BM * MX_BK * 4;  // 8 KB
constexpr int MX_B_TILE = MX_BN * MX_BK * 4;  // 8 KB
constexpr int MX_STAGE_BYTES = MX_PLANES * (MX_A_TILE + MX_B_TILE);  // 64 KB
constexpr int MX_CONV_WARPS = 8;
constexpr int MX_THREADS = 32 * (1 + MX_CONV_WARPS);
constexpr int MX_TMEM_COLS = 512;
constexpr size_t MX_SMEM = (size_t)MX_STAGES * MX_STAGE_BYTES + 1024 + 256;
constexpr unsigned long long MX_TIMEOUT_NS = 2000000000ull;
// A K-block of one operand tile: 4 groups of 32 rows x 4 chunks of 4 K values
// = 16 warp items; A and B together 32, four per converter warp.
constexpr int MX_ITEMS = 2 * (MX_BM / 32) * (MX_BK / 4);
static_assert(MX_ITEMS % MX_CONV_WARPS == 0, "items per converter warp");

struct MixedArgs {
  int m, n, k;
  double2 alpha, beta, diag;
  const double* scale;
  const double2* a;
  long long lda, sa;
  const double2* b;
  long long ldb, sb;
  double2* c;
  const double2* cin;  // C read by the beta term (c when null)
  long long ldc, sc;
  const int* steps;
  int step;
  int* err;
};

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                          int* err) {
  return mbar_wait_bounded(bar, parity, abort_flag, err, MX_TIMEOUT_NS);
}
__device__ __forceinline__ constexpr uint32_t idesc_tf32(bool neg_a) {
  return idesc_tf32_mn(neg_a, MX_BM, MX_BN);
}

// x (FP64) -> hi + lo, hi = x rounded to TF32 (nearest, ties away from zero,
// on the fp32 value), lo = the exact fp32 remainder; the tensor core reads lo
// to TF32 precision.  Together about 22 significant bits, the precision of
// hi*hi + hi*lo + lo*hi.  The TF32 rounding is integer arithmetic on the fp32
// bits (add half a TF32 unit, clear the 13 low mantissa bits).
__device__ __forceinline__ void split_fast(double x, float& hi, float& lo) {
  const float xf = __double2float_rn(x);
  hi = __uint_as_float((__float_as_uint(xf) + 0x1000u) & 0xffffe000u);
  lo = xf - hi;
}

// Byte offset of the 16-byte chunk c (4 K values) of row r in a 64-byte-row
// K-major tile with the 64-byte swizzle (chunk bits 4-5 XOR address bits 7-8;
// tiles are 1024-byte aligned).
__device__ __forceinline__ uint32_t sw64_off(int r, int c) {
  return (uint32_t)(r * 64 + ((c ^ ((r >> 1) & 3)) << 4));
}

__global__ void __launch_bounds__(MX_THREADS, 1) gemm_tf32x3_kernel(MixedArgs p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + MX_STAGES * MX_STAGE_BYTES);
  uint64_t* empty = full + MX_STAGES;
  uint64_t* accum = empty + MX_STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accum + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.z;
  const int m0 = blockIdx.x * MX_BM, n0 = blockIdx.y * MX_BN;
  double2* C = p.c + (long long)b * p.sc;

  if (p.steps != nullptr && p.step >= p.steps[b]) {
    // inactive double-angle step of this batch entry: C = A on this tile
    // (eight loads in flight per thread before their stores: the CTA holds a
    // whole SM's shared memory, so the copy must not wait on each element)
    const double2* A = p.a + (long long)b * p.sa;
    constexpr int U = 8;
    for (int base = 0; base < MX_BM * MX_BN; base += MX_THREADS * U) {
      double2 v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int idx = base + threadIdx.x + u * MX_THREADS;
        const int gi = m0 + idx % MX_BM, gj = n0 + idx / MX_BM;
        v[u] = (idx < MX_BM * MX_BN && gi < p.m && gj < p.n) ? A[gi + (long long)gj * p.lda]
                                                             : make_double2(0.0, 0.0);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int idx = base + threadIdx.x + u * MX_THREADS;
        const int gi = m0 + idx % MX_BM, gj = n0 + idx / MX_BM;
        if (idx < MX_BM * MX_BN && gi < p.m && gj < p.n) C[gi + (long long)gj * p.ldc] = v[u];
      }
    }
    return;
  }

  auto a_tile = [&](int s, int pl) { return smem + s * MX_STAGE_BYTES + pl * MX_A_TILE; };
  auto b_tile = [&](int s, int pl) {
    return smem + s * MX_STAGE_BYTES + MX_PLANES * MX_A_TILE + pl * MX_B_TILE;
  };

  if (threadIdx.x == 0) {
    for (int s = 0; s < MX_STAGES; ++s) {
      mbar_init(&full[s], MX_CONV_WARPS);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accum, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(tmem_slot, MX_TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int nkb = (p.k + MX_BK - 1) / MX_BK;

  if (warp == 0) {
    if (lane == 0) {
      // A planes: 0 Re_hi 1 Re_lo 2 Im_hi 3 Im_lo.  B stage slots: 0 Re_hi,
      // 1 Im_hi, 2 Re_lo, 3 Im_lo ([Br | Bi] of one precision level adjacent:
      // one N = 256 operand).  The FP32 accumulation in TMEM loses precision in
      // proportion to the K it runs over (measured: the error is the same for
      // TF32-exact operands and grows linearly in K), so the K range is split
      // in two halves with their own Re/Im accumulators, summed in FP64 by the
      // epilogue.  Products: Re = +ArBr -AiBi, Im = +ArBi +AiBr, each as
      // hi*hi + hi*lo + lo*hi.  The Ar terms of Re and Im share their A
      // operand: one MMA of N = 256 against [Br | Bi] writes both accumulators
      // (Re and Im of a K half are adjacent TMEM columns); the Ai terms differ
      // in sign and take two N = 128 MMAs each (Re negated).
      const int ar_a[3] = {0, 0, 1}, ar_b[3] = {0, 2, 0};  // B slot of [Br|Bi] hi / lo
      const int ai_a[3] = {2, 2, 3};
      const int ai_bi[3] = {1, 3, 1}, ai_br[3] = {0, 2, 0};  // slots of Bi / Br
      const uint32_t id_pos = idesc_tf32(false), id_neg = idesc_tf32(true);
      const uint32_t id_wide = idesc_tf32_mn(false, MX_BM, 2 * MX_BN);
      const int half = (nkb + 1) / 2;  // k-blocks [0, half) -> set 0, [half, nkb) -> set 1
      for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb % MX_STAGES;
        const uint32_t ph = (uint32_t)((kb / MX_STAGES) & 1);
        if (!mbar_wait(&full[s], ph, abort_flag, p.err)) break;
        tc_fence_after();
        const int set = kb < half ? 0 : 1;
        const uint32_t t_re = tmem + (uint32_t)(2 * set * MX_BN);
        const uint32_t t_im = t_re + (uint32_t)MX_BN;
        const int kb0 = set ? half : 0;
#pragma unroll
        for (int k8 = 0; k8 < MX_BK / 8; ++k8) {
          const uint32_t first = (kb != kb0 || k8) ? 1u : 0u;
#pragma unroll
          for (int q = 0; q < 3; ++q)
            umma_tf32(t_re, umma_desc_sw64(a_tile(s, ar_a[q]) + k8 * 32),
                      umma_desc_sw64(b_tile(s, ar_b[q]) + k8 * 32), id_wide,
                      (first | q) ? 1u : 0u);
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            umma_tf32(t_re, umma_desc_sw64(a_tile(s, ai_a[q]) + k8 * 32),
                      umma_desc_sw64(b_tile(s, ai_bi[q]) + k8 * 32), id_neg, 1u);
            umma_tf32(t_im, umma_desc_sw64(a_tile(s, ai_a[q]) + k8 * 32),
                      umma_desc_sw64(b_tile(s, ai_br[q]) + k8 * 32), id_pos, 1u);
          }
        }
        umma_commit(&empty[s]);  // frees the stage when these MMAs complete
      }
      umma_commit(accum);  // always: the epilogue / teardown waits on it
    }
  } else {
    // ---- converters: warp item it (0..31) of a K-block; items < 16 are A
    // (rows m0 + 32*(it/4) + lane, K chunk it%4), the others B (columns).  Each
    // lane loads the 4 complex values of its chunk (A: 4 columns, 32 lanes =
    // 512 contiguous bytes per load; B: 64 contiguous bytes of one column),
    // splits them and stores one 16-byte chunk per plane.  Every item is
    // loaded before the first store, so the warp has 16 loads in flight.
    const int cw = warp - 1;
    const double2* A = p.a + (long long)b * p.sa;
    const double2* B = p.b + (long long)b * p.sb;
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb % MX_STAGES;
      const uint32_t ph = (uint32_t)((kb / MX_STAGES) & 1);
      const bool got = mbar_wait(&empty[s], ph ^ 1u, abort_flag, p.err);
      if (!__all_sync(0xffffffffu, got)) break;
      const int k0 = kb * MX_BK;
      double2 v[MX_ITEMS / MX_CONV_WARPS][4];
#pragma unroll
      for (int j = 0; j < MX_ITEMS / MX_CONV_WARPS; ++j) {
        const int it = cw + MX_CONV_WARPS * j;
        const int c = it & 3;
        const int row = 32 * ((it & 15) >> 2) + lane;
        const int kc = k0 + 4 * c;
        if (it < 16) {
          const int gm = m0 + row;
#pragma unroll
          for (int e = 0; e < 4; ++e)
            v[j][e] = (gm < p.m && kc + e < p.k) ? __ldg(&A[gm + (long long)(kc + e) * p.lda])
                                                 : make_double2(0.0, 0.0);
        } else {
          const int gn = n0 + row;
          const double2* col = B + (long long)gn * p.ldb + kc;
#pragma unroll
          for (int e = 0; e < 4; ++e)
            v[j][e] = (gn < p.n && kc + e < p.k) ? __ldg(col + e) : make_double2(0.0, 0.0);
        }
      }
#pragma unroll
      for (int j = 0; j < MX_ITEMS / MX_CONV_WARPS; ++j) {
        const int it = cw + MX_CONV_WARPS * j;
        const int c = it & 3;
        const int row = 32 * ((it & 15) >> 2) + lane;
        float4 rh, rl, ih, il;
        split_fast(v[j][0].x, rh.x, rl.x);
        split_fast(v[j][1].x, rh.y, rl.y);
        split_fast(v[j][2].x, rh.z, rl.z);
        split_fast(v[j][3].x, rh.w, rl.w);
        split_fast(v[j][0].y, ih.x, il.x);
        split_fast(v[j][1].y, ih.y, il.y);
        split_fast(v[j][2].y, ih.z, il.z);
        split_fast(v[j][3].y, ih.w, il.w);
        const uint32_t off = sw64_off(row, c);
        if (it < 16) {
          *reinterpret_cast<float4*>(a_tile(s, 0) + off) = rh;
          *reinterpret_cast<float4*>(a_tile(s, 1) + off) = rl;
          *reinterpret_cast<float4*>(a_tile(s, 2) + off) = ih;
          *reinterpret_cast<float4*>(a_tile(s, 3) + off) = il;
        } else {
          *reinterpret_cast<float4*>(b_tile(s, 0) + off) = rh;
          *reinterpret_cast<float4*>(b_tile(s, 1) + off) = ih;
          *reinterpret_cast<float4*>(b_tile(s, 2) + off) = rl;
          *reinterpret_cast<float4*>(b_tile(s, 3) + off) = il;
        }
      }
      // the generic-proxy stores must be visible to the tensor core (async proxy)
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0)
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&full[s]))
                     : "memory");
    }

    // ---- epilogue: warp w reads TMEM lanes 32*(w%4).. (= tile rows) and
    // columns [64*h, 64*h + 64), h = 0 for warps 1..4, 1 for warps 5..8
    const int q = warp & 3;
    const int h = (warp - 1) >> 2;
    const bool waited = mbar_wait(accum, 0u, abort_flag, p.err) && !*abort_flag && nkb > 0;
    const bool ok = __all_sync(0xffffffffu, waited);  // tcgen05.ld below is warp-collective
    tc_fence_after();
    const int row = m0 + q * 32 + lane;
    const double sc = p.scale ? p.scale[b] : 1.0;
    const cplx alpha = mk(p.alpha.x * sc, p.alpha.y * sc);
    const cplx beta = mk(p.beta.x, p.beta.y);
    const bool use_beta = (p.beta.x != 0.0 || p.beta.y != 0.0);
    const double2* Cin = p.cin ? p.cin + (long long)b * p.sc : C;
    const cplx dg = mk(p.diag.x, p.diag.y);
    if (ok) {
      for (int c0 = 64 * h; c0 < 64 * h + 64; c0 += 16) {
        if (n0 + c0 >= p.n) break;  // warp-uniform
        uint32_t vr[16], vi[16], cr[16], ci[16];
        const uint32_t lane_addr = ((uint32_t)(q * 32) << 16);
        tmem_ld16(tmem + lane_addr + (uint32_t)c0, vr);
        tmem_ld16(tmem + lane_addr + (uint32_t)(MX_BN + c0), vi);
        tmem_ld16(tmem + lane_addr + (uint32_t)(2 * MX_BN + c0), cr);
        tmem_ld16(tmem + lane_addr + (uint32_t)(3 * MX_BN + c0), ci);
        tmem_ld_wait();
        if (row < p.m) {
          // all 16 reads of C are issued before the first store: a load after
          // a store through the same pointer type would otherwise wait for it
          double2 old[16];
          if (use_beta) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const int col = n0 + c0 + j;
              old[j] = col < p.n ? Cin[row + (long long)col * p.ldc] : make_double2(0.0, 0.0);
            }
          }
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int col = n0 + c0 + j;
            if (col < p.n) {
              // K halves: set 0 at columns [0, 2BN), set 1 (empty if nkb == 1) at [2BN, 4BN)
              const double s1r = nkb > 1 ? (double)__uint_as_float(cr[j]) : 0.0;
              const double s1i = nkb > 1 ? (double)__uint_as_float(ci[j]) : 0.0;
              cplx v = alpha * mk((double)__uint_as_float(vr[j]) + s1r,
                                  (double)__uint_as_float(vi[j]) + s1i);
              if (use_beta) v = v + beta * mk(old[j].x, old[j].y);
              if (row == col) v = v + dg;
              C[row + (long long)col * p.ldc] = make_double2(v.x, v.y);
            }
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    if (*abort_flag) mbar_drain(accum, 0u, MX_TIMEOUT_NS);  // MMAs in flight finish first
    tmem_dealloc(tmem, MX_TMEM_COLS);
  }
}

// ------------------------------------------------------------------ host
static bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
  const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
  return x < y + nb && y < x + na;
}
static size_t span_bytes(int rows, int cols, long long ld, long long stride, int batch) {
  return ((size_t)(batch - 1) * (size_t)stride + (size_t)(cols - 1) * (size_t)ld + (size_t)rows) *
         sizeof(double2);
}

size_t gemm_mixed_workspace_bytes(int, int, int, int) { return 256; }

int gemm_mixed(int m, int n, int k, cplx alpha, const double* scale, const double2* a,
               long long lda, long long sa, const double2* b, long long ldb, long long sb,
               cplx beta, double2* c, long long ldc, long long sc, cplx diag, int batch,
               const int* steps, int step, void* work, size_t work_bytes, int* status,
               cudaStream_t stream, const double2* cin) {
  if (m <= 0 || n <= 0 || batch <= 0) return EUV_OK;
  if (k <= 0 || batch > 65535) {
    euv_set_error("gemm_mixed: unsupported shape");
    return EUV_ERR_BAD_ARG;
  }
  const size_t cspan = span_bytes(m, n, ldc, sc, batch);
  if (overlaps(c, cspan, a, span_bytes(m, k, lda, sa, batch)) ||
      overlaps(c, cspan, b, span_bytes(k, n, ldb, sb, batch))) {
    euv_set_error("gemm_mixed: C overlaps A or B (m=%d n=%d k=%d)", m, n, k);
    return EUV_ERR_BAD_ARG;
  }
  // the caller's sticky status word, else a per-call word in the workspace
  int* err = status;
  if (err == nullptr) {
    if (work == nullptr || work_bytes < sizeof(int)) {
      euv_set_error("gemm_mixed: workspace too small (%zu bytes; needs %zu without a status word)",
                    work_bytes, gemm_mixed_workspace_bytes(m, n, k, batch));
      return EUV_ERR_WORKSPACE;
    }
    err = reinterpret_cast<int*>(work);
    EUV_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), stream));
  }
  static int smem_done[64];
  EUV_CUDA_TRY(ensure_smem(gemm_tf32x3_kernel, (int)MX_SMEM, smem_done));
  MixedArgs p;
  p.m = m;
  p.n = n;
  p.k = k;
  p.alpha = make_double2(alpha.x, alpha.y);
  p.beta = make_double2(beta.x, beta.y);
  p.diag = make_double2(diag.x, diag.y);
  p.scale = scale;
  p.a = a;
  p.lda = lda;
  p.sa = sa;
  p.b = b;
  p.ldb = ldb;
  p.sb = sb;
  p.c = c;
  p.cin = cin;
  p.ldc = ldc;
  p.sc = sc;
  p.steps = steps;
  p.step = step;
  p.err = err;
  dim3 grid((m + MX_BM - 1) / MX_BM, (n + MX_BN - 1) / MX_BN, batch);
  gemm_tf32x3_kernel<<<grid, MX_THREADS, MX_SMEM, stream>>>(p);
  EUV_LAUNCH_CHECK();
  return EUV_OK;
}

}  // namespace euv

using namespace euv;

extern "C" size_t euv_zgemm_tf32x3_workspace_bytes(int m, int n, int k, int batch) {
  if (m <= 0 || n <= 0 || k <= 0 || batch <= 0) return 0;
  return gemm_mixed_workspace_bytes(m, n, k, batch);
}

extern "C" int euv_zgemm_tf32x3(int m, int n, int k, euv_c64 alpha, const double* d_scale,
                                const euv_c64* d_a, int lda, long long stride_a,
                                const euv_c64* d_b, int ldb, long long stride_b, euv_c64 beta,
                                euv_c64* d_c, int ldc, long long stride_c, euv_c64 diag,
                                int batch, const int* d_steps, int step, void* d_work,
                                size_t work_bytes, int* d_status, void* stream) {
  if (m <= 0 || n <= 0 || k <= 0 || batch <= 0 || lda < m || ldc < m || ldb < k || !d_a ||
      !d_b || !d_c || (d_steps != nullptr && (m != n || m != k))) {
    euv_set_error("euv_zgemm_tf32x3: bad arguments (m=%d n=%d k=%d)", m, n, k);
    return EUV_ERR_BAD_ARG;
  }
  return gemm_mixed(m, n, k, fromc(alpha), d_scale, reinterpret_cast<const double2*>(d_a), lda,
                    stride_a, reinterpret_cast<const double2*>(d_b), ldb, stride_b, fromc(beta),
                    reinterpret_cast<double2*>(d_c), ldc, stride_c, fromc(diag), batch, d_steps,
                    step, d_work, work_bytes, d_status, (cudaStream_t)stream, nullptr);
}
