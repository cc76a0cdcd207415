// Batched complex FP64 GEMM on the B200 FP64 tensor path (DMMA).
//
// Replaces matproduct (header.h:1559-1619: Eigen product for N<=5000, cuBLAS
// Zgemm with host round trips above).  FP64 has no tcgen05 kind on sm_100a, so
// the FP64 form uses mma.sync.m8n8k4.f64 (the FP64 tensor instruction).
//
// Tiling: CTA tile 64x64 complex, K tile 16, 4 warps (2x2), warp tile 32x32
// complex = 4x4 DMMA 8x8 tiles, each with a real and an imaginary accumulator
// (4 DMMA per complex 8x8x4 step).  Operands are staged global->shared with
// 16-byte cp.async (one complex element per copy) in a 3-stage pipeline; the
// shared layout is k-major with a 2-element pad so fragment loads (one 128-bit
// load = re+im) are bank-conflict free.
#include "common.cuh"

namespace euv {

constexpr int GBM = 64;
constexpr int GBN = 64;
constexpr int GBK = 16;
constexpr int GSTAGES = 3;
constexpr int GTHREADS = 128;
constexpr int APAD = GBM + 2;
constexpr int BPAD = GBN + 2;
constexpr size_t GSMEM = (size_t)GSTAGES * GBK * (APAD + BPAD) * sizeof(double2);

struct GemmArgs {
  int m, n, k;
  double2 alpha, beta, diag;
  const double* scale;
  const double2* a;
  long long lda, sa;
  const double2* b;
  long long ldb, sb;
  double2* c;
  long long ldc, sc;
  const int* steps;
  int step;
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// UPD: C -= A B (alpha, beta, scale, diag ignored).  The accumulators start
// from C, whose loads are issued right after the first operand copies, and the
// A fragments are negated: no read of C after the products.
// MI: 8-row blocks per warp (tile BM = 16 MI rows x 64 columns); ST: cp.async stages.
template <bool UPD, int MI, int ST>
__global__ void __launch_bounds__(GTHREADS, MI == 2 ? 4 : 2) zgemm_kernel(GemmArgs p) {
  constexpr int BM = 16 * MI;
  constexpr int AP = BM + 2;
  extern __shared__ double2 smem[];
  double2* As = smem;
  double2* Bs = smem + ST * GBK * AP;
  const int bz = blockIdx.z;
  const int m0 = blockIdx.x * BM;
  const int n0 = blockIdx.y * GBN;
  const double2* A = p.a + (long long)bz * p.sa;
  const double2* B = p.b + (long long)bz * p.sb;
  double2* C = p.c + (long long)bz * p.sc;
  const int tid = threadIdx.x;

  if (p.steps != nullptr && p.step >= p.steps[bz]) {
    // inactive double-angle step for this batch entry: C = A
    // eight loads in flight per thread before their stores
    constexpr int U = 8;
    for (int base = 0; base < BM * GBN; base += GTHREADS * U) {
      double2 v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int idx = base + tid + u * GTHREADS;
        const int gi = m0 + idx % BM, gj = n0 + idx / BM;
        v[u] = (idx < BM * GBN && gi < p.m && gj < p.n) ? A[gi + (long long)gj * p.lda]
                                                         : make_double2(0.0, 0.0);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int idx = base + tid + u * GTHREADS;
        const int gi = m0 + idx % BM, gj = n0 + idx / BM;
        if (idx < BM * GBN && gi < p.m && gj < p.n) C[gi + (long long)gj * p.ldc] = v[u];
      }
    }
    return;
  }

  const int warp = tid >> 5, lane = tid & 31;
  const int wm = (warp & 1) * (8 * MI), wn = (warp >> 1) * 32;
  double accr[MI][4][2], acci[MI][4][2];
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      accr[i][j][0] = accr[i][j][1] = 0.0;
      acci[i][j][0] = acci[i][j][1] = 0.0;
    }

  const int ktiles = (p.k + GBK - 1) / GBK;
  auto load_tile = [&](int stage, int kt) {
    const int k0 = kt * GBK;
    double2* as = As + stage * GBK * AP;
    double2* bs = Bs + stage * GBK * BPAD;
#pragma unroll
    for (int r = 0; r < (BM * GBK) / GTHREADS; ++r) {
      int idx = tid + r * GTHREADS;
      int i = idx % BM, kk = idx / BM;
      int gi = m0 + i, gk = k0 + kk;
      bool ok = gi < p.m && gk < p.k;
      const double2* src = ok ? A + gi + (long long)gk * p.lda : A;
      cp_async16(&as[kk * AP + i], src, ok);
    }
#pragma unroll
    for (int r = 0; r < (GBN * GBK) / GTHREADS; ++r) {
      int idx = tid + r * GTHREADS;
      int kk = idx % GBK, j = idx / GBK;
      int gk = k0 + kk, gj = n0 + j;
      bool ok = gk < p.k && gj < p.n;
      const double2* src = ok ? B + gk + (long long)gj * p.ldb : B;
      cp_async16(&bs[kk * BPAD + j], src, ok);
    }
  };

#pragma unroll
  for (int s = 0; s < ST - 1; ++s) {
    if (s < ktiles) load_tile(s, s);
    cp_async_commit();
  }
  if (UPD) {
#pragma unroll
    for (int mi = 0; mi < MI; ++mi) {
      const int row = m0 + wm + mi * 8 + (lane >> 2);
#pragma unroll
      for (int ni = 0; ni < 4; ++ni)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int col = n0 + wn + ni * 8 + (lane & 3) * 2 + e;
          const double2 v = (row < p.m && col < p.n) ? C[row + (long long)col * p.ldc]
                                                     : make_double2(0.0, 0.0);
          accr[mi][ni][e] = v.x;
          acci[mi][ni][e] = v.y;
        }
    }
  }
  for (int kt = 0; kt < ktiles; ++kt) {
    cp_async_wait<ST - 2>();
    __syncthreads();
    {
      int nk = kt + ST - 1;
      if (nk < ktiles) load_tile(nk % ST, nk);
      cp_async_commit();
    }
    const double2* as = As + (kt % ST) * GBK * AP;
    const double2* bs = Bs + (kt % ST) * GBK * BPAD;
#pragma unroll
    for (int ks = 0; ks < GBK; ks += 4) {
      const int kk = ks + (lane & 3);
      double ar[MI], ai[MI], an[MI], br[4], bi[4];
#pragma unroll
      for (int mi = 0; mi < MI; ++mi) {
        double2 v = as[kk * AP + wm + mi * 8 + (lane >> 2)];
        if (UPD) {
          v.x = -v.x;
          v.y = -v.y;
        }
        ar[mi] = v.x;
        ai[mi] = v.y;
        an[mi] = -v.y;
      }
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
        double2 v = bs[kk * BPAD + wn + ni * 8 + (lane >> 2)];
        br[ni] = v.x;
        bi[ni] = v.y;
      }
#pragma unroll
      for (int mi = 0; mi < MI; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
          dmma(accr[mi][ni][0], accr[mi][ni][1], ar[mi], br[ni]);
          dmma(accr[mi][ni][0], accr[mi][ni][1], an[mi], bi[ni]);
          dmma(acci[mi][ni][0], acci[mi][ni][1], ar[mi], bi[ni]);
          dmma(acci[mi][ni][0], acci[mi][ni][1], ai[mi], br[ni]);
        }
    }
  }
  cp_async_wait<0>();

  if (UPD) {
#pragma unroll
    for (int mi = 0; mi < MI; ++mi) {
      const int row = m0 + wm + mi * 8 + (lane >> 2);
#pragma unroll
      for (int ni = 0; ni < 4; ++ni)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int col = n0 + wn + ni * 8 + (lane & 3) * 2 + e;
          if (row < p.m && col < p.n)
            C[row + (long long)col * p.ldc] = make_double2(accr[mi][ni][e], acci[mi][ni][e]);
        }
    }
    return;
  }

  const double sc = p.scale ? p.scale[bz] : 1.0;
  const cplx alpha = mk(p.alpha.x * sc, p.alpha.y * sc);
  const cplx beta = mk(p.beta.x, p.beta.y);
  const bool use_beta = (p.beta.x != 0.0 || p.beta.y != 0.0);
  const cplx dg = mk(p.diag.x, p.diag.y);
#pragma unroll
  for (int mi = 0; mi < MI; ++mi) {
    const int row = m0 + wm + mi * 8 + (lane >> 2);
    // the 8 reads of C for this row block are issued before its stores (a
    // load after a store through the same pointer type would wait for it)
    double2 old[4][2];
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int col = n0 + wn + ni * 8 + (lane & 3) * 2 + e;
        old[ni][e] = (use_beta && row < p.m && col < p.n) ? C[row + (long long)col * p.ldc]
                                                          : make_double2(0.0, 0.0);
      }
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int col = n0 + wn + ni * 8 + (lane & 3) * 2 + e;
        if (row < p.m && col < p.n) {
          cplx v = alpha * mk(accr[mi][ni][e], acci[mi][ni][e]);
          if (use_beta) v = v + beta * mk(old[ni][e].x, old[ni][e].y);
          if (row == col) v = v + dg;
          C[row + (long long)col * p.ldc] = make_double2(v.x, v.y);
        }
      }
  }
}

template <int MI, int ST>
constexpr size_t zgemm_smem() {
  return (size_t)ST * GBK * (16 * MI + 2 + BPAD) * sizeof(double2);
}

int zgemm_launch(const GemmArgs& p, int batch, cudaStream_t stream, bool upd = false) {
  if (p.m <= 0 || p.n <= 0 || batch <= 0) return EUV_OK;
  static int smem_done[64], smem_done_upd[64], smem_done_rk[64];
  if (upd && p.k <= 2 * GBK) {
    // rank-k update with k <= 32 (the LU's trailing updates): 32 x 64 tiles and
    // two stages (both k tiles in flight at once) for four CTAs per SM
    constexpr size_t sm = zgemm_smem<2, 2>();
    dim3 grid((p.m + 31) / 32, (p.n + GBN - 1) / GBN, batch);
    EUV_CUDA_TRY(ensure_smem(zgemm_kernel<true, 2, 2>, (int)sm, smem_done_rk));
    zgemm_kernel<true, 2, 2><<<grid, GTHREADS, sm, stream>>>(p);
  } else if (upd) {
    constexpr size_t sm = zgemm_smem<4, GSTAGES>();
    dim3 grid((p.m + GBM - 1) / GBM, (p.n + GBN - 1) / GBN, batch);
    EUV_CUDA_TRY(ensure_smem(zgemm_kernel<true, 4, GSTAGES>, (int)sm, smem_done_upd));
    zgemm_kernel<true, 4, GSTAGES><<<grid, GTHREADS, sm, stream>>>(p);
  } else if (tune_lookup(EUV_KNOB_ZGEMM_ROWS, p.m, batch) == 32) {
    // 32 x 64 tiles: twice the CTAs, for shapes that leave SMs idle with 64 rows
    static int smem_done32[64];
    constexpr size_t sm = zgemm_smem<2, GSTAGES>();
    dim3 grid((p.m + 31) / 32, (p.n + GBN - 1) / GBN, batch);
    EUV_CUDA_TRY(ensure_smem(zgemm_kernel<false, 2, GSTAGES>, (int)sm, smem_done32));
    zgemm_kernel<false, 2, GSTAGES><<<grid, GTHREADS, sm, stream>>>(p);
  } else {
    dim3 grid((p.m + GBM - 1) / GBM, (p.n + GBN - 1) / GBN, batch);
    EUV_CUDA_TRY(ensure_smem(zgemm_kernel<false, 4, GSTAGES>, (int)GSMEM, smem_done));
    zgemm_kernel<false, 4, GSTAGES><<<grid, GTHREADS, GSMEM, stream>>>(p);
  }
  EUV_LAUNCH_CHECK();
  return EUV_OK;
}

// C -= A B (the rank-k updates of the blocked LU and its solves)
int zgemm_sub(int m, int n, int k, const double2* a, long long lda, long long sa,
              const double2* b, long long ldb, long long sb, double2* c, long long ldc,
              long long sc, int batch, cudaStream_t stream) {
  GemmArgs p = {};
  p.m = m;
  p.n = n;
  p.k = k;
  p.a = a;
  p.lda = lda;
  p.sa = sa;
  p.b = b;
  p.ldb = ldb;
  p.sb = sb;
  p.c = c;
  p.ldc = ldc;
  p.sc = sc;
  return zgemm_launch(p, batch, stream, true);
}

int zgemm(int m, int n, int k, cplx alpha, const double* scale, const double2* a, long long lda,
          long long sa, const double2* b, long long ldb, long long sb, cplx beta, double2* c,
          long long ldc, long long sc, cplx diag, int batch, const int* steps, int step,
          cudaStream_t stream) {
  GemmArgs p;
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
  p.ldc = ldc;
  p.sc = sc;
  p.steps = steps;
  p.step = step;
  return zgemm_launch(p, batch, stream);
}

}  // namespace euv

extern "C" int euv_zgemm(int m, int n, int k, euv_c64 alpha, const double* d_scale,
                         const euv_c64* d_a, int lda, long long stride_a, const euv_c64* d_b,
                         int ldb, long long stride_b, euv_c64 beta, euv_c64* d_c, int ldc,
                         long long stride_c, euv_c64 diag_add, int batch, const int* d_steps,
                         int step, void* stream) {
  if (m < 0 || n < 0 || k < 0 || batch < 0 || lda < (m > 0 ? m : 1) || ldc < (m > 0 ? m : 1) ||
      ldb < (k > 0 ? k : 1) || d_a == nullptr || d_b == nullptr || d_c == nullptr) {
    euv_set_error("euv_zgemm: bad arguments (m=%d n=%d k=%d lda=%d ldb=%d ldc=%d)", m, n, k, lda,
                  ldb, ldc);
    return EUV_ERR_BAD_ARG;
  }
  if (d_steps != nullptr && (m != n || m != k)) {
    euv_set_error("euv_zgemm: step predication needs square operands");
    return EUV_ERR_BAD_ARG;
  }
  return euv::zgemm(m, n, k, euv::fromc(alpha), d_scale, reinterpret_cast<const double2*>(d_a),
                    lda, stride_a, reinterpret_cast<const double2*>(d_b), ldb, stride_b,
                    euv::fromc(beta), reinterpret_cast<double2*>(d_c), ldc, stride_c,
                    euv::fromc(diag_add), batch, d_steps, step, (cudaStream_t)stream);
}
