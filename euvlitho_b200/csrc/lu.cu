// Batched complex FP64 LU with partial pivoting and triangular solves.
//
// Replaces matinv (header.h:1468-1557: Eigen colPivHouseholderQr for N<=5000,
// cuSOLVER Xgetrf/Xgetrs with host round trips above).  The reference only ever
// applies an inverse to a matrix, so the library factors once and solves with
// the right-hand sides it needs.
//
// Blocked right-looking LU, panel width LU_NB:
//   panel  : columns [j0, j0+nb) of rows [j0, n) (pivot = first max of
//            |re|+|im| as LAPACK izamax, row swap, scale, rank-1 update), the
//            rows in the registers of a cluster of up to 8 CTAs per matrix;
//   laswp  : the panel's row swaps applied to the other columns;
//   trsm   : U12 = L11^-1 A12 (unit lower, L11 staged in shared memory);
//   update : A22 -= L21 U12 with the batched DMMA zgemm;
//   look-ahead: the next panel is factored on a high-priority side stream while
//            the rest of the update runs (the panel alone fills only `batch` SMs).
// Solve: the row swaps on B, then one launch that keeps 8 (or fewer, for large
// n) columns of X in shared memory per CTA through both substitutions.
#include <cooperative_groups.h>

#include "common.cuh"

namespace euv {

namespace cg = cooperative_groups;

int zgemm_sub(int m, int n, int k, const double2* a, long long lda, long long sa,
              const double2* b, long long ldb, long long sb, double2* c, long long ldc,
              long long sc, int batch, cudaStream_t stream);
int zgemm(int m, int n, int k, cplx alpha, const double* scale, const double2* a, long long lda,
          long long sa, const double2* b, long long ldb, long long sb, cplx beta, double2* c,
          long long ldc, long long sc, cplx diag, int batch, const int* steps, int step,
          cudaStream_t stream);

constexpr int LU_NB = 32;
constexpr int LU_PANEL_THREADS = 512;

__device__ __forceinline__ cplx ld2(const double2* p) {
  double2 v = *p;
  return mk(v.x, v.y);
}
__device__ __forceinline__ void st2(double2* p, cplx v) { *p = make_double2(v.x, v.y); }

__global__ void __launch_bounds__(LU_PANEL_THREADS) lu_panel_kernel(int n, int j0, int jb,
                                                                    double2* A, long long lda,
                                                                    long long sa, int* ipiv,
                                                                    int* info) {
  A += (long long)blockIdx.x * sa;
  ipiv += (long long)blockIdx.x * n;
  __shared__ double red_v[LU_PANEL_THREADS / 32];
  __shared__ int red_i[LU_PANEL_THREADS / 32];
  __shared__ int s_piv;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nthr = blockDim.x;
  for (int jj = j0; jj < j0 + jb; ++jj) {
    // pivot search: first index of max |re|+|im| in rows jj..n-1
    double best = -1.0;
    int bidx = n;
    for (int r = jj + tid; r < n; r += nthr) {
      double v = cabs1(ld2(&A[r + (long long)jj * lda]));
      if (v > best) {
        best = v;
        bidx = r;
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      double ov = __shfl_down_sync(0xffffffffu, best, off);
      int oi = __shfl_down_sync(0xffffffffu, bidx, off);
      if (ov > best || (ov == best && oi < bidx)) {
        best = ov;
        bidx = oi;
      }
    }
    if (lane == 0) {
      red_v[warp] = best;
      red_i[warp] = bidx;
    }
    __syncthreads();
    if (tid == 0) {
      double bv = red_v[0];
      int bi = red_i[0];
      for (int w = 1; w < nthr / 32; ++w) {
        if (red_v[w] > bv || (red_v[w] == bv && red_i[w] < bi)) {
          bv = red_v[w];
          bi = red_i[w];
        }
      }
      if (bi >= n) bi = jj;
      s_piv = bi;
      ipiv[jj] = bi;
    }
    __syncthreads();
    const int piv = s_piv;
    if (piv != jj) {
      for (int c = j0 + tid; c < j0 + jb; c += nthr) {
        double2 t = A[jj + (long long)c * lda];
        A[jj + (long long)c * lda] = A[piv + (long long)c * lda];
        A[piv + (long long)c * lda] = t;
      }
    }
    __syncthreads();
    const cplx d = ld2(&A[jj + (long long)jj * lda]);
    if (d.x == 0.0 && d.y == 0.0) {
      if (tid == 0 && info[blockIdx.x] == 0) info[blockIdx.x] = jj + 1;
      __syncthreads();
      continue;
    }
    const cplx inv = cdiv(mk(1.0, 0.0), d);
    for (int r = jj + 1 + tid; r < n; r += nthr) {
      double2* p = &A[r + (long long)jj * lda];
      st2(p, ld2(p) * inv);
    }
    __syncthreads();
    const int rows = n - jj - 1;
    const int cols = j0 + jb - jj - 1;
    if (rows > 0 && cols > 0) {
      for (int idx = tid; idx < rows * cols; idx += nthr) {
        int r = jj + 1 + idx % rows;
        int c = jj + 1 + idx / rows;
        double2* p = &A[r + (long long)c * lda];
        st2(p, ld2(p) - ld2(&A[r + (long long)jj * lda]) * ld2(&A[jj + (long long)c * lda]));
      }
    }
    __syncthreads();
  }
}

// Panel factorisation by a cluster of LC CTAs per matrix with the panel rows
// in registers (n - j0 <= LC * LC_THREADS rows): thread t of cluster rank q
// holds row j0 + q*LC_THREADS + t.  Columns are taken in blocks of LC_BLK
// with the block's columns at compile-time register indices v[0..LC_BLK); the
// register row is rotated by LC_BLK after each block (one block's code for the
// whole panel, no runtime register indexing).  One cluster barrier per column
// jj: before it, every CTA finds its candidate (first max of |re|+|im| in its
// rows >= jj, as izamax; every warp reduces the warp maxima itself) and sends
// the candidate's value, index and row to every CTA through distributed shared
// memory, one column per lane of the warp that holds the row, and rank 0 sends
// row jj the same way; after it, every thread reduces the LC candidates in
// rank order (same pivot in every CTA), takes the pivot row from the winner's
// slot, swaps, scales and applies the rank-1 update to its own row.  The swap
// at column jj exchanges only the columns from jj on (the part of the two rows
// the remaining columns use), so every column c of the panel holds the swaps of
// pivots ..c and lacks exactly those of pivots c+1..: the laswp launch after the
// panel applies them (sub = 1).  Slots alternate by column parity: a slot is
// rewritten two barriers after it was read.  A block's columns are stored when
// it ends, pivots and the singular flag when the panel ends.  Every thread
// executes every barrier the same number of times whatever the data (a zero
// pivot skips only the arithmetic).
constexpr int LC_THREADS = 256;
constexpr int LC_WARPS = LC_THREADS / 32;
constexpr int LC_BLK = 4;
static_assert(LU_NB == 32, "one panel column per lane");
static_assert(LU_NB % LC_BLK == 0, "whole blocks");

__device__ __forceinline__ void argmax_step(double& v, int& i, double ov, int oi) {
  if (ov > v || (ov == v && oi < i)) {
    v = ov;
    i = oi;
  }
}

template <int LC>
__global__ void __cluster_dims__(LC, 1, 1) __launch_bounds__(LC_THREADS, 1)
    lu_panel_cluster_kernel(int n, int j0, int jb, double2* A, long long lda, long long sa,
                            int* ipiv, int* info) {
  cg::cluster_group cluster = cg::this_cluster();
  const int q = (int)cluster.block_rank();
  const int mat = blockIdx.x / LC;
  A += (long long)mat * sa;
  ipiv += (long long)mat * n;
  __shared__ double s_wv[LU_NB][LC_WARPS];
  __shared__ int s_wi[LU_NB][LC_WARPS];
  __shared__ double s_cv[LU_NB][LC];
  __shared__ int s_ci[LU_NB][LC];
  __shared__ double2 s_crow[2][LC][LU_NB];  // candidate rows, by rank
  __shared__ double2 s_rjj[2][LU_NB];       // row jj
  __shared__ int s_piv[LU_NB];
  int zero_col = 0;  // first zero pivot + 1
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r = j0 + q * LC_THREADS + tid;
  const bool own = r < n;
  cplx v[LU_NB];
#pragma unroll
  for (int k = 0; k < LU_NB; ++k)
    v[k] = (own && k < jb) ? ld2(&A[r + (long long)(j0 + k) * lda]) : mk(0.0, 0.0);
#pragma unroll 1
  for (int c0 = 0; c0 < jb; c0 += LC_BLK) {  // jb is the same for every thread
#pragma unroll
    for (int i = 0; i < LC_BLK; ++i) {
      const int c = c0 + i;
      if (c >= jb) break;
      const int jj = j0 + c, buf = c & 1;
      double best = (own && r >= jj) ? cabs1(v[i]) : -1.0;
      int bidx = (own && r >= jj) ? r : n;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1)
        argmax_step(best, bidx, __shfl_xor_sync(0xffffffffu, best, off),
                    __shfl_xor_sync(0xffffffffu, bidx, off));
      if (lane == 0) {
        s_wv[c][warp] = best;
        s_wi[c][warp] = bidx;
      }
      __syncthreads();
      {
        double bv = lane < LC_WARPS ? s_wv[c][lane] : -1.0;
        int bi = lane < LC_WARPS ? s_wi[c][lane] : n;
#pragma unroll
        for (int off = LC_WARPS / 2; off > 0; off >>= 1)
          argmax_step(bv, bi, __shfl_xor_sync(0xffffffffu, bv, off),
                      __shfl_xor_sync(0xffffffffu, bi, off));
        // lane 0 decides (the lanes agree unless a NaN breaks the order)
        bv = __shfl_sync(0xffffffffu, bv, 0);
        bi = __shfl_sync(0xffffffffu, bi, 0);
        if (bi < n && (bi - j0 - q * LC_THREADS) >> 5 == warp) {
          if (r == bi)
#pragma unroll
            for (int k = i; k < LU_NB; ++k) s_crow[buf][q][k] = make_double2(v[k].x, v[k].y);
          __syncwarp();
          if (lane >= i) {
            const double2 x = s_crow[buf][q][lane];
#pragma unroll
            for (int t = 0; t < LC; ++t)
              if (t != q) *cluster.map_shared_rank(&s_crow[buf][q][lane], t) = x;
          }
        }
        if (warp == 0 && lane < LC) {
          *cluster.map_shared_rank(&s_cv[c][q], lane) = bv;
          *cluster.map_shared_rank(&s_ci[c][q], lane) = bi;
        }
      }
      if (q == 0 && warp == 0) {
        if (lane == c)
#pragma unroll
          for (int k = i; k < LU_NB; ++k) s_rjj[buf][k] = make_double2(v[k].x, v[k].y);
        __syncwarp();
        if (lane >= i) {
          const double2 x = s_rjj[buf][lane];
#pragma unroll
          for (int t = 1; t < LC; ++t) *cluster.map_shared_rank(&s_rjj[buf][lane], t) = x;
        }
      }
      cluster.sync();
      double bv = s_cv[c][0];
      int bi = s_ci[c][0], qw = 0;
#pragma unroll
      for (int t = 1; t < LC; ++t) {
        const double ov = s_cv[c][t];
        const int oi = s_ci[c][t];
        if (ov > bv || (ov == bv && oi < bi)) {
          bv = ov;
          bi = oi;
          qw = t;
        }
      }
      const int piv = (bi < jj || bi >= n) ? jj : bi;
      if (tid == 0) s_piv[c] = piv;
      const double2* prow = piv == jj ? s_rjj[buf] : s_crow[buf][qw];
      if (own && piv != jj && (r == jj || r == piv)) {
        const double2* src = r == jj ? prow : s_rjj[buf];
#pragma unroll
        for (int k = i; k < LU_NB; ++k) v[k] = mk(src[k].x, src[k].y);
      }
      const double2 dd = prow[i];
      if (dd.x == 0.0 && dd.y == 0.0) {
        if (zero_col == 0) zero_col = jj + 1;
      } else if (own && r > jj) {
        const cplx l = v[i] * cdiv(mk(1.0, 0.0), mk(dd.x, dd.y));
        v[i] = l;
        // columns c+1 .. jb-1 are v[i+1 .. jb-1-c0]; blocks of 8 past them are skipped
#pragma unroll
        for (int k0 = 0; k0 < LU_NB; k0 += 8) {
          if (k0 + 8 > i + 1 && k0 < jb - c0) {
#pragma unroll
            for (int k = k0; k < k0 + 8; ++k)
              if (k > i) v[k] = v[k] - l * mk(prow[k].x, prow[k].y);
          }
        }
      }
    }
    if (own)
#pragma unroll
      for (int i = 0; i < LC_BLK; ++i)
        if (c0 + i < jb) st2(&A[r + (long long)(j0 + c0 + i) * lda], v[i]);
#pragma unroll
    for (int k = 0; k < LU_NB; ++k) v[k] = k + LC_BLK < LU_NB ? v[k + LC_BLK] : mk(0.0, 0.0);
  }
  __syncthreads();
  if (q == 0) {
    if (tid < jb) ipiv[j0 + tid] = s_piv[tid];
    if (tid == 0 && zero_col != 0 && info[mat] == 0) info[mat] = zero_col;
  }
}

// Row swaps ipiv[j0..j0+jb) applied to every column outside [skip0, skip1).
// Columns in [skip0, skip1) (the panel's own) are skipped when sub == 0; with
// sub > 0 the panel was factored sub columns at a time and already applied to
// each of its columns the swaps up to the end of that column's sub-panel, so
// only the later ones remain.
__global__ void lu_laswp_kernel(int n, int ncols, int j0, int jb, int skip0, int skip1,
                                double2* A, long long lda, long long sa, const int* ipiv,
                                long long ipiv_stride, int sub) {
  const int b = blockIdx.y;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncols) return;
  int first = j0;
  if (c >= skip0 && c < skip1) {
    if (sub <= 0) return;
    first = skip0 + ((c - skip0) / sub + 1) * sub;
  }
  A += (long long)b * sa;
  ipiv += (long long)b * ipiv_stride;
  for (int jj = first; jj < j0 + jb; ++jj) {
    int p = ipiv[jj];
    if (p != jj) {
      double2 t = A[jj + (long long)c * lda];
      A[jj + (long long)c * lda] = A[p + (long long)c * lda];
      A[p + (long long)c * lda] = t;
    }
  }
}

// X = T^-1 X for a jb x jb triangular block T of the factor (unit lower when
// lower != 0, non-unit upper otherwise) and the jb-row slab X of `ncols`
// columns.  One thread per column; T staged in shared memory.
__global__ void lu_trsm_block_kernel(int jb, int ncols, int lower, const double2* T,
                                     long long ldt, long long st, double2* X, long long ldx,
                                     long long sx) {
  __shared__ double2 Ts[LU_NB][LU_NB + 1];
  const int b = blockIdx.y;
  T += (long long)b * st;
  X += (long long)b * sx;
  for (int idx = threadIdx.x; idx < jb * jb; idx += blockDim.x) {
    int r = idx % jb, c = idx / jb;
    Ts[r][c] = T[r + (long long)c * ldt];
  }
  __syncthreads();
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncols) return;
  cplx x[LU_NB];
#pragma unroll
  for (int r = 0; r < LU_NB; ++r)
    if (r < jb) x[r] = ld2(&X[r + (long long)col * ldx]);
  if (lower) {
#pragma unroll
    for (int r = 0; r < LU_NB; ++r) {
      if (r < jb) {
        cplx s = x[r];
#pragma unroll
        for (int q = 0; q < LU_NB; ++q)
          if (q < r) s = s - mk(Ts[r][q].x, Ts[r][q].y) * x[q];
        x[r] = s;
      }
    }
  } else {
#pragma unroll
    for (int r = LU_NB - 1; r >= 0; --r) {
      if (r < jb) {
        cplx s = x[r];
#pragma unroll
        for (int q = 0; q < LU_NB; ++q)
          if (q > r && q < jb) s = s - mk(Ts[r][q].x, Ts[r][q].y) * x[q];
        x[r] = cdiv(s, mk(Ts[r][r].x, Ts[r][r].y));
      }
    }
  }
#pragma unroll
  for (int r = 0; r < LU_NB; ++r)
    if (r < jb) st2(&X[r + (long long)col * ldx], x[r]);
}

// The same solve with one warp per column: lane r holds row r of X; step q
// broadcasts the finished x_q by shuffle and every later (lower) or earlier
// (upper) lane subtracts its term, so a column takes jb short steps instead of
// one thread's chain of jb^2/2 dependent products.  8 columns per CTA.
constexpr int LU_TRSM_WARPS = 8;
__global__ void __launch_bounds__(32 * LU_TRSM_WARPS)
    lu_trsm_warp_kernel(int jb, int ncols, int lower, const double2* T, long long ldt,
                        long long st, double2* X, long long ldx, long long sx) {
  __shared__ double2 Ts[LU_NB][LU_NB + 1];
  const int b = blockIdx.y;
  T += (long long)b * st;
  X += (long long)b * sx;
  for (int idx = threadIdx.x; idx < jb * jb; idx += blockDim.x) {
    const int r = idx % jb, c = idx / jb;
    Ts[r][c] = T[r + (long long)c * ldt];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int col = blockIdx.x * LU_TRSM_WARPS + (threadIdx.x >> 5);
  if (col >= ncols) return;  // whole warps: col is warp-uniform
  double2* Xc = X + (long long)col * ldx;
  cplx x = lane < jb ? ld2(&Xc[lane]) : mk(0.0, 0.0);
  if (lower) {
    for (int q = 0; q < jb; ++q) {
      const cplx xq = mk(__shfl_sync(0xffffffffu, x.x, q), __shfl_sync(0xffffffffu, x.y, q));
      if (lane > q && lane < jb) x = x - mk(Ts[lane][q].x, Ts[lane][q].y) * xq;
    }
  } else {
    for (int q = jb - 1; q >= 0; --q) {
      if (lane == q) x = cdiv(x, mk(Ts[q][q].x, Ts[q][q].y));
      const cplx xq = mk(__shfl_sync(0xffffffffu, x.x, q), __shfl_sync(0xffffffffu, x.y, q));
      if (lane < q) x = x - mk(Ts[lane][q].x, Ts[lane][q].y) * xq;
    }
  }
  if (lane < jb) st2(&Xc[lane], x);
}

static inline dim3 trsm_grid(int ncols, int batch) {
  return dim3((ncols + LU_TRSM_WARPS - 1) / LU_TRSM_WARPS, batch);
}

__global__ void zero_int_kernel(int* p, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = 0;
}

// Side stream (highest priority) and fork/join events of the look-ahead, one
// set per host thread and device, created by the first call (which therefore
// has to come before any stream capture).
struct LuSide {
  cudaStream_t hi = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};
static cudaError_t lu_side(LuSide** out) {
  static thread_local LuSide per_dev[64];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  LuSide& s = per_dev[dev];
  if (s.hi == nullptr) {
    int lo = 0, hi = 0;
    if ((e = cudaDeviceGetStreamPriorityRange(&lo, &hi)) != cudaSuccess) return e;
    if ((e = cudaStreamCreateWithPriority(&s.hi, cudaStreamNonBlocking, hi)) != cudaSuccess) return e;
    if ((e = cudaEventCreateWithFlags(&s.fork, cudaEventDisableTiming)) != cudaSuccess) return e;
    if ((e = cudaEventCreateWithFlags(&s.join, cudaEventDisableTiming)) != cudaSuccess) return e;
  }
  *out = &s;
  return cudaSuccess;
}

// Row-swap granularity the laswp after panel j0 applies to the panel's own
// columns: 1 after the cluster kernel (column c lacks the swaps of pivots
// c+1..), 0 after lu_panel_kernel (the panel's columns are complete).
static int panel_sub(int n, int j0) { return n - j0 <= 8 * LC_THREADS ? 1 : 0; }

static int lu_panel(int n, int j0, int jb, double2* A, long long lda, long long sa, int* ipiv,
                    int* info, int batch, cudaStream_t st) {
  const int rows = n - j0;
  // the tuning table may spread a panel's rows over more CTAs than they need
  const int lc_min = tune_lookup(EUV_KNOB_LU_CLUSTER, n, batch);
  if (rows <= LC_THREADS && lc_min <= 1)
    lu_panel_cluster_kernel<1><<<batch, LC_THREADS, 0, st>>>(n, j0, jb, A, lda, sa, ipiv, info);
  else if (rows <= 2 * LC_THREADS && lc_min <= 2)
    lu_panel_cluster_kernel<2><<<2 * batch, LC_THREADS, 0, st>>>(n, j0, jb, A, lda, sa, ipiv, info);
  else if (rows <= 4 * LC_THREADS && lc_min <= 4)
    lu_panel_cluster_kernel<4><<<4 * batch, LC_THREADS, 0, st>>>(n, j0, jb, A, lda, sa, ipiv, info);
  else if (rows <= 8 * LC_THREADS)
    lu_panel_cluster_kernel<8><<<8 * batch, LC_THREADS, 0, st>>>(n, j0, jb, A, lda, sa, ipiv, info);
  else
    lu_panel_kernel<<<batch, LU_PANEL_THREADS, 0, st>>>(n, j0, jb, A, lda, sa, ipiv, info);
  EUV_LAUNCH_CHECK();
  return EUV_OK;
}

// U12 = L11^-1 A12 and A22 -= L21 U12 of panel [j0, j0+jb) for the columns
// [c0, c0+nc) (rows j0.. of the factor).
static int lu_update(int n, int j0, int jb, int c0, int nc, double2* A, long long lda,
                     long long sa, int batch, cudaStream_t st) {
  if (nc <= 0) return EUV_OK;
  lu_trsm_warp_kernel<<<trsm_grid(nc, batch), 32 * LU_TRSM_WARPS, 0, st>>>(
      jb, nc, 1, A + j0 + (long long)j0 * lda, lda, sa, A + j0 + (long long)c0 * lda, lda, sa);
  EUV_LAUNCH_CHECK();
  const int rest = n - j0 - jb;
  return zgemm_sub(rest, nc, jb, A + (j0 + jb) + (long long)j0 * lda, lda, sa,
                   A + j0 + (long long)c0 * lda, lda, sa, A + (j0 + jb) + (long long)c0 * lda,
                   lda, sa, batch, st);
}

// Right-looking LU with one panel of look-ahead: after panel j, its update of
// the next panel's columns runs first; then the next panel is factored on the
// high-priority side stream (its batch CTAs take SMs as soon as any frees up)
// while the update of the remaining columns runs on the caller's stream.  The
// column sets are disjoint; the laswp of the next panel waits for both.
int lu_factor(int n, double2* A, long long lda, long long sa, int* ipiv, int* info, int batch,
              cudaStream_t stream) {
  if (n <= 0 || batch <= 0) return EUV_OK;
  LuSide* side = nullptr;
  EUV_CUDA_TRY(lu_side(&side));
  zero_int_kernel<<<(batch + 255) / 256, 256, 0, stream>>>(info, batch);
  EUV_LAUNCH_CHECK();
  int j0 = 0, jb = n < LU_NB ? n : LU_NB;
  int rc = lu_panel(n, j0, jb, A, lda, sa, ipiv, info, batch, stream);
  if (rc) return rc;
  for (;;) {
    dim3 gs((n + 127) / 128, batch);
    lu_laswp_kernel<<<gs, 128, 0, stream>>>(n, n, j0, jb, j0, j0 + jb, A, lda, sa, ipiv, n, panel_sub(n, j0));
    EUV_LAUNCH_CHECK();
    const int rest = n - j0 - jb;
    if (rest <= 0) break;
    const int j1 = j0 + jb, nb2 = rest < LU_NB ? rest : LU_NB, rem = rest - nb2;
    if ((rc = lu_update(n, j0, jb, j1, nb2, A, lda, sa, batch, stream))) return rc;
    if (rem > 0) {
      EUV_CUDA_TRY(cudaEventRecord(side->fork, stream));
      EUV_CUDA_TRY(cudaStreamWaitEvent(side->hi, side->fork, 0));
      if ((rc = lu_panel(n, j1, nb2, A, lda, sa, ipiv, info, batch, side->hi))) return rc;
      if ((rc = lu_update(n, j0, jb, j1 + nb2, rem, A, lda, sa, batch, stream))) return rc;
      EUV_CUDA_TRY(cudaEventRecord(side->join, side->hi));
      EUV_CUDA_TRY(cudaStreamWaitEvent(stream, side->join, 0));
    } else if ((rc = lu_panel(n, j1, nb2, A, lda, sa, ipiv, info, batch, stream))) {
      return rc;
    }
    j0 = j1;
    jb = nb2;
  }
  return EUV_OK;
}

// Forward (unit lower L) and backward (upper U) substitution of RC right-hand
// sides per CTA with X resident in shared memory (xs[c*n + r]) for the whole
// solve; L and U are streamed once per CTA in blocks of LS_BLK rows/columns:
//   diagonal block : staged in shared memory (its loads issued during the
//                    previous block's update); warp c solves column c, lane i
//                    = block row i, each solved entry broadcast by shuffle;
//   off-diagonal   : x(r) -= T(r, block) x(block) for the rows below (forward)
//                    or above (backward).  RC = 8 runs it on the FP64 tensor
//                    path: 8-row tiles x 8 right-hand sides x K = 4 DMMAs, four
//                    per complex step, two tiles' loads in flight per warp;
//                    RC = 12 (two column tiles, the second half used) when the
//                    launch then takes fewer waves (24 units x 67 columns: 144
//                    CTAs instead of 216 on 148 SMs).
// Replaces 2*ceil(n/32) trsm launches + as many K=32 GEMMs per solve.
constexpr int LS_THREADS = 512;
constexpr int LS_WARPS = LS_THREADS / 32;
constexpr int LS_BLK = 32;
constexpr size_t LS_SMEM_MAX = 200 * 1024;

__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Two elements per thread of the diagonal block at (j0, j0), zero outside jb.
struct DiagPrefetch {
  double2 v[2];
  __device__ __forceinline__ void load(const double2* LU, long long lda, int j0, int jb, int tid) {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int i = tid + k * LS_THREADS, r = i % LS_BLK, q = i / LS_BLK;
      v[k] = (r < jb && q < jb) ? LU[j0 + r + (long long)(j0 + q) * lda] : make_double2(0.0, 0.0);
    }
  }
  __device__ __forceinline__ void store(double2 (*ds)[LS_BLK + 1], int tid) const {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int i = tid + k * LS_THREADS;
      ds[i % LS_BLK][i / LS_BLK] = v[k];
    }
  }
};
static_assert(2 * LS_THREADS == LS_BLK * LS_BLK, "DiagPrefetch covers the block");

// xs[c*n + r] -= sum_{q<jb} T(r, j0+q) xs[c*n + j0+q], r in [r_lo, r_hi), c < RC
template <int RC>
__device__ __forceinline__ void update_rows(double2* xs, int n, const double2* LU, long long lda,
                                            int j0, int jb, int r_lo, int r_hi, int tid) {
  if constexpr (RC == 8 || RC == 12) {
    // NT column tiles of 8 right-hand sides (RC = 12: the second tile half
    // used); each row tile's L fragment serves all of them.  UT row tiles'
    // loads in flight per warp (one at RC = 12, for the registers).
    constexpr int NT = (RC + 7) / 8, UT = RC == 8 ? 2 : 1;
    const int lane = tid & 31, warp = tid >> 5, kq = lane & 3, g = lane >> 2;
    double br[NT][8], bi[NT][8];  // B fragments: x(j0 + 4ks + kq) of right-hand side 8nt + g
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int ks = 0; ks < 8; ++ks) {
        const int q = 4 * ks + kq, c = 8 * nt + g;
        const double2 v = (q < jb && c < RC) ? xs[c * n + j0 + q] : make_double2(0.0, 0.0);
        br[nt][ks] = v.x;
        bi[nt][ks] = v.y;
      }
    const int ntiles = (r_hi - r_lo + 7) / 8;
    for (int t = warp; t < ntiles; t += UT * LS_WARPS) {
      double2 a[UT][8];
#pragma unroll
      for (int u = 0; u < UT; ++u) {
        const int tt = t + u * LS_WARPS, r = r_lo + tt * 8 + g;
        const bool rok = tt < ntiles && r < r_hi;
#pragma unroll
        for (int ks = 0; ks < 8; ++ks) {
          const int q = 4 * ks + kq;
          a[u][ks] = (rok && q < jb) ? LU[r + (long long)(j0 + q) * lda] : make_double2(0.0, 0.0);
        }
      }
#pragma unroll
      for (int u = 0; u < UT; ++u) {
        const int tt = t + u * LS_WARPS;
        if (tt >= ntiles) break;  // warp-uniform
        const int r = r_lo + tt * 8 + g;
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          double cr0 = 0.0, cr1 = 0.0, ci0 = 0.0, ci1 = 0.0;
#pragma unroll
          for (int ks = 0; ks < 8; ++ks) {
            dmma884(cr0, cr1, a[u][ks].x, br[nt][ks]);
            dmma884(cr0, cr1, -a[u][ks].y, bi[nt][ks]);
            dmma884(ci0, ci1, a[u][ks].x, bi[nt][ks]);
            dmma884(ci0, ci1, a[u][ks].y, br[nt][ks]);
          }
          const int c0 = 8 * nt + 2 * kq;
          if (r < r_hi && c0 < RC) {
            double2* p0 = &xs[c0 * n + r];
            double2* p1 = &xs[(c0 + 1) * n + r];
            const double2 o0 = *p0, o1 = *p1;
            *p0 = make_double2(o0.x - cr0, o0.y - ci0);
            *p1 = make_double2(o1.x - cr1, o1.y - ci1);
          }
        }
      }
    }
  } else {
    for (int r = r_lo + tid; r < r_hi; r += LS_THREADS) {
      cplx acc[RC];
#pragma unroll
      for (int c = 0; c < RC; ++c) acc[c] = mk(0.0, 0.0);
#pragma unroll 8
      for (int q = 0; q < jb; ++q) {
        const cplx lv = ld2(&LU[r + (long long)(j0 + q) * lda]);
#pragma unroll
        for (int c = 0; c < RC; ++c) acc[c] = acc[c] + lv * ld2(&xs[c * n + j0 + q]);
      }
#pragma unroll
      for (int c = 0; c < RC; ++c) st2(&xs[c * n + r], ld2(&xs[c * n + r]) - acc[c]);
    }
  }
}

template <int RC>
__global__ void __launch_bounds__(LS_THREADS) lu_subst_kernel(int n, int nrhs, const double2* LU,
                                                              long long lda, long long sa,
                                                              double2* B, long long ldb,
                                                              long long sb, const int* order,
                                                              long long ostride) {
  extern __shared__ double2 xs[];
  __shared__ double2 ds[LS_BLK][LS_BLK + 1];
  const int b = blockIdx.y, c0 = blockIdx.x * RC;
  const int nc = (nrhs - c0) < RC ? (nrhs - c0) : RC;
  if (order != nullptr) {
    // every column of this CTA is an empty source slot (order < 0): its
    // right-hand sides are zero and so is the solution, already in place
    bool any = false;
    for (int c = 0; c < nc; ++c) any |= order[(long long)b * ostride + c0 + c] >= 0;
    if (!any) return;  // the same for every thread of the CTA
  }
  LU += (long long)b * sa;
  B += (long long)b * sb;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  DiagPrefetch pf;
  pf.load(LU, lda, 0, n < LS_BLK ? n : LS_BLK, tid);
  for (int i = tid; i < RC * n; i += LS_THREADS) {
    const int c = i / n, r = i - c * n;
    xs[i] = c < nc ? B[r + (long long)(c0 + c) * ldb] : make_double2(0.0, 0.0);
  }
  pf.store(ds, tid);
  __syncthreads();
  // ---- forward: L y = b
  for (int j0 = 0; j0 < n; j0 += LS_BLK) {
    const int jb = (n - j0) < LS_BLK ? (n - j0) : LS_BLK;
    if (warp < nc) {
      double2* xc = xs + (long long)warp * n + j0;
      cplx x = lane < jb ? ld2(&xc[lane]) : mk(0.0, 0.0);
#pragma unroll
      for (int q = 0; q < LS_BLK; ++q) {
        const cplx xq = mk(__shfl_sync(0xffffffffu, x.x, q), __shfl_sync(0xffffffffu, x.y, q));
        if (lane > q && lane < jb) x = x - ld2(&ds[lane][q]) * xq;
      }
      if (lane < jb) st2(&xc[lane], x);
    }
    __syncthreads();
    // next diagonal block: the forward pass's successor, or the backward pass's first
    const int jn = j0 + LS_BLK < n ? j0 + LS_BLK : ((n - 1) / LS_BLK) * LS_BLK;
    pf.load(LU, lda, jn, (n - jn) < LS_BLK ? (n - jn) : LS_BLK, tid);
    update_rows<RC>(xs, n, LU, lda, j0, jb, j0 + jb, n, tid);
    pf.store(ds, tid);
    __syncthreads();
  }
  // ---- backward: U x = y
  for (int j0 = ((n - 1) / LS_BLK) * LS_BLK; j0 >= 0; j0 -= LS_BLK) {
    const int jb = (n - j0) < LS_BLK ? (n - j0) : LS_BLK;
    if (warp < nc) {
      double2* xc = xs + (long long)warp * n + j0;
      cplx x = lane < jb ? ld2(&xc[lane]) : mk(0.0, 0.0);
      // each lane's reciprocal pivot, off the serial chain below
      const cplx rinv = lane < jb ? cdiv(mk(1.0, 0.0), ld2(&ds[lane][lane])) : mk(0.0, 0.0);
#pragma unroll
      for (int q = LS_BLK - 1; q >= 0; --q) {
        if (q < jb) {  // warp-uniform
          if (lane == q) x = x * rinv;
          const cplx xq = mk(__shfl_sync(0xffffffffu, x.x, q), __shfl_sync(0xffffffffu, x.y, q));
          if (lane < q) x = x - ld2(&ds[lane][q]) * xq;
        }
      }
      if (lane < jb) st2(&xc[lane], x);
    }
    __syncthreads();
    if (j0 > 0) pf.load(LU, lda, j0 - LS_BLK, LS_BLK, tid);
    update_rows<RC>(xs, n, LU, lda, j0, jb, 0, j0, tid);
    if (j0 > 0) pf.store(ds, tid);
    __syncthreads();
  }
  for (int i = tid; i < RC * n; i += LS_THREADS) {
    const int c = i / n, r = i - c * n;
    if (c < nc) B[r + (long long)(c0 + c) * ldb] = xs[i];
  }
}

template <int RC>
static int launch_subst(int n, int nrhs, const double2* LU, long long lda, long long sa,
                        double2* B, long long ldb, long long sb, int batch, const int* order,
                        long long ostride, cudaStream_t stream) {
  static int smem_done[64];
  const int smem = (int)((size_t)RC * n * sizeof(double2));
  EUV_CUDA_TRY(ensure_smem(lu_subst_kernel<RC>, smem, smem_done));
  dim3 grid((nrhs + RC - 1) / RC, batch);
  lu_subst_kernel<RC><<<grid, LS_THREADS, smem, stream>>>(n, nrhs, LU, lda, sa, B, ldb, sb, order,
                                                          ostride);
  EUV_LAUNCH_CHECK();
  return EUV_OK;
}

int lu_solve(int n, int nrhs, const double2* LU, long long lda, long long sa, const int* ipiv,
             double2* B, long long ldb, long long sb, int batch, cudaStream_t stream,
             const int* order, long long ostride) {
  if (n <= 0 || nrhs <= 0 || batch <= 0) return EUV_OK;
  dim3 gs((nrhs + 127) / 128, batch);
  lu_laswp_kernel<<<gs, 128, 0, stream>>>(n, nrhs, 0, n, 0, 0, B, ldb, sb, ipiv, n, 0);
  EUV_LAUNCH_CHECK();
  if (batch <= 65535) {
    const size_t col = (size_t)n * sizeof(double2);
    // 12 right-hand sides per CTA where that takes fewer waves than 8 (one CTA
    // per SM either way: the resident columns fill its shared memory), or where
    // the tuning table says so
    if (12 * col <= LS_SMEM_MAX && nrhs >= 12) {
      const int tuned = tune_lookup(EUV_KNOB_LU_SUBST_COLS, n, batch);
      bool twelve = tuned == 12;
      if (tuned == 0) {
        int sms = 0, dev = 0;
        EUV_CUDA_TRY(cudaGetDevice(&dev));
        EUV_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const long long w8 = ((long long)((nrhs + 7) / 8) * batch + sms - 1) / sms;
        const long long w12 = ((long long)((nrhs + 11) / 12) * batch + sms - 1) / sms;
        // with empty source slots skipped the launch holds fewer live CTAs than
        // its grid, so a tie in waves goes to 12 (measured: 24 units of N = 961,
        // 96 slots for families of 96, 92 and 12 sources, step 25.35 -> 24.97 ms)
        twelve = sms > 0 && (w12 < w8 || (order != nullptr && w12 == w8));
      }
      if (twelve)
        return launch_subst<12>(n, nrhs, LU, lda, sa, B, ldb, sb, batch, order, ostride, stream);
    }
    if (8 * col <= LS_SMEM_MAX && nrhs >= 8)
      return launch_subst<8>(n, nrhs, LU, lda, sa, B, ldb, sb, batch, order, ostride, stream);
    if (4 * col <= LS_SMEM_MAX && nrhs >= 4)
      return launch_subst<4>(n, nrhs, LU, lda, sa, B, ldb, sb, batch, order, ostride, stream);
    if (2 * col <= LS_SMEM_MAX && nrhs >= 2)
      return launch_subst<2>(n, nrhs, LU, lda, sa, B, ldb, sb, batch, order, ostride, stream);
    if (col <= LS_SMEM_MAX)
      return launch_subst<1>(n, nrhs, LU, lda, sa, B, ldb, sb, batch, order, ostride, stream);
  }
  // n too large for one column of X in shared memory: blocked trsm + GEMM
  // forward: L y = b (unit lower)
  for (int j0 = 0; j0 < n; j0 += LU_NB) {
    const int jb = (n - j0) < LU_NB ? (n - j0) : LU_NB;
    lu_trsm_block_kernel<<<gs, 128, 0, stream>>>(jb, nrhs, 1, LU + j0 + (long long)j0 * lda, lda,
                                                  sa, B + j0, ldb, sb);
    EUV_LAUNCH_CHECK();
    const int rest = n - j0 - jb;
    if (rest > 0) {
      int rc = zgemm_sub(rest, nrhs, jb, LU + (j0 + jb) + (long long)j0 * lda, lda, sa, B + j0,
                         ldb, sb, B + j0 + jb, ldb, sb, batch, stream);
      if (rc != EUV_OK) return rc;
    }
  }
  // backward: U x = y
  const int nblk = (n + LU_NB - 1) / LU_NB;
  for (int bi = nblk - 1; bi >= 0; --bi) {
    const int j0 = bi * LU_NB;
    const int jb = (n - j0) < LU_NB ? (n - j0) : LU_NB;
    lu_trsm_block_kernel<<<gs, 128, 0, stream>>>(jb, nrhs, 0, LU + j0 + (long long)j0 * lda, lda,
                                                  sa, B + j0, ldb, sb);
    EUV_LAUNCH_CHECK();
    if (j0 > 0) {
      int rc = zgemm_sub(j0, nrhs, jb, LU + (long long)j0 * lda, lda, sa, B + j0, ldb, sb, B,
                         ldb, sb, batch, stream);
      if (rc != EUV_OK) return rc;
    }
  }
  return EUV_OK;
}

}  // namespace euv

extern "C" size_t euv_lu_workspace_bytes(int n, int batch) {
  (void)n;
  (void)batch;
  return 0;
}

extern "C" int euv_lu_factor(int n, euv_c64* d_a, int lda, long long stride_a, int* d_ipiv,
                             int* d_info, int batch, void* stream) {
  if (n < 0 || lda < (n > 0 ? n : 1) || batch < 0 || (n > 0 && batch > 0 && (!d_a || !d_ipiv || !d_info))) {
    euv_set_error("euv_lu_factor: bad arguments (n=%d lda=%d batch=%d)", n, lda, batch);
    return EUV_ERR_BAD_ARG;
  }
  return euv::lu_factor(n, reinterpret_cast<double2*>(d_a), lda, stride_a, d_ipiv, d_info, batch,
                        (cudaStream_t)stream);
}

extern "C" int euv_lu_solve(int n, int nrhs, const euv_c64* d_lu, int lda, long long stride_a,
                            const int* d_ipiv, euv_c64* d_b, int ldb, long long stride_b,
                            int batch, void* stream) {
  if (n < 0 || nrhs < 0 || lda < (n > 0 ? n : 1) || ldb < (n > 0 ? n : 1) || batch < 0) {
    euv_set_error("euv_lu_solve: bad arguments (n=%d nrhs=%d lda=%d ldb=%d)", n, nrhs, lda, ldb);
    return EUV_ERR_BAD_ARG;
  }
  return euv::lu_solve(n, nrhs, reinterpret_cast<const double2*>(d_lu), lda, stride_a, d_ipiv,
                       reinterpret_cast<double2*>(d_b), ldb, stride_b, batch,
                       (cudaStream_t)stream, nullptr, 0);
}
