// Hermitian eigendecomposition by parallel cyclic Jacobi rotations.
//
// Replaces the eigh (cupy.linalg.eigh) of the STCC-SOCS transmission
// cross-coefficient matrices (cnn/intensity/stccsocs/eigenfunction.py:128-130):
// a per-configuration step, so simplicity and accuracy matter more than speed.
// The matrix (column-major, n <= a few thousand) stays L2-resident.
//
// A round of a sweep rotates m/2 disjoint index pairs of a round-robin
// tournament over m = n rounded up to even (slot 0 fixed, the others rotating;
// indices >= n are dummies).  For a pair (p, q) with Hermitian 2x2 block
// [[a, b], [conj(b), d]], b = |b| e^{i phi}:
//   J = diag(1, e^{-i phi}) G,  G = [[c, s], [-s, c]],
//   t = sign(tau) / (|tau| + sqrt(1 + tau^2)),  tau = (d - a) / (2 |b|),
// c = 1/sqrt(1 + t^2), s = t c; J^H A J zeroes A(p,q) and gives a - t|b|,
// d + t|b| on the diagonal (the real symmetric Jacobi step after a phase).
// All column updates of a round (A J, V J) commute, then all row updates (J^H .).
// After each sweep the off-diagonal Frobenius norm is compared with tol x the
// full one; once below, a device flag turns the remaining launches into no-ops.
#include "common.cuh"

namespace euv {

struct JacRot {
  double c, s, er, ei;  // J = [[c, s], [-s e, c e]] with e = er + i ei = e^{-i phi}
  double app, aqq;      // the exact new diagonal
  int active;
};

__device__ __forceinline__ int jac_slot(int i, int r, int m) {
  return i == 0 ? 0 : 1 + (i - 1 + r) % (m - 1);
}

__global__ void jac_params_kernel(int n, int m, int r, const double2* A, long long lda,
                                  JacRot* rot, const int* done) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m / 2 || *done) return;
  const int p = jac_slot(k, r, m), q = jac_slot(m - 1 - k, r, m);
  JacRot j;
  j.c = 1.0;
  j.s = 0.0;
  j.er = 1.0;
  j.ei = 0.0;
  j.active = 0;
  j.app = j.aqq = 0.0;
  if (p < n && q < n) {
    const double a = A[p + (long long)p * lda].x, d = A[q + (long long)q * lda].x;
    const double2 b = A[p + (long long)q * lda];
    const double ab = hypot(b.x, b.y);
    if (ab > 1e-300 && ab > 1e-18 * (fabs(a) + fabs(d))) {
      const double tau = (d - a) / (2.0 * ab);
      const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
      j.c = 1.0 / sqrt(1.0 + t * t);
      j.s = t * j.c;
      j.er = b.x / ab;   // e^{-i phi} = conj(b)/|b|
      j.ei = -b.y / ab;
      j.app = a - t * ab;
      j.aqq = d + t * ab;
      j.active = 1;
    }
  }
  rot[k] = j;
}

// columns p, q of A and V: X(:,p) <- c X(:,p) - s e X(:,q),  X(:,q) <- s X(:,p) + c e X(:,q)
__global__ void jac_cols_kernel(int n, int m, int r, double2* A, long long lda, double2* V,
                                long long ldv, const JacRot* rot, const int* done) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (i >= n || *done) return;
  const JacRot j = rot[k];
  if (!j.active) return;
  const int p = jac_slot(k, r, m), q = jac_slot(m - 1 - k, r, m);
  const cplx e = mk(j.er, j.ei);
  {
    double2* xp = A + i + (long long)p * lda;
    double2* xq = A + i + (long long)q * lda;
    const cplx u = mk(xp->x, xp->y), w = mk(xq->x, xq->y);
    const cplx ew = e * w;
    const cplx np_ = j.c * u - j.s * ew, nq = j.s * u + j.c * ew;
    *xp = make_double2(np_.x, np_.y);
    *xq = make_double2(nq.x, nq.y);
  }
  {
    double2* xp = V + i + (long long)p * ldv;
    double2* xq = V + i + (long long)q * ldv;
    const cplx u = mk(xp->x, xp->y), w = mk(xq->x, xq->y);
    const cplx ew = e * w;
    const cplx np_ = j.c * u - j.s * ew, nq = j.s * u + j.c * ew;
    *xp = make_double2(np_.x, np_.y);
    *xq = make_double2(nq.x, nq.y);
  }
}

// rows p, q of A: X(p,:) <- c X(p,:) - s conj(e) X(q,:),  X(q,:) <- s X(p,:) + c conj(e) X(q,:);
// the 2x2 block itself is set to its exact rotated value.
__global__ void jac_rows_kernel(int n, int m, int r, double2* A, long long lda, const JacRot* rot,
                                const int* done) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int col = blockIdx.y;
  if (k >= m / 2 || *done) return;
  const JacRot j = rot[k];
  if (!j.active) return;
  const int p = jac_slot(k, r, m), q = jac_slot(m - 1 - k, r, m);
  double2* xp = A + p + (long long)col * lda;
  double2* xq = A + q + (long long)col * lda;
  if (col == p) {
    *xp = make_double2(j.app, 0.0);
    *xq = make_double2(0.0, 0.0);
    return;
  }
  if (col == q) {
    *xp = make_double2(0.0, 0.0);
    *xq = make_double2(j.aqq, 0.0);
    return;
  }
  const cplx ce = mk(j.er, -j.ei);
  const cplx u = mk(xp->x, xp->y), w = mk(xq->x, xq->y);
  const cplx cw = ce * w;
  const cplx np_ = j.c * u - j.s * cw, nq = j.s * u + j.c * cw;
  *xp = make_double2(np_.x, np_.y);
  *xq = make_double2(nq.x, nq.y);
}

// acc[0] += off-diagonal |A_ij|^2, acc[1] += all |A_ij|^2
__global__ void jac_norm_kernel(int n, const double2* A, long long lda, double* acc,
                                const int* done) {
  if (*done) return;
  __shared__ double so[8], st[8];
  double off = 0.0, tot = 0.0;
  const long long nn = (long long)n * n;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nn;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % n), c = (int)(t / n);
    const double2 v = A[i + (long long)c * lda];
    const double a2 = v.x * v.x + v.y * v.y;
    tot += a2;
    if (i != c) off += a2;
  }
  for (int o = 16; o > 0; o >>= 1) {
    off += __shfl_down_sync(0xffffffffu, off, o);
    tot += __shfl_down_sync(0xffffffffu, tot, o);
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    so[w] = off;
    st[w] = tot;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int u = 0; u < (int)(blockDim.x >> 5); ++u) {
      a += so[u];
      b += st[u];
    }
    atomicAdd(&acc[0], a);
    atomicAdd(&acc[1], b);
  }
}

__global__ void jac_check_kernel(double* acc, double tol2, int* done, int last, int* status,
                                 double* w, const double2* A, long long lda, int n) {
  if (*done == 0 && acc[0] <= tol2 * acc[1]) *done = 1;
  acc[0] = acc[1] = 0.0;
  if (last) {
    if (*done == 0 && status) atomicOr(status, EUV_STATUS_NOT_CONVERGED);
    for (int i = 0; i < n; ++i) w[i] = A[i + (long long)i * lda].x;
  }
}

__global__ void jac_eye_kernel(int n, double2* V, long long ldv) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int i = (int)(t % n), c = (int)(t / n);
  V[i + (long long)c * ldv] = make_double2(i == c ? 1.0 : 0.0, 0.0);
}

__global__ void jac_init_kernel(double* acc, int* done) {
  acc[0] = acc[1] = 0.0;
  *done = 0;
}

}  // namespace euv

using namespace euv;

extern "C" size_t euv_heev_workspace_bytes(int n) {
  if (n <= 0) return 0;
  const int m = n + (n & 1);
  return ((size_t)(m / 2) * sizeof(JacRot) + 255) / 256 * 256 + 256;
}

extern "C" int euv_heev(int n, euv_c64* d_a, int lda, double* d_w, euv_c64* d_v, int ldv,
                        int max_sweeps, double tol, void* d_work, size_t work_bytes, int* d_status,
                        void* stream_) {
  if (n <= 0 || n > 65535 || lda < n || ldv < n || !d_a || !d_w || !d_v || max_sweeps <= 0 ||
      max_sweeps > 100 || !(tol > 0.0) || !d_work) {
    euv_set_error("euv_heev: bad arguments (n=%d lda=%d ldv=%d sweeps=%d)", n, lda, ldv, max_sweeps);
    return EUV_ERR_BAD_ARG;
  }
  if (work_bytes < euv_heev_workspace_bytes(n)) {
    euv_set_error("euv_heev: workspace too small");
    return EUV_ERR_WORKSPACE;
  }
  cudaStream_t stream = (cudaStream_t)stream_;
  const int m = n + (n & 1);
  char* w = reinterpret_cast<char*>(d_work);
  JacRot* rot = reinterpret_cast<JacRot*>(w);
  const size_t rot_bytes = ((size_t)(m / 2) * sizeof(JacRot) + 255) / 256 * 256;
  double* acc = reinterpret_cast<double*>(w + rot_bytes);
  int* done = reinterpret_cast<int*>(w + rot_bytes + 2 * sizeof(double));
  double2* A = reinterpret_cast<double2*>(d_a);
  double2* V = reinterpret_cast<double2*>(d_v);
  jac_init_kernel<<<1, 1, 0, stream>>>(acc, done);
  EUV_LAUNCH_CHECK();
  jac_eye_kernel<<<(unsigned)(((long long)n * n + 255) / 256), 256, 0, stream>>>(n, V, ldv);
  EUV_LAUNCH_CHECK();
  const int pairs = m / 2;
  const dim3 gp((pairs + 127) / 128);
  const dim3 gc((n + 127) / 128, pairs);
  const dim3 gr((pairs + 127) / 128, n);
  const double tol2 = tol * tol;
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    for (int r = 0; r < m - 1; ++r) {
      jac_params_kernel<<<gp, 128, 0, stream>>>(n, m, r, A, lda, rot, done);
      EUV_LAUNCH_CHECK();
      jac_cols_kernel<<<gc, 128, 0, stream>>>(n, m, r, A, lda, V, ldv, rot, done);
      EUV_LAUNCH_CHECK();
      jac_rows_kernel<<<gr, 128, 0, stream>>>(n, m, r, A, lda, rot, done);
      EUV_LAUNCH_CHECK();
    }
    jac_norm_kernel<<<148 * 4, 256, 0, stream>>>(n, A, lda, acc, done);
    EUV_LAUNCH_CHECK();
    jac_check_kernel<<<1, 1, 0, stream>>>(acc, tol2, done, sweep == max_sweeps - 1, d_status, d_w, A,
                                          lda, n);
    EUV_LAUNCH_CHECK();
  }
  return EUV_OK;
}
