// STCC-SOCS imaging from M3D parameters (cnn/intensity/stccsocs/socs.py:12-151).
//
// Per clip the reference forms, for each retained TCC eigenfunction, the pupil
// amplitudes weighted by it, scatters them onto a 64 x 64 frequency grid and
// inverse-FFTs them (100 + 5 x 20 grids), sums alpha |F|^2 and the slope cross
// terms, and Fourier-interpolates the 64 x 64 image to XDIV x YDIV.  Here:
//   socs_rows_kernel   : all rows of all clips scattered onto the grids;
//   2 batched zgemm    : F = E G E with E the 64-point DFT matrix (e^{+2 pi i ab/64});
//   socs_accum_kernel  : the weighted |F|^2 / cross-term sum per grid point;
//   2 batched zgemm    : the interpolation Ky . small^T . Kx^T with the resident
//                        kernels Kx[x][u] = (1/64) sum_{i=-32}^{31} e^{2 pi i i (x/XDIV - u/64)},
//                        written as the complex image [x][y] (its real part is
//                        the reference's output).
#include "common.cuh"

namespace euv {

int zgemm(int m, int n, int k, cplx alpha, const double* scale, const double2* a, long long lda,
          long long sa, const double2* b, long long ldb, long long sb, cplx beta, double2* c,
          long long ldc, long long sc, cplx diag, int batch, const int* steps, int step,
          cudaStream_t stream);

struct SocsArgs {
  int ncut, lpx, lpy, nsocs, nxy, nout, rows;
  const int *lp, *mp;
  double k, dx, dy, kx0, ky0, z0;
  cplx vc, ab, phase0_inv;
  const double2 *phi0, *phix, *phiy;
};

// rows r < nsocs: A0 phi0[r]; then for j < nxy, t = 0..4:
//   A0 phix[j], Ax phix[j], A0 phiy[j], Ay phiy[j], Axy phi0[j]
// with A0 = famp + a0, Ax = ax dx/2pi, Ay = ay dy/2pi, Axy = ax lp/2 + ay mp/2
// (socs.py:84-98).  Grid element (px, py) of row r of clip c at
// G[(c*rows + r)*nout^2 + px + nout*py], px = lp mod nout.
__global__ void socs_rows_kernel(SocsArgs p, const double2* fvac, const double2* a0,
                                 const double2* ax, const double2* ay, double2* G) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y, c = blockIdx.z;
  if (n >= p.ncut) return;
  const int l = p.lp[n], m = p.mp[n];
  const long long nsp = (long long)(2 * p.lpx + 1) * (2 * p.lpy + 1);
  const double2 fv = fvac[c * nsp + (l + p.lpx) + (long long)(2 * p.lpx + 1) * (m + p.lpy)];
  cplx f = (p.vc - p.ab) * mk(fv.x, fv.y);
  if (l == 0 && m == 0) f = f + p.ab;
  const double twopi = 6.283185307179586476925286766559;
  const double kxp = twopi * l / p.dx, kyp = twopi * m / p.dy;
  const double arg = -((p.kx0 * kxp + 0.5 * kxp * kxp) + (p.ky0 * kyp + 0.5 * kyp * kyp)) / p.k * p.z0;
  double sn, cs;
  sincos(arg, &sn, &cs);
  const long long q = (long long)c * p.ncut + n;
  const cplx famp = f * mk(cs, sn) * p.phase0_inv;
  const cplx va0 = mk(a0[q].x, a0[q].y), vax = mk(ax[q].x, ax[q].y), vay = mk(ay[q].x, ay[q].y);
  cplx amp, phi;
  if (r < p.nsocs) {
    amp = famp + va0;
    const double2 v = p.phi0[(long long)r * p.ncut + n];
    phi = mk(v.x, v.y);
  } else {
    const int j = (r - p.nsocs) / 5, t = (r - p.nsocs) % 5;
    const double2* src = (t == 0 || t == 1) ? p.phix : (t == 2 || t == 3) ? p.phiy : p.phi0;
    const double2 v = src[(long long)j * p.ncut + n];
    phi = mk(v.x, v.y);
    if (t == 0 || t == 2) amp = famp + va0;
    else if (t == 1) amp = vax * (p.dx / twopi);
    else if (t == 3) amp = vay * (p.dy / twopi);
    else amp = vax * (0.5 * l) + vay * (0.5 * m);
  }
  const int px = ((l % p.nout) + p.nout) % p.nout, py = ((m % p.nout) + p.nout) % p.nout;
  const cplx v = amp * phi;
  G[((long long)c * p.rows + r) * p.nout * p.nout + px + (long long)p.nout * py] = make_double2(v.x, v.y);
}

// small^T[c][v + nout*u] = sum_r alpha0 |F_r(u,v)|^2 + cross terms (socs.py:99-136)
__global__ void socs_accum_kernel(int nout, int rows, int nsocs, int nxy, const double* al0,
                                  const double* alx, const double* aly, const double2* F,
                                  double2* smallT) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;  // u + nout*v (F's column-major index)
  const int c = blockIdx.y;
  const int nn = nout * nout;
  if (g >= nn) return;
  const double2* f = F + (long long)c * rows * nn + g;
  double s = 0.0;
  for (int r = 0; r < nsocs; ++r) {
    const double2 v = f[(long long)r * nn];
    s += al0[r] * (v.x * v.x + v.y * v.y);
  }
  for (int j = 0; j < nxy; ++j) {
    const double2* b = f + (long long)(nsocs + 5 * j) * nn;
    const double2 f0x = b[0], fx = b[nn], f0y = b[2 * (long long)nn], fy = b[3 * (long long)nn],
                  fxy = b[4 * (long long)nn];
    const double2 f0 = f[(long long)j * nn];
    s += 2.0 * alx[j] * (f0x.x * fx.x + f0x.y * fx.y) + 2.0 * aly[j] * (f0y.x * fy.x + f0y.y * fy.y) +
         2.0 * al0[j] * (f0.x * fxy.x + f0.y * fxy.y);
  }
  const int u = g % nout, v = g / nout;
  smallT[(long long)c * nn + v + (long long)nout * u] = make_double2(s, 0.0);
}

}  // namespace euv

using namespace euv;

static size_t socs_bytes(const euv_socs_desc* d, size_t* g, size_t* sm, size_t* t3) {
  const size_t nn = (size_t)d->nout * d->nout;
  const size_t rows = (size_t)d->nsocs + 5 * (size_t)d->nsocsxy;
  *g = ((size_t)d->n_clips * rows * nn * 16 + 255) / 256 * 256;
  *sm = ((size_t)d->n_clips * nn * 16 + 255) / 256 * 256;
  *t3 = ((size_t)d->n_clips * d->nout * d->xdiv * 16 + 255) / 256 * 256;
  return 2 * *g + *sm + *t3;
}

extern "C" size_t euv_socs_workspace_bytes(const euv_socs_desc* d) {
  if (!d || d->n_clips <= 0 || d->nout <= 0 || d->nsocs <= 0 || d->nsocsxy < 0 ||
      d->nsocsxy > d->nsocs || d->xdiv <= 0)
    return 0;
  size_t g, sm, t3;
  return socs_bytes(d, &g, &sm, &t3);
}

extern "C" int euv_socs_image(const euv_socs_desc* d, const euv_c64* d_fvac, const euv_c64* d_a0,
                              const euv_c64* d_ax, const euv_c64* d_ay, euv_c64* d_image,
                              void* d_work, size_t work_bytes, void* stream_) {
  if (!d || !d_fvac || !d_a0 || !d_ax || !d_ay || !d_image || d->n_clips <= 0 ||
      d->n_clips > 65535 || d->ncut <= 0 || d->lpx < 0 || d->lpy < 0 || d->nsocs <= 0 ||
      d->nsocsxy < 0 || d->nsocsxy > d->nsocs || d->nout <= 0 || d->nout > 1024 ||
      2 * d->lpx + 1 > d->nout || 2 * d->lpy + 1 > d->nout || d->xdiv <= 0 || d->ydiv <= 0 ||
      !d->d_lp || !d->d_mp || !d->d_phi_s0 || (d->nsocsxy > 0 && (!d->d_phi_sx || !d->d_phi_sy)) ||
      !d->d_alpha_s0 || (d->nsocsxy > 0 && (!d->d_alpha_sx || !d->d_alpha_sy)) || !d->d_e ||
      !d->d_kxT || !d->d_ky || (d->amp_vc.re == 0.0 && d->amp_vc.im == 0.0)) {
    euv_set_error("euv_socs_image: bad arguments");
    return EUV_ERR_BAD_ARG;
  }
  const int rows = d->nsocs + 5 * d->nsocsxy;
  if ((long long)rows > 65535) {
    euv_set_error("euv_socs_image: too many kernel rows");
    return EUV_ERR_BAD_ARG;
  }
  size_t gb, smb, t3b;
  if (!d_work || work_bytes < socs_bytes(d, &gb, &smb, &t3b)) {
    euv_set_error("euv_socs_image: workspace too small");
    return EUV_ERR_WORKSPACE;
  }
  cudaStream_t stream = (cudaStream_t)stream_;
  char* w = reinterpret_cast<char*>(d_work);
  double2* G = reinterpret_cast<double2*>(w);
  double2* T = reinterpret_cast<double2*>(w + gb);
  double2* smallT = reinterpret_cast<double2*>(w + 2 * gb);
  double2* T3 = reinterpret_cast<double2*>(w + 2 * gb + smb);
  const int nout = d->nout, nn = nout * nout;
  SocsArgs p;
  p.ncut = d->ncut;
  p.lpx = d->lpx;
  p.lpy = d->lpy;
  p.nsocs = d->nsocs;
  p.nxy = d->nsocsxy;
  p.nout = nout;
  p.rows = rows;
  p.lp = d->d_lp;
  p.mp = d->d_mp;
  p.k = d->k;
  p.dx = d->dx;
  p.dy = d->dy;
  p.kx0 = d->kx0;
  p.ky0 = d->ky0;
  p.z0 = d->z0;
  p.vc = fromc(d->amp_vc);
  p.ab = fromc(d->amp_ab);
  const double av = sqrt(p.vc.x * p.vc.x + p.vc.y * p.vc.y);
  p.phase0_inv = cdiv(mk(1.0, 0.0), mk(p.vc.x / av, p.vc.y / av));
  p.phi0 = reinterpret_cast<const double2*>(d->d_phi_s0);
  p.phix = reinterpret_cast<const double2*>(d->d_phi_sx);
  p.phiy = reinterpret_cast<const double2*>(d->d_phi_sy);
  EUV_CUDA_TRY(cudaMemsetAsync(G, 0, gb, stream));
  socs_rows_kernel<<<dim3((d->ncut + 127) / 128, rows, d->n_clips), 128, 0, stream>>>(
      p, reinterpret_cast<const double2*>(d_fvac), reinterpret_cast<const double2*>(d_a0),
      reinterpret_cast<const double2*>(d_ax), reinterpret_cast<const double2*>(d_ay), G);
  EUV_LAUNCH_CHECK();
  const cplx one = mk(1.0, 0.0), zero = mk(0.0, 0.0);
  const double2* E = reinterpret_cast<const double2*>(d->d_e);
  const int nb = d->n_clips * rows;
  // T = G E (each grid col-major px x py), F = E T  -> F[x][y] = sum G e^{+} e^{+}
  int rc = zgemm(nout, nout, nout, one, nullptr, G, nout, nn, E, nout, 0, zero, T, nout, nn, zero, nb,
                 nullptr, 0, stream);
  if (rc) return rc;
  rc = zgemm(nout, nout, nout, one, nullptr, E, nout, 0, T, nout, nn, zero, G, nout, nn, zero, nb,
             nullptr, 0, stream);
  if (rc) return rc;
  socs_accum_kernel<<<dim3((nn + 127) / 128, d->n_clips), 128, 0, stream>>>(
      nout, rows, d->nsocs, d->nsocsxy, d->d_alpha_s0, d->d_alpha_sx, d->d_alpha_sy, G, smallT);
  EUV_LAUNCH_CHECK();
  // T3 = small^T . Kx^T (nout x XDIV), image^T = Ky . T3 (YDIV x XDIV) = image[x][y]
  const double2* kxT = reinterpret_cast<const double2*>(d->d_kxT);
  const double2* ky = reinterpret_cast<const double2*>(d->d_ky);
  rc = zgemm(nout, d->xdiv, nout, one, nullptr, smallT, nout, nn, kxT, nout, 0, zero, T3, nout,
             (long long)nout * d->xdiv, zero, d->n_clips, nullptr, 0, stream);
  if (rc) return rc;
  rc = zgemm(d->ydiv, d->xdiv, nout, one, nullptr, ky, d->ydiv, 0, T3, nout,
             (long long)nout * d->xdiv, zero, reinterpret_cast<double2*>(d_image), d->ydiv,
             (long long)d->xdiv * d->ydiv, zero, d->n_clips, nullptr, 0, stream);
  return rc;
}
