// Linear Abbe model from M3D parameters (cnn/intensity/linear/linear.py).
//
// The reference builds, per source point of a fine source grid and per pupil
// order, the thin-mask amplitude corrected by the M3D parameters
// (linear.py:120-172), then images it with one FFT Abbe loop per source
// (linear.py:11-43).  Here the amplitudes of every clip x source x pupil point
// are one elementwise launch; the image is the fused Abbe kernel (abbe.cu) with
// identity pupil tables.  HBM-bound: 16 B written per amplitude, the inputs
// (spectrum and parameters per pupil point) are re-read from L2.
#include "common.cuh"

namespace euv {

struct LinearArgs {
  int n_src, ncut, lpx, lpy;
  const int *lp, *mp;
  const double *ls, *ms;
  double k, dx, dy, kx0, ky0, z0;
  cplx vc, ab, phase0_inv;
};

__global__ void linear_amp_kernel(LinearArgs p, const double2* fvac, const double2* a0,
                                  const double2* ax, const double2* ay, double2* amp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y, c = blockIdx.z;
  if (i >= p.ncut) return;
  const int l = p.lp[i], m = p.mp[i];
  const long long nsp = (long long)(2 * p.lpx + 1) * (2 * p.lpy + 1);
  const double2 fv = fvac[c * nsp + (l + p.lpx) + (long long)(2 * p.lpx + 1) * (m + p.lpy)];
  cplx f = (p.vc - p.ab) * mk(fv.x, fv.y);
  if (l == 0 && m == 0) f = f + p.ab;
  const double twopi = 6.283185307179586476925286766559;
  const double kxp = twopi * l / p.dx, kyp = twopi * m / p.dy;
  const double arg = -((p.kx0 * kxp + 0.5 * kxp * kxp) + (p.ky0 * kyp + 0.5 * kyp * kyp)) / p.k * p.z0;
  double sn, cs;
  sincos(arg, &sn, &cs);
  cplx a = f * mk(cs, sn) * p.phase0_inv;
  if (a0 != nullptr) {
    const long long q = (long long)c * p.ncut + i;
    const double ls = p.ls[s] + 0.5 * l, ms = p.ms[s] + 0.5 * m;
    a = a + mk(a0[q].x, a0[q].y) + ls * mk(ax[q].x, ax[q].y) + ms * mk(ay[q].x, ay[q].y);
  }
  amp[((long long)c * p.n_src + s) * p.ncut + i] = make_double2(a.x, a.y);
}

}  // namespace euv

using namespace euv;

extern "C" int euv_linear_amp(const euv_linear_desc* d, const euv_c64* d_fvac, const euv_c64* d_a0,
                              const euv_c64* d_ax, const euv_c64* d_ay, euv_c64* d_amp,
                              void* stream) {
  if (!d || !d_fvac || !d_amp || d->n_clips <= 0 || d->n_clips > 65535 || d->n_src <= 0 ||
      d->n_src > 65535 || d->ncut <= 0 || d->lpx < 0 || d->lpy < 0 || !d->d_lp || !d->d_mp ||
      !d->d_ls || !d->d_ms || d->k <= 0.0 || d->dx <= 0.0 || d->dy <= 0.0 ||
      (d_a0 != nullptr && (!d_ax || !d_ay)) ||
      (d->amp_vc.re == 0.0 && d->amp_vc.im == 0.0)) {
    euv_set_error("euv_linear_amp: bad arguments");
    return EUV_ERR_BAD_ARG;
  }
  LinearArgs p;
  p.n_src = d->n_src;
  p.ncut = d->ncut;
  p.lpx = d->lpx;
  p.lpy = d->lpy;
  p.lp = d->d_lp;
  p.mp = d->d_mp;
  p.ls = d->d_ls;
  p.ms = d->d_ms;
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
  dim3 grid((d->ncut + 255) / 256, d->n_src, d->n_clips);
  linear_amp_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(
      p, reinterpret_cast<const double2*>(d_fvac), reinterpret_cast<const double2*>(d_a0),
      reinterpret_cast<const double2*>(d_ax), reinterpret_cast<const double2*>(d_ay),
      reinterpret_cast<double2*>(d_amp));
  EUV_LAUNCH_CHECK();
  return EUV_OK;
}
