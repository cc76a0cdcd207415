// M3D-parameter extraction (replaces m3d.cpp:240-467), one thread per
// (clip, pupil order).
#include "common.cuh"

namespace euv {

struct M3dParams {
  int n_src, ninput, n_order, n_order_narrow, lpx, lpy, s_center;
  double k, dx, dy, z0, kx0, ky0;
  const int* src_l;
  const int* src_m;
  const int* src_nn;
  const double2* ax_vc;
  const double2* ax_ab;
  const int* lin;
  const int* min_;
  const int* xin;
  const int* pair;
};

__device__ __forceinline__ cplx unit_phase(cplx v) {
  double a = cabs(v);
  return mk(v.x / a, v.y / a);
}

__global__ void m3d_fit_kernel(M3dParams p, int n_clips, const double2* ax_wide,
                               const double2* fmask, double2* a0, double2* ax, double2* ay) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_clips * p.ninput) return;
  const int c = t / p.ninput, n = t % p.ninput;
  const double twopi = 6.283185307179586476925286766559;
  // specular vacuum / absorber amplitudes of the centre source (m3d.cpp:240-258)
  const int sc = p.s_center;
  const double2 vv = p.ax_vc[(long long)sc * p.n_order_narrow + p.src_nn[sc]];
  const double2 aa = p.ax_ab[(long long)sc * p.n_order_narrow + p.src_nn[sc]];
  const cplx vc_c = mk(vv.x, vv.y), ab_c = mk(aa.x, aa.y);
  const cplx ph_c = unit_phase(vc_c);
  const int lp = p.lin[n], mp = p.min_[n];
  const int ip = lp + p.lpx, jp = mp + p.lpy;
  // thin-mask amplitude of the centre source (m3d.cpp:329-356, 384-394)
  const double kxp = twopi * lp / p.dx, kyp = twopi * mp / p.dy;
  const double arg = -(p.kx0 * kxp + kxp * kxp / 2.0 + p.ky0 * kyp + kyp * kyp / 2.0) / p.k * p.z0;
  double sn, cs;
  sincos(arg, &sn, &cs);
  const double2 fm2 = fmask[(long long)c * (2 * p.lpx + 1) * (2 * p.lpy + 1) + ip +
                            (long long)(2 * p.lpx + 1) * jp];
  cplx famp = mk(fm2.x, fm2.y) * mk(cs, sn) * (vc_c - ab_c);
  if (lp == 0 && mp == 0) famp = famp + ab_c;
  famp = cdiv(famp, ph_c);
  // least-squares sums over the sources seeing this pupil order (m3d.cpp:426-450)
  cplx f1 = mk(0, 0), fx = mk(0, 0), fy = mk(0, 0);
  double c1 = 0, cx = 0, cy = 0, cx2 = 0, cy2 = 0, cxy = 0;
  const double2* axc = ax_wide + (long long)c * p.n_src * p.n_order;
  for (int s = 0; s < p.n_src; ++s) {
    const int o = p.pair[(long long)n * p.n_src + s];
    if (o < 0) continue;
    const double2 a2 = axc[(long long)s * p.n_order + o];
    const double2 v2 = p.ax_vc[(long long)s * p.n_order_narrow + p.src_nn[s]];
    const cplx f = cdiv(mk(a2.x, a2.y), unit_phase(mk(v2.x, v2.y))) - famp;  // dampxx
    const double ls = p.src_l[s] + lp / 2.0, ms = p.src_m[s] + mp / 2.0;
    f1 = f1 + f;
    fx = fx + ls * f;
    fy = fy + ms * f;
    c1 += 1;
    cx += ls;
    cy += ms;
    cx2 += ls * ls;
    cy2 += ms * ms;
    cxy += ls * ms;
  }
  cplx r0, rx = mk(0, 0), ry = mk(0, 0);
  if (p.xin[n] == 1) {  // 3x3 Cramer (m3d.cpp:451-461)
    const double cd = c1 * cx2 * cy2 + 2.0 * cx * cxy * cy - c1 * cxy * cxy - cx2 * cy * cy -
                      cy2 * cx * cx;
    r0 = (1.0 / cd) * ((cx2 * cy2 - cxy * cxy) * f1 + (-cx * cy2 + cy * cxy) * fx +
                       (cx * cxy - cy * cx2) * fy);
    rx = (1.0 / cd) * ((-cx * cy2 + cy * cxy) * f1 + (c1 * cy2 - cy * cy) * fx +
                       (-c1 * cxy + cx * cy) * fy);
    ry = (1.0 / cd) * ((cx * cxy - cy * cx2) * f1 + (-c1 * cxy + cx * cy) * fx +
                       (c1 * cx2 - cx * cx) * fy);
  } else {
    r0 = (1.0 / c1) * f1;
  }
  const long long o = (long long)c * p.ninput + n;
  a0[o] = make_double2(r0.x, r0.y);
  ax[o] = make_double2(rx.x, rx.y);
  ay[o] = make_double2(ry.x, ry.y);
}

}  // namespace euv

using namespace euv;

extern "C" int euv_m3d_fit(const euv_m3d_desc* d, const euv_c64* d_ax_wide,
                           const euv_c64* d_fmask, euv_c64* d_a0, euv_c64* d_ax, euv_c64* d_ay,
                           void* stream_) {
  if (!d || !d_ax_wide || !d_fmask || !d_a0 || !d_ax || !d_ay || d->n_clips <= 0 ||
      d->n_src <= 0 || d->ninput <= 0 || d->n_order <= 0 || d->n_order_narrow <= 0 ||
      d->s_center < 0 || d->s_center >= d->n_src || !d->d_src_l || !d->d_src_m ||
      !d->d_src_nidx_narrow || !d->d_ax_vc || !d->d_ax_ab || !d->d_lin || !d->d_min ||
      !d->d_xin || !d->d_pair_order || d->k <= 0) {
    euv_set_error("euv_m3d_fit: bad arguments");
    return EUV_ERR_BAD_ARG;
  }
  M3dParams p;
  p.n_src = d->n_src;
  p.ninput = d->ninput;
  p.n_order = d->n_order;
  p.n_order_narrow = d->n_order_narrow;
  p.lpx = d->lpx;
  p.lpy = d->lpy;
  p.s_center = d->s_center;
  p.k = d->k;
  p.dx = d->dx;
  p.dy = d->dy;
  p.z0 = d->z0;
  p.kx0 = d->kx0;
  p.ky0 = d->ky0;
  p.src_l = d->d_src_l;
  p.src_m = d->d_src_m;
  p.src_nn = d->d_src_nidx_narrow;
  p.ax_vc = reinterpret_cast<const double2*>(d->d_ax_vc);
  p.ax_ab = reinterpret_cast<const double2*>(d->d_ax_ab);
  p.lin = d->d_lin;
  p.min_ = d->d_min;
  p.xin = d->d_xin;
  p.pair = d->d_pair_order;
  const int total = d->n_clips * d->ninput;
  m3d_fit_kernel<<<(total + 127) / 128, 128, 0, (cudaStream_t)stream_>>>(
      p, d->n_clips, reinterpret_cast<const double2*>(d_ax_wide),
      reinterpret_cast<const double2*>(d_fmask), reinterpret_cast<double2*>(d_a0),
      reinterpret_cast<double2*>(d_ax), reinterpret_cast<double2*>(d_ay));
  EUV_LAUNCH_CHECK();
  return EUV_OK;
}
