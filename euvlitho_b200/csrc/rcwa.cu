// RCWA (Fourier-modal) solve of the absorber on the Mo/Si multilayer, batched
// over units (clip, Bloch family, polarisation).  Replaces ampS and its callees
// in header.h (maskamp 1147-1206, multilayerS 5-363, absorberS0 754-1145,
// absorberS 365-752, the tail of ampS 1355-1465).
//
// Formulation.  For a slice with Toeplitz matrix D (header.h:416-443) the
// reference diagonalises D = W diag(al^2) W^-1 and forms the T-matrix blocks
// T1UL..T1BR from W, al, B1 = i(k W - kp/k Sigma W) and gamma = exp(i al d).
// Writing X = W(U1U+U1B), Y = W al (U1U-U1B) and G = i(k I - diag(kp/k) Sigma),
// those blocks collapse to
//     X1 = c (G1^-1 G2 X2) - i s Y2,   Y1 = -i D s (G1^-1 G2 X2) + c Y2,
// with c = cos(sqrt(D) d) and s = sin(sqrt(D) d)/sqrt(D) -- entire functions
// of D, so no eigenvectors, square-root branches or W^-1 are needed.  At the
// bottom (Ru cap, header.h:1292-1303) G2 X2 = diag(Bru (URUU+URUB)) and
// Y2 = diag(alru (URUU-URUB)); at the top (header.h:1355-1391)
// U0 = diag(klm) X + Y and FG = diag(1/klm) Y U0^-1, so
//     Ax[:,s] = -diag(1/klm) Y U0^-1 (2 kz_s e_s) + e_s     (header.h:1394-1465).
// c and s come from a degree-8 Taylor polynomial of A = D h^2 (Paterson-
// Stockmeyer with A^2..A^4) at h = d/2^m, ||A||_1 <= 1, followed by m
// double-angle steps s <- 2 s c, c <- 2 c^2 - I: every step is a GEMM.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>
#include <math.h>
#include "common.cuh"

namespace euv {

int zgemm(int m, int n, int k, cplx alpha, const double* scale, const double2* a, long long lda,
          long long sa, const double2* b, long long ldb, long long sb, cplx beta, double2* c,
          long long ldc, long long sc, cplx diag, int batch, const int* steps, int step,
          cudaStream_t stream);
int lu_factor(int n, double2* A, long long lda, long long sa, int* ipiv, int* info, int batch,
              cudaStream_t stream);
// order (optional): per batch entry, ostride ints whose first nrhs mark the
// right-hand sides; a CTA whose columns are all < 0 (zero columns) is skipped
int lu_solve(int n, int nrhs, const double2* LU, long long lda, long long sa, const int* ipiv,
             double2* B, long long ldb, long long sb, int batch, cudaStream_t stream,
             const int* order = nullptr, long long ostride = 0);
int gemm_mixed(int m, int n, int k, cplx alpha, const double* scale, const double2* a,
               long long lda, long long sa, const double2* b, long long ldb, long long sb,
               cplx beta, double2* c, long long ldc, long long sc, cplx diag, int batch,
               const int* steps, int step, void* work, size_t work_bytes, int* status,
               cudaStream_t stream, int reuse, const double2* cin);
size_t gemm_mixed_workspace_bytes(int m, int n, int k, int batch);

// ||A||_1 bound for the degree-8 Taylor step of cos/sin(sqrt(A)): the dropped
// term is ~theta^9/18!, 1.6e-16 at theta = 1 (FP64) and 2e-8 at theta = 8,
// which the mixed form uses (its split-FP16x3 products carry ~1e-6 relative error,
// and each double-angle step saved also saves its error growth).
constexpr double kThetaFp64 = 1.0;
constexpr double kThetaMixed = 8.0;
inline double theta_for(int precision) {
  return precision == EUV_PREC_MIXED ? kThetaMixed : kThetaFp64;
}
constexpr int kMaxSteps = 40;

// ---------------------------------------------------------------- mask DFT
// The indicator of pattern pixel (x, y), x < FX, y < FY (header.h:1153-1166):
// the mask bit of column x / meshx and row NDIVY-1 - y / meshy + y_offset
// (rows outside the mask read as absorber), inverted unless select_vacuum.
__device__ __forceinline__ double mask_indicator(const uint8_t* bits, int ndivx, int ndivy,
                                                 int meshx, int meshy, int select_vacuum,
                                                 int y_offset, int x, int y) {
  const int ii = x / meshx;
  const int jj = ndivy - 1 - y / meshy + y_offset;
  int b = 0;
  if (jj >= 0 && jj < ndivy) {
    const long long bit = (long long)ndivx * jj + ii;
    b = (bits[bit >> 3] >> (7 - (int)(bit & 7))) & 1;
  }
  return select_vacuum ? (double)b : (double)(1 - b);
}

// Stage 1 of the separable DFT, straight from the packed bits:
//   T[g][m'][x] = sum_y IND_g(x, y) Wy[y + FY m']        (x contiguous)
// CTA tile: 32 x-columns (lanes) x 64 frequencies (8 warps x 8) for one mask,
// y streamed through shared memory in chunks of 32.  The indicator is 0/1, so
// each term is a masked add of a twiddle; one CTA per (x tile, m' tile, mask).
constexpr int SP_X = 32, SP_M = 64, SP_Y = 32;
__global__ void __launch_bounds__(256) spectrum_rows_kernel(
    const uint8_t* bits, long long mask_bytes, int ndivx, int ndivy, int fx, int fy, int mr,
    int select_vacuum, int y_offset, const double2* Wy, double2* T) {
  __shared__ double2 ws[SP_Y][SP_M + 1];
  __shared__ double vs[SP_Y][SP_X];
  const int g = blockIdx.z;
  const int x0 = blockIdx.x * SP_X, m0 = blockIdx.y * SP_M;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint8_t* mb = bits + (long long)g * mask_bytes;
  const int meshx = fx / ndivx, meshy = fy / ndivy;
  double ar[8], ai[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) ar[j] = ai[j] = 0.0;
  for (int y0 = 0; y0 < fy; y0 += SP_Y) {
    for (int i = threadIdx.x; i < SP_Y * SP_M; i += 256) {
      const int yy = i % SP_Y, mm = i / SP_Y, y = y0 + yy, m = m0 + mm;
      ws[yy][mm] = (y < fy && m < mr) ? Wy[y + (long long)fy * m] : make_double2(0.0, 0.0);
    }
    for (int i = threadIdx.x; i < SP_Y * SP_X; i += 256) {
      const int xx = i % SP_X, yy = i / SP_X, x = x0 + xx, y = y0 + yy;
      vs[yy][xx] = (x < fx && y < fy)
                       ? mask_indicator(mb, ndivx, ndivy, meshx, meshy, select_vacuum, y_offset, x, y)
                       : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int yy = 0; yy < SP_Y; ++yy) {
      const double a = vs[yy][lane];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const double2 wv = ws[yy][w + 8 * j];
        ar[j] = fma(a, wv.x, ar[j]);
        ai[j] = fma(a, wv.y, ai[j]);
      }
    }
    __syncthreads();
  }
  const int x = x0 + lane;
  if (x >= fx) return;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int m = m0 + w + 8 * j;
    if (m < mr) T[((long long)g * mr + m) * fx + x] = make_double2(ar[j], ai[j]);
  }
}

// Stage 2:  out[g][l' + LR m'] = sum_x Wx[l' + LR x] T[g][m'][x]
// One CTA per (m', mask); the T row is staged in shared memory, threads own l'.
constexpr int SC_THREADS = 64, SC_X = 256;
__global__ void __launch_bounds__(SC_THREADS) spectrum_cols_kernel(int fx, int lr, int mr,
                                                                   const double2* Wx,
                                                                   const double2* T,
                                                                   double2* out) {
  __shared__ double2 ts[SC_X];
  const int m = blockIdx.x, g = blockIdx.y;
  const double2* t = T + ((long long)g * mr + m) * fx;
  for (int l0 = 0; l0 < lr; l0 += SC_THREADS) {
    const int l = l0 + threadIdx.x;
    double sr = 0.0, si = 0.0;
    for (int x0 = 0; x0 < fx; x0 += SC_X) {
      __syncthreads();
      for (int i = threadIdx.x; i < SC_X; i += SC_THREADS)
        ts[i] = x0 + i < fx ? t[x0 + i] : make_double2(0.0, 0.0);
      __syncthreads();
      if (l < lr) {
        const int xe = fx - x0 < SC_X ? fx - x0 : SC_X;
        const double2* wx = Wx + l + (long long)lr * x0;
#pragma unroll 8
        for (int xx = 0; xx < xe; ++xx) {
          const double2 a = wx[(long long)lr * xx], b = ts[xx];
          sr = fma(a.x, b.x, fma(-a.y, b.y, sr));
          si = fma(a.x, b.y, fma(a.y, b.x, si));
        }
      }
    }
    if (l < lr) out[(long long)g * lr * mr + l + (long long)lr * m] = make_double2(sr, si);
  }
}

// Stage 2 as a split-K DMMA GEMM (out = Wx T^T, K = x in `parts` chunks, one
// batch entry per chunk): the chunk partial sums, added here.
__global__ void spectrum_reduce_kernel(const double2* part, int parts, long long total,
                                       double2* out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  double2 s = part[t];
  for (int p = 1; p < parts; ++p) {
    const double2 v = part[(long long)p * total + t];
    s.x += v.x;
    s.y += v.y;
  }
  out[t] = s;
}

// K chunks of stage 2 (0: the per-column kernel): fx / parts a multiple of 64
static int spectrum_parts(int fx) {
  if (fx % 64) return 0;
  int parts = fx / 64 < 16 ? fx / 64 : 16;
  while ((fx / 64) % parts) --parts;
  return parts;
}

// W[r + rows*c] = scale * exp(-2 pi i ((f*g) mod fdiv)/fdiv) with f = r - roff
// (frequency) and g = c - coff (sample), or transposed roles when `freq_rows`==0.
__global__ void twiddle_kernel(int rows, int cols, int roff, int coff, int fdiv, int freq_rows,
                               double scale, double2* W) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)rows * cols) return;
  int r = (int)(t % rows), c = (int)(t / rows);
  long long f = freq_rows ? (r - roff) : (c - coff);
  long long g = freq_rows ? c : r;
  long long q = (f * g) % fdiv;
  if (q < 0) q += fdiv;
  double s, co;
  sincospi(-2.0 * (double)q / (double)fdiv, &s, &co);
  W[t] = make_double2(scale * co, scale * s);
}

// ---------------------------------------------------------------- D and G
struct SliceParams {
  double k, dx, dy;
  const double* dxs;  // per-unit periods (NULL: dx, dy for every unit)
  const double* dys;
  int n, lmax, mmax, lr2, mr2, n_slices, slice;
  cplx eps_m1;   // eps_abs - 1
  cplx sig_m1;   // 1/eps_abs - 1
  cplx logeps;   // log(eps_abs)
};

// D(i,j) = k^2 eps[..] - i eta[..] kx_j (X) / - i zeta[..] ky_j (Y), minus kxy2_i
// on the diagonal (header.h:416-443); G(i,j) = i(k delta_ij - kp_i/k sigma[..] kp_j)
// (B1 = G W1, header.h:596-623).  want_d/want_g select the outputs.
__global__ void build_dg_kernel(SliceParams p, const double2* spectra, const int* spec_of_unit,
                                const int* lidx, const int* midx, const double* kx0,
                                const double* ky0, const int* polar, double2* D, double2* G,
                                int want_d, int want_g) {
  // grid: x = column j, y = row chunk, z = unit (no 64-bit division per element)
  const int u = blockIdx.z, j = blockIdx.x;
  // the unit's and column's constants once per CTA: no FP64 division per element
  __shared__ double s_c[8];  // 2pi/dx, 2pi/dy, 1/k, kx_j, ky_j, kx0, ky0
  if (threadIdx.x == 0) {
    const double twopi = 6.283185307179586476925286766559;
    const double dxu = p.dxs ? p.dxs[u] : p.dx, dyu = p.dys ? p.dys[u] : p.dy;
    const double gx = twopi / dxu, gy = twopi / dyu;
    s_c[0] = gx;
    s_c[1] = gy;
    s_c[2] = 1.0 / p.k;
    s_c[3] = kx0[u] + gx * lidx[j];
    s_c[4] = ky0[u] + gy * midx[j];
    s_c[5] = kx0[u];
    s_c[6] = ky0[u];
  }
  __syncthreads();
  const int i = blockIdx.y * blockDim.x + threadIdx.x;
  if (i >= p.n) return;
  const long long nn = (long long)p.n * p.n;
  const long long t = (long long)j * p.n + i;
  const int li = lidx[i], mi = midx[i], lj = lidx[j], mj = midx[j];
  const int l = li - lj + 2 * p.lmax, m = mi - mj + 2 * p.mmax;
  const double2* sp = spectra + ((long long)spec_of_unit[u] * p.n_slices + p.slice) * p.lr2 * p.mr2;
  const double2 f2 = sp[l + (long long)p.lr2 * m];
  const cplx F = mk(f2.x, f2.y);
  const bool dc = (l == 2 * p.lmax) && (m == 2 * p.mmax);
  const double gx = s_c[0], gy = s_c[1], ik = s_c[2];
  const double kxi = s_c[5] + gx * li, kyi = s_c[6] + gy * mi;
  const double kxj = s_c[3], kyj = s_c[4];
  const int pol = polar[u];
  if (want_d) {
    cplx eps = p.eps_m1 * F;
    if (dc) eps.x += 1.0;
    cplx leps = p.logeps * F;
    cplx v = (p.k * p.k) * eps;
    if (pol == 0) {
      // -i * eta * kx_j, eta = i 2 pi l / dx * leps  ->  +2 pi l/dx * leps * kx_j
      v = v + (gx * (double)(l - 2 * p.lmax) * kxj) * leps;
    } else {
      v = v + (gy * (double)(m - 2 * p.mmax) * kyj) * leps;
    }
    if (i == j) v.x -= kxi * kxi + kyi * kyi;
    D[(long long)u * nn + t] = make_double2(v.x, v.y);
  }
  if (want_g) {
    cplx sig = p.sig_m1 * F;
    if (dc) sig.x += 1.0;
    const double kpi = pol == 0 ? kxi : kyi, kpj = pol == 0 ? kxj : kyj;
    if (want_g == 2) {
      // E = diag(kp/k) sigma diag(kp/k), with G = i k (I - E)
      cplx v = (kpi * ik * (kpj * ik)) * sig;
      G[(long long)u * nn + t] = make_double2(v.x, v.y);
    } else {
      // G = i (k delta - kp_i/k sig kp_j)
      cplx a = (-kpi * ik * kpj) * sig;
      if (i == j) a.x += p.k;
      cplx v = cmul_i(a);
      G[(long long)u * nn + t] = make_double2(v.x, v.y);
    }
  }
}

// Z = s * (R + E R) with R = diag(v) (dense == 0) or R dense: the first factor
// of the Euler product (I - E)^-1 = (I + E)(I + E^2)(I + E^4)...
__global__ void euler_first_diag_kernel(int n, cplx s, const double2* E, const double2* v,
                                        double2* Z) {
  const long long nn = (long long)n * n;
  const int b = blockIdx.y;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nn) return;
  const long long o = (long long)b * nn + t;
  const int i = (int)(t % n), j = (int)(t / n);
  const double2 vv = v[(long long)b * n + j];
  const double2 e = E[o];
  cplx r = mk(e.x, e.y) * mk(vv.x, vv.y);
  if (i == j) r = r + mk(vv.x, vv.y);
  r = s * r;
  Z[o] = make_double2(r.x, r.y);
}

// ---------------------------------------------------------------- multilayer
struct StackParams {
  double k;
  cplx emo, esi, eru, emosi2, erusi, esio2;
  double dmo, dmosi, dsi, dsimo, dsiru, dru;
  int nml;
  double dx, dy;
  const double* dxs;  // per-unit periods (NULL: dx, dy for every unit)
  const double* dys;
  int n;
};

struct Blk {
  cplx ul, ur, bl, br;
};

__device__ __forceinline__ Blk iface(cplx cj, cplx al_out, cplx al_in, double thick) {
  // 1/2 (Cj +- al_out/al_in Cjp) exp(-+ i al_in d) (header.h:68-92 pattern)
  cplx expz = cexp_(cmul_i(al_in) * thick);
  cplx a = cdiv(al_out, al_in);
  cplx pl = 0.5 * (cj + a), mi = 0.5 * (cj - a);
  Blk b;
  b.ul = cdiv(pl, expz);
  b.ur = cdiv(mi, expz);
  b.bl = mi * expz;
  b.br = pl * expz;
  return b;
}
__device__ __forceinline__ void apply_blk(const Blk& b, cplx& uu, cplx& ub) {
  cplx nu = b.ul * uu + b.ur * ub;
  cplx nb = b.bl * uu + b.br * ub;
  uu = nu;
  ub = nb;
}

// Per order: URUU, URUB (header.h:5-363), alru, Bru (header.h:1292-1303), and
// the bottom boundary data x2 = URUU+URUB, y2 = alru (URUU-URUB),
// gx2 = Bru (URUU+URUB); klm = sqrt(k^2-kxy2) as a real root (header.h:1283).
__global__ void multilayer_kernel(StackParams p, const int* lidx, const int* midx,
                                  const double* kx0, const double* ky0, const int* polar,
                                  double2* x2, double2* y2, double2* gx2, double* klm,
                                  int n_units) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= p.n * n_units) return;
  const int u = t / p.n, i = t % p.n;
  const double twopi = 6.283185307179586476925286766559;
  const double kx = kx0[u] + twopi * lidx[i] / (p.dxs ? p.dxs[u] : p.dx);
  const double ky = ky0[u] + twopi * midx[i] / (p.dys ? p.dys[u] : p.dy);
  const double kxy2 = kx * kx + ky * ky;
  const double k = p.k, k2 = k * k;
  const double kp = polar[u] == 0 ? kx : ky;
  auto al = [&](cplx e) { return csqrt_p(mk(k2 * e.x - kxy2, k2 * e.y)); };
  cplx alsio2 = al(p.esio2), almo = al(p.emo), alsi = al(p.esi), almosi2 = al(p.emosi2),
       alru = al(p.eru), alrusi = al(p.erusi);
  auto ratio = [&](cplx enu, cplx eden) {
    cplx a = mk(k, 0.0) - cdiv(mk(kp * kp / k, 0.0), enu);
    cplx b = mk(k, 0.0) - cdiv(mk(kp * kp / k, 0.0), eden);
    return cdiv(a, b);
  };
  Blk TMO = iface(ratio(p.emosi2, p.emo), almosi2, almo, p.dmo);
  Blk TMOSI = iface(ratio(p.emo, p.emosi2), almo, almosi2, p.dmosi);
  Blk TSI = iface(ratio(p.emosi2, p.esi), almosi2, alsi, p.dsi);
  Blk TSIMO = iface(ratio(p.esi, p.emosi2), alsi, almosi2, p.dsimo);
  Blk TSIRU = iface(ratio(p.esi, p.erusi), alsi, alrusi, p.dsiru);
  Blk TRU = iface(ratio(p.erusi, p.eru), alrusi, alru, p.dru);
  Blk TN = iface(ratio(p.esio2, p.emo), alsio2, almo, p.dmo);
  cplx uu = TN.ul, ub = TN.bl;  // substrate (header.h:294-324)
  for (int l = p.nml - 1; l >= 0; --l) {  // header.h:326-359
    if (l < p.nml - 1) apply_blk(TMO, uu, ub);
    apply_blk(TMOSI, uu, ub);
    apply_blk(TSI, uu, ub);
    if (l > 0)
      apply_blk(TSIMO, uu, ub);
    else
      apply_blk(TSIRU, uu, ub);
  }
  apply_blk(TRU, uu, ub);  // URUU, URUB (header.h:361-362)
  const cplx bru = mk(0.0, k) - cmul_i(cdiv(mk(kp * kp / k, 0.0), p.eru));
  const cplx s = uu + ub, d = uu - ub;
  x2[t] = make_double2(s.x, s.y);
  cplx yv = alru * d;
  y2[t] = make_double2(yv.x, yv.y);
  cplx gv = bru * s;
  gx2[t] = make_double2(gv.x, gv.y);
  klm[t] = sqrt(k2 - kxy2);  // NaN for evanescent orders, as the reference
}

// ---------------------------------------------------------------- matrix functions
__global__ void zero_f64_kernel(double* p, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = 0.0;
}

// norm[b] = max_j sum_i (|re|+|im|)(D[b](i,j)): one warp per column.
__global__ void norm1_kernel(int n, const double2* D, double* norm) {
  const int b = blockIdx.y;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const double2* col = D + (long long)b * n * n + (long long)warp * n;
  double s = 0.0;
  for (int i = lane; i < n; i += 32) s += fabs(col[i].x) + fabs(col[i].y);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if (lane == 0) atomicMax(reinterpret_cast<unsigned long long*>(&norm[b]), __double_as_longlong(s));
}

// m = smallest m >= 0 with norm*(d/2^m)^2 <= theta (capped at m_max); h = d/2^m.
__global__ void scale_kernel(int batch, double theta, const double* norm, const double* thick, int m_max,
                             int* steps, double* h, double* h2, double* h4, int* capped) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  double d = thick[b];
  double v = norm[b] * d * d;
  int m = 0;
  while (v > theta && m < kMaxSteps) {
    v *= 0.25;
    ++m;
  }
  if (m > m_max) {
    m = m_max;
    if (capped) atomicOr(capped, EUV_STATUS_STEPS_CLAMPED);
  }
  double hh = ldexp(d, -m);
  steps[b] = m;
  h[b] = hh;
  h2[b] = hh * hh;
  h4[b] = hh * hh * hh * hh;
}

// Taylor coefficients: cos: (-1)^n/(2n)!, sinc: (-1)^n/(2n+1)!, n = 0..8.
__constant__ double c_cos[9] = {1.0, -1.0 / 2.0, 1.0 / 24.0, -1.0 / 720.0, 1.0 / 40320.0,
                                -1.0 / 3628800.0, 1.0 / 479001600.0, -1.0 / 87178291200.0,
                                1.0 / 20922789888000.0};
__constant__ double c_sin[9] = {1.0, -1.0 / 6.0, 1.0 / 120.0, -1.0 / 5040.0, 1.0 / 362880.0,
                                -1.0 / 39916800.0, 1.0 / 6227020800.0, -1.0 / 1307674368000.0,
                                1.0 / 355687428096000.0};

// With A = h^2 D, P2 = A^2, P3 = A^3, P4 = A^4 (scaled):
//   Cc = sum_{n<4} a_n A^n,  Tc = sum_{n<4} a_{n+4} A^n + a_8 A^4
//   Cs = h sum_{n<4} b_n A^n, Ts = h (sum_{n<4} b_{n+4} A^n + b_8 A^4)
// so that cos = Cc + P4 Tc and sin/sqrt = Cs + P4 Ts.
__global__ void taylor_prep_kernel(int n, int batch, const double2* D, const double2* P2,
                                   const double2* P3, const double2* P4, const double* h,
                                   const double* h2, double2* Cc, double2* Tc, double2* Cs,
                                   double2* Ts) {
  const long long nn = (long long)n * n;
  const int b = blockIdx.y;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nn) return;
  const long long o = (long long)b * nn + t;
  const int i = (int)(t % n), j = (int)(t / n);
  const double e = (i == j) ? 1.0 : 0.0;
  const double hb = h[b], s2 = h2[b];
  const double2 d = D[o], p2 = P2[o], p3 = P3[o], p4 = P4[o];
  const double ax = s2 * d.x, ay = s2 * d.y;
  double ccx = c_cos[0] * e + c_cos[1] * ax + c_cos[2] * p2.x + c_cos[3] * p3.x;
  double ccy = c_cos[1] * ay + c_cos[2] * p2.y + c_cos[3] * p3.y;
  double tcx = c_cos[4] * e + c_cos[5] * ax + c_cos[6] * p2.x + c_cos[7] * p3.x + c_cos[8] * p4.x;
  double tcy = c_cos[5] * ay + c_cos[6] * p2.y + c_cos[7] * p3.y + c_cos[8] * p4.y;
  double csx = c_sin[0] * e + c_sin[1] * ax + c_sin[2] * p2.x + c_sin[3] * p3.x;
  double csy = c_sin[1] * ay + c_sin[2] * p2.y + c_sin[3] * p3.y;
  double tsx = c_sin[4] * e + c_sin[5] * ax + c_sin[6] * p2.x + c_sin[7] * p3.x + c_sin[8] * p4.x;
  double tsy = c_sin[5] * ay + c_sin[6] * p2.y + c_sin[7] * p3.y + c_sin[8] * p4.y;
  Cc[o] = make_double2(ccx, ccy);
  Tc[o] = make_double2(tcx, tcy);
  Cs[o] = make_double2(hb * csx, hb * csy);
  Ts[o] = make_double2(hb * tsx, hb * tsy);
}

// ---------------------------------------------------------------- elementwise
// out[b](i,j) = alpha * A[b](i,j) * v[b][j] + beta * out[b](i,j)
__global__ void colscale_kernel(int n, cplx alpha, const double2* A, const double2* v, cplx beta,
                                double2* out) {
  const long long nn = (long long)n * n;
  const int b = blockIdx.y;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nn) return;
  const long long o = (long long)b * nn + t;
  const int j = (int)(t / n);
  double2 a = A[o], vv = v[(long long)b * n + j];
  cplx r = alpha * (mk(a.x, a.y) * mk(vv.x, vv.y));
  if (beta.x != 0.0 || beta.y != 0.0) {
    double2 q = out[o];
    r = r + beta * mk(q.x, q.y);
  }
  out[o] = make_double2(r.x, r.y);
}

// out[b] = diag(v[b])
__global__ void diag_kernel(int n, const double2* v, double2* out) {
  const long long nn = (long long)n * n;
  const int b = blockIdx.y;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nn) return;
  const int i = (int)(t % n), j = (int)(t / n);
  out[(long long)b * nn + t] = (i == j) ? v[(long long)b * n + i] : make_double2(0.0, 0.0);
}

// U0 = diag(klm) X + Y (header.h:1355-1371 in X,Y form)
__global__ void u0_kernel(int n, const double* klm, const double2* X, const double2* Y,
                          double2* U0) {
  const long long nn = (long long)n * n;
  const int b = blockIdx.y;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nn) return;
  const long long o = (long long)b * nn + t;
  const int i = (int)(t % n);
  const double kl = klm[(long long)b * n + i];
  double2 x = X[o], y = Y[o];
  U0[o] = make_double2(kl * x.x + y.x, kl * x.y + y.y);
}

// E[b](i,s) = 2kz_s if i == src_order[b][s] else 0 (AS of header.h:1402-1409)
__global__ void src_rhs_kernel(int n, int nsrc, const int* src_order, const double* src_2kz,
                               double2* E) {
  const int b = blockIdx.y;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * nsrc) return;
  const int i = (int)(t % n), s = (int)(t / n);
  const int o = src_order[(long long)b * nsrc + s];
  double v = (i == o) ? src_2kz[(long long)b * nsrc + s] : 0.0;
  E[(long long)b * n * nsrc + t] = make_double2(v, 0.0);
}

// Ax[b](i,s) = -(1/klm_i) YZ[b](i,s) + [i == src_order] (header.h:1449-1461)
__global__ void ax_out_kernel(int n, int nsrc, const int* src_order, const double* klm,
                              const double2* YZ, double2* ax) {
  const int b = blockIdx.y;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * nsrc) return;
  const int i = (int)(t % n), s = (int)(t / n);
  const int o = src_order[(long long)b * nsrc + s];
  const long long off = (long long)b * n * nsrc + t;
  if (o < 0) {
    ax[off] = make_double2(0.0, 0.0);
    return;
  }
  const double kl = klm[(long long)b * n + i];
  double2 v = YZ[off];
  double rx = -v.x / kl, ry = -v.y / kl;
  if (i == o) rx += 1.0;
  ax[off] = make_double2(rx, ry);
}

// ---------------------------------------------------------------- workspace
struct Bump {
  char* base;
  size_t cap, off;
  bool ok;
  template <typename T>
  T* take(size_t count) {
    size_t bytes = ((count * sizeof(T)) + 255) & ~(size_t)255;
    if (off + bytes > cap) ok = false;
    T* p = reinterpret_cast<T*>(base + off);
    off += bytes;
    return (ok && base) ? p : nullptr;
  }
};

inline unsigned grid1(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

__global__ void fill_f64_kernel(double* p, int n, double v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// An LU's zero pivots (info != 0) as EUV_STATUS_SINGULAR in the status word.
__global__ void flag_singular_kernel(const int* info, int n, int* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && info[i] != 0) atomicOr(status, EUV_STATUS_SINGULAR);
}

// GEMM dispatch by precision (FP64 DMMA, or split-FP16x3 tcgen05 tensor cores for
// the bulk products of the mixed form; `status` receives EUV_STATUS_TIMEOUT).
// Gemm reuse flags (mixed form only): the previous call through the same Gemm
// split this unchanged operand in the same role and shape, so its fp16 planes
// in the workspace are current.
constexpr int kReuseA = 1;
constexpr int kReuseB = 2;

struct Gemm {
  int precision;
  void* mwork;
  size_t mbytes;
  cudaStream_t stream;
  int* status = nullptr;
  int operator()(int m, int n, int k, cplx alpha, const double* scale, const double2* a,
                 long long lda, long long sa, const double2* b, long long ldb, long long sb,
                 cplx beta, double2* c, long long ldc, long long sc, cplx diag, int batch,
                 const int* steps = nullptr, int step = 0, int reuse = 0,
                 const double2* cin = nullptr) const {
    if (precision == EUV_PREC_MIXED)
      return gemm_mixed(m, n, k, alpha, scale, a, lda, sa, b, ldb, sb, beta, c, ldc, sc, diag,
                        batch, steps, step, mwork, mbytes, status, stream, reuse, cin);
    if (cin != nullptr && cin != c) {
      // FP64 GEMM: the beta term reads C, so C = Cin first (same shape)
      const size_t span = (size_t)(batch - 1) * sc + (size_t)(n - 1) * ldc + m;
      EUV_CUDA_TRY(cudaMemcpyAsync(c, cin, span * sizeof(double2), cudaMemcpyDeviceToDevice, stream));
    }
    return zgemm(m, n, k, alpha, scale, a, lda, sa, b, ldb, sb, beta, c, ldc, sc, diag, batch,
                 steps, step, stream);
  }
};

// Matrix functions for a batch: on return *pc, *ps point to cos / sinc (they
// may be swapped with the temporaries t0, t1).
struct MatfunBufs {
  double2 *P2, *P3, *P4, *T1, *T2;
  double *norm, *h, *h2, *h4;
  int* steps;
  int* capped;
};

int matfun(int n, int batch, const double2* D, const double* thick, double2** pc, double2** ps,
           const MatfunBufs& w, int m_max, const Gemm& gemm, cudaStream_t stream) {
  const long long nn = (long long)n * n;
  const int bs = 256;
  dim3 ge(grid1(nn, bs), batch);
  zero_f64_kernel<<<grid1(batch, 256), 256, 0, stream>>>(w.norm, batch);
  EUV_LAUNCH_CHECK();
  dim3 gn(grid1((long long)n * 32, 256), batch);
  norm1_kernel<<<gn, 256, 0, stream>>>(n, D, w.norm);
  EUV_LAUNCH_CHECK();
  scale_kernel<<<grid1(batch, 128), 128, 0, stream>>>(batch, theta_for(gemm.precision), w.norm,
                                                      thick, m_max, w.steps, w.h,
                                                      w.h2, w.h4, w.capped);
  EUV_LAUNCH_CHECK();
  const cplx one = mk(1.0, 0.0), zero = mk(0.0, 0.0);
  int rc;
  // P2 = h^4 D D, P3 = h^2 P2 D, P4 = P2 P2
  if ((rc = gemm(n, n, n, one, w.h4, D, n, nn, D, n, nn, zero, w.P2, n, nn, zero, batch))) return rc;
  if ((rc = gemm(n, n, n, one, w.h2, w.P2, n, nn, D, n, nn, zero, w.P3, n, nn, zero, batch, nullptr, 0,
                 kReuseB))) return rc;  // D as B again
  if ((rc = gemm(n, n, n, one, nullptr, w.P2, n, nn, w.P2, n, nn, zero, w.P4, n, nn, zero, batch,
                 nullptr, 0, kReuseA))) return rc;  // P2 as A again
  double2* C = *pc;
  double2* S = *ps;
  taylor_prep_kernel<<<ge, bs, 0, stream>>>(n, batch, D, w.P2, w.P3, w.P4, w.h, w.h2, C, w.T1, S,
                                            w.T2);
  EUV_LAUNCH_CHECK();
  if ((rc = gemm(n, n, n, one, nullptr, w.P4, n, nn, w.T1, n, nn, one, C, n, nn, zero, batch))) return rc;
  if ((rc = gemm(n, n, n, one, nullptr, w.P4, n, nn, w.T2, n, nn, one, S, n, nn, zero, batch,
                 nullptr, 0, kReuseA))) return rc;  // P4 as A again
  // double-angle steps; entries with fewer steps copy through (C = A)
  double2* tS = w.P2;
  double2* tC = w.P3;
  for (int step = 0; step < m_max; ++step) {
    if ((rc = gemm(n, n, n, mk(2.0, 0.0), nullptr, S, n, nn, C, n, nn, zero, tS, n, nn, zero,
                   batch, w.steps, step)))
      return rc;
    if ((rc = gemm(n, n, n, mk(2.0, 0.0), nullptr, C, n, nn, C, n, nn, zero, tC, n, nn,
                   mk(-1.0, 0.0), batch, w.steps, step, kReuseB)))  // C as B again
      return rc;
    double2* t = S;
    S = tS;
    tS = t;
    t = C;
    C = tC;
    tC = t;
  }
  *pc = C;
  *ps = S;
  return EUV_OK;
}

// Upper bound of max_b ||D_b||_1 from the config (Parseval: the window sum of
// |F| is at most sqrt(window size)); used to bound the double-angle steps.
static int derive_m_max(const euv_amp_desc* d) {
  const double theta = theta_for(d->precision);
  const double k = d->k;
  const int lr2 = 4 * d->lmax + 1, mr2 = 4 * d->mmax + 1;
  const double S = sqrt((double)lr2 * (double)mr2);
  const double twopi = 6.283185307179586476925286766559;
  // largest |kx|, |ky| over orders and families (family offsets < 2 pi/dx)
  const double k0 = d->k0_max > 0 ? d->k0_max : k;
  double kxm = twopi * (2 * d->lmax + 2) / d->dx + k0;
  double kym = twopi * (2 * d->mmax + 2) / d->dy + k0;
  int mm = 0;
  for (int n = 0; n < d->n_slices; ++n) {
    double er = d->eabs[n].re - 1.0, ei = d->eabs[n].im;
    double ae = sqrt(er * er + ei * ei);
    double lr = 0.5 * log(d->eabs[n].re * d->eabs[n].re + d->eabs[n].im * d->eabs[n].im);
    double li = atan2(d->eabs[n].im, d->eabs[n].re);
    double al = sqrt(lr * lr + li * li);
    double etam = twopi * 2.0 * (d->lmax > d->mmax ? d->lmax : d->mmax) /
                  (d->dx < d->dy ? d->dx : d->dy) * al;
    double bound = 1.4142135623730951 *
                   (k * k * (1.0 + ae * S) + etam * (kxm > kym ? kxm : kym) * S +
                    kxm * kxm + kym * kym);
    double v = bound * d->dabs[n] * d->dabs[n];
    int m = 0;
    while (v > theta && m < kMaxSteps) {
      v *= 0.25;
      ++m;
    }
    if (m > mm) mm = m;
  }
  return mm;
}

// Factors of the Euler product for (I - E)^-1, E = diag(kp/k) Sigma diag(kp/k).
// A finite section of the Toeplitz operator of 1/eps(x) has 2-norm at most
// sup |1/eps| = max(1, 1/|eps_abs|), so ||E||_2 <= (max|kp|/k)^2 max(1, 1/|eps|).
// Returns the F with ||E||^(2^F) <= 1e-7, or 0 (use LU) when the bound is weak.
static int euler_factors(const euv_amp_desc* d) {
  const double twopi = 6.283185307179586476925286766559;
  const double k0 = d->k0_max > 0 ? d->k0_max : d->k;
  const double kpx = k0 + twopi * (d->lmax + 1) / d->dx;
  const double kpy = k0 + twopi * (d->mmax + 1) / d->dy;
  const double kp = kpx > kpy ? kpx : kpy;
  double sup = 1.0;
  for (int n = 0; n < d->n_slices; ++n) {
    const double a = sqrt(d->eabs[n].re * d->eabs[n].re + d->eabs[n].im * d->eabs[n].im);
    if (1.0 / a > sup) sup = 1.0 / a;
  }
  const double e = (kp / d->k) * (kp / d->k) * sup;
  if (!(e < 0.5)) return 0;
  // The product serves the mixed form only, whose split-FP16x3 products carry ~1e-6
  // relative error each: a truncation ||E||^(2^F) <= 1e-7 stays below that.
  // the product of F factors is sum_{j < 2^F} E^j: truncation ||E||^(2^F)
  int f = 1;
  double v = e * e;  // ||E||^(2^f)
  while (v > 1e-7 && f < 8) {
    v = v * v;
    ++f;
  }
  return f;
}

struct AmpLayout {
  size_t bytes;
};

// All workspace carving in one place so the size query and the run agree.
struct AmpWork {
  double2 *D, *G, *P2, *P3, *P4, *T1, *C, *S, *X, *Y, *Z, *W, *Gp;
  double2 *x2, *y2, *gx2, *E, *YZ;
  double *klm, *norm, *h, *h2, *h4, *thick;
  int *steps, *ipiv, *info, *capped;
  void* mwork;
  size_t mbytes;
};

static bool carve(const euv_amp_desc* d, Bump& bp, AmpWork& w) {
  const long long N = d->n_orders, U = d->n_units, nn = N * N;
  w.D = bp.take<double2>(U * nn);
  w.G = bp.take<double2>(U * nn);
  w.P2 = bp.take<double2>(U * nn);
  w.P3 = bp.take<double2>(U * nn);
  w.P4 = bp.take<double2>(U * nn);
  w.T1 = bp.take<double2>(U * nn);
  w.C = bp.take<double2>(U * nn);
  w.S = bp.take<double2>(U * nn);
  w.X = bp.take<double2>(U * nn);
  w.Y = bp.take<double2>(U * nn);
  w.Z = bp.take<double2>(U * nn);
  w.W = bp.take<double2>(U * nn);
  w.Gp = d->refresh_sigma ? bp.take<double2>(U * nn) : nullptr;
  w.x2 = bp.take<double2>(U * N);
  w.y2 = bp.take<double2>(U * N);
  w.gx2 = bp.take<double2>(U * N);
  w.E = bp.take<double2>(U * N * (d->n_src > 0 ? d->n_src : 1));
  w.YZ = bp.take<double2>(U * N * (d->n_src > 0 ? d->n_src : 1));
  w.klm = bp.take<double>(U * N);
  w.norm = bp.take<double>(U);
  w.h = bp.take<double>(U);
  w.h2 = bp.take<double>(U);
  w.h4 = bp.take<double>(U);
  w.thick = bp.take<double>(U * (d->n_slices > 0 ? d->n_slices : 1));
  w.steps = bp.take<int>(U);
  w.ipiv = bp.take<int>(U * N);
  w.info = bp.take<int>(U);
  w.capped = bp.take<int>(1);
  // the mixed products are N x N x N, and N x n_src x N for the interface (n_src may exceed N)
  const int ncol = d->n_src > N ? d->n_src : (int)N;
  w.mbytes = d->precision == EUV_PREC_MIXED ? gemm_mixed_workspace_bytes((int)N, ncol, (int)N, (int)U) : 0;
  w.mwork = w.mbytes ? bp.take<char>(w.mbytes) : nullptr;
  return bp.ok;
}

static int check_desc(const euv_amp_desc* d) {
  if (!d) return 0;
  if (d->n_orders <= 0 || d->n_units <= 0 || d->lmax < 0 || d->mmax < 0 || d->n_slices <= 0 ||
      d->n_slices > EUV_MAX_SLICES || d->n_src < 0 || d->k <= 0 || d->dx <= 0 || d->dy <= 0 ||
      !d->d_lindex || !d->d_mindex || !d->d_kx0 || !d->d_ky0 || !d->d_polar || !d->d_spec ||
      (d->n_src > 0 && (!d->d_src_order || !d->d_src_2kz)) ||
      (d->precision != EUV_PREC_FP64 && d->precision != EUV_PREC_MIXED) || d->euler_f < -1 ||
      d->euler_f > 8)
    return 0;
  for (int n = 0; n < d->n_slices; ++n)
    if (!(d->dabs[n] >= 0.0) || (d->eabs[n].re == 0.0 && d->eabs[n].im == 0.0)) return 0;
  return 1;
}

}  // namespace euv

using namespace euv;

extern "C" int euv_amp_euler_factors(const euv_amp_desc* d) {
  if (!d || !check_desc(d)) {
    euv_set_error("euv_amp_euler_factors: invalid descriptor");
    return -2;
  }
  if (d->precision != EUV_PREC_MIXED) return 0;
  if (d->euler_f != 0) return d->euler_f;
  const int f = euler_factors(d);
  return f > 0 ? f : -1;
}

extern "C" size_t euv_amp_workspace_bytes(const euv_amp_desc* d) {
  if (!check_desc(d)) return 0;
  Bump bp{nullptr, (size_t)-1, 0, true};
  AmpWork w;
  carve(d, bp, w);
  return bp.off;
}

static cplx clog_host(euv_c64 e) {
  return mk(0.5 * log(e.re * e.re + e.im * e.im), atan2(e.im, e.re));
}

extern "C" int euv_amp(const euv_amp_desc* d, const euv_c64* d_spectra, euv_c64* d_ax,
                       void* d_work, size_t work_bytes, void* stream_) {
  if (!check_desc(d) || !d_spectra || !d_ax) {
    euv_set_error("euv_amp: invalid descriptor or null buffer");
    return EUV_ERR_BAD_ARG;
  }
  cudaStream_t stream = (cudaStream_t)stream_;
  Bump bp{reinterpret_cast<char*>(d_work), work_bytes, 0, true};
  AmpWork w;
  if (!d_work || !carve(d, bp, w)) {
    euv_set_error("euv_amp: workspace too small (%zu bytes given, %zu needed)", work_bytes,
                  euv_amp_workspace_bytes(d));
    return EUV_ERR_WORKSPACE;
  }
  const int N = d->n_orders, U = d->n_units, NS = d->n_slices;
  const long long nn = (long long)N * N;
  const int bs = 256;
  const dim3 ge(grid1(nn, bs), U);
  const dim3 gdg((unsigned)N, (unsigned)((N + bs - 1) / bs), U);  // build_dg: column, rows, unit
  const cplx one = mk(1.0, 0.0), zero = mk(0.0, 0.0), mi = mk(0.0, -1.0);
  int m_max = d->m_max > 0 ? d->m_max : derive_m_max(d);
  if (m_max > kMaxSteps) m_max = kMaxSteps;
  // device-detected conditions go to the caller's status word, else to a
  // workspace word nobody reads
  int* status = d->d_status ? d->d_status : w.capped;
  Gemm gemm{d->precision, w.mwork, w.mbytes, stream, status};
  int rc;

  if (!d->d_status) EUV_CUDA_TRY(cudaMemsetAsync(w.capped, 0, sizeof(int), stream));
  // per-slice thickness arrays [slice][unit]
  for (int n = 0; n < NS; ++n) {
    fill_f64_kernel<<<grid1(U, 256), 256, 0, stream>>>(w.thick + (size_t)n * U, U, d->dabs[n]);
    EUV_LAUNCH_CHECK();
  }

  SliceParams sp;
  sp.k = d->k;
  sp.dx = d->dx;
  sp.dy = d->dy;
  sp.dxs = d->d_dx;
  sp.dys = d->d_dy;
  sp.n = N;
  sp.lmax = d->lmax;
  sp.mmax = d->mmax;
  sp.lr2 = 4 * d->lmax + 1;
  sp.mr2 = 4 * d->mmax + 1;
  sp.n_slices = NS;
  auto slice_params = [&](int n) {
    SliceParams q = sp;
    q.slice = n;
    cplx e = fromc(d->eabs[n]);
    q.eps_m1 = e - mk(1.0, 0.0);
    q.sig_m1 = cdiv(mk(1.0, 0.0), e) - mk(1.0, 0.0);
    q.logeps = clog_host(d->eabs[n]);
    return q;
  };

  StackParams stp;
  stp.k = d->k;
  stp.emo = fromc(d->stack.eps_mo);
  stp.esi = fromc(d->stack.eps_si);
  stp.eru = fromc(d->stack.eps_ru);
  stp.emosi2 = fromc(d->stack.eps_mosi2);
  stp.erusi = fromc(d->stack.eps_rusi);
  stp.esio2 = fromc(d->stack.eps_sio2);
  stp.dmo = d->stack.d_mo;
  stp.dmosi = d->stack.d_mosi;
  stp.dsi = d->stack.d_si;
  stp.dsimo = d->stack.d_simo;
  stp.dsiru = d->stack.d_siru;
  stp.dru = d->stack.d_ru;
  stp.nml = d->stack.nml;
  stp.dx = d->dx;
  stp.dy = d->dy;
  stp.dxs = d->d_dx;
  stp.dys = d->d_dy;
  stp.n = N;
  multilayer_kernel<<<grid1((long long)N * U, 128), 128, 0, stream>>>(
      stp, d->d_lindex, d->d_mindex, d->d_kx0, d->d_ky0, d->d_polar, w.x2, w.y2, w.gx2, w.klm, U);
  EUV_LAUNCH_CHECK();

  const double2* spec = reinterpret_cast<const double2*>(d_spectra);
  MatfunBufs mb{w.P2, w.P3, w.P4, w.T1, w.W, w.norm, w.h, w.h2, w.h4, w.steps, status};
  // Mixed form: G^-1 by the Euler product (I - E)^-1 = prod_f (I + E^(2^f)),
  // f < euler_f, when the config bound on ||E||_2 makes it converge fast.
  const int euler_f = d->precision != EUV_PREC_MIXED ? 0
                      : d->euler_f > 0                ? d->euler_f
                      : d->euler_f < 0                ? 0
                                                      : euler_factors(d);
  // factors f = 1..euler_f-1 applied to the partial product held in Zbuf (the
  // f = 0 factor is applied by the caller); E^(2^f) ping-pongs between G and P2
  // g_split: the caller's last GEMM had G as its A operand
  auto euler_tail = [&](double2* Zbuf, bool g_split) -> int {
    double2* P = w.G;
    double2* Pn = w.P2;
    double2* Zc = Zbuf;
    double2* Zt = w.W;
    for (int f = 1; f < euler_f; ++f) {
      // P as A again: split by the previous factor's P Zc (or the caller's G Z)
      const int ru = (f > 1 || g_split) ? kReuseA : 0;
      int r2 = gemm(N, N, N, one, nullptr, P, N, nn, P, N, nn, zero, Pn, N, nn, zero, U, nullptr, 0,
                    ru);
      if (r2) return r2;
      double2* t = P;
      P = Pn;
      Pn = t;
      // Zt = P Zc + Zc (the beta term read from Zc)
      r2 = gemm(N, N, N, one, nullptr, P, N, nn, Zc, N, nn, one, Zt, N, nn, zero, U, nullptr, 0, 0,
                Zc);
      if (r2) return r2;
      t = Zc;
      Zc = Zt;
      Zt = t;
    }
    if (Zc != Zbuf)
      EUV_CUDA_TRY(cudaMemcpyAsync(Zbuf, Zc, (size_t)U * nn * sizeof(double2), cudaMemcpyDeviceToDevice, stream));
    return EUV_OK;
  };
  double2* X = w.X;
  double2* Y = w.Y;
  for (int n = NS - 1; n >= 0; --n) {
    SliceParams q = slice_params(n);
    const bool bottom = (n == NS - 1);
    const bool need_g = bottom || d->refresh_sigma;
    // bottom slice sigma is used for every slice unless refresh_sigma (header.h:1327-1353)
    build_dg_kernel<<<gdg, bs, 0, stream>>>(q, spec, d->d_spec, d->d_lindex, d->d_mindex, d->d_kx0,
                                           d->d_ky0, d->d_polar, w.D, w.G, 1,
                                           need_g ? (euler_f > 0 ? 2 : 1) : 0);
    EUV_LAUNCH_CHECK();
    double2* Zp = X;
    if (bottom && euler_f > 0) {
      // mixed form: Z = G^-1 diag(gx2) = (1/ik) (I - E)^-1 diag(gx2) by the Euler
      // product on the tensor cores (E was built in place of G)
      euler_first_diag_kernel<<<ge, bs, 0, stream>>>(N, cdiv(one, mk(0.0, d->k)), w.G, w.gx2, w.Z);
      EUV_LAUNCH_CHECK();
      if ((rc = euler_tail(w.Z, false))) return rc;
      Zp = w.Z;
    } else if (bottom) {
      // Z = G^-1 diag(Bru (URUU+URUB))
      diag_kernel<<<ge, bs, 0, stream>>>(N, w.gx2, w.Z);
      EUV_LAUNCH_CHECK();
      if ((rc = lu_factor(N, w.G, N, nn, w.ipiv, w.info, U, stream))) return rc;
      flag_singular_kernel<<<grid1(U, 256), 256, 0, stream>>>(w.info, U, status);
      EUV_LAUNCH_CHECK();
      if ((rc = lu_solve(N, N, w.G, N, nn, w.ipiv, w.Z, N, nn, U, stream))) return rc;
      Zp = w.Z;
    } else if (d->refresh_sigma && euler_f > 0) {
      // Z = (I - E_n)^-1 (I - E_{n+1}) X  (= G_n^-1 G_{n+1} X)
      SliceParams qp = slice_params(n + 1);
      build_dg_kernel<<<gdg, bs, 0, stream>>>(qp, spec, d->d_spec, d->d_lindex, d->d_mindex,
                                             d->d_kx0, d->d_ky0, d->d_polar, nullptr, w.Gp, 0, 2);
      EUV_LAUNCH_CHECK();
      if ((rc = gemm(N, N, N, mk(-1.0, 0.0), nullptr, w.Gp, N, nn, X, N, nn, one, w.Z, N, nn, zero,
                     U, nullptr, 0, 0, X))) return rc;  // Z = X - Gp X
      if ((rc = gemm(N, N, N, one, nullptr, w.G, N, nn, w.Z, N, nn, one, w.W, N, nn, zero, U,
                     nullptr, 0, 0, w.Z))) return rc;  // W = Z + G Z
      EUV_CUDA_TRY(cudaMemcpyAsync(w.Z, w.W, (size_t)U * nn * sizeof(double2), cudaMemcpyDeviceToDevice, stream));
      if ((rc = euler_tail(w.Z, true))) return rc;
      Zp = w.Z;
    } else if (d->refresh_sigma) {
      // Z = G_n^-1 G_{n+1} X
      SliceParams qp = slice_params(n + 1);
      build_dg_kernel<<<gdg, bs, 0, stream>>>(qp, spec, d->d_spec, d->d_lindex, d->d_mindex,
                                             d->d_kx0, d->d_ky0, d->d_polar, nullptr, w.Gp, 0, 1);
      EUV_LAUNCH_CHECK();
      if ((rc = gemm(N, N, N, one, nullptr, w.Gp, N, nn, X, N, nn, zero, w.Z, N, nn, zero, U))) return rc;
      if ((rc = lu_factor(N, w.G, N, nn, w.ipiv, w.info, U, stream))) return rc;
      flag_singular_kernel<<<grid1(U, 256), 256, 0, stream>>>(w.info, U, status);
      EUV_LAUNCH_CHECK();
      if ((rc = lu_solve(N, N, w.G, N, nn, w.ipiv, w.Z, N, nn, U, stream))) return rc;
      Zp = w.Z;
    }
    double2* C = w.C;
    double2* S = w.S;
    if ((rc = matfun(N, U, w.D, w.thick + (size_t)n * U, &C, &S, mb, m_max, gemm, stream))) return rc;
    // buffers free after matfun: P2, P3, P4, T1, W minus the two now holding C/S
    double2* pool[7] = {w.P2, w.P3, w.P4, w.T1, w.W, w.C, w.S};
    double2* fr[5];
    int nf = 0;
    for (int i = 0; i < 7; ++i)
      if (pool[i] != C && pool[i] != S && pool[i] != Zp) fr[nf++] = pool[i];
    double2* Wb = fr[0];
    double2* Xn = fr[1];
    double2* Yn = fr[2];
    // W = S Z ; Xn = C Z - i S Y ; Yn = -i D W + C Y, ordered so that three of
    // the five products find one operand already split
    if ((rc = gemm(N, N, N, one, nullptr, S, N, nn, Zp, N, nn, zero, Wb, N, nn, zero, U))) return rc;
    if ((rc = gemm(N, N, N, one, nullptr, C, N, nn, Zp, N, nn, zero, Xn, N, nn, zero, U, nullptr, 0,
                   kReuseB))) return rc;  // Zp as B again
    if (bottom) {
      if ((rc = gemm(N, N, N, mi, nullptr, w.D, N, nn, Wb, N, nn, zero, Yn, N, nn, zero, U))) return rc;
      colscale_kernel<<<ge, bs, 0, stream>>>(N, mi, S, w.y2, one, Xn);
      EUV_LAUNCH_CHECK();
      colscale_kernel<<<ge, bs, 0, stream>>>(N, one, C, w.y2, one, Yn);
      EUV_LAUNCH_CHECK();
    } else {
      if ((rc = gemm(N, N, N, one, nullptr, C, N, nn, Y, N, nn, zero, Yn, N, nn, zero, U, nullptr,
                     0, kReuseA))) return rc;  // C as A again
      if ((rc = gemm(N, N, N, mi, nullptr, S, N, nn, Y, N, nn, one, Xn, N, nn, zero, U, nullptr, 0,
                     kReuseB))) return rc;  // Y as B again
      if ((rc = gemm(N, N, N, mi, nullptr, w.D, N, nn, Wb, N, nn, one, Yn, N, nn, zero, U))) return rc;
    }
    if (n == 0) {
      // top slice: the interface below reads Xn, Yn where they are (nothing
      // after the loop writes the matrix-function buffers)
      X = Xn;
      Y = Yn;
      break;
    }
    // move the new X, Y into the dedicated buffers for the next slice's matfun
    EUV_CUDA_TRY(cudaMemcpyAsync(w.X, Xn, (size_t)U * nn * sizeof(double2),
                                 cudaMemcpyDeviceToDevice, stream));
    EUV_CUDA_TRY(cudaMemcpyAsync(w.Y, Yn, (size_t)U * nn * sizeof(double2),
                                 cudaMemcpyDeviceToDevice, stream));
    X = w.X;
    Y = w.Y;
  }
  // top interface: U0 = klm X + Y, Z = U0^-1 E, Ax = -(1/klm) Y Z + e
  u0_kernel<<<ge, bs, 0, stream>>>(N, w.klm, X, Y, w.G);
  EUV_LAUNCH_CHECK();
  if ((rc = lu_factor(N, w.G, N, nn, w.ipiv, w.info, U, stream))) return rc;
  flag_singular_kernel<<<grid1(U, 256), 256, 0, stream>>>(w.info, U, status);
  EUV_LAUNCH_CHECK();
  const int ns = d->n_src;
  if (ns > 0) {
    dim3 gs(grid1((long long)N * ns, bs), U);
    src_rhs_kernel<<<gs, bs, 0, stream>>>(N, ns, d->d_src_order, d->d_src_2kz, w.E);
    EUV_LAUNCH_CHECK();
    // empty source slots (order < 0, zero columns of E) skip their CTAs
    if ((rc = lu_solve(N, ns, w.G, N, nn, w.ipiv, w.E, N, (long long)N * ns, U, stream,
                       d->d_src_order, ns)))
      return rc;
    // Y Z for the source columns: a product, so the mixed form takes it on the
    // tensor cores (split-FP16x3, ~1e-6 relative) like the matrix functions; the
    // solve above stays FP64
    if ((rc = gemm(N, ns, N, one, nullptr, Y, N, nn, w.E, N, (long long)N * ns, zero, w.YZ, N,
                   (long long)N * ns, zero, U)))
      return rc;
    ax_out_kernel<<<gs, bs, 0, stream>>>(N, ns, d->d_src_order, w.klm, w.YZ,
                                         reinterpret_cast<double2*>(d_ax));
    EUV_LAUNCH_CHECK();
  }
  return EUV_OK;
}

// ------------------------------------------------------------------ spectrum
extern "C" size_t euv_mask_spectrum_workspace_bytes(int n_masks, int ndivx, int ndivy, int fdivx,
                                                    int fdivy, int lh, int mh) {
  (void)ndivx;
  (void)ndivy;
  const size_t lr = 2 * (size_t)lh + 1, mr = 2 * (size_t)mh + 1;
  Bump bp{nullptr, (size_t)-1, 0, true};
  bp.take<double2>((size_t)fdivy * mr);
  bp.take<double2>(lr * (size_t)fdivx);
  const size_t nm = n_masks > 1 ? n_masks : 1;
  bp.take<double2>(nm * mr * fdivx);
  bp.take<double2>(nm * (size_t)spectrum_parts(fdivx) * lr * mr);
  bp.take<char>(256);  // the run's alignment slack between the two arrays
  return bp.off;
}

// Masks are transformed in groups that fit the workspace (all of them when it
// was sized by euv_mask_spectrum_workspace_bytes for n_masks): two launches per
// group after the two twiddle tables.
extern "C" int euv_mask_spectrum(const uint8_t* d_bits, int n_masks, int ndivx, int ndivy,
                                 int fdivx, int fdivy, int lh, int mh, int select_vacuum,
                                 int y_offset, euv_c64* d_out, void* d_work, size_t work_bytes, void* stream_) {
  if (!d_bits || !d_out || n_masks < 0 || ndivx <= 0 || ndivy <= 0 || fdivx <= 0 || fdivy <= 0 ||
      fdivx % ndivx || fdivy % ndivy || lh < 0 || mh < 0 || 2 * lh + 1 > fdivx ||
      2 * mh + 1 > fdivy || ((long long)ndivx * ndivy) % 8) {
    euv_set_error("euv_mask_spectrum: bad arguments");
    return EUV_ERR_BAD_ARG;
  }
  cudaStream_t stream = (cudaStream_t)stream_;
  const int lr = 2 * lh + 1, mr = 2 * mh + 1;
  Bump bp{reinterpret_cast<char*>(d_work), work_bytes, 0, true};
  double2* Wy = bp.take<double2>((size_t)fdivy * mr);
  double2* Wx = bp.take<double2>((size_t)lr * fdivx);
  const int parts = spectrum_parts(fdivx);
  const size_t t_bytes = (size_t)mr * fdivx * sizeof(double2);
  const size_t p_bytes = (size_t)parts * lr * mr * sizeof(double2);
  const size_t left = bp.ok && work_bytes > bp.off + 256 ? work_bytes - bp.off - 256 : 0;
  long long group = (long long)(left / (t_bytes + p_bytes));
  if (group > 65535) group = 65535;  // grid z / y limit
  if (!d_work || !bp.ok || group < 1) {
    euv_set_error("euv_mask_spectrum: workspace too small");
    return EUV_ERR_WORKSPACE;
  }
  double2* T = reinterpret_cast<double2*>(reinterpret_cast<char*>(d_work) + bp.off);
  // Wy[y + FY m'] = exp(-2 pi i m y / FY) ; Wx[l' + LR x] = exp(-2 pi i l x/FX)/(FX FY)
  twiddle_kernel<<<grid1((long long)fdivy * mr, 256), 256, 0, stream>>>(fdivy, mr, 0, mh, fdivy, 0,
                                                                        1.0, Wy);
  EUV_LAUNCH_CHECK();
  twiddle_kernel<<<grid1((long long)lr * fdivx, 256), 256, 0, stream>>>(
      lr, fdivx, lh, 0, fdivx, 1, 1.0 / ((double)fdivx * (double)fdivy), Wx);
  EUV_LAUNCH_CHECK();
  const long long mask_bytes = (long long)ndivx * ndivy / 8;
  for (long long g0 = 0; g0 < n_masks; g0 += group) {
    const int ng = (int)(n_masks - g0 < group ? n_masks - g0 : group);
    dim3 g1((fdivx + SP_X - 1) / SP_X, (mr + SP_M - 1) / SP_M, ng);
    spectrum_rows_kernel<<<g1, 256, 0, stream>>>(d_bits + g0 * mask_bytes, mask_bytes, ndivx,
                                                  ndivy, fdivx, fdivy, mr, select_vacuum,
                                                  y_offset, Wy, T);
    EUV_LAUNCH_CHECK();
    double2* out = reinterpret_cast<double2*>(d_out) + g0 * lr * mr;
    if (parts > 0) {
      // out (lr x ng mr) = Wx (lr x FX) T^T (FX x ng mr), K split in `parts` chunks
      const int kc = fdivx / parts;
      const long long cols = (long long)ng * mr;
      double2* P = reinterpret_cast<double2*>(
          reinterpret_cast<char*>(T) + ((ng * t_bytes + 255) & ~(size_t)255));
      int rc = zgemm(lr, (int)cols, kc, mk(1.0, 0.0), nullptr, Wx, lr, (long long)kc * lr, T,
                     fdivx, kc, mk(0.0, 0.0), P, lr, (long long)lr * cols, mk(0.0, 0.0), parts,
                     nullptr, 0, stream);
      if (rc) return rc;
      const long long total = (long long)lr * cols;
      spectrum_reduce_kernel<<<grid1(total, 256), 256, 0, stream>>>(P, parts, total, out);
    } else {
      spectrum_cols_kernel<<<dim3(mr, ng), SC_THREADS, 0, stream>>>(fdivx, lr, mr, Wx, T, out);
    }
    EUV_LAUNCH_CHECK();
  }
  return EUV_OK;
}

// ------------------------------------------------------------------ matfun
extern "C" size_t euv_matfun_workspace_bytes(int n, int batch) {
  Bump bp{nullptr, (size_t)-1, 0, true};
  const long long nn = (long long)n * n;
  for (int i = 0; i < 5; ++i) bp.take<double2>(nn * batch);
  for (int i = 0; i < 4; ++i) bp.take<double>(batch);
  bp.take<int>(batch);
  bp.take<int>(1);
  bp.take<char>(gemm_mixed_workspace_bytes(n, n, n, batch));
  return bp.off;
}

extern "C" int euv_matfun_cs(int n, const euv_c64* d_d, const double* d_thick, euv_c64* d_cos,
                             euv_c64* d_sin, int batch, int m_max, int precision, void* d_work,
                             size_t work_bytes, void* stream_) {
  if (n <= 0 || batch <= 0 || !d_d || !d_thick || !d_cos || !d_sin || m_max < 0 ||
      m_max > kMaxSteps || (precision != EUV_PREC_FP64 && precision != EUV_PREC_MIXED)) {
    euv_set_error("euv_matfun_cs: bad arguments");
    return EUV_ERR_BAD_ARG;
  }
  cudaStream_t stream = (cudaStream_t)stream_;
  const long long nn = (long long)n * n;
  Bump bp{reinterpret_cast<char*>(d_work), work_bytes, 0, true};
  MatfunBufs mb;
  mb.P2 = bp.take<double2>(nn * batch);
  mb.P3 = bp.take<double2>(nn * batch);
  mb.P4 = bp.take<double2>(nn * batch);
  mb.T1 = bp.take<double2>(nn * batch);
  mb.T2 = bp.take<double2>(nn * batch);
  mb.norm = bp.take<double>(batch);
  mb.h = bp.take<double>(batch);
  mb.h2 = bp.take<double>(batch);
  mb.h4 = bp.take<double>(batch);
  mb.steps = bp.take<int>(batch);
  mb.capped = bp.take<int>(1);
  size_t mbytes = gemm_mixed_workspace_bytes(n, n, n, batch);
  void* mw = bp.take<char>(mbytes);
  if (!d_work || !bp.ok) {
    euv_set_error("euv_matfun_cs: workspace too small");
    return EUV_ERR_WORKSPACE;
  }
  Gemm gemm{precision, mw, mbytes, stream};
  double2* C = reinterpret_cast<double2*>(d_cos);
  double2* S = reinterpret_cast<double2*>(d_sin);
  double2* C0 = C;
  double2* S0 = S;
  int rc = matfun(n, batch, reinterpret_cast<const double2*>(d_d), d_thick, &C, &S, mb, m_max,
                  gemm, stream);
  if (rc) return rc;
  if (C != C0) EUV_CUDA_TRY(cudaMemcpyAsync(C0, C, nn * batch * sizeof(double2), cudaMemcpyDeviceToDevice, stream));
  if (S != S0) EUV_CUDA_TRY(cudaMemcpyAsync(S0, S, nn * batch * sizeof(double2), cudaMemcpyDeviceToDevice, stream));
  return EUV_OK;
}

// ------------------------------------------------------------------ matfun, no allocation
// Scratch of euv_matfun_cs_noalloc: a fixed device array in this library, so the
// entry point needs no workspace from the caller and allocates nothing.  It is
// EUV_NOALLOC_SCRATCH_BYTES on every GPU that loads the library, for the life of
// the process.  Every call uses the same array.
static __device__ __align__(256) unsigned char g_matfun_scratch[EUV_NOALLOC_SCRATCH_BYTES];

namespace {
// Device address of g_matfun_scratch per device, looked up on the first call
// made with that device current (cudaGetSymbolAddress is a host-side query).
void* g_scratch_ptr[64];
int g_scratch_ready[64];

int scratch_for_current_device(void** out) {
  int dev = 0;
  EUV_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    euv_set_error("euv_matfun_cs_noalloc: device ordinal %d out of range", dev);
    return EUV_ERR_BAD_ARG;
  }
  if (!__atomic_load_n(&g_scratch_ready[dev], __ATOMIC_ACQUIRE)) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_matfun_scratch);
    if (e != cudaSuccess || p == nullptr) {
      euv_set_error("euv_matfun_cs_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
                    cudaGetErrorString(e));
      return EUV_ERR_CUDA;
    }
    g_scratch_ptr[dev] = p;
    __atomic_store_n(&g_scratch_ready[dev], 1, __ATOMIC_RELEASE);
  }
  *out = g_scratch_ptr[dev];
  return EUV_OK;
}
}  // namespace

extern "C" int euv_matfun_cs_noalloc(int n, const euv_c64* d_d, const double* d_thick,
                                     euv_c64* d_cos, euv_c64* d_sin, int batch, int m_max,
                                     void* stream_) {
  if (n <= 0 || batch <= 0 || !d_d || !d_thick || !d_cos || !d_sin || m_max < 0 ||
      m_max > kMaxSteps) {
    euv_set_error("euv_matfun_cs_noalloc: bad arguments");
    return EUV_ERR_BAD_ARG;
  }
  size_t need;
  {
    Bump dry{nullptr, (size_t)-1, 0, true};
    const long long nn0 = (long long)n * n;
    for (int i = 0; i < 5; ++i) dry.take<double2>(nn0 * batch);
    for (int i = 0; i < 4; ++i) dry.take<double>(batch);
    dry.take<int>(batch);
    dry.take<int>(1);
    need = dry.off;
  }
  if (need > (size_t)EUV_NOALLOC_SCRATCH_BYTES) {
    euv_set_error("euv_matfun_cs_noalloc: n=%d batch=%d needs %zu bytes of scratch, above the "
                  "fixed %zu bytes (use euv_matfun_cs with a caller workspace)",
                  n, batch, need, (size_t)EUV_NOALLOC_SCRATCH_BYTES);
    return EUV_ERR_BAD_ARG;
  }
  void* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  cudaStream_t stream = (cudaStream_t)stream_;
  const long long nn = (long long)n * n;
  Bump bp{reinterpret_cast<char*>(scratch), (size_t)EUV_NOALLOC_SCRATCH_BYTES, 0, true};
  MatfunBufs mb;
  mb.P2 = bp.take<double2>(nn * batch);
  mb.P3 = bp.take<double2>(nn * batch);
  mb.P4 = bp.take<double2>(nn * batch);
  mb.T1 = bp.take<double2>(nn * batch);
  mb.T2 = bp.take<double2>(nn * batch);
  mb.norm = bp.take<double>(batch);
  mb.h = bp.take<double>(batch);
  mb.h2 = bp.take<double>(batch);
  mb.h4 = bp.take<double>(batch);
  mb.steps = bp.take<int>(batch);
  mb.capped = bp.take<int>(1);
  if (!bp.ok) {
    euv_set_error("euv_matfun_cs_noalloc: scratch layout overflow");
    return EUV_ERR_BAD_ARG;
  }
  // The array keeps the previous call's contents: the only state that must
  // start at zero is the cap flag (the column-norm maxima are cleared by matfun).
  EUV_CUDA_TRY(cudaMemsetAsync(mb.capped, 0, sizeof(int), stream));
  Gemm gemm{EUV_PREC_FP64, nullptr, 0, stream};
  double2* C = reinterpret_cast<double2*>(d_cos);
  double2* S = reinterpret_cast<double2*>(d_sin);
  double2* C0 = C;
  double2* S0 = S;
  rc = matfun(n, batch, reinterpret_cast<const double2*>(d_d), d_thick, &C, &S, mb, m_max, gemm,
              stream);
  if (rc) return rc;
  if (C != C0)
    EUV_CUDA_TRY(cudaMemcpyAsync(C0, C, nn * batch * sizeof(double2), cudaMemcpyDeviceToDevice, stream));
  if (S != S0)
    EUV_CUDA_TRY(cudaMemcpyAsync(S0, S, nn * batch * sizeof(double2), cudaMemcpyDeviceToDevice, stream));
  return EUV_OK;
}
