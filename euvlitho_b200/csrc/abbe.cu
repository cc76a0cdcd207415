// Fused Abbe imaging (replaces intensity.cpp:248-408).
//
// The reference, per source point: builds the E field of every pupil order on
// the host (rotate(), pupil phase, defocus), scatters it into three XDIV^2
// grids, copies each to the GPU, runs a cuFFT Z2Z inverse, copies back and
// accumulates |Ex|^2+|Ey|^2+|Ez|^2.  Here one kernel does all of it on chip:
// a CTA owns a stripe of AB_YS image rows (all x) of one unit and loops over
// that unit's sources:
//   1. E_c(i) = coef_c(s,i) * Ax(s, nidx(s,i)) for the pupil points (smem);
//   2. separable inverse DFT, stage y: G_c(l,y) = sum_m E_c(l,m) e^{2 pi i m y/YDIV}
//      for the stripe (pupil points are stored l-major, so row l is a range);
//   3. stage x: f_c(x,y) = sum_l G_c(l,y) e^{2 pi i l x/XDIV}, with the twiddle
//      advanced by a recurrence from an exact start, and |f|^2 accumulated in
//      registers.
// Only the DFT of the non-zero pupil box is evaluated (the reference FFTs the
// whole zero-padded grid).  Partial images are added with FP64 atomics.
#include "common.cuh"

namespace euv {

// complex arithmetic in the kernel's type R (double: FP64 form; float: the
// mixed form, whose DFT sums need ~1e-6, not 1e-16)
template <typename R>
struct cx {
  R x, y;
};
template <typename R>
__device__ __forceinline__ cx<R> operator+(cx<R> a, cx<R> b);
template <typename R>
__device__ __forceinline__ cx<R> operator*(cx<R> a, cx<R> b);
template <typename R>
__device__ __forceinline__ cx<R> operator+(cx<R> a, cx<R> b) { return {a.x + b.x, a.y + b.y}; }
template <typename R>
__device__ __forceinline__ cx<R> operator*(cx<R> a, cx<R> b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename R>
struct vec2;
template <>
struct vec2<double> {
  using type = double2;
};
template <>
struct vec2<float> {
  using type = float2;
};

constexpr int AB_YS = 4;

constexpr int AB_THREADS = 256;

// f[b][c] += G[lx][b][c] w for the AB_YS x 3 values of G at one lx (16 B
// aligned): FP32 reads them as float4 pairs, FP64 one double2 at a time
__device__ __forceinline__ void stage_x_lx(const float2* gp, cx<float> (&f)[AB_YS][3],
                                           cx<float> w) {
  const float4* q = reinterpret_cast<const float4*>(gp);
#pragma unroll
  for (int k = 0; k < AB_YS * 3 / 2; ++k) {
    const float4 v = q[k];
    const int e0 = 2 * k, e1 = 2 * k + 1;
    f[e0 / 3][e0 % 3] = f[e0 / 3][e0 % 3] + cx<float>{v.x, v.y} * w;
    f[e1 / 3][e1 % 3] = f[e1 / 3][e1 % 3] + cx<float>{v.z, v.w} * w;
  }
}
__device__ __forceinline__ void stage_x_lx(const double2* gp, cx<double> (&f)[AB_YS][3],
                                           cx<double> w) {
#pragma unroll
  for (int e = 0; e < AB_YS * 3; ++e) {
    const double2 v = gp[e];
    f[e / 3][e % 3] = f[e / 3][e % 3] + cx<double>{v.x, v.y} * w;
  }
}
constexpr int AB_XPT = 4;  // x values (groups of four, radix-4) per thread: xdiv <= 1024
constexpr int AB_GP = 4;   // radix-4 layout: zero rows of G before and after the pupil box
static_assert(AB_YS == 4, "accumulators are [AB_XPT][4]");

// the three components G[lx][b][0..2] of one row of the radix-4 layout (four
// slots per (lx, b), 32 B aligned for FP32)
__device__ __forceinline__ void load_g3(const float2* gp, cx<float> (&g)[3]) {
  const float4 v0 = reinterpret_cast<const float4*>(gp)[0];
  const float2 v1 = gp[2];
  g[0] = {v0.x, v0.y};
  g[1] = {v0.z, v0.w};
  g[2] = {v1.x, v1.y};
}
__device__ __forceinline__ void load_g3(const double2* gp, cx<double> (&g)[3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) g[c] = {gp[c].x, gp[c].y};
}

struct AbbeParams {
  int xdiv, ydiv, lpx, lpy, bx, by, ncut, n_src, n_order, nsplit;
  const double2* coef;
  const int* nidx;
  const int* py;
  const int* row_start;
  const int* tab_of_unit;
  const int* img_of_unit;
  const int* nsrc_of_unit;
  const double* inv_weight;
};

// R4 (xdiv and ydiv divisible by 4): both DFT stages as four-way splits.
//   x stage: with t = lx - lpx, f(g + q X/4) = sum_s i^(q s) P_s(g), P_s(g) =
//     sum over t = s (mod 4) of G(lx) e^(2 pi i t g / X): one pass over the
//     pupil box gives four image columns, combined by a radix-4 butterfly.  G
//     has AB_GP zero rows on both sides and four slots per (lx, row), so the
//     pass starts at an lx with t = 0 (mod 4) and needs no bounds test.
//   y stage: the CTA's four rows are y0 + q Y/4 (not four adjacent rows), so
//     with u = E(l, m) e^(2 pi i m y0 / Y) every pupil point adds i^(m q) u to
//     row q: one product per point for the four rows.
template <typename R, bool R4>
__global__ void __launch_bounds__(AB_THREADS) abbe_kernel(AbbeParams p, const double2* ax,
                                                          double* image) {
  using V2 = typename vec2<R>::type;
  using C = cx<R>;
  constexpr int GC = R4 ? 4 : 3;       // slots per (lx, row)
  constexpr int GP = R4 ? AB_GP : 0;   // zero rows before the pupil box
  extern __shared__ __align__(16) unsigned char sm_raw[];
  V2* E = reinterpret_cast<V2*>(sm_raw);              // [ncut][3]
  V2* G = E + (((size_t)p.ncut * 3 + 1) & ~(size_t)1);  // [GP + bx + GP][YS][GC], 16 B aligned
  const int g_rows = p.bx + 2 * GP;
  V2* twy = G + (size_t)g_rows * AB_YS * GC;          // [YS][by]
  int* s_py = reinterpret_cast<int*>(twy + (size_t)AB_YS * p.by);  // [ncut] pupil m + lpy
  const int u = blockIdx.z;
  const int y0 = R4 ? blockIdx.x : blockIdx.x * AB_YS;
  const int ystep = R4 ? p.ydiv / 4 : 1;  // distance between the CTA's image rows
  const int tid = threadIdx.x;
  const int nsrc_u = p.nsrc_of_unit[u];
  const int img = p.img_of_unit[u];
  const int ny = R4 ? AB_YS : ((p.ydiv - y0) < AB_YS ? (p.ydiv - y0) : AB_YS);

  // twiddles of stage y: rows y0 + yy (R4: the one row y0)
  for (int idx = tid; idx < (R4 ? 1 : AB_YS) * p.by; idx += AB_THREADS) {
    int yy = idx / p.by, mm = idx % p.by;
    long long q = ((long long)(mm - p.lpy) * (y0 + yy)) % p.ydiv;
    if (q < 0) q += p.ydiv;
    double s, c;
    sincospi(2.0 * (double)q / (double)p.ydiv, &s, &c);
    twy[idx] = V2{(R)c, (R)s};
  }
  for (int i = tid; i < p.ncut; i += AB_THREADS) s_py[i] = p.py[i] + p.lpy;
  if (R4)  // the pad rows and slots stay zero; stage y writes the rest
    for (int i = tid; i < g_rows * AB_YS * GC; i += AB_THREADS) G[i] = V2{(R)0, (R)0};

  double acc[AB_XPT][4];
#pragma unroll
  for (int a = 0; a < AB_XPT; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;

  for (int s = blockIdx.y; s < nsrc_u; s += p.nsplit) {
    __syncthreads();
    const long long base = ((long long)p.tab_of_unit[u] * p.n_src + s);
    const double2* axs = ax + ((long long)u * p.n_src + s) * p.n_order;
    for (int i = tid; i < p.ncut; i += AB_THREADS) {
      const int n = p.nidx[base * p.ncut + i];
      cplx e0 = mk(0, 0), e1 = mk(0, 0), e2 = mk(0, 0);
      if (n >= 0) {
        double2 a2 = axs[n];
        cplx a = mk(a2.x, a2.y);
        const double2* cf = p.coef + (base * p.ncut + i) * 3;
        e0 = mk(cf[0].x, cf[0].y) * a;
        e1 = mk(cf[1].x, cf[1].y) * a;
        e2 = mk(cf[2].x, cf[2].y) * a;
      }
      E[i * 3 + 0] = V2{(R)e0.x, (R)e0.y};
      E[i * 3 + 1] = V2{(R)e1.x, (R)e1.y};
      E[i * 3 + 2] = V2{(R)e2.x, (R)e2.y};
    }
    __syncthreads();
    // stage y; G[GP + lx][yy][c]: the values stage x reads per lx are contiguous
    if (R4) {
      const int kofs = 4 - (p.lpy & 3);  // (mm + kofs) & 3 = (mm - lpy) mod 4 = m mod 4
      // two lanes per (lx, c): alternate points, summed by a shuffle
      const int nitem2 = 2 * p.bx * 3;
      for (int base = 0; base < nitem2; base += AB_THREADS) {  // uniform trip count
        const int o = base + tid;
        const bool live = o < nitem2;
        const int item = o >> 1, c = item % 3, lx = item / 3;
        C g[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) g[q] = C{(R)0, (R)0};
        const int i0 = live ? p.row_start[lx] + (o & 1) : 0, i1 = live ? p.row_start[lx + 1] : 0;
        for (int i = i0; i < i1; i += 2) {
          const V2 e = E[i * 3 + c];
          const int mm = s_py[i];
          const V2 t = twy[mm];
          const C w = C{e.x, e.y} * C{t.x, t.y};
          const int k = (mm + kofs) & 3;
          // i^k w = sg (i^(k&1) w); (-1)^k w; (-i)^k w = (-1)^k sg (i^(k&1) w)
          const C v = (k & 1) ? C{-w.y, w.x} : w;
          const R sg = (k & 2) ? (R)-1 : (R)1;
          const R sodd = (k & 1) ? (R)-1 : (R)1;
          g[0] = C{g[0].x + w.x, g[0].y + w.y};
          g[1] = C{g[1].x + sg * v.x, g[1].y + sg * v.y};
          g[2] = C{g[2].x + sodd * w.x, g[2].y + sodd * w.y};
          g[3] = C{g[3].x + sodd * sg * v.x, g[3].y + sodd * sg * v.y};
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          g[q].x += __shfl_xor_sync(0xffffffffu, g[q].x, 1);
          g[q].y += __shfl_xor_sync(0xffffffffu, g[q].y, 1);
        }
        if (live && (o & 1) == 0)
#pragma unroll
          for (int q = 0; q < 4; ++q) G[((GP + lx) * AB_YS + q) * GC + c] = V2{g[q].x, g[q].y};
      }
    } else
    for (int o = tid; o < AB_YS * p.bx * 3; o += AB_THREADS) {
      const int c = o % 3, lx = (o / 3) % p.bx, yy = o / (3 * p.bx);
      C g{(R)0, (R)0};
      const int i0 = p.row_start[lx], i1 = p.row_start[lx + 1];
      const V2* ty = twy + yy * p.by;
      for (int i = i0; i < i1; ++i) {
        const V2 e = E[i * 3 + c];
        const V2 t = ty[s_py[i]];
        g = g + C{e.x, e.y} * C{t.x, t.y};
      }
      G[((GP + lx) * AB_YS + yy) * GC + c] = V2{g.x, g.y};
    }
    __syncthreads();
    if (R4) {
      // stage x, radix 4: thread = (column group g, stripe row b)
      const int b = tid & (AB_YS - 1), g0 = tid / AB_YS;
      const int x4 = p.xdiv / 4;
      const int lx0 = (p.lpx & 3) - 4;  // lx0 - lpx = 0 (mod 4); rows lx0 .. -1 are pad
      const int nj = (p.bx - lx0 + 3) / 4;
#pragma unroll
      for (int a = 0; a < AB_XPT; ++a) {
        const int g = g0 + a * (AB_THREADS / AB_YS);
        if (g < x4) {
          long long q0 = ((long long)(lx0 - p.lpx) * g) % p.xdiv;
          if (q0 < 0) q0 += p.xdiv;
          double s0, c0, s1, c1;
          sincospi(2.0 * (double)q0 / (double)p.xdiv, &s0, &c0);
          sincospi(2.0 * (double)g / (double)p.xdiv, &s1, &c1);
          C w{(R)c0, (R)s0};
          const C r{(R)c1, (R)s1};
          C P[4][3];
#pragma unroll
          for (int k = 0; k < 4; ++k) P[k][0] = P[k][1] = P[k][2] = C{(R)0, (R)0};
          const V2* gp = G + ((size_t)(GP + lx0) * AB_YS + b) * GC;
          for (int j = 0; j < nj; ++j) {
#pragma unroll
            for (int k = 0; k < 4; ++k, gp += AB_YS * GC) {
              C gv[3];
              load_g3(gp, gv);
#pragma unroll
              for (int c = 0; c < 3; ++c) P[k][c] = P[k][c] + gv[c] * w;
              w = w * r;
            }
          }
          double e[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const C A{P[0][c].x + P[2][c].x, P[0][c].y + P[2][c].y};
            const C B{P[0][c].x - P[2][c].x, P[0][c].y - P[2][c].y};
            const C S{P[1][c].x + P[3][c].x, P[1][c].y + P[3][c].y};
            const C D{P[1][c].x - P[3][c].x, P[1][c].y - P[3][c].y};
            const C f[4] = {{A.x + S.x, A.y + S.y}, {B.x - D.y, B.y + D.x},
                            {A.x - S.x, A.y - S.y}, {B.x + D.y, B.y - D.x}};
#pragma unroll
            for (int q = 0; q < 4; ++q) e[q] += (double)(f[q].x * f[q].x + f[q].y * f[q].y);
          }
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[a][q] += e[q];
        }
      }
    } else {
      // stage x + |f|^2, one image column per thread
#pragma unroll
      for (int a = 0; a < AB_XPT; ++a) {
        const int x = tid + a * AB_THREADS;
        if (x < p.xdiv) {
          long long q0 = ((long long)(-p.lpx) * x) % p.xdiv;
          if (q0 < 0) q0 += p.xdiv;
          double s0, c0, s1, c1;
          sincospi(2.0 * (double)q0 / (double)p.xdiv, &s0, &c0);
          sincospi(2.0 * (double)x / (double)p.xdiv, &s1, &c1);
          C w{(R)c0, (R)s0};
          const C r{(R)c1, (R)s1};
          C f[AB_YS][3];
#pragma unroll
          for (int b = 0; b < AB_YS; ++b) f[b][0] = f[b][1] = f[b][2] = C{(R)0, (R)0};
          const V2* gp = G;
          for (int lx = 0; lx < p.bx; ++lx, gp += AB_YS * 3) {
            stage_x_lx(gp, f, w);
            w = w * r;
          }
#pragma unroll
          for (int b = 0; b < AB_YS; ++b)
            acc[a][b] += (double)(f[b][0].x * f[b][0].x + f[b][0].y * f[b][0].y +
                                  f[b][1].x * f[b][1].x + f[b][1].y * f[b][1].y +
                                  f[b][2].x * f[b][2].x + f[b][2].y * f[b][2].y);
        }
      }
    }
  }
  const double wgt = p.inv_weight[img];
  double* im = image + (size_t)img * p.xdiv * p.ydiv;
  if (R4) {
    const int b = tid & (AB_YS - 1), g0 = tid / AB_YS, x4 = p.xdiv / 4;
#pragma unroll
    for (int a = 0; a < AB_XPT; ++a) {
      const int g = g0 + a * (AB_THREADS / AB_YS);
      if (g < x4 && b < ny)
#pragma unroll
        for (int q = 0; q < 4; ++q)
          atomicAdd(&im[(size_t)(g + q * x4) * p.ydiv + y0 + b * ystep], acc[a][q] * wgt);
    }
  } else {
#pragma unroll
    for (int a = 0; a < AB_XPT; ++a) {
      const int x = tid + a * AB_THREADS;
      if (x < p.xdiv)
#pragma unroll
        for (int b = 0; b < AB_YS; ++b)
          if (b < ny) atomicAdd(&im[(size_t)x * p.ydiv + y0 + b], acc[a][b] * wgt);
    }
  }
}

}  // namespace euv

using namespace euv;

extern "C" int euv_abbe(const euv_abbe_desc* d, const euv_c64* d_ax, double* d_image,
                        void* stream_) {
  if (!d || !d_ax || !d_image || d->xdiv <= 0 || d->ydiv <= 0 ||
      d->xdiv > AB_THREADS * AB_XPT || d->lpx < 0 || d->lpy < 0 || d->ncut <= 0 ||
      d->n_units <= 0 || d->n_src <= 0 || d->n_order <= 0 || !d->d_coef || !d->d_nidx ||
      !d->d_px || !d->d_py || !d->d_row_start || !d->d_tab_of_unit || !d->d_img_of_unit || !d->d_nsrc_of_unit || !d->d_inv_weight ||
      d->n_images <= 0 || d->n_units > 65535 ||
      (d->precision != EUV_PREC_FP64 && d->precision != EUV_PREC_MIXED)) {
    euv_set_error("euv_abbe: bad arguments");
    return EUV_ERR_BAD_ARG;
  }
  cudaStream_t stream = (cudaStream_t)stream_;
  AbbeParams p;
  p.xdiv = d->xdiv;
  p.ydiv = d->ydiv;
  p.lpx = d->lpx;
  p.lpy = d->lpy;
  p.bx = 2 * d->lpx + 1;
  p.by = 2 * d->lpy + 1;
  p.ncut = d->ncut;
  p.n_src = d->n_src;
  p.n_order = d->n_order;
  p.coef = reinterpret_cast<const double2*>(d->d_coef);
  p.nidx = d->d_nidx;
  p.py = d->d_py;
  p.row_start = d->d_row_start;
  p.tab_of_unit = d->d_tab_of_unit;
  p.img_of_unit = d->d_img_of_unit;
  p.nsrc_of_unit = d->d_nsrc_of_unit;
  p.inv_weight = d->d_inv_weight;
  const int ystripes = (d->ydiv + AB_YS - 1) / AB_YS;
  const bool fp32 = d->precision == EUV_PREC_MIXED;
  const bool r4 = d->xdiv % 4 == 0 && d->ydiv % 4 == 0;
  const size_t g_elems = r4 ? (size_t)(p.bx + 2 * AB_GP) * AB_YS * 4 : (size_t)AB_YS * p.bx * 3;
  size_t smem = ((((size_t)d->ncut * 3 + 1) & ~(size_t)1) + g_elems + (size_t)AB_YS * p.by) *
                    (fp32 ? sizeof(float2) : sizeof(double2)) +
                (size_t)d->ncut * sizeof(int);
  if (smem > 227 * 1024) {
    euv_set_error("euv_abbe: pupil too large for one CTA (%zu bytes of shared memory)", smem);
    return EUV_ERR_BAD_ARG;
  }
  using Kern = void (*)(AbbeParams, const double2*, double*);
  static const Kern kerns[4] = {abbe_kernel<double, false>, abbe_kernel<double, true>,
                                abbe_kernel<float, false>, abbe_kernel<float, true>};
  static int smem_done[4][64];
  const int kv = (fp32 ? 2 : 0) + (r4 ? 1 : 0);
  EUV_CUDA_TRY(ensure_smem(kerns[kv], (int)smem, smem_done[kv]));
  // source split: the CTAs of a unit's row groups take every nsplit-th source.
  // Chosen to minimise (waves of resident CTAs) x (sources per CTA + 1), the
  // 1 standing for a CTA's own setup and atomics, so that the last wave is not
  // left mostly empty without multiplying the CTAs; ties keep the smaller
  // split.
  int dev = 0, sms = 148, per_sm = 1;
  EUV_CUDA_TRY(cudaGetDevice(&dev));
  EUV_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  EUV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kerns[kv], AB_THREADS, smem));
  const long long slots = (long long)sms * (per_sm > 0 ? per_sm : 1);
  const long long groups = (long long)ystripes * d->n_units;
  int nsplit = 1;
  long long best = -1;
  for (int ns = 1; ns <= d->n_src && ns <= 64; ++ns) {
    const long long cost = ((groups * ns + slots - 1) / slots) * ((d->n_src + ns - 1) / ns + 1);
    if (best < 0 || cost < best) {
      best = cost;
      nsplit = ns;
    }
  }
  const int tuned = tune_lookup(EUV_KNOB_ABBE_SPLIT, d->n_units, d->n_src);
  if (tuned > 0) nsplit = tuned < d->n_src ? tuned : d->n_src;
  p.nsplit = nsplit;
  dim3 grid(ystripes, nsplit, d->n_units);
  kerns[kv]<<<grid, AB_THREADS, smem, stream>>>(p, reinterpret_cast<const double2*>(d_ax), d_image);
  EUV_LAUNCH_CHECK();
  return EUV_OK;
}
