/*
 * euvl_b200.h -- C ABI of the B200 EUV mask-3D library (libeuvl_b200.so).
 *
 * Drop-in boundary for the rigorous mask-3D solve and Abbe imaging of
 * takahashi-edalab/EUVlitho.  The reference exposes these as C++ functions in
 * cnn/include/header.h and the main() loops of cnn/intensity/abbe/intensity.cpp
 * and cnn/intensity/m3d/m3d.cpp; each entry point below names the reference
 * code it replaces.
 *
 * Conventions
 *  - Every pointer named d_* is DEVICE memory owned by the caller (e.g. a
 *    torch tensor); h_* is host memory.  The library allocates nothing on the
 *    device: scratch space is a caller-provided workspace whose size is given by
 *    the matching *_workspace_bytes() query.
 *  - Complex numbers are euv_c64 = {re, im} doubles, layout-compatible with
 *    cuDoubleComplex, std::complex<double> and torch.complex128.
 *  - Matrices are column-major (element (i,j) at i + j*ld), batched with an
 *    element stride between consecutive matrices.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *    Work is enqueued asynchronously on it; nothing synchronises the host.
 *  - Every function returns EUV_OK (0) or an error code; euv_last_error()
 *    returns a message for the last failure on the calling thread.
 *  - Thread safety: functions keep no global state besides the per-thread error
 *    message; concurrent calls on different streams with disjoint buffers are
 *    safe.
 */
#ifndef EUVL_B200_H
#define EUVL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EUV_OK 0
#define EUV_ERR_BAD_ARG 1
#define EUV_ERR_CUDA 2
#define EUV_ERR_WORKSPACE 3
#define EUV_ERR_SINGULAR 4
#define EUV_ERR_TIMEOUT 5  /* a bounded device wait expired (euv_wait_probe) */

/* Bits of a caller-owned device status word (euv_amp_desc.d_status, the d_status
 * argument of euv_zgemm_mixed and euv_wait_probe).  The library only ORs bits
 * in; the caller zeroes the word and reads it when the stream is idle (the
 * reference checks none of these conditions, header.h:498,888,1529). */
#define EUV_STATUS_TIMEOUT 1       /* a bounded device wait gave up: that call's results are incomplete */
#define EUV_STATUS_STEPS_CLAMPED 2 /* a unit needed more double-angle steps than m_max */
#define EUV_STATUS_SINGULAR 4      /* an LU met an exactly zero pivot */
#define EUV_STATUS_NOT_CONVERGED 8 /* an eigensolver stopped at its sweep limit */

#define EUV_MAX_SLICES 32

#define EUV_PREC_FP64 0  /* every product in FP64 */
#define EUV_PREC_MIXED 1 /* bulk products as split-FP16x3 on tcgen05 tensor cores, FP64 solves */

typedef struct {
  double re, im;
} euv_c64;

/* Multilayer materials (permittivities) and thicknesses in nm: the constants of
 * header.h:1217-1230, made parameters. */
typedef struct {
  euv_c64 eps_mo, eps_si, eps_ru, eps_mosi2, eps_rusi, eps_sio2;
  double d_mo, d_mosi, d_si, d_simo, d_siru, d_ru;
  int nml; /* Mo/Si periods (header.h NML) */
} euv_stack;

/* Library version, last error, and the number of kernels the library has
 * enqueued in this process (launches captured into a CUDA graph count once,
 * at capture). */
const char* euv_version(void);
const char* euv_last_error(void);
unsigned long long euv_kernel_launches(void);

/* ------------------------------------------------------------------------ */
/* Mask spectrum: replaces maskamp (header.h:1147-1206) with fourier /
 * exponential (header.h:1621-1648), and the thin-mask DFT of m3d.cpp:287-327.
 *
 * d_bits: n_masks packed masks of ndivx*ndivy bits each, MSB first, bit index
 *   ndivx*j + i (j = y), exactly the mask.bin layout (intensity.cpp:20-29).
 * The pattern on the fdivx x fdivy Fourier grid is pixel (i/meshx,
 * ndivy-1-j/meshy + y_offset) (y flipped, header.h:1159); rows outside the
 * mask read as absorber.  y_offset = 0 is the shipped header.h; y_offset = 1
 * reproduces the revision that produced the reference's golden emint.csv /
 * inputxx.csv (its flip is one row off).  select_vacuum = 0 transforms the
 * absorber indicator (bit == 0), 1 the vacuum indicator (bit == 1).
 * d_out[mask][l + (2*lh+1)*m'] = (1/(fdivx*fdivy)) sum_x,y ind(x,y)
 *   exp(-2 pi i (l x/fdivx + m y/fdivy)),  l in [-lh, lh], m in [-mh, mh].
 * The permittivity coefficients of header.h:1236-1251 follow as
 *   eps = 1*delta + (eps_abs - 1) * F,  sigma = delta + (1/eps_abs - 1) * F,
 *   leps = log(eps_abs) * F (F = absorber-indicator spectrum). */
size_t euv_mask_spectrum_workspace_bytes(int n_masks, int ndivx, int ndivy, int fdivx, int fdivy,
                                         int lh, int mh);
int euv_mask_spectrum(const uint8_t* d_bits, int n_masks, int ndivx, int ndivy, int fdivx,
                      int fdivy, int lh, int mh, int select_vacuum, int y_offset, euv_c64* d_out,
                      void* d_work, size_t work_bytes, void* stream);

/* ------------------------------------------------------------------------ */
/* Hermitian eigendecomposition (parallel cyclic Jacobi): replaces the eigh of
 * the STCC-SOCS transmission cross-coefficient matrices
 * (cnn/intensity/stccsocs/eigenfunction.py:128-130; cupy.linalg.eigh there).
 * d_a (n x n, column-major, Hermitian) is overwritten (diagonalised);
 * d_w[i] = eigenvalue i, d_v(:, i) its eigenvector, in no particular order.
 * Stops when the off-diagonal Frobenius norm is <= tol x the full one, or
 * after max_sweeps sweeps (EUV_STATUS_NOT_CONVERGED into *d_status then).
 * A per-configuration step: n - 1 rounds of three launches per sweep. */
size_t euv_heev_workspace_bytes(int n);
int euv_heev(int n, euv_c64* d_a, int lda, double* d_w, euv_c64* d_v, int ldv, int max_sweeps,
             double tol, void* d_work, size_t work_bytes, int* d_status, void* stream);

/* ------------------------------------------------------------------------ */
/* STCC-SOCS image from M3D parameters: replaces intsocs
 * (cnn/intensity/stccsocs/socs.py:12-151).  For clip c with vacuum-indicator
 * spectrum F_c (euv_mask_spectrum, select_vacuum = 1, lh = lpx, mh = lpy) and
 * M3D parameters a0, ax, ay [c][ncut] (ax = ay = 0 without a slope):
 *   A0 = famp + a0 (famp as in euv_linear_amp), Ax = ax dx/2pi, Ay = ay dy/2pi,
 *   Axy = ax lp/2 + ay mp/2;
 *   small = sum_{m<nsocs} alpha_s0[m] |F[A0 phi_s0[m]]|^2
 *         + sum_{m<nsocsxy} 2 Re(alpha_sx[m] F[A0 phi_sx[m]] F*[Ax phi_sx[m]]
 *                               + alpha_sy[m] F[A0 phi_sy[m]] F*[Ay phi_sy[m]]
 *                               + alpha_s0[m] F[A0 phi_s0[m]] F*[Axy phi_s0[m]]),
 * F[v](x, y) = sum_n v_n e^{2 pi i (lp_n x + mp_n y)/nout} on the nout x nout grid;
 * d_image[c][x][y] = sum_{u,v} Kx[x][u] small[u][v] Ky[y][v] (complex; its real
 * part is the image), Kx[x][u] = (1/nout) sum_{i=-nout/2}^{nout/2-1}
 * e^{2 pi i i (x/xdiv - u/nout)} (Ky alike): the Fourier interpolation of
 * socs.py:137-150.  phi_*[m][n]: eigenfunction m of the TCC at pupil point n
 * (euv_heev + sort by |alpha|).  The resident tables d_e, d_kxT, d_ky are
 * config-only. */
typedef struct {
  int n_clips, ncut, lpx, lpy, nsocs, nsocsxy, nout, xdiv, ydiv;
  const int* d_lp;             /* [ncut] pupil orders */
  const int* d_mp;
  double k, dx, dy, kx0, ky0, z0;
  euv_c64 amp_vc, amp_ab;      /* specular amplitudes of the all-vacuum / all-absorber mask */
  const euv_c64* d_phi_s0;     /* [nsocs][ncut] */
  const euv_c64* d_phi_sx;     /* [nsocsxy][ncut] */
  const euv_c64* d_phi_sy;
  const double* d_alpha_s0;    /* [nsocs] */
  const double* d_alpha_sx;    /* [nsocsxy] */
  const double* d_alpha_sy;
  const euv_c64* d_e;          /* [nout][nout] e^{2 pi i a b / nout} */
  const euv_c64* d_kxT;        /* element u + nout x = Kx[x][u] */
  const euv_c64* d_ky;         /* element y + ydiv v = Ky[y][v] */
} euv_socs_desc;
size_t euv_socs_workspace_bytes(const euv_socs_desc* desc);
int euv_socs_image(const euv_socs_desc* desc, const euv_c64* d_fvac, const euv_c64* d_a0,
                   const euv_c64* d_ax, const euv_c64* d_ay, euv_c64* d_image, void* d_work,
                   size_t work_bytes, void* stream);

/* ------------------------------------------------------------------------ */
/* Mask rasteriser: replaces the pixel fill of the reference's mask generator
 * (cnn/intensity/mask/mVBF.h:2-70) and its bit packing (mask.cpp:9-26) for
 * bulk data generation on the device.
 *
 * Every mask starts as vacuum (1); d_rects[r] = {mask, x0, x1, y0, y1}
 * (half-open pixel ranges, clipped to the grid) are painted absorber (0).
 * Slice s is the drawn mask with the absorber eroded by h_erosion[s] steps of
 * the 4-neighbour cross (periodic edges; 0 = as drawn) -- a sloped sidewall
 * (n_slices <= 64).  Output d_bits[mask][slice][ndivx*ndivy/8] in the mask.bin
 * layout (bit ndivx*y + x, MSB first, 1 = vacuum), ready for
 * euv_mask_spectrum.  h_erosion is HOST memory.  Workspace:
 * euv_mask_raster_workspace_bytes (two byte images per mask). */
size_t euv_mask_raster_workspace_bytes(int n_masks, int ndivx, int ndivy);
int euv_mask_raster(int n_masks, int ndivx, int ndivy, int n_rects, const int* d_rects,
                    int n_slices, const int* h_erosion, uint8_t* d_bits, void* d_work,
                    size_t work_bytes, void* stream);

/* ------------------------------------------------------------------------ */
/* CNN predict: replaces predict_m3d (cnn/cnn/predict/predict.py:108-121) with
 * the networks CNNmodel / CNNmodels (predict.py:16-88) and the mask
 * downsampling compmask (cnn/cnn/predict/compmask.py:17-41).
 *
 * A model is the reference's network: five [conv 3x3 circular, ReLU, 2x2
 * max-pool, BatchNorm (running statistics)] stages 1-16-32-64-128-256 on a
 * 512 x 512 input, fc1 65536 -> 4096 + ReLU, fc2 4096 -> n_out.  Weights are
 * the torch tensors of a state_dict, fp32, contiguous, on the device, in torch
 * layout (conv [cout][cin][3][3], linear [out][in]); euv_cnn_pack rewrites
 * them once into a blob (conv weights as TF32 (hi, lo) planes, fc weights
 * fp32 in the kernels' K order; about 1.1 GB per model).
 * The predict takes mask.bin rasters (2048 x 2048 bits, MSB first, 524288
 * bytes per mask), and writes out[model][mask][j] = fc2 output / factor
 * (the division of predict.py:114-119, in double) for j < n_out[model],
 * zero above.  Products are TF32x3 with FP32 accumulation (about FP32
 * accuracy). */
#define EUV_CNN_MAX_MODELS 6
#define EUV_CNN_MAX_OUT 8192
typedef struct euv_cnn_model_weights {
  const float* conv_w[5]; /* conv1..conv5 weight, bias */
  const float* conv_b[5];
  const float* bn_w[5];   /* norm1..norm5 weight, bias, running_mean, running_var */
  const float* bn_b[5];
  const float* bn_mean[5];
  const float* bn_var[5];
  const float* fc1_w;     /* [4096][65536] */
  const float* fc1_b;
  const float* fc2_w;     /* [n_out][4096] */
  const float* fc2_b;
  int n_out;
} euv_cnn_model_weights;

typedef struct euv_cnn_desc {
  int n_models, n_masks, max_out; /* max_out: row stride of d_factors and out */
  int n_out[EUV_CNN_MAX_MODELS];
  const double* d_factors;        /* [n_models][max_out] */
  int* d_status;                  /* EUV_STATUS_* word, or NULL */
} euv_cnn_desc;

size_t euv_cnn_blob_bytes(int n_models, int max_out);
int euv_cnn_pack(int n_models, const euv_cnn_model_weights* h_models, int max_out,
                 double bn_eps, void* d_blob, size_t blob_bytes, void* stream);
size_t euv_cnn_workspace_bytes(int n_models, int n_masks, int max_out);
/* d_blob and d_work 256-byte aligned */
int euv_cnn_predict(const euv_cnn_desc* desc, const uint8_t* d_bits, const void* d_blob,
                    double* d_out, void* d_work, size_t work_bytes, void* stream);
/* compmask alone: d_x0[mask][512][512] = 4 x 4 box means of the bits */
int euv_cnn_downsample(int n_masks, const uint8_t* d_bits, float* d_x0, void* stream);

/* ------------------------------------------------------------------------ */
/* Batched ampS: replaces ampS (header.h:1208-1466) with multilayerS
 * (header.h:5-363), absorberS0 (754-1145), absorberS (365-752), matinv and
 * matproduct (1468-1619), for n_units independent problems that share one
 * order set.  A unit is one (clip, Bloch family, polarisation).
 *
 * Outputs Ax for the requested source orders:
 *   d_ax[u][s][n] = Ax[(ls,ms)](n) of header.h:1394-1465, s < n_src, n < N.
 * Source columns whose order is not in the order set (src_order = -1) get zeros
 * except that they are never referenced by the callers. */
typedef struct {
  int n_orders;          /* Nrange */
  int lmax, mmax;        /* LMAX, MMAX: spectra cover orders -2LMAX..2LMAX x -2MMAX..2MMAX */
  const int* d_lindex;   /* [N] */
  const int* d_mindex;   /* [N] */
  double dx, dy;         /* clip period (nm) */
  double k;              /* 2 pi / lambda */
  int n_slices;          /* NABS; slice 0 = top, n_slices-1 sits on the Ru cap */
  euv_c64 eabs[EUV_MAX_SLICES];
  double dabs[EUV_MAX_SLICES];
  int refresh_sigma;     /* 0: reference behaviour (bottom-slice sigma for all slices) */
  euv_stack stack;
  int n_units;
  const double* d_kx0;   /* [U] incidence kx of the unit's Bloch family (sx0) */
  const double* d_ky0;   /* [U] */
  const int* d_polar;    /* [U] 0 = 'X', 1 = 'Y' */
  const int* d_spec;     /* [U] index c of the unit's clip: slice n spectrum is
                            d_spectra[(c*n_slices + n) * (4lmax+1)(4mmax+1)] */
  int n_src;             /* source columns per unit */
  const int* d_src_order;  /* [U][n_src] order index of each source (-1: none) */
  const double* d_src_2kz; /* [U][n_src] 2*kz of each source (header.h:1401-1409) */
  int precision;         /* EUV_PREC_FP64 or EUV_PREC_MIXED */
  int m_max;             /* upper bound on double-angle steps; <= 0: derived */
  double k0_max;         /* bound on |kx0|, |ky0| over the units (<= 0: k) */
  int* d_status;         /* optional device int: EUV_STATUS_* bits OR-ed in (NULL: none) */
  const double* d_dx;    /* optional [U] clip period of each unit (nm), so that clips of
                            different periods with the same order set share a launch;
                            NULL: dx for every unit.  With it, dx must be the smallest
                            period over the units (it bounds the matrix norms) */
  const double* d_dy;    /* optional [U], as d_dx */
  int euler_f;           /* EUV_PREC_MIXED: factors of the Euler product that inverts the
                            interface matrix (1..8); 0: derived from dx, dy and k0_max so
                            that the truncation is <= 1e-7; -1: an FP64 LU instead.  Fix it
                            to make a unit's result independent of the other units of the
                            launch (the derived count depends on the smallest period) */
} euv_amp_desc;

size_t euv_amp_workspace_bytes(const euv_amp_desc* desc);
/* The Euler factor count a launch with this descriptor uses (the euler_f
 * rule above): 1..8, -1 for the FP64 LU, 0 for EUV_PREC_FP64 (the LU always);
 * -2 for an invalid descriptor.  Host only. */
int euv_amp_euler_factors(const euv_amp_desc* desc);
int euv_amp(const euv_amp_desc* desc, const euv_c64* d_spectra, euv_c64* d_ax, void* d_work,
            size_t work_bytes, void* stream);

/* ------------------------------------------------------------------------ */
/* Linear Abbe model from M3D parameters: replaces the amplitude loop of
 * cnn/intensity/linear/linear.py:120-172 (its image loop, linear.py:11-43, is
 * euv_abbe with identity pupil tables, see below).  For clip c, source s of the
 * linear model's source grid (shifts dsx, dsy, linear.py:47-96) and pupil
 * point i (orders lp, mp):
 *   famp(c,i)  = (ab delta(lp,mp) + (vc - ab) F_c(lp,mp)) phX(lp) phY(mp) / (vc/|vc|),
 *   phX(lp)    = exp(-i (kx0 kxp + kxp^2/2) z0 / k),  kxp = 2 pi lp / dx (y alike),
 *   A[c][s][i] = famp(c,i) + a0[c][i] + ax[c][i] (ls_s + lp/2) + ay[c][i] (ms_s + mp/2),
 * ls_s = dsx_s dx / (2 pi), ms_s = dsy_s dy / (2 pi).  d_a0 == NULL gives the
 * thin-mask (Kirchhoff) amplitude famp (linear.py's intft).  F_c is the
 * vacuum-indicator spectrum of clip c (euv_mask_spectrum, select_vacuum = 1,
 * lh = lpx, mh = lpy).  a0, ax, ay: [c][ncut], ax = ay = 0 where the M3D fit
 * has no slope.  Output d_amp[c][s][i] feeds euv_abbe as its d_ax with
 * n_order = ncut, d_nidx[s][i] = i (-1 outside the pupil) and coefficients
 * i k R(:,0) phase / sqrt(k^2 - (kx0+dsx_s)^2). */
typedef struct {
  int n_clips, n_src, ncut, lpx, lpy;
  const int* d_lp;         /* [ncut] pupil orders */
  const int* d_mp;
  const double* d_ls;      /* [n_src] source shifts in orders */
  const double* d_ms;
  double k, dx, dy, kx0, ky0, z0;
  euv_c64 amp_vc, amp_ab;  /* specular amplitudes of the all-vacuum / all-absorber mask */
} euv_linear_desc;
int euv_linear_amp(const euv_linear_desc* desc, const euv_c64* d_fvac, const euv_c64* d_a0,
                   const euv_c64* d_ax, const euv_c64* d_ay, euv_c64* d_amp, void* stream);

/* ------------------------------------------------------------------------ */
/* Fused Abbe imaging: replaces the per-source loop of intensity.cpp:248-408
 * (E-field through rotate(), pupil phase and defocus, scatter, three cuFFT Z2Z
 * inverse transforms, |Ex|^2+|Ey|^2+|Ez|^2, sum over sources / SDIVSUM) with one
 * kernel that keeps the image on chip.
 *
 * The config-only factors are precomputed tables (resident per plan):
 *   d_coef[((t*n_src + s)*ncut + i)*3 + c]  = i k R(c,.) . (polarisation) * phase
 *                                             / sqrt(k^2 - kx^2)  (or ky)
 *   d_nidx[(t*n_src + s)*ncut + i]          = order index of pupil point i of
 *                                             source s (-1: outside the pupil)
 *   with t = d_tab_of_unit[u] (units of different clips share tables)
 *   d_px[i], d_py[i]                        = pupil frequency indices (linput, minput)
 *   d_row_start[l]                          = first pupil point with linput = l - lpx
 *                                             (points are l-major, as intensity.cpp:166-195
 *                                             enumerates them; [2*lpx+2] entries)
 * Image: d_image[img][x*ydiv + y] += (1/weight[img]) * sum over units u with
 * d_img_of_unit[u] == img, sources s < d_nsrc_of_unit[u], of |f|^2, where f is
 * the unnormalised inverse DFT of the pupil field (intensity.cpp:369-386). The
 * image must be zeroed by the caller. */
typedef struct {
  int xdiv, ydiv;        /* image grid */
  int lpx, lpy;          /* pupil box half sizes (lpmaxX, lpmaxY) */
  int ncut;              /* pupil points */
  int n_units, n_src, n_order;
  const euv_c64* d_coef;
  const int* d_nidx;
  const int* d_px;
  const int* d_py;
  const int* d_row_start;
  const int* d_tab_of_unit;   /* [U] */
  const int* d_img_of_unit;   /* [U] */
  const int* d_nsrc_of_unit;  /* [U] */
  int n_images;
  const double* d_inv_weight; /* [n_images] 1/SDIVSUM */
  int precision;               /* EUV_PREC_FP64, or EUV_PREC_MIXED: DFT sums in FP32 */
} euv_abbe_desc;

int euv_abbe(const euv_abbe_desc* desc, const euv_c64* d_ax, double* d_image, void* stream);

/* ------------------------------------------------------------------------ */
/* M3D parameters: replaces m3d.cpp:240-467 (specular vacuum/absorber
 * amplitudes, thin-mask amplitudes, phase normalisation by the vacuum specular
 * phase, difference dampxx, 3x3 Cramer least squares a0 + ax*ls + ay*ms per
 * pupil order).
 *   d_ax_wide[c][s][n]: rigorous amplitudes of clip c for the NA-circle source
 *     orders s (enumeration of header.h:1394-1397), n < n_order;
 *   d_ax_vc / d_ax_ab [s][n']: the same for the all-vacuum / all-absorber mask
 *     on the narrow order set (m3d.cpp:214-238), n' < n_order_narrow;
 *   d_src_nidx_narrow[s]: order index of source s in the narrow set;
 *   s_center: index of source order (0,0);
 *   d_fmask[c][ip + (2lpx+1)*jp]: vacuum-indicator spectrum (euv_mask_spectrum
 *     with select_vacuum=1, lh=lpx, mh=lpy);
 *   d_lin/d_min/d_xin[n]: pupil orders and the xinput flag (m3d.cpp:160-195);
 *   d_pair_order[n*n_src + s] = wide order index of pupil n seen from source s
 *     (-1 where the source or the diffracted order is outside the NA circle).
 * Outputs a0/ax/ay[c][n], n < ninput (ax, ay are zero where xinput == 0). */
typedef struct {
  int n_clips, n_src, ninput, n_order, n_order_narrow;
  int lpx, lpy;
  double k, dx, dy, z0, kx0, ky0;
  int s_center;
  const int* d_src_l;
  const int* d_src_m;
  const int* d_src_nidx_narrow;
  const euv_c64* d_ax_vc;
  const euv_c64* d_ax_ab;
  const int* d_lin;
  const int* d_min;
  const int* d_xin;
  const int* d_pair_order;
} euv_m3d_desc;

int euv_m3d_fit(const euv_m3d_desc* desc, const euv_c64* d_ax_wide, const euv_c64* d_fmask,
                euv_c64* d_a0, euv_c64* d_ax, euv_c64* d_ay, void* stream);

/* ------------------------------------------------------------------------ */
/* Plans: the configuration of the reference drivers and its tables, for C and
 * C++ callers that port intensity.cpp / m3d.cpp onto the library without any
 * other host code.
 *
 * euv_config holds the constants of intensity.cpp:44-146 / m3d.cpp:34-157 as
 * parameters (euv_config_reference() fills the reference's values).  A plan
 * builds, on the host, every table those drivers compute before their loops:
 *   - the order set (rounded diamond intensity.cpp:148-164, ellipse
 *     m3d.cpp:113-129, or an explicit box), l outer / m inner;
 *   - the pupil set with the xinput flag (intensity.cpp:166-195,
 *     m3d.cpp:160-195), l-major;
 *   - the Bloch families and their source orders (source(),
 *     intensity.cpp:467-502; max_sources keeps the first points);
 *   - per (polarisation, family, source, pupil point) the E-field factor
 *     i k R(.) / sqrt(k^2 - k_s^2) * phase of rotate() and the pupil phase
 *     with defocus (intensity.cpp:276-353, 423-465), and the order index the
 *     point reads (the tables euv_abbe takes);
 *   - the NA-circle source orders of ampS (header.h:1394-1397), the narrow
 *     order set of m3d.cpp:101-129 and the (pupil point, source) -> order
 *     pairs of the M3D fit (m3d.cpp:426-450).
 * euv_plan_create allocates host memory only; euv_plan_upload copies the
 * tables into caller device memory (euv_plan_device_bytes), sized for up to
 * max_clips clips per call, after which the run functions can be called.
 * A plan is read-only after upload except for the M3D narrow solves, which
 * the first euv_plan_m3d call computes into the plan's device tables: make
 * that first call before sharing the plan between streams.  Plans on
 * different devices need their own upload. */
#define EUV_ORDERS_DIAMOND 0
#define EUV_ORDERS_ELLIPSE 1
#define EUV_ORDERS_BOX 2

typedef struct {
  int ndivx, ndivy;        /* clip on the mask grid (pixels of 1 nm: dx = ndivx nm) */
  double delta;            /* Fourier-grid pixel (nm): fdivx = ndivx / delta */
  double wavelength;       /* nm */
  double theta0, azimuth;  /* chief ray (deg): kx0 = k sin(theta0) cos(90 - azimuth) */
  double na;
  int mx, my;              /* demagnification (anamorphic: my = 8) */
  int illum_type;          /* 0 conventional, 1 annular, 2 X dipole, 3 Y dipole */
  double sigma1, sigma2, openangle, sigmadiv;
  int ndivs;               /* Bloch families per axis; <= 0: the reference's rule */
  int max_sources;         /* keep the first max_sources source points; <= 0: all */
  int n_slices;            /* absorber slices (slice 0 = top) */
  euv_c64 eabs[EUV_MAX_SLICES]; /* permittivity of each slice */
  double dabs[EUV_MAX_SLICES];  /* thickness of each slice (nm) */
  double z0_offset;        /* z0 = sum(dabs) + z0_offset (intensity.cpp:80) */
  euv_stack stack;
  int refresh_sigma;       /* 0: the bottom slice's sigma for every slice (reference) */
  int order_kind;          /* EUV_ORDERS_* */
  double cut;              /* order cut of the diamond / ellipse sets */
  int lbox, mbox;          /* half sizes of the box set */
  double z;                /* defocus (nm) */
  int yflip_offset;        /* as in euv_mask_spectrum */
  int n_pols;              /* 1 or 2 */
  int pols[2];             /* 0 = X, 1 = Y */
  int precision;           /* EUV_PREC_FP64 or EUV_PREC_MIXED */
} euv_config;

typedef struct {
  int n_orders, lmax, mmax;   /* order set and its limits (LMAX, MMAX) */
  int ncut, lpx, lpy;         /* pupil points and the pupil box half sizes */
  int lsx, lsy;               /* lsmaxX, lsmaxY */
  int n_na_sources;           /* NA-circle source orders of ampS */
  int ndivs, n_families, n_src_max, sdivsum;
  int n_pols, units_per_clip; /* units = families x polarisations */
  int xdiv, ydiv, fdivx, fdivy;
  int n_orders_narrow;        /* m3d.cpp narrow set (ellipse, cut 1.5) */
  double k, kx0, ky0, z0;
} euv_plan_info;

typedef struct euv_plan euv_plan;

/* The reference configuration (intensity.cpp:44-146, header.h:1217-1230):
 * NA 0.33, 4x, 2048 nm, annular 0.55-0.9, Ta 60 nm, X polarisation, FP64. */
void euv_config_reference(euv_config* cfg);
/* Host tables of cfg; *plan is freed by euv_plan_destroy.  EUV_ERR_BAD_ARG
 * for an invalid configuration (e.g. an order set that misses a diffracted
 * order the Abbe loop reads, or reaches evanescent orders: header.h:1283
 * takes a real square root). */
int euv_plan_create(const euv_config* cfg, euv_plan** plan);
void euv_plan_destroy(euv_plan* plan);
int euv_plan_get_info(const euv_plan* plan, euv_plan_info* info);
/* Host copies of the tables (caller arrays of the sizes in euv_plan_info):
 * orders l, m [n_orders]; pupil l, m, xinput [ncut]; family nsx, nsy, count
 * [n_families] and source orders l, m [sdivsum] family by family; the NA
 * sources l, m [n_na_sources]; Abbe table t = pol_index * n_families + family:
 * coef [n_src_max][ncut][3], nidx [n_src_max][ncut].  NULL arrays are skipped. */
int euv_plan_get_orders(const euv_plan* plan, int* h_l, int* h_m);
int euv_plan_get_pupil(const euv_plan* plan, int* h_l, int* h_m, int* h_xinput);
int euv_plan_get_sources(const euv_plan* plan, int* h_nsx, int* h_nsy, int* h_count, int* h_l,
                         int* h_m);
int euv_plan_get_na_sources(const euv_plan* plan, int* h_l, int* h_m);
int euv_plan_get_abbe_table(const euv_plan* plan, int t, euv_c64* h_coef, int* h_nidx);
/* Device tables for up to max_clips clips per call. */
size_t euv_plan_device_bytes(const euv_plan* plan, int max_clips);
int euv_plan_upload(euv_plan* plan, int max_clips, void* d_tables, size_t bytes, void* stream);
/* Reads and clears the plan's device status word (synchronises the stream):
 * EUV_ERR_TIMEOUT / EUV_ERR_SINGULAR if a run since the last check reported
 * one (EUV_STATUS_* bits in *bits), else EUV_OK. */
int euv_plan_check(const euv_plan* plan, int* bits, void* stream);

/* The Abbe images of n_clips clips (intensity.cpp:219-408 for every
 * polarisation of the plan): d_masks [clip][n_mask_slices][ndivx*ndivy/8]
 * mask.bin bits (n_mask_slices 1 = one mask for all slices, the reference;
 * or one per slice); d_image [clip][pol][xdiv][ydiv], I[x][y], overwritten.
 * One batched ampS of all (clip, family, polarisation) units, then the fused
 * Abbe kernel. */
size_t euv_plan_intensity_workspace_bytes(const euv_plan* plan, int n_clips, int n_mask_slices);
int euv_plan_intensity(const euv_plan* plan, const uint8_t* d_masks, int n_clips,
                       int n_mask_slices, double* d_image, void* d_work, size_t work_bytes,
                       void* stream);
/* ampS at one incidence for the NA-circle source orders (header.h:1394-1465):
 * d_ax [clip][na source][n_orders]. */
size_t euv_plan_amp_workspace_bytes(const euv_plan* plan, int n_clips, int n_mask_slices);
int euv_plan_amp(const euv_plan* plan, int polar, double kx0, double ky0, const uint8_t* d_masks,
                 int n_clips, int n_mask_slices, euv_c64* d_ax, void* d_work, size_t work_bytes,
                 void* stream);
/* M3D parameters of m3d.cpp:197-558 for polarisation pols[0]: d_a0, d_ax,
 * d_ay [clip][ncut] (ax, ay zero where xinput == 0). */
size_t euv_plan_m3d_workspace_bytes(const euv_plan* plan, int n_clips, int n_mask_slices);
int euv_plan_m3d(euv_plan* plan, const uint8_t* d_masks, int n_clips, int n_mask_slices,
                 euv_c64* d_a0, euv_c64* d_ax, euv_c64* d_ay, void* d_work, size_t work_bytes,
                 void* stream);

/* ------------------------------------------------------------------------ */
/* Building blocks, exported for tests and for callers composing their own
 * pipelines. */

/* C[b] = alpha*scale[b] * A[b] B[b] + beta C[b] + diag_add * I  (complex FP64,
 * column-major, batched by element strides).  Replaces matproduct
 * (header.h:1559-1619).  `d_scale` may be NULL (= 1).  If d_steps is not NULL
 * and step >= d_steps[b], batch b instead copies A into C (M == N == K). */
int euv_zgemm(int m, int n, int k, euv_c64 alpha, const double* d_scale, const euv_c64* d_a,
              int lda, long long stride_a, const euv_c64* d_b, int ldb, long long stride_b,
              euv_c64 beta, euv_c64* d_c, int ldc, long long stride_c, euv_c64 diag_add,
              int batch, const int* d_steps, int step, void* stream);

/* The bulk product of EUV_PREC_MIXED: same contract as euv_zgemm, computed on
 * the tcgen05 tensor cores as split-FP16x3: each row of A and column of B is
 * scaled by a power of two into fp16's range, each scaled FP64 value split
 * into two fp16 terms, three fp16 products per real product (kind::f16, FP32
 * accumulation), the scaling undone in FP64 (~1e-6 relative error per product,
 * about that of TF32x3 at twice its tensor rate).  Needs a workspace for the
 * split operands.  d_status (optional device int): EUV_STATUS_TIMEOUT is
 * OR-ed in if one of the kernel's bounded waits (about 2 s) gave up. */
size_t euv_zgemm_mixed_workspace_bytes(int m, int n, int k, int batch);
int euv_zgemm_mixed(int m, int n, int k, euv_c64 alpha, const double* d_scale,
                     const euv_c64* d_a, int lda, long long stride_a, const euv_c64* d_b, int ldb,
                     long long stride_b, euv_c64 beta, euv_c64* d_c, int ldc, long long stride_c,
                     euv_c64 diag, int batch, const int* d_steps, int step, void* d_work,
                     size_t work_bytes, int* d_status, void* stream);

/* Tuning table: per problem shape, a pick that overrides a kernel's built-in
 * choice (no reference counterpart; the reference's library calls tune
 * themselves).  The autotuner (euvlitho_b200.autotune) times the candidates
 * on the device and writes its picks here; value 0 clears an entry, get
 * returns 0 when there is none.  Process-wide, all devices. */
#define EUV_KNOB_ABBE_SPLIT 1 /* key (n_units, n_src) of euv_abbe: CTAs sharing a unit's
                                 sources, 1..64 (built in: fills the waves of resident CTAs) */
#define EUV_KNOB_LU_CLUSTER 2 /* key (n, batch) of the LU: smallest CTA cluster of a panel,
                                 1, 2, 4 or 8 (built in: the fewest CTAs that hold the rows) */
#define EUV_KNOB_ZGEMM_ROWS 3 /* key (m, batch) of the FP64 GEMM: row tile 64 or 32 */
#define EUV_KNOB_LU_SUBST_COLS 4 /* key (n, batch) of an LU solve: right-hand sides per CTA,
                                    8 or 12 (built in: 12 where that takes fewer waves,
                                    or as many when empty source slots are skipped) */
int euv_tune_set(int knob, int k0, int k1, int value);
int euv_tune_get(int knob, int k0, int k1);
void euv_tune_clear(void);

/* One device thread waits until *d_flag != 0, with the bounded spin that every
 * device wait of the library uses (limit_ns, at most 2e9); on expiry it ORs
 * EUV_STATUS_TIMEOUT into *d_status and returns.  No reference counterpart:
 * it lets a caller check that an expired wait comes back as a status while
 * the context stays usable. */
int euv_wait_probe(const int* d_flag, long long limit_ns, int* d_status, void* stream);

/* Batched LU with partial pivoting, in place (replaces the getrf branch of
 * matinv, header.h:1518-1529).  d_ipiv[b][j] (0-based row swapped with j);
 * d_info[b] = 0 or 1 + first zero pivot column. */
size_t euv_lu_workspace_bytes(int n, int batch);
int euv_lu_factor(int n, euv_c64* d_a, int lda, long long stride_a, int* d_ipiv, int* d_info,
                  int batch, void* stream);
/* Solve A X = B with the factors (replaces getrs, header.h:1531-1533). */
int euv_lu_solve(int n, int nrhs, const euv_c64* d_lu, int lda, long long stride_a,
                 const int* d_ipiv, euv_c64* d_b, int ldb, long long stride_b, int batch,
                 void* stream);

/* Matrix functions of a slice: for each b, C[b] = cos(sqrt(D) d[b]) and
 * S[b] = sin(sqrt(D) d[b]) / sqrt(D), by Taylor series and double-angle steps.
 * The outputs of absorberS0 / absorberS depend on their eigen-decomposition
 * D = W diag(al^2) W^-1 only through these two entire functions of D.
 * At most m_max double-angle steps are taken; a matrix whose norm asks for
 * more gets m_max, and this call reports that nowhere (euv_amp reports it as
 * EUV_STATUS_STEPS_CLAMPED): choose m_max with 2^m_max >= ||D||_1 d^2. */
size_t euv_matfun_workspace_bytes(int n, int batch);
int euv_matfun_cs(int n, const euv_c64* d_d, const double* d_thick, euv_c64* d_cos,
                  euv_c64* d_sin, int batch, int m_max, int precision, void* d_work,
                  size_t work_bytes, void* stream);

/* Same as euv_matfun_cs (FP64), but without a workspace: no counterpart in
 * the reference, which allocates on every call.
 *
 * For callers that cannot allocate device memory: plug-ins whose host
 * application owns all device memory through its own allocator and hands out
 * none for scratch, hosts with a fixed device-memory budget set at start-up,
 * and latency-critical loops that must not call cudaMalloc/cudaFree because
 * those calls can synchronise the whole device.  The caller passes only the
 * inputs and outputs; the scratch space is a fixed array of
 * EUV_NOALLOC_SCRATCH_BYTES (16 MiB) inside the library, resident on every GPU
 * that loads it until the process exits.  The function calls no allocator.
 *
 *  - Limit: 5*n*n*batch*16 bytes (+ a few hundred) must fit in the array, e.g.
 *    n = 121 up to batch 14, n = 256 up to batch 3.  Larger requests return
 *    EUV_ERR_BAD_ARG with a message and launch nothing.
 *  - The first call on each device looks up the array's device address
 *    (cudaGetSymbolAddress, with that device current); make that first call
 *    before any stream capture.  The address is kept for the life of the
 *    process: after cudaDeviceReset (or any teardown of the device's primary
 *    context) it is stale, so do not call this entry point after a reset.
 *  - As in euv_matfun_cs, the double-angle steps are capped at m_max and a
 *    call that needed more is not reported (no status word): pass an m_max
 *    with 2^m_max >= ||D||_1 * max(d)^2 (about 8 covers an absorber slice of
 *    tens of nm).
 *  - All calls share the one array and it keeps the last call's contents (the
 *    function clears what must start at zero).  Calls whose GPU work overlaps,
 *    e.g. on two streams at once, race on it: order them on one stream or
 *    with events. */
#define EUV_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
int euv_matfun_cs_noalloc(int n, const euv_c64* d_d, const double* d_thick, euv_c64* d_cos,
                          euv_c64* d_sin, int batch, int m_max, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* EUVL_B200_H */
