// The reference-side binding of ampS (cnn/include/header.h:1208-1213): the body
// of ampS replaced by calls into libeuvl_b200.so, keeping the reference's
// signature so that intensity.cpp and m3d.cpp compile unchanged around it.
// Eigen is not needed: the amplitudes are std::vector<std::complex<double>>
// where the reference has Eigen::VectorXcd (Ax[ls + lsmaxX][ms + lsmaxY][n]).
//
// Build: g++ -std=c++17 -I<repo>/include -I<cuda>/include ... -L<repo>/euvlitho_b200
//        -leuvl_b200 -L<cuda>/lib64 -lcudart
#include "ampS_shim.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>

#include "euvl_b200.h"

namespace {

void cuda_ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}
void euv_ok(int rc, const char* what) {
  if (rc != EUV_OK) throw std::runtime_error(std::string(what) + ": " + euv_last_error());
}

// A device buffer released at scope exit.
struct Dev {
  void* p = nullptr;
  explicit Dev(size_t bytes) { cuda_ok(cudaMalloc(&p, bytes ? bytes : 1), "cudaMalloc"); }
  ~Dev() { cudaFree(p); }
  Dev(const Dev&) = delete;
  Dev& operator=(const Dev&) = delete;
  template <typename T>
  T* as() const { return reinterpret_cast<T*>(p); }
};

template <typename T>
void upload(Dev& d, const T* h, size_t n) {
  cuda_ok(cudaMemcpy(d.p, h, n * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
}

euv_c64 c64(std::complex<double> z) { return euv_c64{z.real(), z.imag()}; }

}  // namespace

// The multilayer of header.h:1217-1230 (refractive indices; permittivity = n^2).
euv_stack reference_stack(int NML) {
  auto eps = [](double re, double im) { return c64(std::complex<double>(re, im) * std::complex<double>(re, im)); };
  euv_stack s;
  s.eps_mo = eps(0.9238, 0.006435);
  s.eps_si = eps(0.999, 0.001826);
  s.eps_ru = eps(0.8863, 0.01706);
  s.eps_mosi2 = eps(0.9693, 0.004333);
  s.eps_rusi = eps(0.9099, 0.01547);
  s.eps_sio2 = eps(0.978, 0.01083);
  s.d_mo = 2.052;
  s.d_mosi = 1.661;
  s.d_si = 2.283;
  s.d_simo = 1.045;
  s.d_siru = 0.8;
  s.d_ru = 2.5;
  s.nml = NML;
  return s;
}

void ampS(char polar, AmpGrid& Ax, int NDIVX, int NDIVY, int* mask2d, int LMAX, int Lrange2,
          int MMAX, int Mrange2, int Nrange, std::vector<int>& lindex, std::vector<int>& mindex,
          int FDIVX, int FDIVY, double NA, int MX, int MY, double dx, double dy, double lambda,
          int NABS, int NML, int lsmaxX, int lsmaxY, double k, double kx0, double ky0,
          std::vector<std::complex<double>>& eabs, std::vector<double>& dabs,
          std::vector<std::complex<double>>& cexpX, std::vector<std::complex<double>>& cexpY) {
  (void)Lrange2;
  (void)Mrange2;
  (void)cexpX;  // the library forms its own DFT twiddles
  (void)cexpY;
  if (NABS < 1 || NABS > EUV_MAX_SLICES) throw std::runtime_error("ampS: NABS out of range");
  // 1. mask2d (one int per pixel, index NDIVX*j + i) -> mask.bin bits, MSB first
  std::vector<uint8_t> bits((size_t)NDIVX * NDIVY / 8, 0);
  for (size_t i = 0; i < (size_t)NDIVX * NDIVY; ++i)
    if (mask2d[i]) bits[i >> 3] |= (uint8_t)(0x80u >> (i & 7));
  Dev d_bits(bits.size());
  upload(d_bits, bits.data(), bits.size());

  // 2. absorber-indicator spectrum at orders -2LMAX..2LMAX x -2MMAX..2MMAX; the
  //    reference uses the one mask for every slice (header.h:1243-1251)
  const int lh = 2 * LMAX, mh = 2 * MMAX;
  const size_t S = (size_t)(2 * lh + 1) * (2 * mh + 1);
  Dev d_spec(sizeof(euv_c64) * S * NABS);
  {
    const size_t wb = euv_mask_spectrum_workspace_bytes(1, NDIVX, NDIVY, FDIVX, FDIVY, lh, mh);
    Dev d_w(wb);
    euv_ok(euv_mask_spectrum(d_bits.as<uint8_t>(), 1, NDIVX, NDIVY, FDIVX, FDIVY, lh, mh, 0, 0,
                             d_spec.as<euv_c64>(), d_w.p, wb, nullptr),
           "euv_mask_spectrum");
    for (int n = 1; n < NABS; ++n)
      cuda_ok(cudaMemcpy(d_spec.as<euv_c64>() + (size_t)n * S, d_spec.p, S * sizeof(euv_c64),
                         cudaMemcpyDeviceToDevice),
              "cudaMemcpy D2D");
  }

  // 3. source columns: the NA circle of header.h:1394-1397, with 2 kz (1401-1409)
  std::vector<int> src, ls_of, ms_of;
  std::vector<double> kz2;
  const double pi = std::atan(1.0) * 4.0;
  for (int ls = -lsmaxX; ls <= lsmaxX; ls++)
    for (int ms = -lsmaxY; ms <= lsmaxY; ms++) {
      const double a = ls * MX / dx, b = ms * MY / dy, r = NA / lambda;
      if (a * a + b * b > r * r) continue;
      int idx = -1;
      for (int i = 0; i < Nrange; i++)
        if (lindex[i] == ls && mindex[i] == ms) idx = i;
      const double kx = kx0 + ls * 2. * pi / dx, ky = ky0 + ms * 2. * pi / dy;
      src.push_back(idx);
      kz2.push_back(2. * std::sqrt(k * k - kx * kx - ky * ky));
      ls_of.push_back(ls);
      ms_of.push_back(ms);
    }
  const int ns = (int)src.size();

  // 4. one unit (this family and polarisation) on the device
  Dev d_l(sizeof(int) * Nrange), d_m(sizeof(int) * Nrange);
  upload(d_l, lindex.data(), Nrange);
  upload(d_m, mindex.data(), Nrange);
  const double h_kx0 = kx0, h_ky0 = ky0;
  const int h_pol = polar == 'X' ? 0 : 1, h_spec = 0, h_zero = 0;
  Dev d_kx0(sizeof(double)), d_ky0(sizeof(double)), d_pol(sizeof(int)), d_sp(sizeof(int));
  upload(d_kx0, &h_kx0, 1);
  upload(d_ky0, &h_ky0, 1);
  upload(d_pol, &h_pol, 1);
  upload(d_sp, &h_spec, 1);
  Dev d_src(sizeof(int) * ns), d_kz2(sizeof(double) * ns), d_status(sizeof(int));
  upload(d_src, src.data(), ns);
  upload(d_kz2, kz2.data(), ns);
  upload(d_status, &h_zero, 1);

  euv_amp_desc d;
  std::memset(&d, 0, sizeof(d));
  d.n_orders = Nrange;
  d.lmax = LMAX;
  d.mmax = MMAX;
  d.d_lindex = d_l.as<int>();
  d.d_mindex = d_m.as<int>();
  d.dx = dx;
  d.dy = dy;
  d.k = k;
  d.n_slices = NABS;
  for (int n = 0; n < NABS; ++n) {
    d.eabs[n] = c64(eabs[n]);
    d.dabs[n] = dabs[n];
  }
  d.refresh_sigma = 0;  // the reference's sigma quirk (header.h:1327-1353)
  d.stack = reference_stack(NML);
  d.n_units = 1;
  d.d_kx0 = d_kx0.as<double>();
  d.d_ky0 = d_ky0.as<double>();
  d.d_polar = d_pol.as<int>();
  d.d_spec = d_sp.as<int>();
  d.n_src = ns;
  d.d_src_order = d_src.as<int>();
  d.d_src_2kz = d_kz2.as<double>();
  d.precision = EUV_PREC_FP64;
  d.m_max = 0;
  d.k0_max = std::max(std::fabs(kx0), std::fabs(ky0));
  d.d_status = d_status.as<int>();
  const size_t wa = euv_amp_workspace_bytes(&d);
  if (wa == 0) throw std::runtime_error(std::string("euv_amp_workspace_bytes: ") + euv_last_error());
  Dev d_wa(wa), d_ax(sizeof(euv_c64) * (size_t)Nrange * ns);
  euv_ok(euv_amp(&d, d_spec.as<euv_c64>(), d_ax.as<euv_c64>(), d_wa.p, wa, nullptr), "euv_amp");

  // 5. back into the caller's layout; a device-side failure raises
  std::vector<std::complex<double>> h((size_t)Nrange * ns);
  cuda_ok(cudaMemcpy(h.data(), d_ax.p, h.size() * sizeof(euv_c64), cudaMemcpyDeviceToHost),
          "cudaMemcpy D2H");
  int status = 0;
  cuda_ok(cudaMemcpy(&status, d_status.p, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
  if (status) throw std::runtime_error("euv_amp reported device status " + std::to_string(status));
  for (int s = 0; s < ns; ++s) {
    std::vector<std::complex<double>>& v = Ax[ls_of[s] + lsmaxX][ms_of[s] + lsmaxY];
    v.assign(h.begin() + (size_t)s * Nrange, h.begin() + (size_t)(s + 1) * Nrange);
  }
}
