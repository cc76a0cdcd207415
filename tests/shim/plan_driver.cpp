// The reference drivers ported onto the library's C ABI, with no Python:
// intensity.cpp main (Abbe image -> emint.csv), m3d.cpp main (M3D parameters)
// through the plan API, and the ampS shim (ampS_shim.cpp) called the way
// intensity.cpp:241-246 calls ampS.  The tests compile and run it.
//
//   plan_driver intensity <config.bin> <mask.bin> <outdir>
//       every clip of mask.bin (back-to-back rasters): image.bin (doubles
//       [clip][pol][xdiv][ydiv]) and emint.csv of clip 0, polarisation 0 in the
//       reference's format (intensity.cpp:390-408)
//   plan_driver m3d <config.bin> <mask.bin> <outdir>
//       m3d.bin: a0, ax, ay [clip][ncut] complex (m3d.cpp:197-558)
//   plan_driver amps <config.bin> <mask.bin> <outdir>
//       ax.bin: ampS of the first clip at the chief ray for polarisation
//       pols[0], Ax[na source][n_orders] complex, NA sources ls outer / ms inner
// config.bin holds one euv_config (the bytes of the C struct).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "ampS_shim.h"
#include "euvl_b200.h"

namespace {

void cuda_ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}
void euv_ok(int rc, const char* what) {
  if (rc != EUV_OK) throw std::runtime_error(std::string(what) + ": " + euv_last_error());
}

struct Dev {
  void* p = nullptr;
  explicit Dev(size_t bytes) { cuda_ok(cudaMalloc(&p, bytes ? bytes : 1), "cudaMalloc"); }
  ~Dev() { cudaFree(p); }
  Dev(const Dev&) = delete;
  Dev& operator=(const Dev&) = delete;
};

std::vector<char> read_file(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot read " + path);
  return std::vector<char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

void write_file(const std::string& path, const void* data, size_t bytes) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(data), (std::streamsize)bytes);
  if (!f) throw std::runtime_error("cannot write " + path);
}

struct Plan {
  euv_plan* p = nullptr;
  ~Plan() { euv_plan_destroy(p); }
};

int run(const std::string& mode, const std::string& cfg_path, const std::string& mask_path,
        const std::string& out) {
  const std::vector<char> cb = read_file(cfg_path);
  if (cb.size() != sizeof(euv_config)) throw std::runtime_error("config.bin has the wrong size");
  euv_config cfg;
  std::memcpy(&cfg, cb.data(), sizeof(cfg));
  const std::vector<char> mask = read_file(mask_path);
  const size_t nb = (size_t)cfg.ndivx * cfg.ndivy / 8;
  if (mask.empty() || mask.size() % nb) throw std::runtime_error("mask.bin size");
  const int n_clips = (int)(mask.size() / nb);

  Plan plan;
  euv_ok(euv_plan_create(&cfg, &plan.p), "euv_plan_create");
  euv_plan_info I;
  euv_ok(euv_plan_get_info(plan.p, &I), "euv_plan_get_info");

  if (mode == "amps") {
    // intensity.cpp calls ampS with its own order set and optics: take them
    // from the plan's tables and the configuration
    std::vector<int> lindex(I.n_orders), mindex(I.n_orders);
    euv_ok(euv_plan_get_orders(plan.p, lindex.data(), mindex.data()), "euv_plan_get_orders");
    std::vector<int> mask2d((size_t)cfg.ndivx * cfg.ndivy);
    for (size_t i = 0; i < mask2d.size(); ++i)
      mask2d[i] = (mask[i >> 3] >> (7 - (i & 7))) & 1;
    std::vector<std::complex<double>> eabs(cfg.n_slices);
    std::vector<double> dabs(cfg.n_slices);
    for (int n = 0; n < cfg.n_slices; ++n) {
      eabs[n] = {cfg.eabs[n].re, cfg.eabs[n].im};
      dabs[n] = cfg.dabs[n];
    }
    std::vector<std::complex<double>> cexpX, cexpY;
    AmpGrid Ax(2 * I.lsx + 1, std::vector<std::vector<std::complex<double>>>(2 * I.lsy + 1));
    ampS(cfg.pols[0] == 0 ? 'X' : 'Y', Ax, cfg.ndivx, cfg.ndivy, mask2d.data(), I.lmax,
         4 * I.lmax + 1, I.mmax, 4 * I.mmax + 1, I.n_orders, lindex, mindex, I.fdivx, I.fdivy,
         cfg.na, cfg.mx, cfg.my, (double)cfg.ndivx, (double)cfg.ndivy, cfg.wavelength,
         cfg.n_slices, cfg.stack.nml, I.lsx, I.lsy, I.k, I.kx0, I.ky0, eabs, dabs, cexpX, cexpY);
    std::vector<int> nl(I.n_na_sources), nm(I.n_na_sources);
    euv_ok(euv_plan_get_na_sources(plan.p, nl.data(), nm.data()), "euv_plan_get_na_sources");
    std::vector<std::complex<double>> flat;
    for (int s = 0; s < I.n_na_sources; ++s) {
      const auto& v = Ax[nl[s] + I.lsx][nm[s] + I.lsy];
      if ((int)v.size() != I.n_orders) throw std::runtime_error("ampS left a source column empty");
      flat.insert(flat.end(), v.begin(), v.end());
    }
    write_file(out + "/ax.bin", flat.data(), flat.size() * sizeof(flat[0]));
    return 0;
  }

  cudaStream_t stream;
  cuda_ok(cudaStreamCreate(&stream), "cudaStreamCreate");
  const size_t tb = euv_plan_device_bytes(plan.p, n_clips);
  Dev d_tables(tb), d_masks(mask.size());
  euv_ok(euv_plan_upload(plan.p, n_clips, d_tables.p, tb, stream), "euv_plan_upload");
  cuda_ok(cudaMemcpyAsync(d_masks.p, mask.data(), mask.size(), cudaMemcpyHostToDevice, stream),
          "cudaMemcpyAsync");
  const uint8_t* dm = reinterpret_cast<const uint8_t*>(d_masks.p);
  if (mode == "intensity") {
    const size_t wb = euv_plan_intensity_workspace_bytes(plan.p, n_clips, 1);
    const size_t n_img = (size_t)n_clips * I.n_pols * I.xdiv * I.ydiv;
    Dev d_work(wb), d_img(n_img * sizeof(double));
    euv_ok(euv_plan_intensity(plan.p, dm, n_clips, 1, reinterpret_cast<double*>(d_img.p),
                              d_work.p, wb, stream),
           "euv_plan_intensity");
    std::vector<double> img(n_img);
    cuda_ok(cudaMemcpyAsync(img.data(), d_img.p, n_img * sizeof(double), cudaMemcpyDeviceToHost,
                            stream),
            "cudaMemcpyAsync");
    euv_ok(euv_plan_check(plan.p, nullptr, stream), "euv_plan_check");
    write_file(out + "/image.bin", img.data(), n_img * sizeof(double));
    // emint.csv of clip 0, polarisation 0: rows y = YDIV-1 .. 0, each value
    // followed by a comma, 6 significant digits (ostream default)
    std::ofstream f(out + "/emint.csv");
    for (int j = I.ydiv - 1; j >= 0; j--) {
      for (int i = 0; i < I.xdiv; i++) f << img[(size_t)i * I.ydiv + j] << ",";
      f << std::endl;
    }
  } else if (mode == "m3d") {
    const size_t wb = euv_plan_m3d_workspace_bytes(plan.p, n_clips, 1);
    const size_t n = (size_t)n_clips * I.ncut;
    Dev d_work(wb), d_out(3 * n * sizeof(euv_c64));
    euv_c64* o = reinterpret_cast<euv_c64*>(d_out.p);
    euv_ok(euv_plan_m3d(plan.p, dm, n_clips, 1, o, o + n, o + 2 * n, d_work.p, wb, stream),
           "euv_plan_m3d");
    std::vector<euv_c64> h(3 * n);
    cuda_ok(cudaMemcpyAsync(h.data(), o, h.size() * sizeof(euv_c64), cudaMemcpyDeviceToHost,
                            stream),
            "cudaMemcpyAsync");
    euv_ok(euv_plan_check(plan.p, nullptr, stream), "euv_plan_check");
    write_file(out + "/m3d.bin", h.data(), h.size() * sizeof(euv_c64));
  } else {
    throw std::runtime_error("unknown mode " + mode);
  }
  cuda_ok(cudaStreamDestroy(stream), "cudaStreamDestroy");
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: %s intensity|m3d|amps <config.bin> <mask.bin> <outdir>\n", argv[0]);
    return 2;
  }
  try {
    return run(argv[1], argv[2], argv[3], argv[4]);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "plan_driver: %s\n", e.what());
    return 1;
  }
}
