// ampS with the reference's signature (cnn/include/header.h:1208-1213), its
// amplitudes as std::vector<std::complex<double>> in place of Eigen::VectorXcd:
// Ax[ls + lsmaxX][ms + lsmaxY][n] for the NA-circle source orders (ls, ms).
#pragma once
#include <complex>
#include <vector>

#include "euvl_b200.h"

using AmpGrid = std::vector<std::vector<std::vector<std::complex<double>>>>;

euv_stack reference_stack(int NML);

void ampS(char polar, AmpGrid& Ax, int NDIVX, int NDIVY, int* mask2d, int LMAX, int Lrange2,
          int MMAX, int Mrange2, int Nrange, std::vector<int>& lindex, std::vector<int>& mindex,
          int FDIVX, int FDIVY, double NA, int MX, int MY, double dx, double dy, double lambda,
          int NABS, int NML, int lsmaxX, int lsmaxY, double k, double kx0, double ky0,
          std::vector<std::complex<double>>& eabs, std::vector<double>& dabs,
          std::vector<std::complex<double>>& cexpX, std::vector<std::complex<double>>& cexpY);
