// Mixed-precision complex GEMM (bulk products of the mixed form).
#include "common.cuh"

namespace euv {

size_t gemm_mixed_workspace_bytes(int m, int n, int k, int batch) {
  (void)m; (void)n; (void)k; (void)batch;
  return 0;
}

int gemm_mixed(int, int, int, cplx, const double*, const double2*, long long, long long,
               const double2*, long long, long long, cplx, double2*, long long, long long, cplx,
               int, const int*, int, void*, size_t, cudaStream_t) {
  euv_set_error("mixed precision GEMM is not available in this build");
  return EUV_ERR_BAD_ARG;
}

}  // namespace euv
