// Blackwell (sm_100a) tensor-core plumbing shared by the tcgen05 kernels (the
// mixed-precision complex GEMM, the CNN's convolutions and dense layers):
// mbarriers with bounded waits, TMA tensor loads, UMMA shared-memory
// descriptors for 64-byte-swizzled K-major tiles, tcgen05.mma of kind tf32
// (the CNN; the mixed GEMM issues kind::f16 itself), TMEM loads, the
// FP64/FP32 -> (hi, lo) TF32 split and the driver's tensor-map encoder.
#pragma once
#include <cuda.h>
#include "common.cuh"

namespace euv {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: false after limit_ns (the status word gets EUV_STATUS_TIMEOUT
// and the CTA's abort flag is raised) or when another role already gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  volatile int* abort_flag, int* err,
                                                  unsigned long long limit_ns) {
  const int r = bounded_spin([&] { return mbar_try(bar, parity); },
                             [&] { return *abort_flag != 0; }, limit_ns);
  if (r == 1) return true;
  if (r < 0) {
    *abort_flag = 1;
    atomicOr(err, EUV_STATUS_TIMEOUT);
  }
  return false;
}
// Wait that only gives up on the clock (teardown: copies / MMAs in flight).
__device__ __forceinline__ void mbar_drain(uint64_t* bar, uint32_t parity,
                                           unsigned long long limit_ns) {
  const unsigned long long t0 = globaltimer();
  while (!mbar_try(bar, parity) && globaltimer() - t0 < limit_ns) {
  }
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, int c3, int c4, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4),
      "r"(smem_u32(bar))
      : "memory");
}
// K-major operand, 64-byte swizzle: 8-row atoms of 512 B (SBO), version 1.
__device__ __forceinline__ uint64_t umma_desc_sw64(const void* tile) {
  const uint64_t addr = smem_u32(tile);
  uint64_t d = 0;
  d |= (addr >> 4) & 0x3FFFull;          // start address
  d |= (uint64_t)1 << 16;                // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;       // stride byte offset: 8 rows x 64 B
  d |= (uint64_t)1 << 46;                // descriptor version (sm_100)
  d |= (uint64_t)4 << 61;                // SWIZZLE_64B
  return d;
}
// Instruction descriptor: D f32, A and B tf32 (both K-major), M x N tile.
__host__ __device__ __forceinline__ constexpr uint32_t idesc_tf32_mn(bool neg_a, int m, int n) {
  return (1u << 4)                        // D: F32
         | (2u << 7) | (2u << 10)         // A, B: TF32
         | ((neg_a ? 1u : 0u) << 13)      // negate A
         | ((uint32_t)(n >> 3) << 17)     // N
         | ((uint32_t)(m >> 4) << 24);    // M
}
__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(slot)),
               "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t tmem, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols)
               : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// x = hi + lo with hi = x rounded to TF32 (nearest, ties away) and lo the
// remainder rounded to TF32: hi*hi + hi*lo + lo*hi then carries about 22
// significant bits of each product.
__device__ __forceinline__ float tf32_round(float f) {
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(f));
  return __uint_as_float(h);
}
__device__ __forceinline__ void split_tf32(double x, float& hi, float& lo) {
  hi = tf32_round((float)x);
  lo = (float)(x - (double)hi);
}
__device__ __forceinline__ void split_tf32f(float x, float& hi, float& lo) {
  hi = tf32_round(x);
  lo = tf32_round(x - hi);  // x - hi is exact in fp32
}

// ------------------------------------------------------------------ host
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static inline EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// fp32 tensor map, 64-byte swizzle, zero fill outside the tensor.  dims[0] is
// the contiguous K (channel) axis; strides are in bytes for dims 1..rank-1.
static inline int make_map_f32(CUtensorMap* map, void* base, int rank, const cuuint64_t* dims,
                               const cuuint64_t* strides, const cuuint32_t* box) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) {
    euv_set_error("cuTensorMapEncodeTiled is not available from the driver");
    return EUV_ERR_CUDA;
  }
  cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (cuuint32_t)rank, base, dims, strides,
                   box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    euv_set_error("cuTensorMapEncodeTiled failed (%d), rank %d, dims %llu x %llu", (int)r, rank,
                  (unsigned long long)dims[0], (unsigned long long)dims[1]);
    return EUV_ERR_CUDA;
  }
  return EUV_OK;
}

}  // namespace euv
