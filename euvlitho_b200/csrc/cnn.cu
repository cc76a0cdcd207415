// CNN predict of the M3D parameters: the six networks of
// cnn/cnn/predict/predict.py (re0, im0, rex, imx, rey, imy; classes CNNmodel
// and CNNmodels, predict.py:16-88), run on masks downsampled as compmask
// (cnn/cnn/predict/compmask.py:17-41: 2048^2 bits -> 512^2 box means), with
// the outputs divided by the per-order factors (predict.py:108-121).
//
// Network (per model, input 1 x 512 x 512 fp32):
//   5 x [conv 3x3, circular padding 1, + bias -> ReLU -> max-pool 2x2 ->
//        BatchNorm (eval: running statistics)]      channels 1-16-32-64-128-256
//   flatten (c, h, w) of 256 x 16 x 16 -> fc1 65536 -> 4096, ReLU -> fc2 -> n_out.
//
// B200 form:
//   cnn_input_kernel   bits -> 512^2 box means (popcount of 4x4 bit boxes / 16);
//   cnn_conv1_kernel   conv1 (one input channel, 9 taps: CUDA cores, FP32) for all
//                      models at once, fused bias/ReLU/pool/BN;
//   cnn_conv_kernel    conv2..conv5 as persistent implicit GEMMs on tcgen05: M = 128
//                      output pixels (an 8 x 16 block), N = output channels,
//                      K = 9 taps x input channels.  Activations live as TF32
//                      (hi, lo) planes in NHWC with a one-pixel circular halo,
//                      so each K block (one tap, 16 channels) is one 5-D TMA box
//                      of the padded planes at the tap's offset.  The epilogue
//                      takes the 2 x 2 pool maxima across lanes (shuffles),
//                      adds bias, ReLU, BN, splits into (hi, lo) and writes the
//                      next layer's padded planes including the halo copies;
//   cnn_fc_kernel      fc1 and fc2 as split-K GEMMs (A = weight planes, N =
//                      masks), FP32 partial sums reduced by cnn_fc*_finish.
// Products are TF32x3 (hi*hi + hi*lo + lo*hi, FP32 accumulation), about FP32
// accuracy; split-K keeps each accumulator's K run short (the tensor-core FP32
// accumulation error grows with it).
#include "tcgen05.cuh"

namespace euv {

constexpr int CNN_BITS_SIDE = 2048;
constexpr int CNN_IN = 512;
constexpr int CNN_FC1_K = 16 * 16 * 256;
constexpr int CNN_FC1_N = 4096;
constexpr int CNN_FC1_SPLIT = 16;
constexpr int CNN_FC2_SPLIT = 4;
constexpr int CNN_THREADS = 192;
constexpr int CNN_BK = 16;
constexpr int CNN_A_TILE = 128 * CNN_BK * 4;  // 8 KB per plane
constexpr unsigned long long CNN_TIMEOUT_NS = 2000000000ull;

__host__ __device__ constexpr int cnn_cin(int l) { return l == 0 ? 1 : 8 << l; }
__host__ __device__ constexpr int cnn_cout(int l) { return 16 << l; }
// conv input (= pre-pool output) side of layer l
__host__ __device__ constexpr int cnn_side(int l) { return CNN_IN >> l; }

static inline size_t al256(size_t n) { return (n + 255) / 256 * 256; }  // in floats: 1 KB

// Packed weights (floats, sections 1 KB aligned), every section [model]-major:
//   conv1 w [M][16][9]; per layer l: (l >= 1) w planes [M][2][cout][9 cin] with
//   K = (ky*3 + kx)*cin + c, then bias, bn scale, bn shift [M][cout];
//   fc1 w [M][4096][65536] fp32 (K in (h, w, c) order), bias [M][4096];
//   fc2 w [M][OP][4096] fp32 (rows >= n_out zero), bias [M][OP].
// The fc weights stay fp32 (the fc kernel splits them in shared memory: half
// the HBM stream of stored planes); the conv weights are stored as planes.
struct CnnBlob {
  size_t w[5], bias[5], scale[5], shift[5];
  size_t fc1, fc1_b, fc2, fc2_b, total;
  int op;
};
static CnnBlob cnn_blob(int M, int max_out) {
  CnnBlob b;
  b.op = (max_out + 127) / 128 * 128;
  size_t o = 0;
  for (int l = 0; l < 5; ++l) {
    b.w[l] = o;
    o += al256((size_t)M * (l ? 2 : 1) * cnn_cout(l) * 9 * cnn_cin(l));
    b.bias[l] = o;
    o += al256((size_t)M * cnn_cout(l));
    b.scale[l] = o;
    o += al256((size_t)M * cnn_cout(l));
    b.shift[l] = o;
    o += al256((size_t)M * cnn_cout(l));
  }
  b.fc1 = o;
  o += al256((size_t)M * CNN_FC1_N * CNN_FC1_K);
  b.fc1_b = o;
  o += al256((size_t)M * CNN_FC1_N);
  b.fc2 = o;
  o += al256((size_t)M * b.op * CNN_FC1_N);
  b.fc2_b = o;
  o += al256((size_t)M * b.op);
  b.total = o;
  return b;
}

// Workspace (floats): x0, padded activation planes of conv1..conv4, conv5
// planes (= fc1 input), fc1 partials, fc1 output planes, fc2 partials, status.
struct CnnWork {
  size_t x0, act[5], part1, h, part2, status, total;
};
static CnnWork cnn_work(int M, int B, int op) {
  CnnWork w;
  size_t o = 0;
  w.x0 = o;
  o += al256((size_t)B * CNN_IN * CNN_IN);
  for (int l = 0; l < 5; ++l) {
    const size_t so = (size_t)cnn_side(l) / 2, pad = l < 4 ? 2 : 0;
    w.act[l] = o;
    o += al256((size_t)M * 2 * B * (so + pad) * (so + pad) * cnn_cout(l));
  }
  w.part1 = o;
  o += al256((size_t)CNN_FC1_SPLIT * M * B * CNN_FC1_N);
  w.h = o;
  o += al256((size_t)M * 2 * B * CNN_FC1_N);
  w.part2 = o;
  o += al256((size_t)CNN_FC2_SPLIT * M * B * op);
  w.status = o;
  o += 256;
  w.total = o;
  return w;
}

// ------------------------------------------------------------------ packing

__global__ void cnn_pack_conv1_kernel(const float* w, float* dst) {
  const int t = threadIdx.x;  // 16 x 9
  if (t < 144) dst[t] = w[t];  // torch [16][1][3][3] is already [o][ky*3+kx]
}

// torch [cout][cin][3][3] -> planes [2][cout][9 cin], K = tap*cin + c
__global__ void cnn_pack_conv_kernel(int cout, int cin, const float* w, float* dst) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int kk = 9 * cin;
  if (t >= cout * kk) return;
  const int o = t / kk, k = t % kk, tap = k / cin, c = k % cin;
  float hi, lo;
  split_tf32f(w[((long long)o * cin + c) * 9 + tap], hi, lo);
  dst[t] = hi;
  dst[(long long)cout * kk + t] = lo;
}

// torch [rows][K] -> fp32 [rows_pad][K] (rows >= rows zero); perm: K from
// (c, h, w) of a 256 x 16 x 16 map to (h, w, c)
__global__ void cnn_pack_fc_kernel(int rows, int rows_pad, int K, int perm, const float* w,
                                   float* dst) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)rows_pad * K;
  if (t >= n) return;
  const int r = (int)(t / K), kn = (int)(t % K);
  float v = 0.0f;
  if (r < rows) {
    const int ko = perm ? (kn % 256) * 256 + kn / 256 : kn;
    v = w[(long long)r * K + ko];
  }
  dst[t] = v;
}

// bias (zero beyond n), BN eval as scale = gamma / sqrt(var + eps),
// shift = beta - mean * scale
__global__ void cnn_pack_vec_kernel(int n, int n_pad, const float* bias, const float* gamma,
                                    const float* beta, const float* mean, const float* var,
                                    double eps, float* d_bias, float* d_scale, float* d_shift) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_pad) return;
  d_bias[t] = t < n ? bias[t] : 0.0f;
  if (d_scale) {
    const double s = (double)gamma[t] / sqrt((double)var[t] + eps);
    d_scale[t] = (float)s;
    d_shift[t] = (float)((double)beta[t] - (double)mean[t] * s);
  }
}

// ------------------------------------------------------------------ input + conv1

// compmask: x0[r][c] = (1/16) * number of set bits in rows 4r..4r+3, columns
// 4c..4c+3 of the MSB-first 2048 x 2048 bit raster (a nibble of 4 bytes).
__global__ void cnn_input_kernel(const uint8_t* bits, float* x0) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= CNN_IN * CNN_IN) return;
  const int img = blockIdx.y;
  const int r = t / CNN_IN, c = t % CNN_IN;
  const uint8_t* m = bits + (size_t)img * (CNN_BITS_SIDE * CNN_BITS_SIDE / 8);
  int cnt = 0;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const uint32_t byte = m[(size_t)(4 * r + a) * (CNN_BITS_SIDE / 8) + (c >> 1)];
    cnt += __popc((c & 1) ? (byte & 0xFu) : (byte >> 4));
  }
  x0[(size_t)img * CNN_IN * CNN_IN + t] = (float)cnt * 0.0625f;
}

// Writes 16 channels [c0, c0+16) of pooled pixel (py, px) to the (hi, lo)
// planes of an activation [img][so+2p][so+2p][C] (plane stride `plane`), with
// the circular halo copies when padded.
__device__ __forceinline__ void cnn_store16(float* hi_base, long long plane, int so, int pad,
                                            int cch, int py, int px, int c0, const float* hi,
                                            const float* lo) {
  int ry[2], rx[2], nr = 1, nc = 1;
  ry[0] = py + pad;
  rx[0] = px + pad;
  if (pad) {
    if (py == 0) ry[nr++] = so + 1;
    if (py == so - 1) ry[nr++] = 0;
    if (px == 0) rx[nc++] = so + 1;
    if (px == so - 1) rx[nc++] = 0;
  }
  const int hp = so + 2 * pad;
  for (int i = 0; i < nr; ++i)
    for (int j = 0; j < nc; ++j) {
      float* d = hi_base + ((long long)ry[i] * hp + rx[j]) * cch + c0;
      float4* dh = reinterpret_cast<float4*>(d);
      float4* dl = reinterpret_cast<float4*>(d + plane);
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        dh[v] = make_float4(hi[4 * v], hi[4 * v + 1], hi[4 * v + 2], hi[4 * v + 3]);
        dl[v] = make_float4(lo[4 * v], lo[4 * v + 1], lo[4 * v + 2], lo[4 * v + 3]);
      }
    }
}

// conv1 (1 -> 16 channels, 512^2) + bias, ReLU, 2x2 max-pool, BN for pooled
// pixel (py, px) of image blockIdx.y, model blockIdx.z.
__global__ void cnn_conv1_kernel(int B, const float* x0, const float* w, const float* bias,
                                 const float* scale, const float* shift, float* out) {
  __shared__ float sw[144], sb[16], ss[16], sh[16];
  const int m = blockIdx.z, img = blockIdx.y;
  for (int i = threadIdx.x; i < 144; i += blockDim.x) sw[i] = w[m * 144 + i];
  if (threadIdx.x < 16) {
    sb[threadIdx.x] = bias[m * 16 + threadIdx.x];
    ss[threadIdx.x] = scale[m * 16 + threadIdx.x];
    sh[threadIdx.x] = shift[m * 16 + threadIdx.x];
  }
  __syncthreads();
  constexpr int SO = CNN_IN / 2;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= SO * SO) return;
  const int py = t / SO, px = t % SO;
  const float* X = x0 + (size_t)img * CNN_IN * CNN_IN;
  float win[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int r = (2 * py - 1 + a) & (CNN_IN - 1);
#pragma unroll
    for (int b = 0; b < 4; ++b) win[a][b] = X[r * CNN_IN + ((2 * px - 1 + b) & (CNN_IN - 1))];
  }
  float hi[16], lo[16];
#pragma unroll
  for (int o = 0; o < 16; ++o) {
    float best = -INFINITY;
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dx = 0; dx < 2; ++dx) {
        float acc = 0.0f;
#pragma unroll
        for (int ky = 0; ky < 3; ++ky)
#pragma unroll
          for (int kx = 0; kx < 3; ++kx) acc = fmaf(sw[o * 9 + ky * 3 + kx], win[dy + ky][dx + kx], acc);
        best = fmaxf(best, acc);
      }
    const float y = fmaxf(best + sb[o], 0.0f) * ss[o] + sh[o];
    split_tf32f(y, hi[o], lo[o]);
  }
  const long long plane = (long long)B * (SO + 2) * (SO + 2) * 16;
  float* base = out + ((long long)m * 2 * B + img) * (SO + 2) * (SO + 2) * 16;
  cnn_store16(base, plane, SO, 1, 16, py, px, 0, hi, lo);
}

// ------------------------------------------------------------------ tcgen05 GEMM

// Shared-memory ring of a TF32x3 GEMM: per stage A (hi, lo) 128 x 16 fp32 and
// B (hi, lo) bn x 16 fp32, 64-byte swizzled K-major.
struct CnnRing {
  uint8_t* base;
  int stage_bytes, b_bytes;
  __device__ uint8_t* a(int s, int pl) const { return base + s * stage_bytes + pl * CNN_A_TILE; }
  __device__ uint8_t* b(int s, int pl) const {
    return base + s * stage_bytes + 2 * CNN_A_TILE + pl * b_bytes;
  }
};

// hi*hi + hi*lo + lo*hi of one 16-wide K block into the accumulator at tmem
__device__ __forceinline__ void cnn_mma_block(const CnnRing& r, int s, uint32_t tmem,
                                              uint32_t idesc, bool first) {
#pragma unroll
  for (int k8 = 0; k8 < CNN_BK / 8; ++k8) {
    const uint64_t ah = umma_desc_sw64(r.a(s, 0) + k8 * 32);
    const uint64_t al = umma_desc_sw64(r.a(s, 1) + k8 * 32);
    const uint64_t bh = umma_desc_sw64(r.b(s, 0) + k8 * 32);
    const uint64_t bl = umma_desc_sw64(r.b(s, 1) + k8 * 32);
    umma_tf32(tmem, ah, bh, idesc, (first && k8 == 0) ? 0u : 1u);
    umma_tf32(tmem, ah, bl, idesc, 1u);
    umma_tf32(tmem, al, bh, idesc, 1u);
  }
}

struct CnnConvArgs {
  int models, batch, side, tiles_x, tiles_img, total_tiles;
  int cin, cout, mt, nbuf, a_stages, b_stages, out_pad;
  const float *bias, *scale, *shift;
  float* out;
  int* err;
};

// bytes of one A plane of a conv stage: the (8 mt + 2) x 16 pixel halo block
// of 16 channels (64 B rows)
__host__ __device__ constexpr int cnn_conv_a_plane(int mt) { return (8 * mt + 2) * 16 * 64; }

// Persistent implicit-GEMM convolution.  A CTA tile is mt blocks of 8 x 16
// output pixels stacked in y (M = 128 pixels each, one TMEM accumulator of
// cout columns each), walked as blockIdx.x, + gridDim.x, ... over (model,
// mask, tile).  Per tile and per (kx, 16-channel chunk) warp 0 loads one
// (8 mt + 2) x 16 halo block of the padded input planes (hi, lo) at x offset
// kx; the three ky taps are that block shifted by ky rows of 16 pixels (a
// 1 KB descriptor offset, a whole number of 64-byte swizzle atoms), each with
// its own weight tile (hi, lo) from a second ring.  Warp 1 issues the TF32x3
// MMAs of all mt blocks against each weight tile; warps 2..5 run the fused
// epilogue of the previous tile meanwhile (nbuf = 2 accumulator sets when
// TMEM holds them).  Barriers: full/empty per A and per B stage, tfull (MMA ->
// epilogue) and tempty (epilogue, 4 warps -> MMA) per accumulator set.  All
// waits bounded; a timeout raises EUV_STATUS_TIMEOUT.
__global__ void __launch_bounds__(CNN_THREADS) cnn_conv_kernel(
    const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
    CnnConvArgs p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const int bn = p.cout, mt = p.mt;
  const int a_plane = cnn_conv_a_plane(mt), b_plane = bn * CNN_BK * 4;
  uint8_t* a_ring = smem;
  uint8_t* b_ring = smem + p.a_stages * 2 * a_plane;
  uint64_t* afull = reinterpret_cast<uint64_t*>(b_ring + p.b_stages * 2 * b_plane);
  uint64_t* aempty = afull + p.a_stages;
  uint64_t* bfull = aempty + p.a_stages;
  uint64_t* bempty = bfull + p.b_stages;
  uint64_t* tfull = bempty + p.b_stages;
  uint64_t* tempty = tfull + 2;
  uint64_t* done = tempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  // epilogue constants of every model: bias | bn scale | bn shift, [models][cout] each
  float* s_vec = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(afull) + 512);
  const int nvec = p.models * bn;
  for (int i = threadIdx.x; i < nvec; i += blockDim.x) {
    s_vec[i] = p.bias[i];
    s_vec[nvec + i] = p.scale[i];
    s_vec[2 * nvec + i] = p.shift[i];
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t tcols = 32;
  while ((int)tcols < p.nbuf * mt * bn) tcols <<= 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < p.a_stages; ++s) {
      mbar_init(&afull[s], 1);
      mbar_init(&aempty[s], 1);
    }
    for (int s = 0; s < p.b_stages; ++s) {
      mbar_init(&bfull[s], 1);
      mbar_init(&bempty[s], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&tfull[i], 1);
      mbar_init(&tempty[i], 4);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(tmem_slot, tcols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int cchunks = p.cin / CNN_BK;
  // tile -> (model, img, y0, x0), model slowest so that concurrent CTAs share weights
  auto decode = [&](int t, int& model, int& img, int& y0, int& x0) {
    const int pt = t % p.tiles_img, mi = t / p.tiles_img;
    img = mi % p.batch;
    model = mi / p.batch;
    y0 = 8 * mt * (pt / p.tiles_x);
    x0 = 16 * (pt % p.tiles_x);
  };

  if (warp == 0) {
    if (lane == 0) {
      int ia = 0, ib = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < p.total_tiles && ok; t += gridDim.x) {
        int model, img, y0, x0;
        decode(t, model, img, y0, x0);
        for (int kx = 0; kx < 3 && ok; ++kx)
          for (int cc = 0; cc < cchunks && ok; ++cc, ++ia) {
            const int sa = ia % p.a_stages;
            if (!mbar_wait_bounded(&aempty[sa], (uint32_t)(((ia / p.a_stages) & 1) ^ 1),
                                   abort_flag, p.err, CNN_TIMEOUT_NS)) {
              ok = false;
              break;
            }
            mbar_expect_tx(&afull[sa], (uint32_t)(2 * a_plane));
            for (int pl = 0; pl < 2; ++pl)
              tma_load_5d(a_ring + (sa * 2 + pl) * a_plane, &tmA, cc * CNN_BK, x0 + kx, y0, img,
                          2 * model + pl, &afull[sa]);
            for (int ky = 0; ky < 3; ++ky, ++ib) {
              const int sb = ib % p.b_stages;
              if (!mbar_wait_bounded(&bempty[sb], (uint32_t)(((ib / p.b_stages) & 1) ^ 1),
                                     abort_flag, p.err, CNN_TIMEOUT_NS)) {
                ok = false;
                break;
              }
              mbar_expect_tx(&bfull[sb], (uint32_t)(2 * b_plane));
              const int k0 = (3 * ky + kx) * p.cin + cc * CNN_BK;
              for (int pl = 0; pl < 2; ++pl)
                tma_load_3d(b_ring + (sb * 2 + pl) * b_plane, &tmB, k0, 0, 2 * model + pl,
                            &bfull[sb]);
            }
          }
      }
      if (!ok) {
        // drain this thread's copies in flight (bounded) before the CTA exits
        for (int j = (ia > p.a_stages ? ia - p.a_stages : 0); j < ia; ++j)
          mbar_drain(&afull[j % p.a_stages], (uint32_t)((j / p.a_stages) & 1), CNN_TIMEOUT_NS);
        for (int j = (ib > p.b_stages ? ib - p.b_stages : 0); j < ib; ++j)
          mbar_drain(&bfull[j % p.b_stages], (uint32_t)((j / p.b_stages) & 1), CNN_TIMEOUT_NS);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_tf32_mn(false, 128, bn);
      int ia = 0, ib = 0, local = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < p.total_tiles && ok; t += gridDim.x, ++local) {
        const int ab = local % p.nbuf, use = local / p.nbuf;
        if (!mbar_wait_bounded(&tempty[ab], (uint32_t)((use & 1) ^ 1), abort_flag, p.err,
                               CNN_TIMEOUT_NS)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t acc = tmem + (uint32_t)(ab * mt * bn);
        for (int kx = 0; kx < 3 && ok; ++kx)
          for (int cc = 0; cc < cchunks && ok; ++cc, ++ia) {
            const int sa = ia % p.a_stages;
            if (!mbar_wait_bounded(&afull[sa], (uint32_t)((ia / p.a_stages) & 1), abort_flag,
                                   p.err, CNN_TIMEOUT_NS)) {
              ok = false;
              break;
            }
            for (int ky = 0; ky < 3; ++ky, ++ib) {
              const int sb = ib % p.b_stages;
              if (!mbar_wait_bounded(&bfull[sb], (uint32_t)((ib / p.b_stages) & 1), abort_flag,
                                     p.err, CNN_TIMEOUT_NS)) {
                ok = false;
                break;
              }
              tc_fence_after();
              const bool first = kx == 0 && cc == 0 && ky == 0;
              const uint8_t* bh = b_ring + (sb * 2) * b_plane;
              const uint8_t* bl = bh + b_plane;
              for (int m = 0; m < mt; ++m) {
                // rows (8 m + ky) * 16 .. + 127 of the halo block
                const uint8_t* ah = a_ring + (sa * 2) * a_plane + (8 * m + ky) * 16 * 64;
                const uint8_t* al = ah + a_plane;
                const uint32_t d = acc + (uint32_t)(m * bn);
#pragma unroll
                for (int k8 = 0; k8 < CNN_BK / 8; ++k8) {
                  const uint64_t dah = umma_desc_sw64(ah + k8 * 32);
                  const uint64_t dal = umma_desc_sw64(al + k8 * 32);
                  const uint64_t dbh = umma_desc_sw64(bh + k8 * 32);
                  const uint64_t dbl = umma_desc_sw64(bl + k8 * 32);
                  umma_tf32(d, dah, dbh, idesc, (first && k8 == 0) ? 0u : 1u);
                  umma_tf32(d, dah, dbl, idesc, 1u);
                  umma_tf32(d, dal, dbh, idesc, 1u);
                }
              }
              umma_commit(&bempty[sb]);
            }
            umma_commit(&aempty[sa]);
          }
        if (ok) umma_commit(&tfull[ab]);
      }
      umma_commit(done);  // always: teardown waits for the MMAs in flight
    }
  } else {
    const int q = warp & 3;
    const uint32_t lane_addr = (uint32_t)(q * 32) << 16;
    // TMEM lane = pixel h*16 + w of an 8 x 16 block: a warp holds rows 2q, 2q+1
    const int h = 2 * q + (lane >> 4), w = lane & 15;
    const bool owner = (lane & 17) == 0;
    const int so = p.side / 2, pad = p.out_pad, hp = so + 2 * pad;
    const long long img_elems = (long long)hp * hp * p.cout;
    const long long plane = (long long)p.batch * img_elems;
    int local = 0;
    for (int t = blockIdx.x; t < p.total_tiles; t += gridDim.x, ++local) {
      const int ab = local % p.nbuf, use = local / p.nbuf;
      const bool waited = mbar_wait_bounded(&tfull[ab], (uint32_t)(use & 1), abort_flag, p.err,
                                            CNN_TIMEOUT_NS) && !*abort_flag;
      if (!__all_sync(0xffffffffu, waited)) break;
      tc_fence_after();
      int model, img, y0, x0;
      decode(t, model, img, y0, x0);
      float* base = p.out + (long long)model * 2 * plane + (long long)img * img_elems;
      const float* bias = s_vec + model * bn;
      const float* scale = bias + nvec;
      const float* shift = scale + nvec;
      for (int m = 0; m < mt; ++m) {
        const int py = (y0 + 8 * m + h) >> 1, px = (x0 + w) >> 1;
        const uint32_t col = (uint32_t)((ab * mt + m) * bn);
        for (int c0 = 0; c0 < p.cout; c0 += 16) {
          uint32_t v[16];
          tmem_ld16(tmem + lane_addr + col + (uint32_t)c0, v);
          tmem_ld_wait();
          float hi[16], lo[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            float f = __uint_as_float(v[j]);
            f = fmaxf(f, __shfl_xor_sync(0xffffffffu, f, 1));
            f = fmaxf(f, __shfl_xor_sync(0xffffffffu, f, 16));
            const int c = c0 + j;
            const float y = fmaxf(f + bias[c], 0.0f) * scale[c] + shift[c];
            split_tf32f(y, hi[j], lo[j]);
          }
          if (owner) cnn_store16(base, plane, so, pad, p.cout, py, px, c0, hi, lo);
        }
      }
      // this warp's TMEM reads are complete: hand the accumulator set back
      tc_fence_before();
      __syncwarp();
      if (lane == 0)
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&tempty[ab]))
                     : "memory");
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    // the MMAs in flight (after an abort) and the final commit's arrival
    mbar_drain(done, 0u, CNN_TIMEOUT_NS);
    tmem_dealloc(tmem, tcols);
  }
}

// Conv stage plan: two accumulator sets (the epilogue of one tile overlaps
// the MMAs of the next), mt = 2 blocks per tile (each weight tile serves 256
// pixels) when TMEM holds 2 x 2 x cout columns, else 1; ring depths from a
// shared-memory budget (two CTAs per SM for the small layers).
struct CnnConvPlan {
  int mt, nbuf, a_stages, b_stages;
  size_t smem;
};
static CnnConvPlan cnn_conv_plan(int cout, int models) {
  CnnConvPlan c;
  c.nbuf = 2;
  c.mt = 2 * 2 * cout <= 512 ? 2 : 1;
  const size_t a = 2 * (size_t)cnn_conv_a_plane(c.mt), b = 2 * (size_t)cout * CNN_BK * 4;
  const size_t fixed = 1024 + 512 + (size_t)12 * models * cout;  // align slack, barriers, table
  const size_t budget = cout <= 64 ? 110 * 1024 : 222 * 1024;
  c.a_stages = 2;
  size_t rest = budget - fixed - c.a_stages * a;
  int bs = (int)(rest / b);
  c.b_stages = bs < 2 ? 2 : (bs > 8 ? 8 : bs);
  c.smem = fixed + c.a_stages * a + c.b_stages * b;
  return c;
}

struct CnnFcArgs {
  int models, batch;
  int bn, nkb, stages;
  int rows, nsplit;
  float* part;
  int* err;
};

// Split-K fully connected layer: A = fp32 weights [M][rows][K] (128 rows per
// CTA), B = activation planes [2M][batch][K] (bn masks per CTA), K range
// split blockIdx.y % nsplit; FP32 partial sums to part[split][model][mask][row].
// The TMA writes the fp32 weight tile into the stage's hi tile; warps 2..5
// split it in place (hi) and into the lo tile (same swizzled positions:
// the transform is elementwise), fence the generic-proxy writes for the
// tensor core and arrive on conv[s]; the MMA warp waits on conv[s].  After
// the K loop the same warps run the epilogue.
__global__ void __launch_bounds__(CNN_THREADS) cnn_fc_kernel(
    const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
    CnnFcArgs p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  CnnRing ring{smem, 2 * CNN_A_TILE + 2 * p.bn * CNN_BK * 4, p.bn * CNN_BK * 4};
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + p.stages * ring.stage_bytes);
  uint64_t* conv = full + p.stages;
  uint64_t* empty = conv + p.stages;
  uint64_t* accum = empty + p.stages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accum + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int model = blockIdx.z;
  const int m0 = 128 * blockIdx.x;
  const int split = blockIdx.y % p.nsplit;
  const int n0 = p.bn * (blockIdx.y / p.nsplit);
  uint32_t tcols = 32;
  while ((int)tcols < p.bn) tcols <<= 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < p.stages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&conv[s], 2);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accum, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(tmem_slot, tcols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int nkb = p.nkb;

  if (warp == 0) {
    if (lane == 0) {
      int issued = 0;
      for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb % p.stages;
        const uint32_t ph = (uint32_t)((kb / p.stages) & 1);
        if (!mbar_wait_bounded(&empty[s], ph ^ 1u, abort_flag, p.err, CNN_TIMEOUT_NS)) break;
        mbar_expect_tx(&full[s], (uint32_t)(CNN_A_TILE + 2 * ring.b_bytes));
        const int k0 = (split * nkb + kb) * CNN_BK;
        tma_load_3d(ring.a(s, 0), &tmA, k0, m0, model, &full[s]);
        for (int pl = 0; pl < 2; ++pl)
          tma_load_3d(ring.b(s, pl), &tmB, k0, n0, 2 * model + pl, &full[s]);
        issued = kb + 1;
      }
      if (*abort_flag) {
        for (int kb = (issued > p.stages ? issued - p.stages : 0); kb < issued; ++kb)
          mbar_drain(&full[kb % p.stages], (uint32_t)((kb / p.stages) & 1), CNN_TIMEOUT_NS);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_tf32_mn(false, 128, p.bn);
      for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb % p.stages;
        const uint32_t ph = (uint32_t)((kb / p.stages) & 1);
        if (!mbar_wait_bounded(&conv[s], ph, abort_flag, p.err, CNN_TIMEOUT_NS)) break;
        tc_fence_after();
        cnn_mma_block(ring, s, tmem, idesc, kb == 0);
        umma_commit(&empty[s]);
      }
      umma_commit(accum);
    }
  } else {
    // weight split, 2048 fp32 of a stage's A tile: warps 2-3 take the even K
    // blocks, warps 4-5 the odd ones (two stages converting at once), 32 per thread
    const int grp = (warp - 2) >> 1;
    const int et = threadIdx.x - 64 - 64 * grp;  // 0..63
    for (int kb = grp; kb < nkb; kb += 2) {
      const int s = kb % p.stages;
      const uint32_t ph = (uint32_t)((kb / p.stages) & 1);
      const bool got = mbar_wait_bounded(&full[s], ph, abort_flag, p.err, CNN_TIMEOUT_NS);
      if (!__all_sync(0xffffffffu, got)) break;
      float4* hi = reinterpret_cast<float4*>(ring.a(s, 0));
      float4* lo = reinterpret_cast<float4*>(ring.a(s, 1));
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int i = et + 64 * u;
        const float4 x = hi[i];
        float4 h, l;
        split_tf32f(x.x, h.x, l.x);
        split_tf32f(x.y, h.y, l.y);
        split_tf32f(x.z, h.z, l.z);
        split_tf32f(x.w, h.w, l.w);
        hi[i] = h;
        lo[i] = l;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0)
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&conv[s]))
                     : "memory");
    }
    const int q = warp & 3;
    const bool waited =
        mbar_wait_bounded(accum, 0u, abort_flag, p.err, CNN_TIMEOUT_NS) && !*abort_flag;
    const bool ok = __all_sync(0xffffffffu, waited);
    tc_fence_after();
    const uint32_t lane_addr = (uint32_t)(q * 32) << 16;
    if (ok) {
      const int row = m0 + q * 32 + lane;
      float* part = p.part + ((long long)split * p.models + model) * p.batch * p.rows;
      for (int c0 = 0; c0 < p.bn; c0 += 16) {
        if (n0 + c0 >= p.batch) break;  // warp-uniform
        uint32_t v[16];
        tmem_ld16(tmem + lane_addr + (uint32_t)c0, v);
        tmem_ld_wait();
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int b = n0 + c0 + j;
          if (b < p.batch) part[(long long)b * p.rows + row] = __uint_as_float(v[j]);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    if (*abort_flag) mbar_drain(accum, 0u, CNN_TIMEOUT_NS);
    tmem_dealloc(tmem, tcols);
  }
}

// h = ReLU(sum of fc1 partials + bias) as (hi, lo) planes [M][2][B][4096]
__global__ void cnn_fc1_finish_kernel(int M, int B, const float* part, const float* bias,
                                      float* h) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)M * B * CNN_FC1_N;
  if (t >= n) return;
  const int o = (int)(t % CNN_FC1_N);
  const long long mb = t / CNN_FC1_N;
  const int m = (int)(mb / B), b = (int)(mb % B);
  float v = 0.0f;
  for (int s = 0; s < CNN_FC1_SPLIT; ++s) v += part[(long long)s * n + t];
  v = fmaxf(v + bias[(long long)m * CNN_FC1_N + o], 0.0f);
  float hi, lo;
  split_tf32f(v, hi, lo);
  const long long pl = (long long)B * CNN_FC1_N;
  float* d = h + (long long)m * 2 * pl + (long long)b * CNN_FC1_N + o;
  d[0] = hi;
  d[pl] = lo;
}

// out[m][b][j] = (sum of fc2 partials + bias) / factor[m][j], j < n_out[m]
struct CnnOutArgs {
  int n_out[EUV_CNN_MAX_MODELS];
};
__global__ void cnn_fc2_finish_kernel(int M, int B, int op, int max_out, CnnOutArgs no,
                                      const float* part, const float* bias,
                                      const double* factors, double* out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)M * B * max_out;
  if (t >= n) return;
  const int j = (int)(t % max_out);
  const long long mb = t / max_out;
  const int m = (int)(mb / B);
  if (j >= no.n_out[m]) {
    out[t] = 0.0;
    return;
  }
  const long long src = mb * op + j, np = (long long)M * B * op;
  float v = 0.0f;
  for (int s = 0; s < CNN_FC2_SPLIT; ++s) v += part[(long long)s * np + src];
  v += bias[(long long)m * op + j];
  out[t] = (double)v / factors[(long long)m * max_out + j];
}

// ------------------------------------------------------------------ host

static int cnn_stages(int bn) {
  const int stage = 2 * CNN_A_TILE + 2 * bn * CNN_BK * 4;
  const int budget = stage <= 24 * 1024 ? 110 * 1024 : 200 * 1024;  // two CTAs / SM when small
  int s = budget / stage;
  return s < 2 ? 2 : (s > 6 ? 6 : s);
}
static size_t cnn_smem(int bn, int stages) {
  return (size_t)stages * (2 * CNN_A_TILE + 2 * bn * CNN_BK * 4) + 1024 + 256;
}

template <class Kern, class Args>
static int cnn_launch(Kern kernel, dim3 grid, size_t smem, const CUtensorMap& ta,
                      const CUtensorMap& tb, const Args& p, cudaStream_t stream, int* done) {
  EUV_CUDA_TRY(ensure_smem(kernel, (int)smem, done));
  kernel<<<grid, CNN_THREADS, smem, stream>>>(ta, tb, p);
  EUV_LAUNCH_CHECK();
  return EUV_OK;
}

// persistent grid of the conv kernel: resident CTAs per SM by shared memory
// (with the 1 KB the runtime reserves per CTA) and registers, capped by TMEM
// (tmem_cols accumulator columns, allocated as a power of two)
static int cnn_conv_grid(int total, int tmem_cols, size_t smem) {
  static int done[64];
  int dev = 0, nsm = 148, sm_smem = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  if (ensure_smem(cnn_conv_kernel, (int)smem, done) != cudaSuccess ||
      cudaFuncSetAttribute(cnn_conv_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                           (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess)
    return -1;
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, cnn_conv_kernel) != cudaSuccess ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sm_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) !=
          cudaSuccess)
    return -1;
  int occ = sm_smem / (int)(smem + 1024 + fa.sharedSizeBytes);
  const int regs = ((fa.numRegs + 7) / 8) * 8 * CNN_THREADS;
  if (regs > 0 && occ > 65536 / regs) occ = 65536 / regs;
  int tcols = 32;
  while (tcols < tmem_cols) tcols <<= 1;
  if (occ > 512 / tcols) occ = 512 / tcols;
  if (occ < 1) occ = 1;
  const long long g = (long long)nsm * occ;
  return (int)(g < total ? g : total);
}

}  // namespace euv

using namespace euv;

extern "C" size_t euv_cnn_blob_bytes(int n_models, int max_out) {
  if (n_models < 1 || n_models > EUV_CNN_MAX_MODELS || max_out < 1 || max_out > EUV_CNN_MAX_OUT)
    return 0;
  return cnn_blob(n_models, max_out).total * sizeof(float);
}

extern "C" size_t euv_cnn_workspace_bytes(int n_models, int n_masks, int max_out) {
  if (n_models < 1 || n_models > EUV_CNN_MAX_MODELS || n_masks < 1 || n_masks > 65535 ||
      max_out < 1 || max_out > EUV_CNN_MAX_OUT)
    return 0;
  return cnn_work(n_models, n_masks, cnn_blob(n_models, max_out).op).total * sizeof(float);
}

extern "C" int euv_cnn_pack(int n_models, const euv_cnn_model_weights* w, int max_out,
                            double bn_eps, void* d_blob, size_t blob_bytes, void* stream_) {
  if (n_models < 1 || n_models > EUV_CNN_MAX_MODELS || !w || !d_blob || max_out < 1 ||
      max_out > EUV_CNN_MAX_OUT || !(bn_eps >= 0.0)) {
    euv_set_error("euv_cnn_pack: bad arguments (models=%d max_out=%d)", n_models, max_out);
    return EUV_ERR_BAD_ARG;
  }
  const CnnBlob L = cnn_blob(n_models, max_out);
  if (blob_bytes < L.total * sizeof(float) || (reinterpret_cast<uintptr_t>(d_blob) & 255u)) {
    euv_set_error("euv_cnn_pack: blob too small or not 256-byte aligned");
    return EUV_ERR_WORKSPACE;
  }
  for (int m = 0; m < n_models; ++m) {
    const euv_cnn_model_weights& mw = w[m];
    if (mw.n_out < 1 || mw.n_out > max_out || !mw.fc1_w || !mw.fc1_b || !mw.fc2_w || !mw.fc2_b) {
      euv_set_error("euv_cnn_pack: model %d: bad fc tensors or n_out=%d", m, mw.n_out);
      return EUV_ERR_BAD_ARG;
    }
    for (int l = 0; l < 5; ++l)
      if (!mw.conv_w[l] || !mw.conv_b[l] || !mw.bn_w[l] || !mw.bn_b[l] || !mw.bn_mean[l] ||
          !mw.bn_var[l]) {
        euv_set_error("euv_cnn_pack: model %d layer %d: missing tensor", m, l + 1);
        return EUV_ERR_BAD_ARG;
      }
  }
  cudaStream_t stream = (cudaStream_t)stream_;
  float* blob = reinterpret_cast<float*>(d_blob);
  for (int m = 0; m < n_models; ++m) {
    const euv_cnn_model_weights& mw = w[m];
    for (int l = 0; l < 5; ++l) {
      const int co = cnn_cout(l), ci = cnn_cin(l);
      if (l == 0) {
        cnn_pack_conv1_kernel<<<1, 160, 0, stream>>>(mw.conv_w[0], blob + L.w[0] + m * 144);
      } else {
        const int n = co * 9 * ci;
        cnn_pack_conv_kernel<<<(n + 255) / 256, 256, 0, stream>>>(
            co, ci, mw.conv_w[l], blob + L.w[l] + (size_t)m * 2 * n);
      }
      EUV_LAUNCH_CHECK();
      cnn_pack_vec_kernel<<<(co + 255) / 256, 256, 0, stream>>>(
          co, co, mw.conv_b[l], mw.bn_w[l], mw.bn_b[l], mw.bn_mean[l], mw.bn_var[l], bn_eps,
          blob + L.bias[l] + m * co, blob + L.scale[l] + m * co, blob + L.shift[l] + m * co);
      EUV_LAUNCH_CHECK();
    }
    const long long n1 = (long long)CNN_FC1_N * CNN_FC1_K;
    cnn_pack_fc_kernel<<<(unsigned)((n1 + 255) / 256), 256, 0, stream>>>(
        CNN_FC1_N, CNN_FC1_N, CNN_FC1_K, 1, mw.fc1_w, blob + L.fc1 + (size_t)m * n1);
    EUV_LAUNCH_CHECK();
    cnn_pack_vec_kernel<<<CNN_FC1_N / 256, 256, 0, stream>>>(
        CNN_FC1_N, CNN_FC1_N, mw.fc1_b, nullptr, nullptr, nullptr, nullptr, 0.0,
        blob + L.fc1_b + (size_t)m * CNN_FC1_N, nullptr, nullptr);
    EUV_LAUNCH_CHECK();
    const long long n2 = (long long)L.op * CNN_FC1_N;
    cnn_pack_fc_kernel<<<(unsigned)((n2 + 255) / 256), 256, 0, stream>>>(
        mw.n_out, L.op, CNN_FC1_N, 0, mw.fc2_w, blob + L.fc2 + (size_t)m * n2);
    EUV_LAUNCH_CHECK();
    cnn_pack_vec_kernel<<<(L.op + 255) / 256, 256, 0, stream>>>(
        mw.n_out, L.op, mw.fc2_b, nullptr, nullptr, nullptr, nullptr, 0.0,
        blob + L.fc2_b + (size_t)m * L.op, nullptr, nullptr);
    EUV_LAUNCH_CHECK();
  }
  return EUV_OK;
}

extern "C" int euv_cnn_downsample(int n_masks, const uint8_t* d_bits, float* d_x0, void* stream) {
  if (n_masks < 1 || n_masks > 65535 || !d_bits || !d_x0) {
    euv_set_error("euv_cnn_downsample: bad arguments (n_masks=%d)", n_masks);
    return EUV_ERR_BAD_ARG;
  }
  dim3 g((CNN_IN * CNN_IN + 255) / 256, n_masks);
  cnn_input_kernel<<<g, 256, 0, (cudaStream_t)stream>>>(d_bits, d_x0);
  EUV_LAUNCH_CHECK();
  return EUV_OK;
}

extern "C" int euv_cnn_predict(const euv_cnn_desc* d, const uint8_t* d_bits, const void* d_blob,
                               double* d_out, void* d_work, size_t work_bytes, void* stream_) {
  if (!d || d->n_models < 1 || d->n_models > EUV_CNN_MAX_MODELS || d->n_masks < 1 ||
      d->n_masks > 65535 || d->max_out < 1 || d->max_out > EUV_CNN_MAX_OUT || !d_bits ||
      !d_blob || !d_out || !d->d_factors || !d_work) {
    euv_set_error("euv_cnn_predict: bad arguments");
    return EUV_ERR_BAD_ARG;
  }
  for (int m = 0; m < d->n_models; ++m)
    if (d->n_out[m] < 1 || d->n_out[m] > d->max_out) {
      euv_set_error("euv_cnn_predict: model %d: n_out=%d outside [1, %d]", m, d->n_out[m],
                    d->max_out);
      return EUV_ERR_BAD_ARG;
    }
  const int M = d->n_models, B = d->n_masks;
  const CnnBlob L = cnn_blob(M, d->max_out);
  const CnnWork W = cnn_work(M, B, L.op);
  if (work_bytes < W.total * sizeof(float) || (reinterpret_cast<uintptr_t>(d_work) & 255u) ||
      (reinterpret_cast<uintptr_t>(d_blob) & 255u)) {
    euv_set_error("euv_cnn_predict: workspace too small or blob/workspace not 256-byte aligned");
    return EUV_ERR_WORKSPACE;
  }
  cudaStream_t stream = (cudaStream_t)stream_;
  const float* blob = reinterpret_cast<const float*>(d_blob);
  float* work = reinterpret_cast<float*>(d_work);
  int* err = d->d_status;
  if (!err) {
    err = reinterpret_cast<int*>(work + W.status);
    EUV_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), stream));
  }
  // input + conv1
  {
    dim3 g((CNN_IN * CNN_IN + 255) / 256, B);
    cnn_input_kernel<<<g, 256, 0, stream>>>(d_bits, work + W.x0);
    EUV_LAUNCH_CHECK();
    dim3 g1((CNN_IN / 2) * (CNN_IN / 2) / 256, B, M);
    cnn_conv1_kernel<<<g1, 256, 0, stream>>>(B, work + W.x0, blob + L.w[0], blob + L.bias[0],
                                             blob + L.scale[0], blob + L.shift[0],
                                             work + W.act[0]);
    EUV_LAUNCH_CHECK();
  }
  // conv2..conv5
  for (int l = 1; l < 5; ++l) {
    const int S = cnn_side(l), ci = cnn_cin(l), co = cnn_cout(l);
    float* in = work + W.act[l - 1];
    CUtensorMap ta, tb;
    const cuuint64_t sp = (cuuint64_t)S + 2;
    const cuuint64_t adims[5] = {(cuuint64_t)ci, sp, sp, (cuuint64_t)B, (cuuint64_t)2 * M};
    const cuuint64_t astr[4] = {(cuuint64_t)ci * 4, sp * ci * 4, sp * sp * ci * 4,
                                (cuuint64_t)B * sp * sp * ci * 4};
    const CnnConvPlan cp = cnn_conv_plan(co, M);
    const cuuint32_t abox[5] = {CNN_BK, 16, (cuuint32_t)(8 * cp.mt + 2), 1, 1};
    int rc = make_map_f32(&ta, in, 5, adims, astr, abox);
    if (rc) return rc;
    const cuuint64_t bdims[3] = {(cuuint64_t)9 * ci, (cuuint64_t)co, (cuuint64_t)2 * M};
    const cuuint64_t bstr[2] = {(cuuint64_t)9 * ci * 4, (cuuint64_t)co * 9 * ci * 4};
    const cuuint32_t bbox[3] = {CNN_BK, (cuuint32_t)co, 1};
    rc = make_map_f32(&tb, const_cast<float*>(blob + L.w[l]), 3, bdims, bstr, bbox);
    if (rc) return rc;
    CnnConvArgs p = {};
    p.models = M;
    p.batch = B;
    p.side = S;
    p.tiles_x = S / 16;
    p.tiles_img = (S / (8 * cp.mt)) * (S / 16);
    const long long total = (long long)M * B * p.tiles_img;
    if (total > 0x7fffffffLL) {
      euv_set_error("euv_cnn_predict: too many conv tiles (%lld)", total);
      return EUV_ERR_BAD_ARG;
    }
    p.total_tiles = (int)total;
    p.cin = ci;
    p.cout = co;
    p.mt = cp.mt;
    p.nbuf = cp.nbuf;
    p.a_stages = cp.a_stages;
    p.b_stages = cp.b_stages;
    p.out_pad = l < 4 ? 1 : 0;
    p.bias = blob + L.bias[l];
    p.scale = blob + L.scale[l];
    p.shift = blob + L.shift[l];
    p.out = work + W.act[l];
    p.err = err;
    const size_t smem = cp.smem;
    const int grid = cnn_conv_grid(p.total_tiles, cp.nbuf * cp.mt * co, smem);
    if (grid < 1) {
      euv_set_error("euv_cnn_predict: conv kernel setup failed");
      return EUV_ERR_CUDA;
    }
    cnn_conv_kernel<<<grid, CNN_THREADS, smem, stream>>>(ta, tb, p);
    EUV_LAUNCH_CHECK();
  }
  // fc1, fc2: A = weight planes [M*2][rows][K], B = activation planes [M*2][B][K]
  const int bn = B >= 256 ? 256 : (B + 15) / 16 * 16;
  const int ntiles = (B + bn - 1) / bn;
  for (int f = 0; f < 2; ++f) {
    const int K = f == 0 ? CNN_FC1_K : CNN_FC1_N;
    const int rows = f == 0 ? CNN_FC1_N : L.op;
    const int nsplit = f == 0 ? CNN_FC1_SPLIT : CNN_FC2_SPLIT;
    float* wa = const_cast<float*>(blob + (f == 0 ? L.fc1 : L.fc2));
    float* act = work + (f == 0 ? W.act[4] : W.h);
    CUtensorMap ta, tb;
    const cuuint64_t adims[3] = {(cuuint64_t)K, (cuuint64_t)rows, (cuuint64_t)M};
    const cuuint64_t astr[2] = {(cuuint64_t)K * 4, (cuuint64_t)rows * K * 4};
    const cuuint32_t abox[3] = {CNN_BK, 128, 1};
    int rc = make_map_f32(&ta, wa, 3, adims, astr, abox);
    if (rc) return rc;
    const cuuint64_t bdims[3] = {(cuuint64_t)K, (cuuint64_t)B, (cuuint64_t)2 * M};
    const cuuint64_t bstr[2] = {(cuuint64_t)K * 4, (cuuint64_t)B * K * 4};
    const cuuint32_t bbox[3] = {CNN_BK, (cuuint32_t)bn, 1};
    rc = make_map_f32(&tb, act, 3, bdims, bstr, bbox);
    if (rc) return rc;
    CnnFcArgs p = {};
    p.models = M;
    p.batch = B;
    p.bn = bn;
    p.nkb = K / CNN_BK / nsplit;
    p.stages = cnn_stages(bn);
    p.rows = rows;
    p.nsplit = nsplit;
    p.part = work + (f == 0 ? W.part1 : W.part2);
    p.err = err;
    dim3 grid(rows / 128, ntiles * nsplit, M);
    static int fc_done[64];
    if ((rc = cnn_launch(cnn_fc_kernel, grid, cnn_smem(bn, p.stages), ta, tb, p, stream,
                         fc_done)))
      return rc;
    if (f == 0) {
      const long long n = (long long)M * B * CNN_FC1_N;
      cnn_fc1_finish_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(
          M, B, work + W.part1, blob + L.fc1_b, work + W.h);
    } else {
      CnnOutArgs no;
      for (int m = 0; m < EUV_CNN_MAX_MODELS; ++m) no.n_out[m] = m < M ? d->n_out[m] : 0;
      const long long n = (long long)M * B * d->max_out;
      cnn_fc2_finish_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(
          M, B, L.op, d->max_out, no, work + W.part2, blob + L.fc2_b, d->d_factors, d_out);
    }
    EUV_LAUNCH_CHECK();
  }
  return EUV_OK;
}
