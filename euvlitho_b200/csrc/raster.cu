// Mask rasteriser: axis-aligned absorber rectangles -> packed mask.bin bits on
// the device, with per-slice sidewall erosion.
//
// Replaces the pixel loops and the bit packing of the reference's mask
// generator (cnn/intensity/mask/mVBF.h:2-70 fills an int per pixel,
// mask.cpp:9-26 packs them MSB first) for bulk data generation: the layout
// (rectangles) comes from the host, every pixel and bit is produced here, and
// the packed masks stay on the device for the mask spectrum.  HBM-bound: one
// byte per pixel written and read per erosion step, one bit per pixel out.
#include "common.cuh"

namespace euv {

__global__ void raster_fill_kernel(uint8_t* img, long long n, uint8_t v) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) img[i] = v;
}

// One CTA per rectangle (mask, x0, x1, y0, y1; half-open, clamped to the grid)
// paints 0 (absorber).  Rectangles may overlap: every writer stores the same 0.
__global__ void raster_paint_kernel(const int* rects, int ndivx, int ndivy, int n_masks,
                                    uint8_t* img) {
  const int* r = rects + 5 * (long long)blockIdx.x;
  const int m = r[0];
  if (m < 0 || m >= n_masks) return;
  const int x0 = max(r[1], 0), x1 = min(r[2], ndivx);
  const int y0 = max(r[3], 0), y1 = min(r[4], ndivy);
  if (x0 >= x1 || y0 >= y1) return;
  const int w = x1 - x0;
  const long long area = (long long)w * (y1 - y0);
  uint8_t* base = img + (long long)m * ndivx * ndivy;
  for (long long t = threadIdx.x; t < area; t += blockDim.x) {
    const int y = y0 + (int)(t / w), x = x0 + (int)(t % w);
    base[(long long)y * ndivx + x] = 0;
  }
}

// One step of absorber erosion with the 4-neighbour cross, periodic edges:
// a pixel stays absorber (0) only if it and its four neighbours are absorber.
__global__ void raster_erode_kernel(const uint8_t* in, uint8_t* out, int ndivx, int ndivy,
                                    int n_masks) {
  const long long npix = (long long)ndivx * ndivy;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npix * n_masks) return;
  const long long m = t / npix, p = t - m * npix;
  const int y = (int)(p / ndivx), x = (int)(p - (long long)y * ndivx);
  const uint8_t* b = in + m * npix;
  const int xl = x == 0 ? ndivx - 1 : x - 1, xr = x == ndivx - 1 ? 0 : x + 1;
  const int yd = y == 0 ? ndivy - 1 : y - 1, yu = y == ndivy - 1 ? 0 : y + 1;
  const uint8_t v = b[p] | b[(long long)y * ndivx + xl] | b[(long long)y * ndivx + xr] |
                    b[(long long)yd * ndivx + x] | b[(long long)yu * ndivx + x];
  out[t] = v ? 1 : 0;
}

// 8 pixels (one byte of mask.bin, bit index ndivx*y + x, MSB first) per thread.
__global__ void raster_pack_kernel(const uint8_t* img, long long nbytes_per_mask, int n_masks,
                                   int n_slices, int slice, uint8_t* bits) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nbytes_per_mask * n_masks) return;
  const long long m = t / nbytes_per_mask, q = t - m * nbytes_per_mask;
  const uint8_t* p = img + m * nbytes_per_mask * 8 + q * 8;
  uint8_t v = 0;
#pragma unroll
  for (int b = 0; b < 8; ++b) v |= (uint8_t)((p[b] ? 1 : 0) << (7 - b));
  bits[(m * n_slices + slice) * nbytes_per_mask + q] = v;
}

inline unsigned blocks_for(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace euv

using namespace euv;

extern "C" size_t euv_mask_raster_workspace_bytes(int n_masks, int ndivx, int ndivy) {
  if (n_masks <= 0 || ndivx <= 0 || ndivy <= 0) return 0;
  const size_t img = ((size_t)n_masks * ndivx * ndivy + 255) & ~(size_t)255;
  return 2 * img;
}

extern "C" int euv_mask_raster(int n_masks, int ndivx, int ndivy, int n_rects, const int* d_rects,
                               int n_slices, const int* h_erosion, uint8_t* d_bits, void* d_work,
                               size_t work_bytes, void* stream_) {
  const long long npix = (long long)ndivx * ndivy;
  if (n_masks <= 0 || ndivx <= 0 || ndivy <= 0 || npix % 8 || n_rects < 0 ||
      (n_rects > 0 && !d_rects) || n_slices <= 0 || n_slices > 64 || !h_erosion || !d_bits ||
      !d_work ||
      n_rects > 2147483647 / 5) {
    euv_set_error("euv_mask_raster: bad arguments");
    return EUV_ERR_BAD_ARG;
  }
  for (int s = 0; s < n_slices; ++s)
    if (h_erosion[s] < 0 || h_erosion[s] > ndivx || h_erosion[s] > ndivy) {
      euv_set_error("euv_mask_raster: erosion radius %d of slice %d out of range", h_erosion[s], s);
      return EUV_ERR_BAD_ARG;
    }
  if (work_bytes < euv_mask_raster_workspace_bytes(n_masks, ndivx, ndivy)) {
    euv_set_error("euv_mask_raster: workspace too small");
    return EUV_ERR_WORKSPACE;
  }
  cudaStream_t stream = (cudaStream_t)stream_;
  const long long total = npix * n_masks;
  const size_t img_bytes = ((size_t)total + 255) & ~(size_t)255;
  uint8_t* img = reinterpret_cast<uint8_t*>(d_work);
  uint8_t* tmp = img + img_bytes;
  raster_fill_kernel<<<blocks_for(total, 256), 256, 0, stream>>>(img, total, 1);
  EUV_LAUNCH_CHECK();
  if (n_rects > 0) {
    raster_paint_kernel<<<n_rects, 256, 0, stream>>>(d_rects, ndivx, ndivy, n_masks, img);
    EUV_LAUNCH_CHECK();
  }
  // slices in increasing erosion radius: erosion by r+1 is one cross step
  // applied to erosion by r, so max(r) steps in all, ping-pong img <-> tmp
  const long long nbytes = npix / 8;
  int order[64];
  const int ns = n_slices < 64 ? n_slices : 64;
  for (int s = 0; s < ns; ++s) order[s] = s;
  for (int a = 1; a < ns; ++a)
    for (int c = a; c > 0 && h_erosion[order[c]] < h_erosion[order[c - 1]]; --c) {
      const int t = order[c];
      order[c] = order[c - 1];
      order[c - 1] = t;
    }
  uint8_t* cur = img;
  uint8_t* other = tmp;
  int r_cur = 0;
  for (int oi = 0; oi < ns; ++oi) {
    const int s = order[oi];
    for (; r_cur < h_erosion[s]; ++r_cur) {
      raster_erode_kernel<<<blocks_for(total, 256), 256, 0, stream>>>(cur, other, ndivx, ndivy,
                                                                       n_masks);
      EUV_LAUNCH_CHECK();
      uint8_t* t = cur;
      cur = other;
      other = t;
    }
    raster_pack_kernel<<<blocks_for(nbytes * n_masks, 256), 256, 0, stream>>>(
        cur, nbytes, n_masks, n_slices, s, d_bits);
    EUV_LAUNCH_CHECK();
  }
  return EUV_OK;
}
