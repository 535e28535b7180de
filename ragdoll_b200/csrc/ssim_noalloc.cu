// SSIM / MS-SSIM of two device planes without allocating any device memory
// (rg_ssim_plane_device_noalloc in include/ragdoll_cuda.h).
//
// Who needs this: callers that are not allowed to call cudaMalloc / cudaFree at the time they
// measure quality -- a frame loop with a fixed memory budget whose device memory is already
// reserved by another allocator (a framework's caching pool), or a latency-critical loop where
// an allocation would synchronise the device and stall the other streams. They pass the two
// planes and a two-double output buffer that they own; the working memory (the 2x2-decimated
// pyramid and the per-row sums) lives in one file-scope __device__ array instead.
//
// That array is shared by every call on a device and keeps the last call's contents; nothing in
// it has to start at zero (every byte read is written first by the same call). Calls that
// overlap on the GPU (on different streams, or on different host threads) race on it and must
// be serialised by the caller. Its size bounds the planes: width and height 8..4096 and at most
// 1920 x 1088 samples.
//
// The arithmetic is that of the allocating path (ssim_kernels.cu): per-window f32 ssim_end1
// without fused multiply-add, a sequential f32 sum per window row, an f64 sum of the rows
// (crates/ragdoll-simd/src/metrics.rs:417, :637), and the 5-scale product of
// crates/ragdoll-pix/src/metrics.rs:154, here evaluated on the device.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/ragdoll_cuda.h"

namespace rg {
void set_last_error(const char* msg);
}

namespace {

constexpr long kNaMaxPixels = 1920L * 1088L;
constexpr int kNaMaxDim = 4096;
constexpr int kNaRowsPerBlock = 8;
constexpr size_t kNaPyrBytes = 2 * (kNaMaxPixels / 4 + kNaMaxPixels / 16 + kNaMaxPixels / 64 + kNaMaxPixels / 256) + 4096;
constexpr size_t kNaRowFloats = 2 * (kNaMaxDim / 4) + 64;
constexpr size_t kNaScratchBytes = kNaPyrBytes + kNaRowFloats * sizeof(float) + 16 * sizeof(double);

// The working memory of every call on this device: pyramid planes, then row sums, then the five
// per-scale SSIM values.
__device__ __align__(256) uint8_t g_noalloc_scratch[kNaScratchBytes];

struct NaLevel {
  const uint8_t* a;
  const uint8_t* b;
  long sa, sb;
  int w, h;
  float* rows;
};
struct NaPack {
  NaLevel lv[5];
  int levels;
  int want_ms;
  double* scale_ssim;  // 5 doubles in the scratch
  double* out;         // caller's [ssim, ms_ssim]
};

__device__ __forceinline__ float na_ssim_end1(int s1, int s2, int ss, int s12) {
  int vars = ss * 64 - s1 * s1 - s2 * s2;
  int covar = s12 * 64 - s1 * s2;
  float num = __fmul_rn(__int2float_rn(2 * s1 * s2 + 416), __int2float_rn(2 * covar + 235963));
  float den = __fmul_rn(__int2float_rn(s1 * s1 + s2 * s2 + 416), __int2float_rn(vars + 235963));
  return __fdiv_rn(num, den);
}

__global__ void na_decimate_kernel(NaLevel src, uint8_t* da, uint8_t* db) {
  int dw = src.w >> 1, dh = src.h >> 1;
  int n = dw * dh;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int dy = i / dw, dx = i - dy * dw;
    const uint8_t* ra = src.a + (long)(2 * dy) * src.sa + 2 * dx;
    const uint8_t* rb = src.b + (long)(2 * dy) * src.sb + 2 * dx;
    da[(long)dy * dw + dx] = (uint8_t)((ra[0] + ra[1] + ra[src.sa] + ra[src.sa + 1] + 2) >> 2);
    db[(long)dy * dw + dx] = (uint8_t)((rb[0] + rb[1] + rb[src.sb] + rb[src.sb + 1] + 2) >> 2);
  }
}

__global__ void na_rows_kernel(NaLevel j) {
  int bw = j.w >> 2, bh = j.h >> 2;
  if (bw < 2 || bh < 2) return;
  int nrows = bh - 1;
  int r0 = blockIdx.x * kNaRowsPerBlock;
  if (r0 >= nrows) return;
  int rn = min(kNaRowsPerBlock, nrows - r0);
  extern __shared__ int na_sums[];
  float* vals = (float*)(na_sums + (size_t)(rn + 1) * bw * 4);
  for (int i = threadIdx.x; i < (rn + 1) * bw; i += blockDim.x) {
    int br = i / bw, bx = i - br * bw;
    int y = (r0 + br) * 4, x = bx * 4;
    int s1 = 0, s2 = 0, ss = 0, s12 = 0;
    for (int dy = 0; dy < 4; dy++)
      for (int k = 0; k < 4; k++) {
        int va = j.a[(long)(y + dy) * j.sa + x + k], vb = j.b[(long)(y + dy) * j.sb + x + k];
        s1 += va; s2 += vb; ss += va * va + vb * vb; s12 += va * vb;
      }
    int* o = na_sums + (size_t)i * 4;
    o[0] = s1; o[1] = s2; o[2] = ss; o[3] = s12;
  }
  __syncthreads();
  int nwin = bw - 1;
  for (int i = threadIdx.x; i < rn * nwin; i += blockDim.x) {
    int r = i / nwin, bx = i - r * nwin;
    const int* a0 = na_sums + ((size_t)r * bw + bx) * 4;
    const int* b0 = na_sums + ((size_t)(r + 1) * bw + bx) * 4;
    int v[4];
    for (int k = 0; k < 4; k++) v[k] = a0[k] + a0[4 + k] + b0[k] + b0[4 + k];
    vals[i] = na_ssim_end1(v[0], v[1], v[2], v[3]);
  }
  __syncthreads();
  if ((int)threadIdx.x < rn) {
    float row = 0.0f;
    for (int k = 0; k < nwin; k++) row = __fadd_rn(row, vals[(size_t)threadIdx.x * nwin + k]);
    j.rows[r0 + threadIdx.x] = row;
  }
}

__global__ void na_finish_kernel(NaPack p) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double w5[5] = {0.0448, 0.2856, 0.3001, 0.2363, 0.1333};
  for (int l = 0; l < p.levels; l++) {
    const NaLevel& j = p.lv[l];
    int bw = j.w >> 2, bh = j.h >> 2;
    double s;
    if (bw < 2 || bh < 2) {
      int s1 = 0, s2 = 0, ss = 0, s12 = 0;
      for (int y = 0; y < 8; y++)
        for (int x = 0; x < 8; x++) {
          int va = j.a[(long)y * j.sa + x], vb = j.b[(long)y * j.sb + x];
          s1 += va; s2 += vb; ss += va * va + vb * vb; s12 += va * vb;
        }
      s = (double)na_ssim_end1(s1, s2, ss, s12);
    } else {
      double t = 0.0;
      for (int r = 0; r < bh - 1; r++) t = __dadd_rn(t, (double)j.rows[r]);
      s = __ddiv_rn(t, (double)((bw - 1) * (bh - 1)));
    }
    p.scale_ssim[l] = s;
  }
  double s0 = p.scale_ssim[0];
  p.out[0] = s0;
  double c0 = fmin(1.0, fmax(0.0, s0));
  if (!p.want_ms || fabs(1.0 - c0) < 1e-12 || p.levels == 1) {
    p.out[1] = c0;
    return;
  }
  double wsum = 0.0;
  for (int l = 0; l < p.levels; l++) wsum += w5[l];
  double prod = 1.0;
  for (int l = 0; l < p.levels; l++) {
    double sc = l == 0 ? c0 : fmin(1.0, fmax(0.0, p.scale_ssim[l]));
    prod *= pow(fmax(sc, 1e-9), w5[l] / wsum);
  }
  p.out[1] = fmin(1.0, fmax(0.0, prod));
}

int na_fail(int code, const char* fmt, ...) {
  char buf[384];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  rg::set_last_error(buf);
  return code;
}

// Device address of g_noalloc_scratch per device, found once per device with that device
// current. In host code the array's name is only a stand-in for the symbol, never an address.
std::mutex na_mu;
uint8_t* na_scratch_ptr[64] = {nullptr};

int na_setup(int dev, uint8_t** out) {
  std::lock_guard<std::mutex> lock(na_mu);
  if (dev < 0 || dev >= 64) return na_fail(RG_ERR_INVALID, "rg_ssim_plane_device_noalloc: device %d out of range", dev);
  if (!na_scratch_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return na_fail(RG_ERR_CUDA, "rg_ssim_plane_device_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
    e = cudaFuncSetAttribute(na_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess)
      return na_fail(RG_ERR_CUDA, "rg_ssim_plane_device_noalloc: cudaFuncSetAttribute failed: %s", cudaGetErrorString(e));
    na_scratch_ptr[dev] = (uint8_t*)p;
  }
  *out = na_scratch_ptr[dev];
  return RG_OK;
}

}  // namespace

extern "C" int rg_ssim_plane_device_noalloc(const uint8_t* dev_a, size_t stride_a, const uint8_t* dev_b,
                                            size_t stride_b, int32_t width, int32_t height, double* dev_out,
                                            void* cuda_stream) {
  if (!dev_a || !dev_b || !dev_out) return na_fail(RG_ERR_INVALID, "rg_ssim_plane_device_noalloc: null pointer");
  if (width < 8 || height < 8)
    return na_fail(RG_ERR_INVALID, "rg_ssim_plane_device_noalloc: %dx%d is smaller than one 8x8 window", width, height);
  if (width > kNaMaxDim || height > kNaMaxDim || (long)width * height > kNaMaxPixels)
    return na_fail(RG_ERR_INVALID,
                   "rg_ssim_plane_device_noalloc: %dx%d exceeds the fixed working memory (width and height <= %d, "
                   "at most %ld samples); use rg_ssim_plane",
                   width, height, kNaMaxDim, kNaMaxPixels);
  if (stride_a < (size_t)width || stride_b < (size_t)width)
    return na_fail(RG_ERR_INVALID, "rg_ssim_plane_device_noalloc: stride smaller than width");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return na_fail(RG_ERR_CUDA, "rg_ssim_plane_device_noalloc: %s", cudaGetErrorString(e));
  uint8_t* scratch = nullptr;
  int r = na_setup(dev, &scratch);
  if (r) return r;
  cudaStream_t st = (cudaStream_t)cuda_stream;

  NaPack p{};
  p.want_ms = 1;
  p.out = dev_out;
  float* rows = (float*)(scratch + kNaPyrBytes);
  p.scale_ssim = (double*)(scratch + kNaPyrBytes + kNaRowFloats * sizeof(float));
  p.lv[0] = NaLevel{dev_a, dev_b, (long)stride_a, (long)stride_b, width, height, rows};
  size_t rofs = (size_t)(height / 4) + 1, pofs = 0;
  p.levels = 1;
  // pyramid levels while the next one is at least 8x8 (ms_ssim_plane_u8); none when the first
  // level already decides the result (tiny plane)
  if ((width >> 1) >= 8 && (height >> 1) >= 8) {
    int w = width, h = height;
    for (int l = 1; l < 5; l++) {
      int nw = w >> 1, nh = h >> 1;
      if (nw < 8 || nh < 8) break;
      uint8_t* da = scratch + pofs;
      uint8_t* db = da + (size_t)nw * nh;
      pofs += 2 * (size_t)nw * nh;
      na_decimate_kernel<<<(nw * nh + 255) / 256 < 1024 ? (nw * nh + 255) / 256 : 1024, 256, 0, st>>>(p.lv[l - 1], da, db);
      p.lv[l] = NaLevel{da, db, nw, nw, nw, nh, rows + rofs};
      rofs += (size_t)(nh / 4) + 1;
      p.levels++;
      w = nw;
      h = nh;
    }
  }
  for (int l = 0; l < p.levels; l++) {
    const NaLevel& j = p.lv[l];
    int bw = j.w >> 2, bh = j.h >> 2;
    if (bw < 2 || bh < 2) continue;
    int strips = (bh - 1 + kNaRowsPerBlock - 1) / kNaRowsPerBlock;
    size_t smem = (size_t)(kNaRowsPerBlock + 1) * bw * 4 * sizeof(int) + (size_t)kNaRowsPerBlock * (bw - 1) * sizeof(float);
    na_rows_kernel<<<strips, 256, smem, st>>>(j);
  }
  na_finish_kernel<<<1, 32, 0, st>>>(p);
  e = cudaGetLastError();
  if (e != cudaSuccess) return na_fail(RG_ERR_CUDA, "rg_ssim_plane_device_noalloc: launch failed: %s", cudaGetErrorString(e));
  return RG_OK;
}
