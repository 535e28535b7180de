// SSIM / MS-SSIM / PSNR of 8-bit planes on the device (FFmpeg vf_ssim 4x4-sum reuse), with the
// reference's floating-point order reproduced exactly:
//   crates/ragdoll-simd/src/metrics.rs:417  ssim_end1_8bit: integer sums, two f32 products, one
//                                           f32 division (no fused multiply-add)
//   crates/ragdoll-simd/src/metrics.rs:667  row_ssim: sequential f32 sum over the windows of a row
//   crates/ragdoll-simd/src/metrics.rs:675  total: f64 sum of the rows in order
//   crates/ragdoll-pix/src/metrics.rs:87    decimate_2x2_u8: (a + b + c + d + 2) >> 2
// One block computes a strip of window rows: the 4x4 sums of its block rows, the window values
// of each row, then one thread per row adds them up in order.
//
// VMAF-Lite (crates/ragdoll-pix/src/metrics.rs:218 vmaf_lite_plane_u8): per non-overlapping 4x4
// block the local SSIM term and the VIF information terms in f64 (the same expressions, no fused
// multiply-add); one block per block row sums its terms, rows are added in order, and the host
// forms the score. The reference adds all blocks in one raster-order sum; the row-wise sum here
// differs from it only in rounding (about 1e-13 of the score).
#include <cmath>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "ssim_kernels.h"

namespace rg {

namespace {

constexpr int kC1 = 416;
constexpr int kC2 = 235963;
constexpr int kRowsPerBlock = 8;
constexpr int kThreads = 256;

__device__ __forceinline__ float ssim_end1(int s1, int s2, int ss, int s12) {
  int vars = ss * 64 - s1 * s1 - s2 * s2;
  int covar = s12 * 64 - s1 * s2;
  float num = __fmul_rn(__int2float_rn(2 * s1 * s2 + kC1), __int2float_rn(2 * covar + kC2));
  float den = __fmul_rn(__int2float_rn(s1 * s1 + s2 * s2 + kC1), __int2float_rn(vars + kC2));
  return __fdiv_rn(num, den);
}

// Window rows [r0, r0 + kRowsPerBlock) of job blockIdx.y; window row k covers 4x4-block rows
// k and k + 1 (k = by - 1 of ssim_plane_8bit). Writes one f32 per window row.
__global__ void ssim_rows_kernel(const SsimJob* __restrict__ jobs) {
  const SsimJob& j = jobs[blockIdx.y];
  int bw = j.width >> 2, bh = j.height >> 2;
  if (bw < 2 || bh < 2) return;
  int nrows = bh - 1;
  int r0 = blockIdx.x * kRowsPerBlock;
  if (r0 >= nrows) return;
  int rn = min(kRowsPerBlock, nrows - r0);
  extern __shared__ int sums[];        // (rn + 1) block rows x bw x 4
  float* vals = (float*)(sums + (size_t)(rn + 1) * bw * 4);  // rn x (bw - 1)
  int total_blocks = (rn + 1) * bw;
  for (int i = threadIdx.x; i < total_blocks; i += blockDim.x) {
    int br = i / bw, bx = i - br * bw;
    int y = (r0 + br) * 4, x = bx * 4;
    int s1 = 0, s2 = 0, ss = 0, s12 = 0;
#pragma unroll
    for (int dy = 0; dy < 4; dy++) {
      const uint8_t* pa = j.a + (long)(y + dy) * j.stride_a + x;
      const uint8_t* pb = j.b + (long)(y + dy) * j.stride_b + x;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        int va = pa[k], vb = pb[k];
        s1 += va; s2 += vb; ss += va * va + vb * vb; s12 += va * vb;
      }
    }
    int* o = sums + (size_t)i * 4;
    o[0] = s1; o[1] = s2; o[2] = ss; o[3] = s12;
  }
  __syncthreads();
  int nwin = bw - 1;
  for (int i = threadIdx.x; i < rn * nwin; i += blockDim.x) {
    int r = i / nwin, bx = i - r * nwin;
    const int* a0 = sums + ((size_t)r * bw + bx) * 4;
    const int* a1 = a0 + 4;
    const int* b0 = sums + ((size_t)(r + 1) * bw + bx) * 4;
    const int* b1 = b0 + 4;
    int v[4];
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] = a0[k] + a1[k] + b0[k] + b1[k];
    vals[i] = ssim_end1(v[0], v[1], v[2], v[3]);
  }
  __syncthreads();
  if ((int)threadIdx.x < rn) {
    const float* rv = vals + (size_t)threadIdx.x * nwin;
    float row = 0.0f;
    for (int k = 0; k < nwin; k++) row = __fadd_rn(row, rv[k]);
    j.rows[r0 + threadIdx.x] = row;
  }
}

// f64 sum of the row values in order and the final division; also the small-plane fallback
// (one 8x8 window at the origin).
__global__ void ssim_finish_kernel(const SsimJob* __restrict__ jobs, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const SsimJob& j = jobs[i];
  int bw = j.width >> 2, bh = j.height >> 2;
  if (bw < 2 || bh < 2) {
    int s1 = 0, s2 = 0, ss = 0, s12 = 0;
    for (int y = 0; y < 8; y++)
      for (int x = 0; x < 8; x++) {
        int va = j.a[(long)y * j.stride_a + x], vb = j.b[(long)y * j.stride_b + x];
        s1 += va; s2 += vb; ss += va * va + vb * vb; s12 += va * vb;
      }
    *j.out = (double)ssim_end1(s1, s2, ss, s12);
    return;
  }
  double total = 0.0;
  for (int r = 0; r < bh - 1; r++) total = __dadd_rn(total, (double)j.rows[r]);
  *j.out = __ddiv_rn(total, (double)((bw - 1) * (bh - 1)));
}

__global__ void sse_kernel(const SsimJob* __restrict__ jobs) {
  const SsimJob& j = jobs[blockIdx.y];
  unsigned long long acc = 0;
  long n = (long)j.width * j.height;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    long y = i / j.width, x = i - y * j.width;
    int d = (int)j.a[y * j.stride_a + x] - (int)j.b[y * j.stride_b + x];
    acc += (unsigned long long)(d * d);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && j.sse) atomicAdd(j.sse, acc);
}

// 2x2 decimation of a and b of job blockIdx.y into the next pyramid level.
__global__ void decimate_kernel(const DecimateJob* __restrict__ jobs) {
  const DecimateJob& j = jobs[blockIdx.y];
  int dw = j.src_w >> 1, dh = j.src_h >> 1;
  int n = dw * dh;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int dy = i / dw, dx = i - dy * dw;
    for (int p = 0; p < 2; p++) {
      const uint8_t* s = p ? j.src_b : j.src_a;
      long ss = p ? j.stride_b : j.stride_a;
      const uint8_t* r0 = s + (long)(2 * dy) * ss + 2 * dx;
      int sum = r0[0] + r0[1] + r0[ss] + r0[ss + 1];
      (p ? j.dst_b : j.dst_a)[(long)dy * dw + dx] = (uint8_t)((sum + 2) >> 2);
    }
  }
}

// One 4-row strip of 4x4 blocks of job blockIdx.y: its three f64 sums into rows[3 * by ..].
__global__ void vmaf_rows_kernel(const VmafJob* __restrict__ jobs) {
  const VmafJob& j = jobs[blockIdx.y];
  const int bw = j.width >> 2, bh = j.height >> 2, by = blockIdx.x;
  if (by >= bh) return;
  const double kSigmaNsq = 2.0 * 256.0, kEps = 1.0e-10, kGainLimit = 100.0, c1 = 26.0, c2 = 234.0;
  double num = 0.0, den = 0.0, ssim = 0.0;
  for (int bx = threadIdx.x; bx < bw; bx += blockDim.x) {
    int s1 = 0, s2 = 0, ss = 0, s12 = 0;
#pragma unroll
    for (int dy = 0; dy < 4; dy++) {
      const uint8_t* pa = j.a + (long)(by * 4 + dy) * j.stride_a + bx * 4;
      const uint8_t* pb = j.b + (long)(by * 4 + dy) * j.stride_b + bx * 4;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        int va = pa[k], vb = pb[k];
        s1 += va; s2 += vb; ss += va * va + vb * vb; s12 += va * vb;
      }
    }
    const double mean_sq_sum = (double)(s1 * s1 + s2 * s2);
    const double total_var = (double)max(ss * 16 - s1 * s1 - s2 * s2, 0);
    const double covar = (double)(s12 * 16 - s1 * s2);
    const double blk = ((2.0 * (double)s1 * (double)s2 + c1) * (2.0 * covar + c2)) / ((mean_sq_sum + c1) * (total_var + c2));
    ssim += fmin(1.0, fmax(0.0, blk));
    double err_var = (double)max(ss - 2 * s12, 0) * 16.0 - (double)((s1 - s2) * (s1 - s2));
    err_var = fmax(err_var, 0.0);
    const double sigma1_sq = fmax((total_var - err_var) * 0.5, fmax(covar, 0.0));
    const double sigma2_sq = fmax(total_var - sigma1_sq, 0.0);
    const double sigma12 = fmax(covar, 0.0);
    double g, sv_sq;
    if (sigma1_sq < kEps) {
      g = 0.0;
      sv_sq = sigma2_sq;
    } else if (sigma2_sq < kEps) {
      g = 0.0;
      sv_sq = 0.0;
    } else {
      const double g_raw = sigma12 / (sigma1_sq + kEps);
      if (g_raw < 0.0) {
        g = 0.0;
        sv_sq = sigma2_sq;
      } else {
        g = fmin(g_raw, kGainLimit);
        sv_sq = fmax(sigma2_sq - g_raw * sigma12, kEps);
      }
    }
    sv_sq = fmax(sv_sq, kEps);
    g = fmin(g, kGainLimit);
    num += log2(1.0 + (g * g * sigma1_sq) / (sv_sq + kSigmaNsq));
    den += log2(1.0 + sigma1_sq / kSigmaNsq);
  }
  __shared__ double part[3][32];
  for (int o = 16; o > 0; o >>= 1) {
    num += __shfl_xor_sync(0xffffffffu, num, o);
    den += __shfl_xor_sync(0xffffffffu, den, o);
    ssim += __shfl_xor_sync(0xffffffffu, ssim, o);
  }
  const int warp = threadIdx.x >> 5, nwarps = (blockDim.x + 31) >> 5;
  if ((threadIdx.x & 31) == 0) {
    part[0][warp] = num;
    part[1][warp] = den;
    part[2][warp] = ssim;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double acc = 0.0;
    for (int w = 0; w < nwarps; w++) acc += part[threadIdx.x][w];
    j.rows[3 * by + threadIdx.x] = acc;
  }
}

// Rows of each job added in order; also |a - prev| over the plane when prev is given.
__global__ void vmaf_finish_kernel(const VmafJob* __restrict__ jobs, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const VmafJob& j = jobs[i];
  double acc[3] = {0.0, 0.0, 0.0};
  for (int by = 0; by < (j.height >> 2); by++)
    for (int k = 0; k < 3; k++) acc[k] += j.rows[3 * by + k];
  for (int k = 0; k < 3; k++) j.out[k] = acc[k];
}

__global__ void sad_kernel(const VmafJob* __restrict__ jobs) {
  const VmafJob& j = jobs[blockIdx.y];
  if (!j.prev || !j.sad) return;
  unsigned long long acc = 0;
  long n = (long)j.width * j.height;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    long y = i / j.width, x = i - y * j.width;
    acc += (unsigned long long)abs((int)j.a[y * j.stride_a + x] - (int)j.prev[y * j.stride_prev + x]);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(j.sad, acc);
}

}  // namespace

void launch_vmaf(const VmafJob* d_jobs, int n_jobs, int max_height, cudaStream_t st) {
  dim3 grid(std::max(max_height >> 2, 1), n_jobs);
  vmaf_rows_kernel<<<grid, 128, 0, st>>>(d_jobs);
  vmaf_finish_kernel<<<(n_jobs + 63) / 64, 64, 0, st>>>(d_jobs, n_jobs);
  sad_kernel<<<dim3(64, n_jobs), 256, 0, st>>>(d_jobs);
}

double vmaf_lite_score(double info_num, double info_den, double ssim_sum, long blocks, bool have_prev,
                       unsigned long long sad, long pixels) {
  if (blocks <= 0) return 100.0;
  const double mean_ssim = ssim_sum / (double)blocks;
  if (std::fabs(1.0 - mean_ssim) < 1e-9) return 100.0;
  const double vif = info_den <= 1e-9 ? mean_ssim : std::fmin(1.0, std::fmax(0.0, info_num / info_den));
  double boost = 0.0;
  if (have_prev) boost = std::fmin((double)sad / (double)pixels / 255.0 * 0.08, 0.05);
  const double raw = (0.65 * std::pow(mean_ssim, 0.85) + 0.35 * vif + boost) * 100.0;
  return std::fmin(100.0, std::fmax(0.0, raw));
}

size_t ssim_rows_smem(int width) {
  int bw = width >> 2;
  return (size_t)(kRowsPerBlock + 1) * bw * 4 * sizeof(int) + (size_t)kRowsPerBlock * (bw > 1 ? bw - 1 : 1) * sizeof(float);
}

void launch_ssim(const SsimJob* d_jobs, int n_jobs, int max_width, int max_height, cudaStream_t st) {
  int bh = max_height >> 2;
  int strips = (bh > 1 ? bh - 1 + kRowsPerBlock - 1 : 1) / kRowsPerBlock;
  if (strips < 1) strips = 1;
  size_t smem = ssim_rows_smem(max_width);
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(ssim_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  dim3 grid(strips, n_jobs);
  ssim_rows_kernel<<<grid, kThreads, smem, st>>>(d_jobs);
  ssim_finish_kernel<<<(n_jobs + 63) / 64, 64, 0, st>>>(d_jobs, n_jobs);
}

void launch_sse(const SsimJob* d_jobs, int n_jobs, cudaStream_t st) {
  dim3 grid(64, n_jobs);
  sse_kernel<<<grid, 256, 0, st>>>(d_jobs);
}

void launch_decimate(const DecimateJob* d_jobs, int n_jobs, int max_dst_pixels, cudaStream_t st) {
  int blocks = (max_dst_pixels + 255) / 256;
  if (blocks > 1024) blocks = 1024;
  if (blocks < 1) blocks = 1;
  dim3 grid(blocks, n_jobs);
  decimate_kernel<<<grid, 256, 0, st>>>(d_jobs);
}

}  // namespace rg
