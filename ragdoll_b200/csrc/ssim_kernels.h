// Device SSIM / MS-SSIM / PSNR jobs (ssim_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace rg {

// One plane pair. rows: device scratch of (height / 4) floats; out: device f64 result.
struct SsimJob {
  const uint8_t* a;
  const uint8_t* b;
  long stride_a, stride_b;
  int width, height;
  float* rows;
  double* out;
  unsigned long long* sse;  // optional SSE accumulator (PSNR)
};

// One 2x2 decimation of a plane pair into compact planes (stride = src_w / 2).
struct DecimateJob {
  const uint8_t* src_a;
  const uint8_t* src_b;
  long stride_a, stride_b;
  int src_w, src_h;
  uint8_t* dst_a;
  uint8_t* dst_b;
};

// VMAF-Lite of one plane pair (ref a, distorted b; prev: the previous reference frame or null).
// rows: device scratch of 3 * (height / 4) doubles; out: device {info_num, info_den, ssim_sum};
// sad: optional accumulator of |a - prev| over the plane.
struct VmafJob {
  const uint8_t* a;
  const uint8_t* b;
  const uint8_t* prev;
  long stride_a, stride_b, stride_prev;
  int width, height;
  double* rows;
  double* out;
  unsigned long long* sad;
};

size_t ssim_rows_smem(int width);
void launch_vmaf(const VmafJob* d_jobs, int n_jobs, int max_height, cudaStream_t st);
// The score from the sums (crates/ragdoll-pix/src/metrics.rs:301-324); host code.
double vmaf_lite_score(double info_num, double info_den, double ssim_sum, long blocks, bool have_prev,
                       unsigned long long sad, long pixels);
void launch_ssim(const SsimJob* d_jobs, int n_jobs, int max_width, int max_height, cudaStream_t st);
void launch_sse(const SsimJob* d_jobs, int n_jobs, cudaStream_t st);
void launch_decimate(const DecimateJob* d_jobs, int n_jobs, int max_dst_pixels, cudaStream_t st);

}  // namespace rg
