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

size_t ssim_rows_smem(int width);
void launch_ssim(const SsimJob* d_jobs, int n_jobs, int max_width, int max_height, cudaStream_t st);
void launch_sse(const SsimJob* d_jobs, int n_jobs, cudaStream_t st);
void launch_decimate(const DecimateJob* d_jobs, int n_jobs, int max_dst_pixels, cudaStream_t st);

}  // namespace rg
