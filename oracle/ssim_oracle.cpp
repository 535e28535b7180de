// TEST INFRASTRUCTURE ONLY -- not part of the product path.
//
// CPU oracle of ragdoll's SSIM / MS-SSIM / PSNR (FFmpeg vf_ssim 4x4-sum reuse):
//   crates/ragdoll-simd/src/metrics.rs:409-423  SSIM_C1_8BIT, SSIM_C2_8BIT, ssim_end1_8bit
//   crates/ragdoll-simd/src/metrics.rs:505      ssim_4x4xn_u8_scalar
//   crates/ragdoll-simd/src/metrics.rs:637      ssim_plane_8bit (f32 per row, f64 across rows)
//   crates/ragdoll-pix/src/metrics.rs:87,154    decimate_2x2_u8_scalar, ms_ssim_plane_u8
// Built with -ffp-contract=off so no product is fused into an add, as in the reference.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

const int kC1 = 416;
const int kC2 = 235963;
const double kMsWeights[5] = {0.0448, 0.2856, 0.3001, 0.2363, 0.1333};

float ssim_end1(int s1, int s2, int ss, int s12) {
  int vars = ss * 64 - s1 * s1 - s2 * s2;
  int covar = s12 * 64 - s1 * s2;
  float num = (float)(2 * s1 * s2 + kC1) * (float)(2 * covar + kC2);
  float den = (float)(s1 * s1 + s2 * s2 + kC1) * (float)(vars + kC2);
  return num / den;
}

void sums4x4(const uint8_t* a, long sa, const uint8_t* b, long sb, int n, int (*out)[4]) {
  for (int k = 0; k < n; k++) {
    int s1 = 0, s2 = 0, ss = 0, s12 = 0;
    for (int y = 0; y < 4; y++)
      for (int x = 0; x < 4; x++) {
        int va = a[y * sa + k * 4 + x], vb = b[y * sb + k * 4 + x];
        s1 += va; s2 += vb; ss += va * va + vb * vb; s12 += va * vb;
      }
    out[k][0] = s1; out[k][1] = s2; out[k][2] = ss; out[k][3] = s12;
  }
}

}  // namespace

extern "C" {

double oracle_ssim_plane(const uint8_t* a, long sa, const uint8_t* b, long sb, int width, int height) {
  int bw = width >> 2, bh = height >> 2;
  if (bw < 2 || bh < 2) {
    int s1 = 0, s2 = 0, ss = 0, s12 = 0;
    for (int y = 0; y < 8; y++)
      for (int x = 0; x < 8; x++) {
        int va = a[y * sa + x], vb = b[y * sb + x];
        s1 += va; s2 += vb; ss += va * va + vb * vb; s12 += va * vb;
      }
    return (double)ssim_end1(s1, s2, ss, s12);
  }
  std::vector<int> r0((size_t)bw * 4), r1((size_t)bw * 4);
  sums4x4(a, sa, b, sb, bw, (int(*)[4])r0.data());
  double total = 0.0;
  for (int by = 1; by < bh; by++) {
    sums4x4(a + (long)by * 4 * sa, sa, b + (long)by * 4 * sb, sb, bw, (int(*)[4])r1.data());
    float row = 0.0f;
    for (int bx = 0; bx < bw - 1; bx++) {
      int v[4];
      for (int k = 0; k < 4; k++) v[k] = r0[bx * 4 + k] + r0[(bx + 1) * 4 + k] + r1[bx * 4 + k] + r1[(bx + 1) * 4 + k];
      row += ssim_end1(v[0], v[1], v[2], v[3]);
    }
    total += (double)row;
    std::swap(r0, r1);
  }
  return total / (double)((bw - 1) * (bh - 1));
}

static void decimate2x2(const uint8_t* src, long ss, uint8_t* dst, long ds, int sw, int sh) {
  for (int dy = 0; dy < (sh >> 1); dy++)
    for (int dx = 0; dx < (sw >> 1); dx++) {
      int s = src[(2 * dy) * ss + 2 * dx] + src[(2 * dy) * ss + 2 * dx + 1] + src[(2 * dy + 1) * ss + 2 * dx] +
              src[(2 * dy + 1) * ss + 2 * dx + 1];
      dst[dy * ds + dx] = (uint8_t)((s + 2) >> 2);
    }
}

double oracle_ms_ssim_plane(const uint8_t* a, long sa, const uint8_t* b, long sb, int width, int height) {
  double s0 = std::min(1.0, std::max(0.0, oracle_ssim_plane(a, sa, b, sb, width, height)));
  if (std::fabs(1.0 - s0) < 1e-12 || (width >> 1) < 8 || (height >> 1) < 8) return s0;
  double scores[5] = {s0, s0, s0, s0, s0};
  int active = 1, cw = width, ch = height;
  std::vector<uint8_t> ba, bb;
  for (int sc = 1; sc < 5; sc++) {
    int nw = cw >> 1, nh = ch >> 1;
    if (nw < 8 || nh < 8) break;
    std::vector<uint8_t> na((size_t)nw * nh), nb((size_t)nw * nh);
    if (sc == 1) {
      decimate2x2(a, sa, na.data(), nw, cw, ch);
      decimate2x2(b, sb, nb.data(), nw, cw, ch);
    } else {
      decimate2x2(ba.data(), cw, na.data(), nw, cw, ch);
      decimate2x2(bb.data(), cw, nb.data(), nw, cw, ch);
    }
    scores[sc] = std::min(1.0, std::max(0.0, oracle_ssim_plane(na.data(), nw, nb.data(), nw, nw, nh)));
    ba.swap(na); bb.swap(nb);
    cw = nw; ch = nh;
    active++;
  }
  double wsum = 0.0;
  for (int s = 0; s < active; s++) wsum += kMsWeights[s];
  double prod = 1.0;
  for (int s = 0; s < active; s++) prod *= std::pow(std::max(scores[s], 1e-9), kMsWeights[s] / wsum);
  return std::min(1.0, std::max(0.0, prod));
}

// crates/ragdoll-pix/src/metrics.rs:336-351 (plane SSE -> PSNR)
double oracle_psnr_plane(const uint8_t* a, long sa, const uint8_t* b, long sb, int width, int height) {
  uint64_t sse = 0;
  for (int y = 0; y < height; y++)
    for (int x = 0; x < width; x++) {
      int d = (int)a[y * sa + x] - (int)b[y * sb + x];
      sse += (uint64_t)(d * d);
    }
  if (sse == 0) return INFINITY;
  double mse = (double)sse / ((double)width * height);
  return 10.0 * std::log10((255.0 * 255.0) / mse);
}

}  // extern "C"
