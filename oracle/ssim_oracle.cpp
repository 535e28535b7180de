// TEST INFRASTRUCTURE ONLY -- not part of the product path.
//
// CPU oracle of ragdoll's SSIM / MS-SSIM / PSNR / VMAF-Lite (FFmpeg vf_ssim 4x4-sum reuse):
//   crates/ragdoll-simd/src/metrics.rs:409-423  SSIM_C1_8BIT, SSIM_C2_8BIT, ssim_end1_8bit
//   crates/ragdoll-simd/src/metrics.rs:505      ssim_4x4xn_u8_scalar
//   crates/ragdoll-simd/src/metrics.rs:637      ssim_plane_8bit (f32 per row, f64 across rows)
//   crates/ragdoll-pix/src/metrics.rs:87,154    decimate_2x2_u8_scalar, ms_ssim_plane_u8
//   crates/ragdoll-pix/src/metrics.rs:218       vmaf_lite_plane_u8 (per-4x4 SSIM / VIF terms, f64
//                                               sums in raster order, motion term from the plane SAD)
//   crates/ragdoll-simd/src/metrics.rs:60,221   sad_plane_u8_scalar, sse_plane_u8_scalar
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

// crates/ragdoll-simd/src/metrics.rs:221 sse_plane_u8_scalar
uint64_t oracle_sse_plane(const uint8_t* a, long sa, const uint8_t* b, long sb, int width, int height) {
  uint64_t sse = 0;
  for (int y = 0; y < height; y++)
    for (int x = 0; x < width; x++) {
      int d = (int)a[y * sa + x] - (int)b[y * sb + x];
      sse += (uint64_t)(d * d);
    }
  return sse;
}

// crates/ragdoll-pix/src/metrics.rs:218 vmaf_lite_plane_u8; prev may be NULL (no motion term).
double oracle_vmaf_lite_plane(const uint8_t* ref, long sr, const uint8_t* dist, long sd, int width, int height,
                              const uint8_t* prev, long sp) {
  int bw = width >> 2, bh = height >> 2;
  if (bw == 0 || bh == 0) return 100.0;
  const double kSigmaNsq = 2.0 * 256.0, kEps = 1.0e-10, kGainLimit = 100.0;
  std::vector<int> sums((size_t)bw * 4);
  double info_num = 0.0, info_den = 0.0, ssim_acc = 0.0;
  long blocks = 0;
  for (int by = 0; by < bh; by++) {
    sums4x4(ref + (long)by * 4 * sr, sr, dist + (long)by * 4 * sd, sd, bw, (int(*)[4])sums.data());
    for (int bx = 0; bx < bw; bx++) {
      int s1 = sums[bx * 4], s2 = sums[bx * 4 + 1], ss = sums[bx * 4 + 2], s12 = sums[bx * 4 + 3];
      double mean_sq_sum = (double)(s1 * s1 + s2 * s2);
      double total_var = (double)std::max(ss * 16 - s1 * s1 - s2 * s2, 0);
      double covar = (double)(s12 * 16 - s1 * s2);
      const double c1 = 26.0, c2 = 234.0;
      double blk = ((2.0 * (double)s1 * (double)s2 + c1) * (2.0 * covar + c2)) / ((mean_sq_sum + c1) * (total_var + c2));
      ssim_acc += std::min(1.0, std::max(0.0, blk));
      double err_var = (double)std::max(ss - 2 * s12, 0) * 16.0 - (double)((s1 - s2) * (s1 - s2));
      err_var = std::max(err_var, 0.0);
      double sigma1_sq = std::max((total_var - err_var) * 0.5, std::max(covar, 0.0));
      double sigma2_sq = std::max(total_var - sigma1_sq, 0.0);
      double sigma12 = std::max(covar, 0.0);
      double g, sv_sq;
      if (sigma1_sq < kEps) {
        g = 0.0; sv_sq = sigma2_sq;
      } else if (sigma2_sq < kEps) {
        g = 0.0; sv_sq = 0.0;
      } else {
        double g_raw = sigma12 / (sigma1_sq + kEps);
        if (g_raw < 0.0) { g = 0.0; sv_sq = sigma2_sq; }
        else { g = std::min(g_raw, kGainLimit); sv_sq = std::max(sigma2_sq - g_raw * sigma12, kEps); }
      }
      sv_sq = std::max(sv_sq, kEps);
      g = std::min(g, kGainLimit);
      info_num += std::log2(1.0 + (g * g * sigma1_sq) / (sv_sq + kSigmaNsq));
      info_den += std::log2(1.0 + sigma1_sq / kSigmaNsq);
      blocks++;
    }
  }
  double mean_ssim = ssim_acc / (double)std::max(blocks, 1L);
  if (std::fabs(1.0 - mean_ssim) < 1e-9) return 100.0;
  double vif = info_den <= 1e-9 ? mean_ssim : std::min(1.0, std::max(0.0, info_num / info_den));
  double boost = 0.0;
  if (prev) {
    uint64_t sad = 0;
    for (int y = 0; y < height; y++)
      for (int x = 0; x < width; x++) sad += (uint64_t)std::abs((int)ref[y * sr + x] - (int)prev[y * sp + x]);
    double mad = (double)sad / ((double)width * height);
    boost = std::min(mad / 255.0 * 0.08, 0.05);
  }
  double raw = (0.65 * std::pow(mean_ssim, 0.85) + 0.35 * vif + boost) * 100.0;
  return std::min(100.0, std::max(0.0, raw));
}

}  // extern "C"
