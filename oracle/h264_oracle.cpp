// TEST INFRASTRUCTURE ONLY -- not part of the product path.
//
// CPU oracle: a scalar C++ restatement of ragdoll's Balanced H.264 encoder (analysis,
// reconstruction, deblocking, CAVLC and CABAC slice writers, SPS/PPS/slice headers, NAL packing). The GPU
// engine's decisions, levels and reconstructions are checked against it, and it is itself pinned
// byte for byte to the reference's committed encoder output (qa/corpus/synth/clip_160x90_30fps.mp4)
// by tests/test_oracle_golden.py. Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg load it.
//
// Each function cites the reference code it restates (paths inside oddurs/ragdoll).
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../include/ragdoll_cuda.h"
#include "oracle_tables.h"

namespace oracle {

// enc.rs:56-61
static const int PAD_Y = 48;
static const int PAD_C = 16;
static const int MV_MARGIN = 28;
static const int MV_COST_RANGE = 4096;

static inline int clamp255(int v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }
static inline int16_t clamp_i16(int64_t v) {
  return (int16_t)(v < -32768 ? -32768 : (v > 32767 ? 32767 : v));
}
static inline int iabs(int v) { return v < 0 ? -v : v; }
static inline int clz32(uint32_t v) { return v ? __builtin_clz(v) : 32; }

// ---------------------------------------------------------------------------------------------
// Padded planes (enc.rs:100-213)
struct Plane {
  std::vector<uint8_t> buf;
  int stride = 0, w = 0, h = 0, pad = 0;
  void alloc(int w_, int h_, int pad_) {
    w = w_; h = h_; pad = pad_;
    stride = (w + 2 * pad + 31) & ~31;
    buf.assign((size_t)stride * (h + 2 * pad), 0);
  }
  int at(int x, int y) const { return (y + pad) * stride + x + pad; }
  uint8_t* ptr(int x, int y) { return &buf[at(x, y)]; }
  const uint8_t* ptr(int x, int y) const { return &buf[at(x, y)]; }
  // enc.rs:165 extend_borders
  void extend_borders() {
    int p = pad, s = stride;
    for (int y = p; y < p + h; y++) {
      uint8_t* row = &buf[(size_t)y * s];
      uint8_t l = row[p], r = row[p + w - 1];
      memset(row, l, p);
      memset(row + p + w, r, s - p - w);
    }
    for (int y = 0; y < p; y++) {
      memcpy(&buf[(size_t)y * s], &buf[(size_t)p * s], s);
      memcpy(&buf[(size_t)(p + h + y) * s], &buf[(size_t)(p + h - 1) * s], s);
    }
  }
};
struct Pic {
  Plane y, u, v;
  void alloc(int w, int h) { y.alloc(w, h, PAD_Y); u.alloc(w / 2, h / 2, PAD_C); v.alloc(w / 2, h / 2, PAD_C); }
};

// enc.rs:522 blk_xy: column and row of 4x4 block b (decoding order)
static inline void blk_xy(int b, int& x, int& y) {
  x = (b & 1) + ((b >> 1) & 2);
  y = ((b >> 1) & 1) + ((b >> 2) & 2);
}
static inline int chroma_qp(int qp, int off) {
  int i = qp + off;
  return kChromaQp[i < 0 ? 0 : (i > 51 ? 51 : i)];
}
// enc.rs:546 se_bits
static inline uint32_t se_bits(int d) {
  uint32_t v = (uint32_t)iabs(d) * 2 - (d > 0 ? 1 : 0);
  return 2 * (32 - clz32(v + 1)) - 1;
}
// enc.rs:559 decimate_score
static uint32_t decimate_score(const int16_t* s, int n) {
  const uint8_t* table = n == 64 ? kDecimate8 : kDecimate4;
  int idx = n;
  while (idx > 0 && s[idx - 1] == 0) idx--;
  uint32_t score = 0;
  while (idx > 0) {
    idx--;
    if (iabs(s[idx]) > 1) return 9;
    int run = 0;
    while (idx > 0 && s[idx - 1] == 0) { idx--; run++; }
    score += table[run];
  }
  return score;
}

// ---------------------------------------------------------------------------------------------
// Integer work actually evaluated by the decisions: pixel differences of every SAD, SSD and SATD
// (a SATD of n samples counts n; the three-way I16 SATD counts 3 x 256). Counted per encoding
// thread and added to the process total after each frame (a measurement, not part of the
// algorithm).
static thread_local uint64_t t_pixel_ops = 0;
static std::atomic<uint64_t> g_pixel_ops{0};

// ---------------------------------------------------------------------------------------------
// Pixel kernels (crates/ragdoll-simd, the _scalar functions)
static uint32_t sad(const uint8_t* a, int sa, const uint8_t* b, int sb, int w, int h) {
  t_pixel_ops += (uint64_t)w * h;
  uint32_t s = 0;
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) s += (uint32_t)iabs((int)a[y * sa + x] - (int)b[y * sb + x]);
  return s;
}
static uint32_t ssd(const uint8_t* a, int sa, const uint8_t* b, int sb, int n) {
  t_pixel_ops += (uint64_t)n * n;
  uint32_t s = 0;
  for (int y = 0; y < n; y++)
    for (int x = 0; x < n; x++) {
      int d = (int)a[y * sa + x] - (int)b[y * sb + x];
      s += (uint32_t)(d * d);
    }
  return s;
}
// fixed.rs:104 forward_dct4x4_scalar
static void fdct4(const int16_t* in, int16_t* out) {
  int t[16];
  for (int r = 0; r < 4; r++) {
    const int16_t* b = in + r * 4;
    int s03 = b[0] + b[3], s12 = b[1] + b[2], d03 = b[0] - b[3], d12 = b[1] - b[2];
    t[r * 4 + 0] = s03 + s12;
    t[r * 4 + 1] = (d03 << 1) + d12;
    t[r * 4 + 2] = s03 - s12;
    t[r * 4 + 3] = d03 - (d12 << 1);
  }
  for (int c = 0; c < 4; c++) {
    int s03 = t[c] + t[c + 12], s12 = t[c + 4] + t[c + 8];
    int d03 = t[c] - t[c + 12], d12 = t[c + 4] - t[c + 8];
    out[c] = (int16_t)(s03 + s12);
    out[c + 4] = (int16_t)((d03 << 1) + d12);
    out[c + 8] = (int16_t)(s03 - s12);
    out[c + 12] = (int16_t)(d03 - (d12 << 1));
  }
}
// fixed.rs:192 inverse_idct4x4_scalar
static void idct4(const int16_t* c, int16_t* out) {
  int t[16];
  for (int r = 0; r < 4; r++) {
    const int16_t* b = c + r * 4;
    int e0 = b[0] + b[2], e1 = b[0] - b[2];
    int e2 = (b[1] >> 1) - b[3], e3 = b[1] + (b[3] >> 1);
    t[r * 4 + 0] = e0 + e3;
    t[r * 4 + 1] = e1 + e2;
    t[r * 4 + 2] = e1 - e2;
    t[r * 4 + 3] = e0 - e3;
  }
  for (int k = 0; k < 4; k++) {
    int e0 = t[k] + t[k + 8], e1 = t[k] - t[k + 8];
    int e2 = (t[k + 4] >> 1) - t[k + 12], e3 = t[k + 4] + (t[k + 12] >> 1);
    out[k] = (int16_t)((e0 + e3 + 32) >> 6);
    out[k + 4] = (int16_t)((e1 + e2 + 32) >> 6);
    out[k + 8] = (int16_t)((e1 - e2 + 32) >> 6);
    out[k + 12] = (int16_t)((e0 - e3 + 32) >> 6);
  }
}
// h264_enc.rs:497 add_idct4x4_8x8_scalar (one block)
static void add_idct4(uint8_t* dst, int ds, const int16_t* c) {
  int16_t r[16];
  idct4(c, r);
  for (int y = 0; y < 4; y++)
    for (int x = 0; x < 4; x++) dst[y * ds + x] = (uint8_t)clamp255(dst[y * ds + x] + r[y * 4 + x]);
}
// fixed.rs:322 hadamard4x4_scalar (output >> 1)
static void hadamard4_dc(const int16_t* in, int16_t* out) {
  int t[16];
  for (int r = 0; r < 4; r++) {
    const int16_t* b = in + r * 4;
    int s03 = b[0] + b[3], s12 = b[1] + b[2], d03 = b[0] - b[3], d12 = b[1] - b[2];
    t[r * 4 + 0] = s03 + s12;
    t[r * 4 + 1] = d03 + d12;
    t[r * 4 + 2] = s03 - s12;
    t[r * 4 + 3] = d03 - d12;
  }
  for (int c = 0; c < 4; c++) {
    int s03 = t[c] + t[c + 12], s12 = t[c + 4] + t[c + 8];
    int d03 = t[c] - t[c + 12], d12 = t[c + 4] - t[c + 8];
    out[c] = (int16_t)((s03 + s12) >> 1);
    out[c + 4] = (int16_t)((d03 + d12) >> 1);
    out[c + 8] = (int16_t)((s03 - s12) >> 1);
    out[c + 12] = (int16_t)((d03 - d12) >> 1);
  }
}
// fixed.rs:392 forward_dct8x8
static void fdct8(const int16_t* in, int16_t* out) {
  int t[64];
  auto pass = [](const int* a, int* o) {
    int a0 = a[0] + a[7], a1 = a[1] + a[6], a2 = a[2] + a[5], a3 = a[3] + a[4];
    int a4 = a[0] - a[7], a5 = a[1] - a[6], a6 = a[2] - a[5], a7 = a[3] - a[4];
    int b0 = a0 + a3, b1 = a1 + a2, b2 = a0 - a3, b3 = a1 - a2;
    int b4 = a5 + a6 + ((a4 >> 1) + a4);
    int b5 = a4 - a7 - ((a6 >> 1) + a6);
    int b6 = a4 + a7 - ((a5 >> 1) + a5);
    int b7 = a5 - a6 + ((a7 >> 1) + a7);
    o[0] = b0 + b1;
    o[1] = b4 + (b7 >> 2);
    o[2] = b2 + (b3 >> 1);
    o[3] = b5 + (b6 >> 2);
    o[4] = b0 - b1;
    o[5] = b6 - (b5 >> 2);
    o[6] = (b2 >> 1) - b3;
    o[7] = (b4 >> 2) - b7;
  };
  for (int r = 0; r < 8; r++) {
    int a[8], o[8];
    for (int k = 0; k < 8; k++) a[k] = in[r * 8 + k];
    pass(a, o);
    for (int k = 0; k < 8; k++) t[r * 8 + k] = o[k];
  }
  for (int c = 0; c < 8; c++) {
    int a[8], o[8];
    for (int k = 0; k < 8; k++) a[k] = t[k * 8 + c];
    pass(a, o);
    for (int k = 0; k < 8; k++) out[k * 8 + c] = (int16_t)o[k];
  }
}
// h264_idct.rs:225 idct8_1d (wrapping i32)
static void idct8_1d(const int32_t* d, int32_t* o) {
  auto W = [](int64_t v) { return (int32_t)(uint32_t)v; };
  int32_t a0 = W((int64_t)d[0] + d[4]);
  int32_t a1 = W((int64_t)d[5] - d[3] - d[7] - (d[7] >> 1));
  int32_t a2 = W((int64_t)d[0] - d[4]);
  int32_t a3 = W((int64_t)d[1] + d[7] - d[3] - (d[3] >> 1));
  int32_t a4 = W((int64_t)(d[2] >> 1) - d[6]);
  int32_t a5 = W((int64_t)d[7] - d[1] + d[5] + (d[5] >> 1));
  int32_t a6 = W((int64_t)d[2] + (d[6] >> 1));
  int32_t a7 = W((int64_t)d[3] + d[5] + d[1] + (d[1] >> 1));
  int32_t b0 = W((int64_t)a0 + a6), b1 = W((int64_t)a1 + (a7 >> 2));
  int32_t b2 = W((int64_t)a2 + a4), b3 = W((int64_t)a3 + (a5 >> 2));
  int32_t b4 = W((int64_t)a2 - a4), b5 = W((int64_t)(a3 >> 2) - a5);
  int32_t b6 = W((int64_t)a0 - a6), b7 = W((int64_t)a7 - (a1 >> 2));
  o[0] = W((int64_t)b0 + b7); o[1] = W((int64_t)b2 + b5);
  o[2] = W((int64_t)b4 + b3); o[3] = W((int64_t)b6 + b1);
  o[4] = W((int64_t)b6 - b1); o[5] = W((int64_t)b4 - b3);
  o[6] = W((int64_t)b2 - b5); o[7] = W((int64_t)b0 - b7);
}
// h264_idct.rs:268 h264_idct8_add_scalar
static void idct8_add(uint8_t* dst, int stride, const int32_t* d) {
  int32_t g[64];
  for (int i = 0; i < 8; i++) idct8_1d(d + i * 8, g + i * 8);
  for (int j = 0; j < 8; j++) {
    int32_t col[8], o[8];
    for (int i = 0; i < 8; i++) col[i] = g[i * 8 + j];
    idct8_1d(col, o);
    for (int i = 0; i < 8; i++) {
      int32_t v = (int32_t)((uint32_t)o[i] + 32u) >> 6;
      dst[i * stride + j] = (uint8_t)clamp255((int32_t)((uint32_t)dst[i * stride + j] + (uint32_t)v));
    }
  }
}
// metrics.rs:705 satd_4x4_u8_scalar (halved)
static uint32_t satd4(const uint8_t* a, int sa, const uint8_t* b, int sb) {
  t_pixel_ops += 16;
  int t[4][4];
  for (int y = 0; y < 4; y++) {
    int d0 = a[y * sa] - b[y * sb], d1 = a[y * sa + 1] - b[y * sb + 1];
    int d2 = a[y * sa + 2] - b[y * sb + 2], d3 = a[y * sa + 3] - b[y * sb + 3];
    int s03 = d0 + d3, s12 = d1 + d2, d03 = d0 - d3, d12 = d1 - d2;
    t[y][0] = s03 + s12; t[y][1] = d03 + d12; t[y][2] = s03 - s12; t[y][3] = d03 - d12;
  }
  uint32_t s = 0;
  for (int x = 0; x < 4; x++) {
    int s03 = t[0][x] + t[3][x], s12 = t[1][x] + t[2][x], d03 = t[0][x] - t[3][x], d12 = t[1][x] - t[2][x];
    s += iabs(s03 + s12) + iabs(d03 + d12) + iabs(s03 - s12) + iabs(d03 - d12);
  }
  return s >> 1;
}
// The unhalved sum of one 4x4 transform (the search forms halve the sum over a partition's blocks).
static uint32_t satd4_raw(const uint8_t* a, int sa, const uint8_t* b, int sb) {
  t_pixel_ops += 16;
  int t[4][4];
  for (int y = 0; y < 4; y++) {
    int d0 = a[y * sa] - b[y * sb], d1 = a[y * sa + 1] - b[y * sb + 1];
    int d2 = a[y * sa + 2] - b[y * sb + 2], d3 = a[y * sa + 3] - b[y * sb + 3];
    int s03 = d0 + d3, s12 = d1 + d2, d03 = d0 - d3, d12 = d1 - d2;
    t[y][0] = s03 + s12; t[y][1] = d03 + d12; t[y][2] = s03 - s12; t[y][3] = d03 - d12;
  }
  uint32_t s = 0;
  for (int x = 0; x < 4; x++) {
    int s03 = t[0][x] + t[3][x], s12 = t[1][x] + t[2][x], d03 = t[0][x] - t[3][x], d12 = t[1][x] - t[2][x];
    s += iabs(s03 + s12) + iabs(d03 + d12) + iabs(s03 - s12) + iabs(d03 - d12);
  }
  return s;
}
// h264_enc.rs:167 pixel_satd_16x16_scalar (sum of 4x4 transforms, halved once)
static uint32_t satd16(const uint8_t* a, int sa, const uint8_t* b, int sb) {
  t_pixel_ops += 256;
  uint32_t sum = 0;
  for (int by = 0; by < 4; by++)
    for (int bx = 0; bx < 4; bx++) {
      int d[4][4];
      for (int y = 0; y < 4; y++)
        for (int x = 0; x < 4; x++)
          d[y][x] = a[(by * 4 + y) * sa + bx * 4 + x] - b[(by * 4 + y) * sb + bx * 4 + x];
      for (int y = 0; y < 4; y++) {
        int s01 = d[y][0] + d[y][1], d01 = d[y][0] - d[y][1];
        int s23 = d[y][2] + d[y][3], d23 = d[y][2] - d[y][3];
        d[y][0] = s01 + s23; d[y][1] = s01 - s23; d[y][2] = d01 + d23; d[y][3] = d01 - d23;
      }
      for (int c = 0; c < 4; c++) {
        int s01 = d[0][c] + d[1][c], d01 = d[0][c] - d[1][c];
        int s23 = d[2][c] + d[3][c], d23 = d[2][c] - d[3][c];
        sum += iabs(s01 + s23) + iabs(s01 - s23) + iabs(d01 + d23) + iabs(d01 - d23);
      }
    }
  return sum >> 1;
}
// h264_mc.rs:148 h264_luma_mc_scalar; src points at the integer sample of the block origin.
static void luma_mc(const uint8_t* src, int ss, int w, int h, int mx, int my, uint8_t* dst, int ds) {
  auto at = [&](int r, int c) { return (int)src[r * ss + c]; };
  auto tap = [](int a, int b, int c, int d, int e, int f) { return a - 5 * b + 20 * c + 20 * d - 5 * e + f; };
  auto hraw = [&](int r, int c) { return tap(at(r, c - 2), at(r, c - 1), at(r, c), at(r, c + 1), at(r, c + 2), at(r, c + 3)); };
  auto G = [&](int r, int c) { return at(r, c); };
  auto B = [&](int r, int c) { return clamp255((hraw(r, c) + 16) >> 5); };
  auto V = [&](int r, int c) {
    return clamp255((tap(at(r - 2, c), at(r - 1, c), at(r, c), at(r + 1, c), at(r + 2, c), at(r + 3, c)) + 16) >> 5);
  };
  auto J = [&](int r, int c) {
    return clamp255((tap(hraw(r - 2, c), hraw(r - 1, c), hraw(r, c), hraw(r + 1, c), hraw(r + 2, c), hraw(r + 3, c)) + 512) >> 10);
  };
  auto avg = [](int a, int b) { return (a + b + 1) >> 1; };
  for (int r = 0; r < h; r++)
    for (int c = 0; c < w; c++) {
      int v;
      switch ((mx & 3) | ((my & 3) << 2)) {
        case 0: v = G(r, c); break;
        case 1: v = avg(G(r, c), B(r, c)); break;
        case 2: v = B(r, c); break;
        case 3: v = avg(B(r, c), G(r, c + 1)); break;
        case 4: v = avg(G(r, c), V(r, c)); break;
        case 5: v = avg(B(r, c), V(r, c)); break;
        case 6: v = avg(B(r, c), J(r, c)); break;
        case 7: v = avg(B(r, c), V(r, c + 1)); break;
        case 8: v = V(r, c); break;
        case 9: v = avg(V(r, c), J(r, c)); break;
        case 10: v = J(r, c); break;
        case 11: v = avg(J(r, c), V(r, c + 1)); break;
        case 12: v = avg(V(r, c), G(r + 1, c)); break;
        case 13: v = avg(V(r, c), B(r + 1, c)); break;
        case 14: v = avg(J(r, c), B(r + 1, c)); break;
        default: v = avg(V(r, c + 1), B(r + 1, c)); break;
      }
      dst[r * ds + c] = (uint8_t)v;
    }
}
// h264_enc.rs:1279 chroma_mc_8x8_x2_scalar (one plane)
static void chroma_mc(const uint8_t* src, int ss, int fx, int fy, uint8_t* out) {
  int wa = (8 - fx) * (8 - fy), wb = fx * (8 - fy), wc = (8 - fx) * fy, wd = fx * fy;
  for (int r = 0; r < 8; r++)
    for (int c = 0; c < 8; c++) {
      int x = wa * src[r * ss + c] + wb * src[r * ss + c + 1] + wc * src[(r + 1) * ss + c] + wd * src[(r + 1) * ss + c + 1];
      out[r * 8 + c] = (uint8_t)((x + 32) >> 6);
    }
}
// h264_dsp.rs:799 predict_intra_4x4_u8_scalar
static void pred4x4(int mode, const uint8_t* top /*8 or null*/, const uint8_t* left /*4 or null*/, int tl, uint8_t* dst) {
  uint8_t t[8], l[4];
  for (int i = 0; i < 8; i++) t[i] = top ? top[i] : 128;
  for (int i = 0; i < 4; i++) l[i] = left ? left[i] : 128;
  int a = t[0], b = t[1], c = t[2], d = t[3], e = t[4], f = t[5], g = t[6], h = t[7];
  int i = l[0], j = l[1], k = l[2], ls = l[3], m = tl;
  auto a2 = [](int x, int y) { return (uint8_t)((x + y + 1) >> 1); };
  auto a3 = [](int x, int y, int z) { return (uint8_t)((x + 2 * y + z + 2) >> 2); };
  uint8_t o[16];
  switch (mode) {
    case 0: for (int y = 0; y < 4; y++) for (int x = 0; x < 4; x++) o[y * 4 + x] = t[x]; break;
    case 1: for (int y = 0; y < 4; y++) for (int x = 0; x < 4; x++) o[y * 4 + x] = l[y]; break;
    case 2: {
      int dc;
      if (top && left) dc = (a + b + c + d + i + j + k + ls + 4) >> 3;
      else if (top) dc = (a + b + c + d + 2) >> 2;
      else if (left) dc = (i + j + k + ls + 2) >> 2;
      else dc = 128;
      for (int q = 0; q < 16; q++) o[q] = (uint8_t)dc;
      break;
    }
    case 3: {
      uint8_t p[7] = {a3(a, b, c), a3(b, c, d), a3(c, d, e), a3(d, e, f), a3(e, f, g), a3(f, g, h), a3(g, h, h)};
      for (int y = 0; y < 4; y++) for (int x = 0; x < 4; x++) o[y * 4 + x] = p[x + y];
      break;
    }
    case 4: {
      uint8_t lm = a3(k, j, i), kj = a3(ls, k, j), ji = a3(j, i, m), im = a3(i, m, a), ma = a3(m, a, b), ab = a3(a, b, c), bc = a3(b, c, d);
      uint8_t r[4][4] = {{im, ma, ab, bc}, {ji, im, ma, ab}, {lm, ji, im, ma}, {kj, lm, ji, im}};
      memcpy(o, r, 16);
      break;
    }
    case 5: {
      uint8_t r0[4] = {a2(m, a), a2(a, b), a2(b, c), a2(c, d)};
      uint8_t r1[4] = {a3(i, m, a), a3(m, a, b), a3(a, b, c), a3(b, c, d)};
      uint8_t r2[4] = {a3(j, i, m), r0[0], r0[1], r0[2]};
      uint8_t r3[4] = {a3(k, j, i), r1[0], r1[1], r1[2]};
      memcpy(o, r0, 4); memcpy(o + 4, r1, 4); memcpy(o + 8, r2, 4); memcpy(o + 12, r3, 4);
      break;
    }
    case 6: {
      uint8_t r0[4] = {a2(m, i), a3(i, m, a), a3(m, a, b), a3(a, b, c)};
      uint8_t r1[4] = {a2(i, j), a3(m, i, j), r0[0], r0[1]};
      uint8_t r2[4] = {a2(j, k), a3(i, j, k), r1[0], r1[1]};
      uint8_t r3[4] = {a2(k, ls), a3(j, k, ls), r2[0], r2[1]};
      memcpy(o, r0, 4); memcpy(o + 4, r1, 4); memcpy(o + 8, r2, 4); memcpy(o + 12, r3, 4);
      break;
    }
    case 7: {
      uint8_t r0[4] = {a2(a, b), a2(b, c), a2(c, d), a2(d, e)};
      uint8_t r1[4] = {a3(a, b, c), a3(b, c, d), a3(c, d, e), a3(d, e, f)};
      uint8_t r2[4] = {r0[1], r0[2], r0[3], a2(e, f)};
      uint8_t r3[4] = {r1[1], r1[2], r1[3], a3(e, f, g)};
      memcpy(o, r0, 4); memcpy(o + 4, r1, 4); memcpy(o + 8, r2, 4); memcpy(o + 12, r3, 4);
      break;
    }
    default: {
      uint8_t p0 = a2(i, j), p1 = a3(i, j, k), p2 = a2(j, k), p3 = a3(j, k, ls), p4 = a2(k, ls), p5 = a3(k, ls, ls), p6 = l[3];
      uint8_t r[4][4] = {{p0, p1, p2, p3}, {p2, p3, p4, p5}, {p4, p5, p6, p6}, {p6, p6, p6, p6}};
      memcpy(o, r, 16);
      break;
    }
  }
  memcpy(dst, o, 16);
}
// h264.rs:1715 predict_intra_16x16_scalar / enc.rs:1561 pred16
static void pred16(int mode, const uint8_t* top, const uint8_t* left, int tl, uint8_t* dst) {
  uint8_t t[16], l[16];
  for (int q = 0; q < 16; q++) { t[q] = top ? top[q] : 128; l[q] = left ? left[q] : 128; }
  if (mode == 0) { for (int y = 0; y < 16; y++) memcpy(dst + y * 16, t, 16); return; }
  if (mode == 1) { for (int y = 0; y < 16; y++) memset(dst + y * 16, l[y], 16); return; }
  if (mode == 2) {
    int dc;
    uint32_t st = 0, sl = 0;
    for (int q = 0; q < 16; q++) { st += t[q]; sl += l[q]; }
    if (top && left) dc = (st + sl + 16) >> 5;
    else if (top) dc = (st + 8) >> 4;
    else if (left) dc = (sl + 8) >> 4;
    else dc = 128;
    memset(dst, dc, 256);
    return;
  }
  int H = 0, Vv = 0;
  for (int q = 0; q < 8; q++) {
    int pt = q == 7 ? tl : t[6 - q], pl = q == 7 ? tl : l[6 - q];
    H += (q + 1) * (t[8 + q] - pt);
    Vv += (q + 1) * (l[8 + q] - pl);
  }
  int a = 16 * (t[15] + l[15]), b = (5 * H + 32) >> 6, c = (5 * Vv + 32) >> 6;
  for (int y = 0; y < 16; y++)
    for (int x = 0; x < 16; x++) dst[y * 16 + x] = (uint8_t)clamp255((a + b * (x - 7) + c * (y - 7) + 16) >> 5);
}
// h264.rs:1967 predict_intra_chroma_8x8_scalar / enc.rs:1586 pred_chroma
static void pred_chroma(int mode, const uint8_t* top, const uint8_t* left, int tl, uint8_t* dst) {
  uint8_t t[8], l[8];
  for (int q = 0; q < 8; q++) { t[q] = top ? top[q] : 128; l[q] = left ? left[q] : 128; }
  if (mode == 0) {
    int d00, d01, d10, d11;
    int st0 = t[0] + t[1] + t[2] + t[3], st1 = t[4] + t[5] + t[6] + t[7];
    int sl0 = l[0] + l[1] + l[2] + l[3], sl1 = l[4] + l[5] + l[6] + l[7];
    if (top && left) {
      d00 = (st0 + sl0 + 4) >> 3; d01 = (st1 + 2) >> 2; d10 = (sl1 + 2) >> 2; d11 = (st1 + sl1 + 4) >> 3;
    } else if (top) {
      d00 = d10 = (st0 + 2) >> 2; d01 = d11 = (st1 + 2) >> 2;
    } else if (left) {
      d00 = d01 = (sl0 + 2) >> 2; d10 = d11 = (sl1 + 2) >> 2;
    } else {
      d00 = d01 = d10 = d11 = 128;
    }
    for (int y = 0; y < 8; y++)
      for (int x = 0; x < 8; x++) dst[y * 8 + x] = (uint8_t)(y < 4 ? (x < 4 ? d00 : d01) : (x < 4 ? d10 : d11));
    return;
  }
  if (mode == 1) { for (int y = 0; y < 8; y++) memset(dst + y * 8, l[y], 8); return; }
  if (mode == 2) { for (int y = 0; y < 8; y++) memcpy(dst + y * 8, t, 8); return; }
  int H = 0, Vv = 0;
  for (int q = 0; q < 4; q++) {
    int pt = q == 3 ? tl : t[2 - q], pl = q == 3 ? tl : l[2 - q];
    H += (q + 1) * (t[4 + q] - pt);
    Vv += (q + 1) * (l[4 + q] - pl);
  }
  int a = 16 * (t[7] + l[7]), b = (17 * H + 16) >> 5, c = (17 * Vv + 16) >> 5;
  for (int y = 0; y < 8; y++)
    for (int x = 0; x < 8; x++) dst[y * 8 + x] = (uint8_t)clamp255((a + b * (x - 3) + c * (y - 3) + 16) >> 5);
}
// h264_enc.rs:355 hadamard4x4_16x4_scalar for one 4x4 block: out[4v + h]
static void hadamard_src4(const uint8_t* s, int ss, int16_t* out) {
  auto h1 = [](const int* x, int* o) {
    int s01 = x[0] + x[1], d01 = x[0] - x[1], s23 = x[2] + x[3], d23 = x[2] - x[3];
    o[0] = s01 + s23; o[1] = s01 - s23; o[2] = d01 + d23; o[3] = d01 - d23;
  };
  int rows[4][4];
  for (int y = 0; y < 4; y++) {
    int x[4] = {s[y * ss], s[y * ss + 1], s[y * ss + 2], s[y * ss + 3]};
    h1(x, rows[y]);
  }
  for (int h = 0; h < 4; h++) {
    int col[4] = {rows[0][h], rows[1][h], rows[2][h], rows[3][h]}, o[4];
    h1(col, o);
    for (int v = 0; v < 4; v++) out[4 * v + h] = (int16_t)o[v];
  }
}
static void hadamard_edge(const uint8_t* x, int* o) {
  int s01 = x[0] + x[1], d01 = x[0] - x[1], s23 = x[2] + x[3], d23 = x[2] - x[3];
  o[0] = 4 * (s01 + s23); o[1] = 4 * (s01 - s23); o[2] = 4 * (d01 + d23); o[3] = 4 * (d01 - d23);
}
// h264_enc.rs:628 intra_satd_x3_16x16_scalar -> [v, h, dc]
static void intra_satd_x3_16(const uint8_t* src, const uint8_t* top, const uint8_t* left, int dc, uint32_t out[3]) {
  t_pixel_ops += 3 * 256;
  int tv[4][4], th[4][4];
  for (int b = 0; b < 4; b++) { hadamard_edge(top + b * 4, tv[b]); hadamard_edge(left + b * 4, th[b]); }
  uint32_t s[3] = {0, 0, 0};
  for (int by = 0; by < 4; by++)
    for (int bx = 0; bx < 4; bx++) {
      int16_t blk[16];
      hadamard_src4(src + by * 64 + bx * 4, 16, blk);
      for (int k = 0; k < 16; k++) {
        int v = k / 4, h = k % 4, c = blk[k];
        int pv = v == 0 ? tv[bx][h] : 0, ph = h == 0 ? th[by][v] : 0, pd = k == 0 ? 16 * dc : 0;
        s[0] += iabs(c - pv); s[1] += iabs(c - ph); s[2] += iabs(c - pd);
      }
    }
  for (int q = 0; q < 3; q++) out[q] = s[q] >> 1;
}

// ---------------------------------------------------------------------------------------------
// Quantisation (enc.rs:1703-1779, h264_enc.rs:408, h264_dct8.rs:84, h264.rs:1245-1420)
struct Quant4 { uint16_t mf[16]; uint32_t bias, shift; };
static inline int pos4(int i) {
  int r = i >> 2, c = i & 3;
  if (!(r & 1) && !(c & 1)) return 0;
  if ((r & 1) && (c & 1)) return 1;
  return 2;
}
static inline int pos8(int i) {
  int r = (i >> 3) & 3, c = (i & 7) & 3;
  if (r == 0 && c == 0) return 0;
  if ((r == 1 || r == 3) && (c == 1 || c == 3)) return 1;
  if (r == 2 && c == 2) return 2;
  if ((r == 0 && (c == 1 || c == 3)) || ((r == 1 || r == 3) && c == 0)) return 3;
  if ((r == 0 && c == 2) || (r == 2 && c == 0)) return 4;
  return 5;
}
static Quant4 quant4(int qp, bool intra) {
  Quant4 q;
  qp = std::min(qp, 51);
  q.shift = 15 + qp / 6;
  for (int i = 0; i < 16; i++) q.mf[i] = (uint16_t)kQuant4Mf[qp % 6][pos4(i)];
  q.bias = (1u << q.shift) / (intra ? 3 : 6);
  return q;
}
static void dequant4_scale(int qp, int32_t* s) {
  qp = std::min(qp, 51);
  for (int i = 0; i < 16; i++) s[i] = kDequant4Init[qp % 6][pos4(i)] << (qp / 6);
}
// quant_4x4_x4_scalar on one block: bit 0 any level, bit 1 a level above 1.
static int quant_block(int16_t* c, const Quant4& q) {
  int nz = 0;
  for (int i = 0; i < 16; i++) {
    uint64_t lv = ((uint64_t)iabs(c[i]) * q.mf[i] + q.bias) >> q.shift;
    if (lv > 32767) lv = 32767;
    c[i] = c[i] < 0 ? -(int16_t)lv : (int16_t)lv;
    if (lv) nz |= 1;
    if (lv > 1) nz |= 2;
  }
  return nz;
}
static void dequant_block(int16_t* c, const int32_t* s) {
  for (int i = 0; i < 16; i++) c[i] = clamp_i16((int64_t)c[i] * s[i]);
}
static inline void zigzag16(const int16_t* raster, int16_t* zz) {
  for (int i = 0; i < 16; i++) zz[i] = raster[kZigzag4[i]];
}
// enc.rs:1938 quant_chroma_dc
static void quant_chroma_dc(const int16_t* dc, int qpc, int16_t* out) {
  int d0 = dc[0], d1 = dc[1], d2 = dc[2], d3 = dc[3];
  int had[4] = {d0 + d1 + d2 + d3, d0 - d1 + d2 - d3, d0 + d1 - d2 - d3, d0 - d1 - d2 + d3};
  qpc = std::min(qpc, 51);
  int qbits = 16 + qpc / 6, mf = kQuant4Mf[qpc % 6][0], f = (1 << qbits) / 3;
  for (int i = 0; i < 4; i++) {
    int l = (iabs(had[i]) * mf + f) >> qbits;
    out[i] = (int16_t)(had[i] < 0 ? -l : l);
  }
}
// enc.rs:1960 quant_luma_dc
static void quant_luma_dc(const int16_t* dc, int qp, int16_t* out) {
  int16_t had[16];
  hadamard4_dc(dc, had);
  qp = std::min(qp, 51);
  int qbits = 16 + qp / 6, mf = kQuant4Mf[qp % 6][0], f = (1 << qbits) / 3;
  for (int i = 0; i < 16; i++) {
    int l = (iabs(had[i]) * mf + f) >> qbits;
    out[i] = (int16_t)(had[i] < 0 ? -l : l);
  }
}
// h264.rs:1645 dequantize_idct_luma_dc4x4
static void dequant_idct_luma_dc(const int16_t* lv, int qp, int16_t* out) {
  qp = std::min(qp, 51);
  int qmul = (kDequant4Init[qp % 6][0] * 16) << (qp / 6 + 2);
  int t[16];
  for (int i = 0; i < 4; i++) {
    int z0 = lv[4 * i] + lv[4 * i + 1], z1 = lv[4 * i] - lv[4 * i + 1];
    int z2 = lv[4 * i + 2] - lv[4 * i + 3], z3 = lv[4 * i + 2] + lv[4 * i + 3];
    t[4 * i] = z0 + z3; t[4 * i + 1] = z0 - z3; t[4 * i + 2] = z1 - z2; t[4 * i + 3] = z1 + z2;
  }
  for (int i = 0; i < 4; i++) {
    int z0 = t[i] + t[8 + i], z1 = t[i] - t[8 + i], z2 = t[4 + i] - t[12 + i], z3 = t[4 + i] + t[12 + i];
    out[i] = (int16_t)(((z0 + z3) * qmul + 128) >> 8);
    out[4 + i] = (int16_t)(((z1 + z2) * qmul + 128) >> 8);
    out[8 + i] = (int16_t)(((z1 - z2) * qmul + 128) >> 8);
    out[12 + i] = (int16_t)(((z0 - z3) * qmul + 128) >> 8);
  }
}
// h264.rs:1674 dequantize_idct_chroma_dc2x2
static void dequant_idct_chroma_dc(const int16_t* lv, int qpc, int16_t* out) {
  qpc = std::min(qpc, 51);
  int qmul = (kDequant4Init[qpc % 6][0] * 16) << (qpc / 6 + 2);
  int a = lv[0], b = lv[1], c = lv[2], d = lv[3];
  int e = a - b, apb = a + b, cmd = c - d, cpd = c + d;
  out[0] = (int16_t)(((apb + cpd) * qmul) >> 7);
  out[1] = (int16_t)(((e + cmd) * qmul) >> 7);
  out[2] = (int16_t)(((apb - cpd) * qmul) >> 7);
  out[3] = (int16_t)(((e - cmd) * qmul) >> 7);
}
// h264.rs:1403 dequantize_block8x8
static void dequant8(const int16_t* lv, int qp, int32_t* out) {
  qp = std::min(qp, 51);
  int qdiv = qp / 6, rem = qp % 6;
  for (int i = 0; i < 64; i++) {
    int v = kDequant8Init[rem][pos8(i)];
    int d;
    if (qdiv >= 2) d = lv[i] * (v << (qdiv - 2));
    else { int rs = 2 - qdiv; d = (lv[i] * v + (1 << (rs - 1))) >> rs; }
    out[i] = clamp_i16(d);
  }
}

// ---------------------------------------------------------------------------------------------
// Bit writer (enc.rs:2674 Bits; ragdoll-core BitWriter): MSB first.
struct BitWriter {
  std::vector<uint8_t> out;
  uint64_t acc = 0;
  int n = 0;
  void put(uint32_t val, int len) {  // len <= 32
    if (len == 0) return;
    acc = (acc << len) | (uint64_t)(len == 32 ? val : (val & ((1u << len) - 1)));
    n += len;
    while (n >= 8) { n -= 8; out.push_back((uint8_t)(acc >> n)); }
  }
  void bit(bool b) { put(b ? 1 : 0, 1); }
  void ue(uint64_t v) {
    uint64_t code = v + 1;
    int len = 64 - __builtin_clzll(code);
    put(0, len - 1 > 32 ? 32 : len - 1);
    if (len - 1 > 32) put(0, len - 1 - 32);
    if (len > 32) { put((uint32_t)(code >> 32), len - 32); put((uint32_t)code, 32); }
    else put((uint32_t)code, len);
  }
  void se(int64_t v) { ue(v > 0 ? (uint64_t)(2 * v - 1) : (uint64_t)(-2 * v)); }
  size_t bits() const { return out.size() * 8 + n; }
  void align_zero() { if (n & 7) put(0, 8 - (n & 7)); }
  void trailing() { bit(true); align_zero(); }
  std::vector<uint8_t> finish() { align_zero(); return out; }
};
// h264.rs:189 encode_annex_b_nal / ragdoll-core escape_rbsp
static void append_nal(std::vector<uint8_t>& dst, int ref_idc, int type, const std::vector<uint8_t>& rbsp) {
  dst.insert(dst.end(), {0, 0, 0, 1, (uint8_t)(((ref_idc & 3) << 5) | type)});
  int zeros = 0;
  for (uint8_t b : rbsp) {
    if (zeros == 2 && b <= 3) { dst.push_back(3); zeros = 0; }
    dst.push_back(b);
    zeros = b == 0 ? zeros + 1 : 0;
  }
}

// ---------------------------------------------------------------------------------------------
// CABAC (crates/ragdoll-codec/src/cabac.rs): the x264-style M-coder and the binarisations of the
// syntax elements the Balanced encoder writes.
struct CabacEnc {
  uint32_t low = 0, range = 510;
  int queue = -9;
  uint32_t outstanding = 0;
  std::vector<uint8_t> out;
  uint8_t ctx[460];  // 2 * pStateIdx + valMPS (cabac.rs:324)

  // cabac.rs:427 init_cabac_contexts, :354 CabacContext::from_mn_qp
  void init(int slice_qp, bool islice, int idc) {
    int t = islice ? 0 : 1 + std::min(idc, 2);
    for (int i = 0; i < 460; i++) {
      int m = kCabacInitMN[(t * 460 + i) * 2], n = kCabacInitMN[(t * 460 + i) * 2 + 1];
      int pre = std::max(1, std::min(126, ((m * std::min(slice_qp, 51)) >> 4) + n));
      ctx[i] = pre <= 63 ? (uint8_t)((63 - pre) << 1) : (uint8_t)(((pre - 64) << 1) | 1);
    }
  }
  // cabac.rs:524 putbyte
  void putbyte() {
    if (queue < 0) return;
    uint32_t o = low >> (queue + 10);
    low &= (0x400u << queue) - 1;
    queue -= 8;
    if ((o & 0xFF) == 0xFF) {
      outstanding++;
    } else {
      uint32_t carry = o >> 8;
      if (!out.empty()) out.back() = (uint8_t)(out.back() + carry);
      uint8_t fill = carry ? 0x00 : 0xFF;
      for (; outstanding; outstanding--) out.push_back(fill);
      out.push_back((uint8_t)(o & 0xFF));
    }
  }
  // cabac.rs:549 renormalize
  void renorm() {
    int shift = __builtin_clz(range) - 23;
    range <<= shift;
    low <<= shift;
    queue += shift;
    if (queue >= 0) putbyte();
  }
  // cabac.rs:562 encode_decision (9.3.3.2.1)
  void decision(int ci, int bin) {
    int st = ctx[ci] >> 1, mps = ctx[ci] & 1;
    uint32_t rl = kCabacRangeLps[st * 4 + ((range >> 6) & 3)];
    range -= rl;
    if (bin != mps) {
      low += range;
      range = rl;
      if (st == 0) mps ^= 1;
      st = kCabacTransLps[st];
    } else {
      st = std::min(st + 1, 62);
    }
    ctx[ci] = (uint8_t)((st << 1) | mps);
    renorm();
  }
  // cabac.rs:578 encode_bypass
  void bypass(int bin) {
    low <<= 1;
    if (bin) low += range;
    queue++;
    if (queue >= 0) putbyte();
  }
  // cabac.rs:591 encode_terminate
  void terminate(int bin) {
    range -= 2;
    if (bin) {
      low += range;
      low = (low << 9) | 0x200;
      queue += 9;
      putbyte();
      putbyte();
      low <<= -queue;
      queue = 0;
      putbyte();
      for (; outstanding; outstanding--) out.push_back(0xFF);
    } else {
      renorm();
    }
  }
  // cabac.rs:738 encode_intra_mb_type (ctx_base 3: I slice, 17: suffix in a P slice)
  void intra_mb_type(int ctx_base, int ca, int cb, int t) {
    bool islice = ctx_base == 3;
    int c0 = islice ? 3 + ca + cb : ctx_base;
    if (t == 0) { decision(c0, 0); return; }
    decision(c0, 1);
    terminate(0);  // never I_PCM here (QP >= 1)
    int code = t - 1, luma_mode = code % 4, cbpc = (code / 4) % 3, cbpl = code >= 12;
    if (islice) {
      decision(6, cbpl);
      decision(7, cbpc > 0);
      if (cbpc > 0) decision(8, cbpc == 2);
      decision(9, (luma_mode >> 1) & 1);
      decision(10, luma_mode & 1);
    } else {
      decision(ctx_base + 1, cbpl);
      decision(ctx_base + 2, cbpc > 0);
      if (cbpc > 0) decision(ctx_base + 2, cbpc == 2);
      decision(ctx_base + 3, (luma_mode >> 1) & 1);
      decision(ctx_base + 3, luma_mode & 1);
    }
  }
  // cabac.rs:787 encode_p_mb_type (0 = P_L0_16x16, >= 5 intra)
  void p_mb_type(int t) {
    if (t >= 5) { decision(14, 1); intra_mb_type(17, 0, 0, t - 5); return; }
    decision(14, 0);
    decision(15, 0);
    decision(16, 0);
  }
  // cabac.rs:819 encode_intra4x4_pred_mode
  void i4_mode(bool prev, int rem) {
    if (prev) { decision(68, 1); return; }
    decision(68, 0);
    decision(69, rem & 1);
    decision(69, (rem >> 1) & 1);
    decision(69, (rem >> 2) & 1);
  }
  // cabac.rs:836 encode_chroma_pred_mode
  void chroma_mode(int ca, int cb, int mode) {
    int c0 = 64 + ca + cb;
    if (mode == 0) { decision(c0, 0); return; }
    decision(c0, 1);
    if (mode == 1) { decision(67, 0); return; }
    decision(67, 1);
    decision(67, mode >= 3);
  }
  // cabac.rs:891 encode_mb_qp_delta
  void qp_delta(int prev_nz, int d) {
    int c0 = 60 + (prev_nz != 0);
    if (d == 0) { decision(c0, 0); return; }
    unsigned code = d > 0 ? 2 * d - 1 : -2 * d;
    decision(c0, 1);
    if (code == 1) { decision(62, 0); return; }
    decision(62, 1);
    for (unsigned k = 2; k < code; k++) decision(63, 1);
    decision(63, 0);
  }
  // cabac.rs:940 encode_mvd
  void mvd(int comp, uint32_t abs_sum, int v) {
    int base = comp == 0 ? 40 : 47;
    int inc0 = abs_sum < 3 ? 0 : (abs_sum <= 32 ? 1 : 2);
    uint32_t a = (uint32_t)std::abs(v);
    if (a == 0) { decision(base + inc0, 0); return; }
    decision(base + inc0, 1);
    uint32_t prefix = std::min(a, 9u);
    for (uint32_t i = 1; i < prefix; i++) decision(base + 3 + std::min((int)i - 1, 3), 1);
    if (a < 9) {
      decision(base + 3 + std::min((int)a - 1, 3), 0);
    } else {
      uint32_t rem = a - 9;
      int k = 3;
      while (rem >= (1u << k)) { bypass(1); rem -= 1u << k; k++; }
      bypass(0);
      for (int b = k - 1; b >= 0; b--) bypass((rem >> b) & 1);
    }
    bypass(v < 0);
  }
  // cabac.rs:981 encode_residual_block_cat, :1030 encode_sig_and_levels, :1059 sig_map, :1090 levels
  void residual(int cat, int cbf_inc, const int16_t* c, int n) {
    static const int kCbf[5] = {85, 89, 93, 97, 101};
    static const int kSig[6] = {105, 120, 134, 149, 152, 402};
    static const int kLast[6] = {166, 181, 195, 210, 213, 417};
    static const int kLvl[6] = {227, 237, 247, 257, 266, 426};
    int last = -1;
    for (int i = n - 1; i >= 0; i--) if (c[i]) { last = i; break; }
    if (cat < 5) {
      if (last < 0) { decision(kCbf[cat] + cbf_inc, 0); return; }
      decision(kCbf[cat] + cbf_inc, 1);
    } else if (last < 0) {
      last = 0;
    }
    int flagged = std::min(last, n - 2);
    for (int i = 0; i <= flagged; i++) {
      int so = cat == 5 ? kCabacSigOff8x8[i] : i, lo = cat == 5 ? kCabacLastOff8x8[i] : i;
      if (c[i] == 0) {
        decision(kSig[cat] + so, 0);
      } else {
        decision(kSig[cat] + so, 1);
        decision(kLast[cat] + lo, i == last);
      }
    }
    int gt_max = cat == 3 ? 3 : 4, eq1 = 0, gt1 = 0, lv = kLvl[cat];
    for (int i = last; i >= 0; i--) {
      if (c[i] == 0) continue;
      uint32_t m1 = (uint32_t)std::abs(c[i]) - 1;
      int c0 = gt1 > 0 ? 0 : std::min(1 + eq1, 4);
      if (m1 == 0) {
        decision(lv + c0, 0);
        eq1++;
      } else {
        decision(lv + c0, 1);
        int c1 = 5 + std::min(gt1, gt_max);
        uint32_t prefix = std::min(m1, 14u);
        for (uint32_t k = 1; k < prefix; k++) decision(lv + c1, 1);
        if (m1 < 14) {
          decision(lv + c1, 0);
        } else {
          uint32_t rem = m1 - 14;
          int k = 0;
          while (rem >= (1u << k)) { bypass(1); rem -= 1u << k; k++; }
          bypass(0);
          for (int b = k - 1; b >= 0; b--) bypass((rem >> b) & 1);
        }
        gt1++;
      }
      bypass(c[i] < 0);
    }
  }
};

// h264.rs:2215 encode_cavlc_block
static void cavlc_block(BitWriter& w, const int16_t* sc, int max_coeff, int nc, bool chroma_dc) {
  int tbl = nc <= 1 ? 0 : (nc <= 3 ? 1 : (nc <= 7 ? 2 : 3));
  int last = -1;
  for (int i = max_coeff - 1; i >= 0; i--) if (sc[i]) { last = i; break; }
  if (last < 0) {
    if (chroma_dc) w.put(kChromaDcTokenBits[0], kChromaDcTokenLen[0]);
    else w.put(kCoeffTokenBits[tbl][0], kCoeffTokenLen[tbl][0]);
    return;
  }
  int levels[16], runs[16], nlev = 0, nrun = 0, total_zeros = 0, cur_run = 0;
  for (int i = last; i >= 0; i--) {
    if (sc[i]) {
      if (nlev) { runs[nrun++] = cur_run; total_zeros += cur_run; }
      levels[nlev++] = sc[i];
      cur_run = 0;
    } else cur_run++;
  }
  runs[nrun++] = cur_run;
  total_zeros += cur_run;
  int total_coeff = nlev, t1 = 0;
  for (int q = 0; q < std::min(3, nlev); q++) { if (iabs(levels[q]) == 1) t1++; else break; }
  int tok = total_coeff * 4 + t1;
  if (chroma_dc) w.put(kChromaDcTokenBits[tok], kChromaDcTokenLen[tok]);
  else w.put(kCoeffTokenBits[tbl][tok], kCoeffTokenLen[tbl][tok]);
  for (int q = 0; q < t1; q++) w.bit(levels[q] < 0);
  uint32_t suffix = (total_coeff > 10 && t1 < 3) ? 1 : 0;
  for (int idx = t1; idx < nlev; idx++) {
    int lv = levels[idx];
    int code = lv > 0 ? (lv << 1) - 2 : (-lv << 1) - 1;
    if (idx == t1 && t1 < 3) code -= 2;
    uint32_t cu = (uint32_t)code;
    if (cu < (14u << suffix)) {
      w.put(0, cu >> suffix);
      w.bit(true);
      if (suffix > 0) w.put(cu & ((1u << suffix) - 1), suffix);
    } else if (suffix == 0 && cu < 30) {
      w.put(0, 14); w.bit(true); w.put(cu - 14, 4);
    } else if (suffix > 0 && cu < (15u << suffix)) {
      w.put(0, 14); w.bit(true); w.put(cu - (14u << suffix), suffix);
    } else {
      uint32_t esc = cu - (15u << suffix);
      if (suffix == 0) esc -= 15;
      w.put(0, 15); w.bit(true); w.put(esc & 0xFFF, 12);
    }
    if (suffix == 0) suffix = 1;
    if ((uint32_t)iabs(lv) > (3u << (suffix - 1)) && suffix < 6) suffix++;
  }
  if (total_coeff < max_coeff) {
    if (chroma_dc) w.put(kChromaDcTotalZerosBits[total_coeff - 1][total_zeros], kChromaDcTotalZerosLen[total_coeff - 1][total_zeros]);
    else w.put(kTotalZerosBits[total_coeff - 1][total_zeros], kTotalZerosLen[total_coeff - 1][total_zeros]);
  }
  int zl = total_zeros;
  for (int q = 0; q < total_coeff - 1 && zl > 0; q++) {
    int vi = std::min(zl - 1, 6);
    w.put(kRunBits[vi][runs[q]], kRunLen[vi][runs[q]]);
    zl -= runs[q];
  }
}

// ---------------------------------------------------------------------------------------------
// Encoder state (enc.rs:218-387) and frame coder.
struct MbSrc { uint8_t y[256], u[64], v[64]; };

struct Encoder {
  int width = 0, height = 0, mb_w = 0, mb_h = 0, profile = 0, qp = 26, keyint = 30;
  int fps_num = 30, fps_den = 1;
  bool cabac = false, t8x8 = false;
  uint32_t frame_count = 0;
  bool has_ref = false;
  Pic cur, refp;
  std::vector<int8_t> ref_grid;           // per 4x4
  std::vector<int16_t> mv_grid;           // per 4x4, 2 comps
  std::vector<int16_t> prev_mb_mv;        // per MB, 2 comps
  std::vector<uint8_t> intra4x4_modes;    // per 4x4
  std::vector<uint8_t> tc_nnz;            // per 4x4: total_coeff (CAVLC nC)
  std::vector<uint8_t> tc_cnnz[2];        // per chroma 4x4
  std::vector<uint16_t> nz16;             // per MB: 4x4 blocks holding levels (deblocking)
  std::vector<uint8_t> mb_intra, mb_cbp_luma, mb_t8, mb_qp, mb_skip;
  std::vector<rg_mb_out> recs;
  std::vector<uint8_t> recon_unfiltered[3];
  int cur_qp = 0;
  uint32_t skip_run = 0;
  bool is_idr = false;
  // skip bounds (enc.rs:2104)
  uint32_t sb_luma, sb_luma_ssd, sb_chroma, sb_chroma_ssd, sb_probe;

  void init(int w, int h, int prof, int q, int kint, int fn, int fd) {
    width = w; height = h; profile = prof; qp = std::max(0, std::min(q, 51)); keyint = kint;
    fps_num = fn; fps_den = fd;
    cabac = prof != 0;
    t8x8 = prof == 2;
    mb_w = (w + 15) / 16; mb_h = (h + 15) / 16;
    cur.alloc(mb_w * 16, mb_h * 16);
    refp.alloc(mb_w * 16, mb_h * 16);
    int n4 = mb_w * mb_h * 16, n = mb_w * mb_h;
    ref_grid.assign(n4, -2);
    mv_grid.assign(n4 * 2, 0);
    prev_mb_mv.assign(n * 2, 0);
    recs.assign(n, rg_mb_out());
  }

  // ---- SPS / PPS (h264.rs:556-660, 806-832) ----
  std::vector<uint8_t> sps_rbsp() const {
    BitWriter w;
    int pidc = profile == 0 ? 66 : (profile == 1 ? 77 : 100);
    int flags = profile == 0 ? 0xC0 : (profile == 1 ? 0x40 : 0x00);
    w.put(pidc, 8); w.put(flags, 8); w.put(40, 8); w.ue(0);
    if (pidc == 100) { w.ue(1); w.ue(0); w.ue(0); w.bit(false); w.bit(false); }
    w.ue(0);  // log2_max_frame_num - 4 (4)
    w.ue(0);  // pic_order_cnt_type
    w.ue(2);  // log2_max_pic_order_cnt_lsb - 4 (6)
    w.ue(2);  // max_num_ref_frames
    w.bit(false);
    w.ue(mb_w - 1); w.ue(mb_h - 1);
    w.bit(true);   // frame_mbs_only
    w.bit(true);   // direct_8x8_inference
    int crop_r = (mb_w * 16 - width) / 2, crop_b = (mb_h * 16 - height) / 2;
    bool crop = crop_r || crop_b;
    w.bit(crop);
    if (crop) { w.ue(0); w.ue(crop_r); w.ue(0); w.ue(crop_b); }
    w.bit(true);             // vui
    w.bit(true); w.put(1, 8);  // aspect ratio 1:1
    w.bit(false);            // overscan
    w.bit(true); w.put(5, 3); w.bit(false);  // video signal: unspecified format, limited range
    w.bit(true); w.put(1, 8); w.put(1, 8); w.put(1, 8);  // BT.709
    w.bit(false);            // chroma loc
    w.bit(true); w.put((uint32_t)fps_den, 32); w.put((uint32_t)(fps_num * 2), 32); w.bit(true);
    w.bit(false); w.bit(false); w.bit(false); w.bit(false);
    w.trailing();
    return w.finish();
  }
  std::vector<uint8_t> pps_rbsp() const {
    BitWriter w;
    w.ue(0); w.ue(0); w.bit(cabac); w.bit(false); w.ue(0); w.ue(0); w.ue(0);
    w.bit(false); w.put(0, 2);
    w.se(qp - 26); w.se(0); w.se(0);
    w.bit(true); w.bit(false); w.bit(false);
    if (t8x8) { w.bit(true); w.bit(false); w.se(0); }
    w.trailing();
    return w.finish();
  }

  // ---- source load (enc.rs:400, h264.rs:3660) ----
  void load_src(const uint8_t* Y, const uint8_t* U, const uint8_t* V, int sy, int suv, int mbx, int mby, MbSrc& s) const {
    int cw = (width + 1) / 2, ch = (height + 1) / 2;
    for (int r = 0; r < 16; r++)
      for (int c = 0; c < 16; c++) {
        int yy = std::min(mby * 16 + r, height - 1), xx = std::min(mbx * 16 + c, width - 1);
        s.y[r * 16 + c] = Y[(size_t)yy * sy + xx];
      }
    for (int r = 0; r < 8; r++)
      for (int c = 0; c < 8; c++) {
        int yy = std::min(mby * 8 + r, ch - 1), xx = std::min(mbx * 8 + c, cw - 1);
        s.u[r * 8 + c] = U[(size_t)yy * suv + xx];
        s.v[r * 8 + c] = V[(size_t)yy * suv + xx];
      }
  }

  // ---- helpers on grids ----
  int gstride() const { return mb_w * 4; }
  void fill_motion(int mbx, int mby, int ref, int mx, int my) {
    int g = gstride();
    for (int y = 0; y < 4; y++)
      for (int x = 0; x < 4; x++) {
        int i = (mby * 4 + y) * g + mbx * 4 + x;
        ref_grid[i] = (int8_t)ref;
        mv_grid[2 * i] = (int16_t)mx;
        mv_grid[2 * i + 1] = (int16_t)my;
      }
  }
  // h264.rs:3577 pred_motion_partition (16x16 partition, ref 0)
  void mvp16(int gx, int gy, int16_t out[2]) const {
    int g = gstride();
    int lref = -2, tref = -2, dref = -2;
    int a[2] = {0, 0}, b[2] = {0, 0}, c[2] = {0, 0};
    if (gx > 0) { int i = gy * g + gx - 1; lref = ref_grid[i]; a[0] = mv_grid[2 * i]; a[1] = mv_grid[2 * i + 1]; }
    if (gy > 0) { int i = (gy - 1) * g + gx; tref = ref_grid[i]; b[0] = mv_grid[2 * i]; b[1] = mv_grid[2 * i + 1]; }
    int tr = gx + 4;
    bool tr_avail = gy > 0 && tr < g;  // 16x16 at a macroblock corner: only the picture bounds matter
    if (tr_avail && ref_grid[(gy - 1) * g + tr] != -2) {
      int i = (gy - 1) * g + tr; dref = ref_grid[i]; c[0] = mv_grid[2 * i]; c[1] = mv_grid[2 * i + 1];
    } else if (gy > 0 && gx > 0) {
      int i = (gy - 1) * g + gx - 1; dref = ref_grid[i]; c[0] = mv_grid[2 * i]; c[1] = mv_grid[2 * i + 1];
    }
    auto med = [](int x, int y, int z) { return std::min(std::max(x, y), std::max(std::min(x, y), z)); };
    int m = (lref == 0) + (tref == 0) + (dref == 0);
    if (m > 1) { out[0] = (int16_t)med(a[0], b[0], c[0]); out[1] = (int16_t)med(a[1], b[1], c[1]); }
    else if (m == 1) {
      const int* s = lref == 0 ? a : (tref == 0 ? b : c);
      out[0] = (int16_t)s[0]; out[1] = (int16_t)s[1];
    } else if (tref == -2 && dref == -2 && lref != -2) { out[0] = (int16_t)a[0]; out[1] = (int16_t)a[1]; }
    else { out[0] = (int16_t)med(a[0], b[0], c[0]); out[1] = (int16_t)med(a[1], b[1], c[1]); }
  }
  // h264.rs:3283 pred_intra4x4_mode
  int pred_i4_mode(int gx, int gy) const {
    if (gx == 0 || gy == 0) return 2;
    int g = gstride();
    return std::min(intra4x4_modes[gy * g + gx - 1], intra4x4_modes[(gy - 1) * g + gx]);
  }

  // ---- edges (enc.rs:1459-1521) from the unfiltered reconstruction ----
  void i16_edges(int mbx, int mby, uint8_t* top, uint8_t* left, bool& ht, bool& hl, int& tl) const {
    const Plane& p = cur.y;
    ht = mby > 0; hl = mbx > 0;
    if (ht) memcpy(top, p.ptr(mbx * 16, mby * 16 - 1), 16);
    if (hl) for (int r = 0; r < 16; r++) left[r] = *p.ptr(mbx * 16 - 1, mby * 16 + r);
    tl = (ht && hl) ? *p.ptr(mbx * 16 - 1, mby * 16 - 1) : 128;
  }
  void chroma_edges(const Plane& p, int mbx, int mby, uint8_t* top, uint8_t* left, bool& ht, bool& hl, int& tl) const {
    ht = mby > 0; hl = mbx > 0;
    if (ht) memcpy(top, p.ptr(mbx * 8, mby * 8 - 1), 8);
    if (hl) for (int r = 0; r < 8; r++) left[r] = *p.ptr(mbx * 8 - 1, mby * 8 + r);
    tl = (ht && hl) ? *p.ptr(mbx * 8 - 1, mby * 8 - 1) : 128;
  }

  // enc.rs:1637 analyse_i16_edges -> (satd, mode)
  void analyse_i16(int mbx, int mby, const MbSrc& src, uint32_t& best_cost, int& best_mode) const {
    uint8_t top[16] = {0}, left[16] = {0};
    bool ht, hl; int tl;
    i16_edges(mbx, mby, top, left, ht, hl, tl);
    int dc;
    {
      uint32_t st = 0, sl = 0;
      for (int q = 0; q < 16; q++) { st += top[q]; sl += left[q]; }
      if (ht && hl) dc = (st + sl + 16) >> 5;
      else if (ht) dc = (st + 8) >> 4;
      else if (hl) dc = (sl + 8) >> 4;
      else dc = 128;
    }
    uint8_t zt[16] = {0}, zl[16] = {0};
    uint32_t s3[3];
    intra_satd_x3_16(src.y, ht ? top : zt, hl ? left : zl, dc, s3);
    best_cost = s3[2]; best_mode = 2;
    if (ht && s3[0] < best_cost) { best_cost = s3[0]; best_mode = 0; }
    if (hl && s3[1] < best_cost) { best_cost = s3[1]; best_mode = 1; }
    if (ht && hl) {
      uint8_t pred[256];
      pred16(3, top, left, tl, pred);
      uint32_t c = satd16(src.y, 16, pred, 16);
      if (c < best_cost) { best_cost = c; best_mode = 3; }
    }
  }
  // enc.rs:1526 analyse_chroma_intra
  int analyse_chroma(int mbx, int mby, const MbSrc& src, uint8_t* pu, uint8_t* pv) const {
    uint8_t tu[8], lu[8], tv[8], lv[8];
    bool htu, hlu, htv, hlv; int tlu, tlv;
    chroma_edges(cur.u, mbx, mby, tu, lu, htu, hlu, tlu);
    chroma_edges(cur.v, mbx, mby, tv, lv, htv, hlv, tlv);
    uint32_t best = UINT32_MAX; int bm = 0;
    for (int mode = 0; mode < 4; mode++) {
      bool ok = mode == 1 ? hlu : (mode == 2 ? htu : (mode == 3 ? (htu && hlu) : true));
      if (!ok) continue;
      uint8_t a[64], b[64];
      pred_chroma(mode, htu ? tu : nullptr, hlu ? lu : nullptr, tlu, a);
      pred_chroma(mode, htv ? tv : nullptr, hlv ? lv : nullptr, tlv, b);
      uint32_t c = sad(src.u, 8, a, 8, 8, 8) + sad(src.v, 8, b, 8, 8, 8) + (mode == 0 ? 0 : 8);
      if (c < best) { best = c; bm = mode; memcpy(pu, a, 64); memcpy(pv, b, 64); }
    }
    return bm;
  }

  // ---- chroma residual (enc.rs:1854-1934) ----
  struct Chroma {
    int16_t dc[2][4];
    int16_t ac[2][4][16];    // zig-zag, slot 0 unused
    uint32_t mask[2][4];     // non-zero AC levels (bit i-1 for zig-zag slot i)
    int16_t raster[2][4][16];
  };
  void quant_chroma(const MbSrc& src, const uint8_t* pu, const uint8_t* pv, int qpc, bool intra, Chroma& c) const {
    Quant4 q = quant4(qpc, intra);
    for (int p = 0; p < 2; p++) {
      const uint8_t* s = p ? src.v : src.u;
      const uint8_t* pr = p ? pv : pu;
      int16_t blk[4][16], dcraw[4];
      for (int b = 0; b < 4; b++) {
        int16_t d[16];
        int o = (b >> 1) * 32 + (b & 1) * 4;
        for (int y = 0; y < 4; y++) for (int x = 0; x < 4; x++) d[y * 4 + x] = (int16_t)(s[o + y * 8 + x] - pr[o + y * 8 + x]);
        fdct4(d, blk[b]);
        dcraw[b] = blk[b][0];
      }
      int nz = 0;
      for (int b = 0; b < 4; b++) nz |= quant_block(blk[b], q);
      if (nz) {
        for (int b = 0; b < 4; b++) {
          int16_t zz[16];
          zigzag16(blk[b], zz);
          uint32_t m = 0;
          for (int i = 1; i < 16; i++) if (zz[i]) m |= 1u << (i - 1);
          c.mask[p][b] = m;
          memcpy(c.ac[p][b], zz, sizeof zz);
          c.ac[p][b][0] = 0;
          memcpy(c.raster[p][b], blk[b], sizeof blk[b]);
        }
      } else {
        memset(c.mask[p], 0, sizeof c.mask[p]);
        memset(c.ac[p], 0, sizeof c.ac[p]);
        memset(c.raster[p], 0, sizeof c.raster[p]);
      }
      quant_chroma_dc(dcraw, qpc, c.dc[p]);
    }
  }
  uint32_t chroma_ac_score(const Chroma& c, int p) const {
    uint32_t s = 0;
    for (int b = 0; b < 4; b++) s += decimate_score(c.ac[p][b] + 1, 15);
    return s;
  }
  static int chroma_cbp(const Chroma& c) {
    uint32_t m = 0;
    for (int p = 0; p < 2; p++) for (int b = 0; b < 4; b++) m |= c.mask[p][b];
    if (m) return 2;
    for (int p = 0; p < 2; p++) for (int b = 0; b < 4; b++) if (c.dc[p][b]) return 1;
    return 0;
  }
  // enc.rs:1992 recon_chroma
  void recon_chroma(uint8_t* pu, uint8_t* pv, const Chroma& c, int cbpc, int qpc) const {
    if (cbpc == 0) return;
    int32_t sc[16];
    dequant4_scale(qpc, sc);
    for (int p = 0; p < 2; p++) {
      uint8_t* pred = p ? pv : pu;
      int16_t dcr[4];
      dequant_idct_chroma_dc(c.dc[p], qpc, dcr);
      for (int b = 0; b < 4; b++) {
        int16_t blk[16] = {0};
        if (cbpc >= 2) { memcpy(blk, c.raster[p][b], sizeof blk); dequant_block(blk, sc); }
        blk[0] = dcr[b];
        add_idct4(pred + (b >> 1) * 32 + (b & 1) * 4, 8, blk);
      }
    }
  }

  // luma residual of a 16x16 prediction: 16 blocks, decoding order (enc.rs:1794 dct_luma)
  static void dct_luma(const uint8_t* src, const uint8_t* pred, int16_t out[16][16]) {
    for (int b = 0; b < 16; b++) {
      int bx, by; blk_xy(b, bx, by);
      int o = by * 64 + bx * 4;
      int16_t d[16];
      for (int y = 0; y < 4; y++) for (int x = 0; x < 4; x++) d[y * 4 + x] = (int16_t)(src[o + y * 16 + x] - pred[o + y * 16 + x]);
      fdct4(d, out[b]);
    }
  }
  // enc.rs:1810 quant_luma_4x4_inter -> cbp, q4 quantised & decimated (raster per block)
  int quant_luma_inter(const uint8_t* src, const uint8_t* pred, int q_, int16_t q4[16][16]) const {
    dct_luma(src, pred, q4);
    Quant4 q = quant4(q_, false);
    int cbp = 0; uint32_t total = 0;
    for (int g = 0; g < 4; g++) {
      int nz = 0;
      for (int k = 0; k < 4; k++) nz |= quant_block(q4[g * 4 + k], q);
      if (!(nz & 1)) continue;
      if (nz & 2) { cbp |= 1 << g; total += 9; continue; }
      uint32_t score = 0;
      for (int k = 0; k < 4; k++) { int16_t zz[16]; zigzag16(q4[g * 4 + k], zz); score += decimate_score(zz, 16); }
      if (score < 4) { for (int k = 0; k < 4; k++) memset(q4[g * 4 + k], 0, 32); }
      else cbp |= 1 << g;
      total += score;
    }
    if (total < 6 && cbp) { memset(q4, 0, 16 * 16 * 2); cbp = 0; }
    return cbp;
  }
  // enc.rs:2041 quant_luma_8x8_inter -> cbp8, q8 (raster per 8x8 block)
  static int quant_luma_8x8(const uint8_t* src, const uint8_t* pred, int q_, int16_t q8[4][64], bool fine = false) {
    int qq = std::min(q_, 51);
    uint32_t shift = 16 + qq / 6, bias = (1u << shift) / (fine ? 3 : 6);
    int cbp = 0; uint32_t total = 0;
    for (int b = 0; b < 4; b++) {
      int o = (b >> 1) * 128 + (b & 1) * 8;
      int16_t d[64];
      for (int y = 0; y < 8; y++) for (int x = 0; x < 8; x++) d[y * 8 + x] = (int16_t)(src[o + y * 16 + x] - pred[o + y * 16 + x]);
      fdct8(d, q8[b]);
      int nz = 0;
      for (int i = 0; i < 64; i++) {
        int16_t c = q8[b][i];
        uint64_t lv = ((uint64_t)iabs(c) * (uint32_t)kQuant8Mf[qq % 6][pos8(i)] + bias) >> shift;
        if (lv > 32767) lv = 32767;
        q8[b][i] = c < 0 ? -(int16_t)lv : (int16_t)lv;
        if (lv) nz |= 1;
        if (lv > 1) nz |= 2;
      }
      uint32_t score;
      if (nz == 0) score = 0;
      else if (nz == 1) { int16_t zz[64]; for (int i = 0; i < 64; i++) zz[i] = q8[b][kZigzag8[i]]; score = decimate_score(zz, 64); }
      else score = 9;
      total += score;
      if (score >= 4) cbp |= 1 << b;
      else memset(q8[b], 0, 128);
    }
    if (total < 6 && cbp) { memset(q8, 0, 4 * 64 * 2); cbp = 0; }
    return cbp;
  }

  // ---- motion search (enc.rs:1099-1449) ----
  struct Bounds { int min[2], max[2]; };
  Bounds mv_bounds(int x0, int y0) const {
    int w = refp.y.w, h = refp.y.h;
    Bounds b;
    b.min[0] = -4 * (x0 + MV_MARGIN);
    b.min[1] = std::max(-4 * (y0 + MV_MARGIN), -2048);
    b.max[0] = 4 * (w - 16 - x0 + MV_MARGIN);
    b.max[1] = std::min(4 * (h - 16 - y0 + MV_MARGIN), 2044);
    return b;
  }
  static bool in_bounds(const Bounds& b, int mx, int my) {
    return mx >= b.min[0] && mx <= b.max[0] && my >= b.min[1] && my <= b.max[1];
  }
  uint32_t mvd_cost(int d, int lambda) const {
    if (d >= -MV_COST_RANGE && d <= MV_COST_RANGE) return (uint16_t)(lambda * se_bits(d));
    return lambda * se_bits(d);
  }
  // qpel prediction of the 16x16 block at (x0,y0) displaced by mv (enc.rs:1058 mc_luma)
  void mc_luma16(int x0, int y0, int mx, int my, uint8_t* dst) const {
    const uint8_t* s = refp.y.ptr(x0 + (mx >> 2), y0 + (my >> 2));
    luma_mc(s, refp.y.stride, 16, 16, mx & 3, my & 3, dst, 16);
  }
  void mc_chroma8(int mbx, int mby, int mx, int my, uint8_t* pu, uint8_t* pv) const {
    int cx = mbx * 8 + (mx >> 3), cy = mby * 8 + (my >> 3);
    int fx = mx & 7, fy = my & 7;
    chroma_mc(refp.u.ptr(cx, cy), refp.u.stride, fx, fy, pu);
    chroma_mc(refp.v.ptr(cx, cy), refp.v.stride, fx, fy, pv);
  }

  // ---- deblocking (enc.rs:3776-3942, h264_deblock.rs:71,187) ----
  static void luma_edge(uint8_t* buf, int xs, int ys, int alpha, int beta, const int* tc0v, bool strong) {
    for (int k = 0; k < 16; k++) {
      int tc0 = tc0v[k / 4];
      if (!strong && tc0 < 0) continue;
      uint8_t* o = buf + k * ys;
      int p0 = o[-xs], q0 = o[0], p1 = o[-2 * xs], q1 = o[xs];
      if (iabs(p0 - q0) >= alpha || iabs(p1 - p0) >= beta || iabs(q1 - q0) >= beta) continue;
      int p2 = o[-3 * xs], q2 = o[2 * xs];
      bool ap = iabs(p2 - p0) < beta, aq = iabs(q2 - q0) < beta;
      if (!strong) {
        int tc = tc0 + ap + aq;
        int d = std::max(-tc, std::min(tc, (((q0 - p0) << 2) + (p1 - q1) + 4) >> 3));
        o[-xs] = (uint8_t)clamp255(p0 + d);
        o[0] = (uint8_t)clamp255(q0 - d);
        if (ap) o[-2 * xs] = (uint8_t)(p1 + std::max(-tc0, std::min(tc0, (p2 + ((p0 + q0 + 1) >> 1) - (p1 << 1)) >> 1)));
        if (aq) o[xs] = (uint8_t)(q1 + std::max(-tc0, std::min(tc0, (q2 + ((p0 + q0 + 1) >> 1) - (q1 << 1)) >> 1)));
      } else {
        int p3 = o[-4 * xs], q3 = o[3 * xs];
        bool small = iabs(p0 - q0) < ((alpha >> 2) + 2);
        if (ap && small) {
          o[-xs] = (uint8_t)((p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3);
          o[-2 * xs] = (uint8_t)((p2 + p1 + p0 + q0 + 2) >> 2);
          o[-3 * xs] = (uint8_t)((2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3);
        } else o[-xs] = (uint8_t)((2 * p1 + p0 + q1 + 2) >> 2);
        if (aq && small) {
          o[0] = (uint8_t)((p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2 + 4) >> 3);
          o[xs] = (uint8_t)((p0 + q0 + q1 + q2 + 2) >> 2);
          o[2 * xs] = (uint8_t)((2 * q3 + 3 * q2 + q1 + q0 + p0 + 4) >> 3);
        } else o[0] = (uint8_t)((2 * q1 + q0 + p1 + 2) >> 2);
      }
    }
  }
  static void chroma_edge(uint8_t* buf, int xs, int ys, int alpha, int beta, const int* tc0v, bool strong) {
    for (int k = 0; k < 8; k++) {
      int tc0 = tc0v[k / 2];
      if (!strong && tc0 < 0) continue;
      uint8_t* o = buf + k * ys;
      int p1 = o[-2 * xs], p0 = o[-xs], q0 = o[0], q1 = o[xs];
      if (iabs(p0 - q0) >= alpha || iabs(p1 - p0) >= beta || iabs(q1 - q0) >= beta) continue;
      if (strong) {
        o[-xs] = (uint8_t)((2 * p1 + p0 + q1 + 2) >> 2);
        o[0] = (uint8_t)((2 * q1 + q0 + p1 + 2) >> 2);
      } else {
        int tc = tc0 + 1;
        int d = std::max(-tc, std::min(tc, (((q0 - p0) << 2) + (p1 - q1) + 4) >> 3));
        o[-xs] = (uint8_t)clamp255(p0 + d);
        o[0] = (uint8_t)clamp255(q0 - d);
      }
    }
  }
  static bool edge_filter(int qpv, const int* bs, int& alpha, int& beta, int* tc0, bool& strong) {
    int ia = std::max(0, std::min(51, qpv));
    alpha = kAlpha[ia]; beta = kBeta[ia];
    if (!alpha || !beta) return false;
    for (int k = 0; k < 4; k++) {
      int b = std::min(bs[k], 4);
      tc0[k] = b == 0 ? -1 : (b == 4 ? 0 : kTc0[ia][b - 1]);
    }
    strong = bs[0] == 4;
    return true;
  }
  void deblock() {
    int g = gstride();
    auto quiet = [&](int m) { return !mb_intra[m] && mb_cbp_luma[m] == 0; };
    auto mv_of = [&](int mbx, int mby, int c) { return mv_grid[2 * ((mby * 4) * g + mbx * 4) + c]; };
    for (int mby = 0; mby < mb_h; mby++)
      for (int mbx = 0; mbx < mb_w; mbx++) {
        int m = mby * mb_w + mbx;
        auto same_mv = [&](int ox, int oy) { return mv_of(ox, oy, 0) == mv_of(mbx, mby, 0) && mv_of(ox, oy, 1) == mv_of(mbx, mby, 1); };
        bool split = form && mb_split[m];
        bool nsplit = form && ((mbx > 0 && mb_split[m - 1]) || (mby > 0 && mb_split[m - mb_w]));
        if (!split && !nsplit && quiet(m) && (mbx == 0 || (quiet(m - 1) && same_mv(mbx - 1, mby))) &&
            (mby == 0 || (quiet(m - mb_w) && same_mv(mbx, mby - 1))))
          continue;
        bool intra = mb_intra[m];
        bool internal = intra || mb_cbp_luma[m] != 0 || split;
        bool skip_odd = mb_t8[m];
        int qpq = mb_qp[m], qpcq = chroma_qp(qpq, 0);
        for (int dir = 0; dir < 2; dir++)
          for (int e = 0; e < 4; e++) {
            int pm;
            if (e == 0) {
              if (dir == 0 && mbx > 0) pm = m - 1;
              else if (dir == 1 && mby > 0) pm = m - mb_w;
              else continue;
            } else {
              if (!internal || ((e & 1) && skip_odd)) continue;
              pm = m;
            }
            int bs[4];
            if (intra || mb_intra[pm]) {
              for (int k = 0; k < 4; k++) bs[k] = e == 0 ? 4 : 3;
            } else {
              // segment k: 4x4 blocks on either side hold levels
              auto nzq = [&](int bx, int by) { int b = ((by >> 1) << 3) | ((bx >> 1) << 2) | ((by & 1) << 1) | (bx & 1); return (nz16[m] >> b) & 1; };
              auto nzp = [&](int mm, int bx, int by) { int b = ((by >> 1) << 3) | ((bx >> 1) << 2) | ((by & 1) << 1) | (bx & 1); return (nz16[mm] >> b) & 1; };
              int coded[4];
              for (int k = 0; k < 4; k++) {
                if (dir == 0) coded[k] = nzq(e, k) | (e == 0 ? nzp(pm, 3, k) : nzq(e - 1, k));
                else coded[k] = nzq(k, e) | (e == 0 ? nzp(pm, k, 3) : nzq(k, e - 1));
              }
              bool mot[4] = {false, false, false, false};
              for (int k = 0; k < 4; k++) {
                // 4x4 blocks q (this side) and p (across the edge) of segment k; the plain form's
                // vectors are one per macroblock, so only its edge 0 can differ
                if (!form && (e != 0 || k != 0)) { mot[k] = mot[0]; continue; }
                int qx = dir == 0 ? e : k, qy = dir == 0 ? k : e;
                int gq = (mby * 4 + qy) * g + mbx * 4 + qx;
                int gp = dir == 0 ? gq - 1 : gq - g;
                mot[k] = ref_grid[gq] != ref_grid[gp] || iabs(mv_grid[2 * gq] - mv_grid[2 * gp]) >= 4 ||
                         iabs(mv_grid[2 * gq + 1] - mv_grid[2 * gp + 1]) >= 4;
              }
              if (!coded[0] && !coded[1] && !coded[2] && !coded[3] && !mot[0] && !mot[1] && !mot[2] && !mot[3]) continue;
              for (int k = 0; k < 4; k++) bs[k] = coded[k] ? 2 : (mot[k] ? 1 : 0);
            }
            int qpv, qpc;
            if (pm == m) { qpv = qpq; qpc = qpcq; }
            else {
              int qpp = mb_qp[pm];
              qpv = (qpq + qpp + 1) >> 1;
              qpc = (qpcq + chroma_qp(qpp, 0) + 1) >> 1;
            }
            int x = dir == 0 ? mbx * 16 + e * 4 : mbx * 16, y = dir == 0 ? mby * 16 : mby * 16 + e * 4;
            int alpha, beta, tc0[4]; bool strong;
            if (edge_filter(qpv, bs, alpha, beta, tc0, strong)) {
              Plane& p = cur.y;
              int xs = dir == 0 ? 1 : p.stride, ys = dir == 0 ? p.stride : 1;
              luma_edge(p.ptr(x, y), xs, ys, alpha, beta, tc0, strong);
            }
            if (!(e & 1) && edge_filter(qpc, bs, alpha, beta, tc0, strong)) {
              for (int pl = 0; pl < 2; pl++) {
                Plane& p = pl ? cur.v : cur.u;
                int xs = dir == 0 ? 1 : p.stride, ys = dir == 0 ? p.stride : 1;
                chroma_edge(p.ptr(x / 2, y / 2), xs, ys, alpha, beta, tc0, strong);
              }
            }
          }
      }
  }

  // ---- CAVLC macroblock writers (enc.rs:989-1054, 3260-3285, 3540-3577, 3736-3750) ----
  int nc_luma(int gx, int gy) const {
    int g = gstride();
    bool ha = gx > 0, hb = gy > 0;
    int a = ha ? tc_nnz[gy * g + gx - 1] : 0, b = hb ? tc_nnz[(gy - 1) * g + gx] : 0;
    if (ha && hb) return (a + b + 1) >> 1;
    if (ha) return a;
    if (hb) return b;
    return 0;
  }
  int nc_chroma(int p, int cgx, int cgy) const {
    int cg = mb_w * 2;
    bool ha = cgx > 0, hb = cgy > 0;
    int a = ha ? tc_cnnz[p][cgy * cg + cgx - 1] : 0, b = hb ? tc_cnnz[p][(cgy - 1) * cg + cgx] : 0;
    if (ha && hb) return (a + b + 1) >> 1;
    if (ha) return a;
    if (hb) return b;
    return 0;
  }
  void write_chroma_cavlc(BitWriter& w, int mbx, int mby, const rg_mb_out& r) {
    int cbpc = r.cbp >> 4;
    if (cbpc >= 1)
      for (int p = 0; p < 2; p++) cavlc_block(w, r.chroma_dc[p], 4, 0, true);
    if (cbpc >= 2) {
      int cg = mb_w * 2;
      for (int p = 0; p < 2; p++)
        for (int b = 0; b < 4; b++) {
          int cgx = mbx * 2 + (b & 1), cgy = mby * 2 + (b >> 1);
          int nc = nc_chroma(p, cgx, cgy);
          cavlc_block(w, r.chroma_ac[p][b] + 1, 15, nc, false);
          int cnt = 0;
          for (int i = 1; i < 16; i++) cnt += r.chroma_ac[p][b][i] != 0;
          tc_cnnz[p][cgy * cg + cgx] = (uint8_t)cnt;
        }
    }
  }
  void write_luma4x4_cavlc(BitWriter& w, int mbx, int mby, const rg_mb_out& r) {
    int g = gstride();
    for (int b = 0; b < 16; b++) {
      int bx, by; blk_xy(b, bx, by);
      int gx = mbx * 4 + bx, gy = mby * 4 + by;
      if (!(r.cbp & (1 << (b >> 2)))) { tc_nnz[gy * g + gx] = 0; continue; }
      int nc = nc_luma(gx, gy);
      cavlc_block(w, r.luma + b * 16, 16, nc, false);
      int cnt = 0;
      for (int i = 0; i < 16; i++) cnt += r.luma[b * 16 + i] != 0;
      tc_nnz[gy * g + gx] = (uint8_t)cnt;
    }
  }
  void write_mb_cavlc(BitWriter& w, int mbx, int mby, const rg_mb_out& r) {
    int g = gstride();
    if (r.mb_type == RG_MB_P_SKIP) { skip_run++; return; }
    if (!is_idr) { w.ue(skip_run); skip_run = 0; }
    if (r.mb_type == RG_MB_P_L0_16X16) {
      w.ue(0); w.se(r.mvd[0]); w.se(r.mvd[1]);
      int code = 0;
      for (int i = 0; i < 48; i++) if (kGolombToInterCbp[i] == r.cbp) { code = i; break; }
      w.ue(code);
      if (r.cbp) {
        if (t8x8) w.bit(false);
        w.se(r.qp_delta);
        write_luma4x4_cavlc(w, mbx, mby, r);
        write_chroma_cavlc(w, mbx, mby, r);
      }
    } else if (r.mb_type == RG_MB_I16X16) {
      int cbpl = r.cbp & 15, cbpc = r.cbp >> 4;
      int mbt = 1 + r.i16_mode + 4 * cbpc + (cbpl ? 12 : 0);
      w.ue((is_idr ? 0 : 5) + mbt);
      w.ue(r.chroma_mode);
      w.se(r.qp_delta);
      cavlc_block(w, r.luma_dc, 16, nc_luma(mbx * 4, mby * 4), false);
      if (cbpl) {
        for (int b = 0; b < 16; b++) {
          int bx, by; blk_xy(b, bx, by);
          int gx = mbx * 4 + bx, gy = mby * 4 + by;
          int nc = nc_luma(gx, gy);
          cavlc_block(w, r.luma + b * 16 + 1, 15, nc, false);
          int cnt = 0;
          for (int i = 1; i < 16; i++) cnt += r.luma[b * 16 + i] != 0;
          tc_nnz[gy * g + gx] = (uint8_t)cnt;
        }
      }
      write_chroma_cavlc(w, mbx, mby, r);
    } else {  // I4x4
      w.ue(is_idr ? 0 : 5);
      if (t8x8) w.bit(false);
      // predicted modes see neighbours' modes and this MB's earlier blocks
      for (int b = 0; b < 16; b++) {
        int bx, by; blk_xy(b, bx, by);
        intra4x4_modes[(mby * 4 + by) * g + mbx * 4 + bx] = 2;
      }
      for (int b = 0; b < 16; b++) {
        int bx, by; blk_xy(b, bx, by);
        int gx = mbx * 4 + bx, gy = mby * 4 + by;
        int pm = pred_i4_mode(gx, gy), m = r.i4_modes[b];
        if (m == pm) w.bit(true);
        else { w.bit(false); w.put(m < pm ? m : m - 1, 3); }
        intra4x4_modes[gy * g + gx] = (uint8_t)m;
      }
      w.ue(r.chroma_mode);
      int code = 3;
      for (int i = 0; i < 48; i++) if (kGolombToIntra4x4Cbp[i] == r.cbp) { code = i; break; }
      w.ue(code);
      if (r.cbp) {
        w.se(r.qp_delta);
        write_luma4x4_cavlc(w, mbx, mby, r);
        write_chroma_cavlc(w, mbx, mby, r);
      }
    }
  }

  // ---- CABAC macroblock layer (enc.rs:2779 begin_coded_mb, :2877 code_skip, :3196 code_inter,
  // :3442 code_i4, :3587 code_i16; h264.rs:3293-3553 the coded_block_pattern / residual glue).
  // Neighbour state as EncState keeps it for the CABAC writer (enc.rs:218-276).
  CabacEnc ce;
  std::vector<uint8_t> cb_nnz, cb_cnnz[2], cb_intra, cb_i16, cb_skip, cb_cbpl, cb_cbpc, cb_cmode, cb_ldc, cb_cdc[2], cb_t8;
  std::vector<int16_t> cb_mvd;
  bool prev_qp_delta_nz = false;

  void cabac_prepare() {
    int n = mb_w * mb_h, n4 = n * 16;
    cb_nnz.assign(n4, 0);
    cb_cnnz[0].assign(n * 4, 0); cb_cnnz[1].assign(n * 4, 0);
    for (auto* v : {&cb_intra, &cb_i16, &cb_skip, &cb_cbpl, &cb_cbpc, &cb_cmode, &cb_ldc, &cb_cdc[0], &cb_cdc[1], &cb_t8})
      v->assign(n, 0);
    cb_mvd.assign(n4 * 2, 0);
    prev_qp_delta_nz = false;
    ce = CabacEnc();
    ce.init(qp, is_idr, 0);
  }
  // h264.rs:2139 cabac_cbf_ctx_inc (-1: neighbour unavailable)
  static int cbf_inc(int l, int t, bool intra) {
    int a = l < 0 ? intra : l, b = t < 0 ? intra : t;
    return a + 2 * b;
  }
  // h264.rs:3293 luma_neighbor_cbf
  int luma_nb(int gx, int gy, bool left) const {
    if (left ? gx == 0 : gy == 0) return -1;
    int ngx = left ? gx - 1 : gx, ngy = left ? gy : gy - 1;
    int nm = (ngy / 4) * mb_w + ngx / 4;
    if (cb_skip[nm]) return 0;
    if (!cb_i16[nm]) {
      int n8 = (ngy & 2) + ((ngx & 2) >> 1);
      if (!((cb_cbpl[nm] >> n8) & 1) && !cb_intra[nm]) return 0;
    }
    return cb_nnz[ngy * gstride() + ngx] > 0;
  }
  // h264.rs:3492 encode_cabac_chroma_residuals
  void cabac_chroma(int mbx, int mby, bool intra, int cbpc, const rg_mb_out& r) {
    int m = mby * mb_w + mbx, cg = mb_w * 2;
    if (cbpc >= 1)
      for (int p = 0; p < 2; p++) {
        int l = mbx > 0 ? (!cb_skip[m - 1] && cb_cdc[p][m - 1]) : -1;
        int t = mby > 0 ? (!cb_skip[m - mb_w] && cb_cdc[p][m - mb_w]) : -1;
        ce.residual(3, cbf_inc(l, t, intra), r.chroma_dc[p], 4);
        cb_cdc[p][m] = r.chroma_dc[p][0] || r.chroma_dc[p][1] || r.chroma_dc[p][2] || r.chroma_dc[p][3];
      }
    if (cbpc >= 2)
      for (int p = 0; p < 2; p++)
        for (int b = 0; b < 4; b++) {
          int cx = mbx * 2 + (b & 1), cy = mby * 2 + (b >> 1);
          int l = cx > 0 ? cb_cnnz[p][cy * cg + cx - 1] > 0 : -1;
          int t = cy > 0 ? cb_cnnz[p][(cy - 1) * cg + cx] > 0 : -1;
          const int16_t* ac = r.chroma_ac[p][b] + 1;
          ce.residual(4, cbf_inc(l, t, intra), ac, 15);
          int cnt = 0;
          for (int i = 0; i < 15; i++) cnt += ac[i] != 0;
          cb_cnnz[p][cy * cg + cx] = (uint8_t)cnt;
        }
  }
  // h264.rs:3327 encode_cabac_cbp_and_residuals
  void cabac_cbp_residuals(int mbx, int mby, bool intra, bool write8, const rg_mb_out& r) {
    int m = mby * mb_w + mbx, g = gstride();
    int cbpl = r.cbp & 15, cbpc = r.cbp >> 4;
    for (int i8 = 0; i8 < 4; i8++) {
      int bx8 = i8 & 1, by8 = i8 >> 1;
      bool lnz = bx8 ? (cbpl >> (i8 - 1)) & 1 : (mbx > 0 ? !cb_skip[m - 1] && ((cb_cbpl[m - 1] >> (by8 * 2 + 1)) & 1) : true);
      bool tnz = by8 ? (cbpl >> (i8 - 2)) & 1 : (mby > 0 ? !cb_skip[m - mb_w] && ((cb_cbpl[m - mb_w] >> (2 + bx8)) & 1) : true);
      ce.decision(73 + !lnz + 2 * !tnz, (cbpl >> i8) & 1);
    }
    int lc = mbx > 0 && !cb_skip[m - 1] ? cb_cbpc[m - 1] : 0;
    int tc = mby > 0 && !cb_skip[m - mb_w] ? cb_cbpc[m - mb_w] : 0;
    int c0 = 77 + (lc != 0) + 2 * (tc != 0);
    if (cbpc == 0) {
      ce.decision(c0, 0);
    } else {
      ce.decision(c0, 1);
      ce.decision(81 + (lc == 2) + 2 * (tc == 2), cbpc == 2);
    }
    cb_cbpl[m] = (uint8_t)cbpl;
    cb_cbpc[m] = (uint8_t)cbpc;
    if (cbpl == 0 && cbpc == 0) { prev_qp_delta_nz = false; return; }
    if (write8 && cbpl && !intra) {
      int l8 = mbx > 0 && cb_t8[m - 1], t8 = mby > 0 && cb_t8[m - mb_w];
      ce.decision(399 + l8 + t8, r.transform_8x8 != 0);
    }
    ce.qp_delta(prev_qp_delta_nz, r.qp_delta);
    prev_qp_delta_nz = r.qp_delta != 0;
    if (r.transform_8x8) {
      for (int i8 = 0; i8 < 4; i8++) {
        int gx = mbx * 4 + (i8 & 1) * 2, gy = mby * 4 + (i8 >> 1) * 2;
        bool coded = (cbpl >> i8) & 1;
        if (coded) ce.residual(5, 0, r.luma + i8 * 64, 64);
        for (int y = 0; y < 2; y++)
          for (int x = 0; x < 2; x++) cb_nnz[(gy + y) * g + gx + x] = coded;
      }
    } else {
      for (int b = 0; b < 16; b++) {
        int bx, by; blk_xy(b, bx, by);
        int gx = mbx * 4 + bx, gy = mby * 4 + by;
        if ((cbpl >> (b >> 2)) & 1) {
          const int16_t* c = r.luma + b * 16;
          ce.residual(2, cbf_inc(luma_nb(gx, gy, true), luma_nb(gx, gy, false), intra), c, 16);
          int cnt = 0;
          for (int i = 0; i < 16; i++) cnt += c[i] != 0;
          cb_nnz[gy * g + gx] = (uint8_t)cnt;
        } else {
          cb_nnz[gy * g + gx] = 0;
        }
      }
    }
    cabac_chroma(mbx, mby, intra, cbpc, r);
  }
  void write_mb_cabac(int mbx, int mby, const rg_mb_out& r) {
    int m = mby * mb_w + mbx, g = gstride();
    int sl = mbx > 0 && !cb_skip[m - 1], st = mby > 0 && !cb_skip[m - mb_w];
    if (r.mb_type == RG_MB_P_SKIP) {
      ce.decision(11 + sl + st, 1);
      cb_skip[m] = 1;
      prev_qp_delta_nz = false;
      return;
    }
    if (!is_idr) ce.decision(11 + sl + st, 0);
    int li = mbx > 0 && cb_i16[m - 1], ti = mby > 0 && cb_i16[m - mb_w];
    if (r.mb_type == RG_MB_P_L0_16X16) {
      if (r.transform_8x8) cb_t8[m] = 1;
      ce.p_mb_type(0);
      uint32_t ax = 0, ay = 0;
      int gx0 = mbx * 4, gy0 = mby * 4;
      if (gx0 > 0) { int i = gy0 * g + gx0 - 1; ax += std::abs(cb_mvd[2 * i]); ay += std::abs(cb_mvd[2 * i + 1]); }
      if (gy0 > 0) { int i = (gy0 - 1) * g + gx0; ax += std::abs(cb_mvd[2 * i]); ay += std::abs(cb_mvd[2 * i + 1]); }
      ce.mvd(0, ax, r.mvd[0]);
      ce.mvd(1, ay, r.mvd[1]);
      cabac_cbp_residuals(mbx, mby, false, t8x8, r);
      for (int y = 0; y < 4; y++)
        for (int x = 0; x < 4; x++) {
          int i = (gy0 + y) * g + gx0 + x;
          cb_mvd[2 * i] = r.mvd[0];
          cb_mvd[2 * i + 1] = r.mvd[1];
        }
      return;
    }
    cb_intra[m] = 1;
    cb_cmode[m] = r.chroma_mode;
    int lcm = mbx > 0 && cb_intra[m - 1] && cb_cmode[m - 1] != 0;
    int tcm = mby > 0 && cb_intra[m - mb_w] && cb_cmode[m - mb_w] != 0;
    if (r.mb_type == RG_MB_I4X4) {
      for (int b = 0; b < 16; b++) {
        int bx, by; blk_xy(b, bx, by);
        intra4x4_modes[(mby * 4 + by) * g + mbx * 4 + bx] = 2;
      }
      if (!is_idr) ce.p_mb_type(5);
      else ce.intra_mb_type(3, li, ti, 0);
      if (t8x8) ce.decision(399 + (mbx > 0 && cb_t8[m - 1]) + (mby > 0 && cb_t8[m - mb_w]), 0);
      for (int b = 0; b < 16; b++) {
        int bx, by; blk_xy(b, bx, by);
        int gx = mbx * 4 + bx, gy = mby * 4 + by;
        int pm = pred_i4_mode(gx, gy), md = r.i4_modes[b];
        ce.i4_mode(md == pm, md < pm ? md : std::max(md - 1, 0));
        intra4x4_modes[gy * g + gx] = (uint8_t)md;
      }
      ce.chroma_mode(lcm, tcm, r.chroma_mode);
      cabac_cbp_residuals(mbx, mby, true, false, r);
      return;
    }
    // I_16x16
    int cbpl = r.cbp & 15, cbpc = r.cbp >> 4;
    cb_i16[m] = 1;
    cb_cbpl[m] = (uint8_t)cbpl;
    cb_cbpc[m] = (uint8_t)cbpc;
    int mbt = 1 + r.i16_mode + 4 * cbpc + (cbpl ? 12 : 0);
    if (!is_idr) ce.p_mb_type(5 + mbt);
    else ce.intra_mb_type(3, li, ti, mbt);
    ce.chroma_mode(lcm, tcm, r.chroma_mode);
    ce.qp_delta(prev_qp_delta_nz, r.qp_delta);
    prev_qp_delta_nz = r.qp_delta != 0;
    int ldc = mbx > 0 ? cb_ldc[m - 1] : -1, tdc = mby > 0 ? cb_ldc[m - mb_w] : -1;
    ce.residual(0, cbf_inc(ldc, tdc, true), r.luma_dc, 16);
    bool any = false;
    for (int i = 0; i < 16; i++) any |= r.luma_dc[i] != 0;
    cb_ldc[m] = any;
    if (cbpl)
      for (int b = 0; b < 16; b++) {
        int bx, by; blk_xy(b, bx, by);
        int gx = mbx * 4 + bx, gy = mby * 4 + by;
        const int16_t* ac = r.luma + b * 16 + 1;
        ce.residual(1, cbf_inc(luma_nb(gx, gy, true), luma_nb(gx, gy, false), true), ac, 15);
        int cnt = 0;
        for (int i = 0; i < 15; i++) cnt += ac[i] != 0;
        cb_nnz[gy * g + gx] = (uint8_t)cnt;
      }
    cabac_chroma(mbx, mby, true, cbpc, r);
  }

  // ---- macroblock coding ----
  void store_mb(int mbx, int mby, const uint8_t* y, const uint8_t* u, const uint8_t* v) {
    for (int r = 0; r < 16; r++) memcpy(cur.y.ptr(mbx * 16, mby * 16 + r), y + r * 16, 16);
    for (int r = 0; r < 8; r++) {
      memcpy(cur.u.ptr(mbx * 8, mby * 8 + r), u + r * 8, 8);
      memcpy(cur.v.ptr(mbx * 8, mby * 8 + r), v + r * 8, 8);
    }
  }
  void set_mb_state(int m, bool intra, int cbpl, bool t8, uint16_t nzm) {
    mb_intra[m] = intra; mb_cbp_luma[m] = (uint8_t)cbpl; mb_t8[m] = t8; nz16[m] = nzm; mb_qp[m] = (uint8_t)cur_qp;
  }

  // enc.rs:3587 code_i16 (mode chosen)
  void code_i16(int mbx, int mby, const MbSrc& src, int mode, rg_mb_out& r) {
    int m = mby * mb_w + mbx;
    uint8_t top[16], left[16]; bool ht, hl; int tl;
    i16_edges(mbx, mby, top, left, ht, hl, tl);
    uint8_t pred[256], pu[64], pv[64];
    pred16(mode, ht ? top : nullptr, hl ? left : nullptr, tl, pred);
    int cm = analyse_chroma(mbx, mby, src, pu, pv);
    fill_motion(mbx, mby, -1, 0, 0);
    int q_ = cur_qp, qpc = chroma_qp(q_, 0);
    int16_t ac[16][16], dcraw[16];
    dct_luma(src.y, pred, ac);
    static const int z2r[16] = {0, 1, 4, 5, 2, 3, 6, 7, 8, 9, 12, 13, 10, 11, 14, 15};
    for (int b = 0; b < 16; b++) dcraw[z2r[b]] = ac[b][0];
    Quant4 q = quant4(q_, true);
    bool any_ac = false;
    int16_t aczz[16][16];
    memset(aczz, 0, sizeof aczz);
    for (int gi = 0; gi < 4; gi++) {
      int nz = 0;
      for (int k = 0; k < 4; k++) nz |= quant_block(ac[gi * 4 + k], q);
      if (nz) {
        for (int k = 0; k < 4; k++) {
          ac[gi * 4 + k][0] = 0;
          zigzag16(ac[gi * 4 + k], aczz[gi * 4 + k]);
          for (int i = 1; i < 16; i++) if (aczz[gi * 4 + k][i]) any_ac = true;
        }
      }
    }
    int16_t dcq[16];
    quant_luma_dc(dcraw, q_, dcq);
    int cbpl = any_ac ? 15 : 0;
    Chroma c;
    quant_chroma(src, pu, pv, qpc, true, c);
    int cbpc = chroma_cbp(c);
    // record
    r.mb_type = RG_MB_I16X16; r.i16_mode = (uint8_t)mode; r.chroma_mode = (uint8_t)cm;
    r.cbp = (uint8_t)(cbpl | (cbpc << 4));
    uint16_t nzm = 0;
    for (int b = 0; b < 16; b++) {
      memcpy(r.luma + b * 16, aczz[b], 32);
      if (cbpl) for (int i = 1; i < 16; i++) if (aczz[b][i]) nzm |= 1 << b;
    }
    zigzag16(dcq, r.luma_dc);
    memcpy(r.chroma_dc, c.dc, sizeof c.dc);
    memcpy(r.chroma_ac, c.ac, sizeof c.ac);
    set_mb_state(m, true, cbpl, false, nzm);
    // recon
    int16_t dcr[16];
    dequant_idct_luma_dc(dcq, q_, dcr);
    int32_t sc[16];
    dequant4_scale(q_, sc);
    for (int gi = 0; gi < 4; gi++) {
      bool any = false;
      for (int k = 0; k < 4; k++) {
        int16_t* blk = ac[gi * 4 + k];
        if (cbpl) dequant_block(blk, sc);
        blk[0] = dcr[z2r[gi * 4 + k]];
        for (int i = 0; i < 16; i++) any |= blk[i] != 0;
      }
      if (any)
        for (int k = 0; k < 4; k++) {
          int bx, by; blk_xy(gi * 4 + k, bx, by);
          add_idct4(pred + by * 64 + bx * 4, 16, ac[gi * 4 + k]);
        }
    }
    recon_chroma(pu, pv, c, cbpc, qpc);
    store_mb(mbx, mby, pred, pu, pv);
  }

  // enc.rs:3336 analyse_i4; returns false when the budget is exceeded. Writes recon into cur.y.
  bool analyse_i4(int mbx, int mby, const MbSrc& src, uint32_t budget, rg_mb_out& r, uint8_t* recon, int16_t q4[16][16], int& cbpl,
                  const uint16_t* masks = nullptr) {
    int g = gstride();
    int q_ = cur_qp;
    uint32_t lambda = kLambda[q_];
    uint8_t saved[16];
    for (int b = 0; b < 16; b++) { int bx, by; blk_xy(b, bx, by); saved[b] = intra4x4_modes[(mby * 4 + by) * g + mbx * 4 + bx]; }
    int16_t had[16][16];
    for (int by = 0; by < 4; by++) for (int bx = 0; bx < 4; bx++) hadamard_src4(src.y + by * 64 + bx * 4, 16, had[by * 4 + bx]);
    Quant4 quant = quant4(q_, true);
    int32_t sc[16];
    dequant4_scale(q_, sc);
    uint32_t total = lambda * 24;
    cbpl = 0;
    for (int b = 0; b < 16; b++) {
      int bx, by; blk_xy(b, bx, by);
      int px = mbx * 16 + bx * 4, py = mby * 16 + by * 4, gx = mbx * 4 + bx, gy = mby * 4 + by;
      // enc.rs:1493 i4_edges
      uint8_t top[8], left[4]; bool ht = py > 0, hl = px > 0; int tl;
      if (ht) {
        memcpy(top, cur.y.ptr(px, py - 1), 4);
        bool tr = !(b == 3 || b == 7 || b == 11 || b == 13 || b == 15) && (b != 5 || mbx + 1 < mb_w);
        if (tr) memcpy(top + 4, cur.y.ptr(px + 4, py - 1), 4);
        else memset(top + 4, top[3], 4);
      }
      if (hl) for (int k = 0; k < 4; k++) left[k] = *cur.y.ptr(px - 1, py + k);
      tl = (ht && hl) ? *cur.y.ptr(px - 1, py - 1) : 128;
      int pm = pred_i4_mode(gx, gy);
      auto bits = [&](int md) { return lambda * (md == pm ? 1u : 4u); };
      // enc.rs:1671 intra_satd_x3_4x4
      const int16_t* h = had[by * 4 + bx];
      int total_abs = 0;
      for (int k = 0; k < 16; k++) total_abs += iabs(h[k]);
      int dc;
      {
        int st = ht ? top[0] + top[1] + top[2] + top[3] : 0, sl = hl ? left[0] + left[1] + left[2] + left[3] : 0;
        if (ht && hl) dc = (st + sl + 4) >> 3;
        else if (ht) dc = (st + 2) >> 2;
        else if (hl) dc = (sl + 2) >> 2;
        else dc = 128;
      }
      int sd = total_abs - iabs(h[0]) + iabs(h[0] - 16 * dc), sv = 0, sh = 0;
      if (ht) { int p[4]; hadamard_edge(top, p); sv = total_abs; for (int k = 0; k < 4; k++) sv += iabs(h[k] - p[k]) - iabs(h[k]); }
      if (hl) { int p[4]; hadamard_edge(left, p); sh = total_abs; for (int k = 0; k < 4; k++) sh += iabs(h[4 * k] - p[k]) - iabs(h[4 * k]); }
      uint32_t s3[3] = {(uint32_t)(sv >> 1), (uint32_t)(sh >> 1), (uint32_t)(sd >> 1)};
      uint32_t best = UINT32_MAX; int bm = 2;
      // learned form: only the hinted modes available here (DC when none is)
      uint32_t allow = 0x1ff;
      if (masks) {
        uint32_t avail = 0x4u | (ht ? 0x89u : 0u) | (hl ? 0x102u : 0u) | (ht && hl ? 0x70u : 0u);
        allow = masks[b] & avail;
        if (!allow) allow = 0x4u;
      }
      bool ok3[3] = {ht, hl, true};
      for (int md = 0; md < 3; md++)
        if (ok3[md] && ((allow >> md) & 1) && s3[md] + bits(md) < best) { best = s3[md] + bits(md); bm = md; }
      uint8_t t8[8], l4[4];
      for (int k = 0; k < 8; k++) t8[k] = ht ? top[k] : 128;
      for (int k = 0; k < 4; k++) l4[k] = hl ? left[k] : 128;
      uint8_t dirs[6][16];
      for (int md = 3; md <= 8; md++) pred4x4(md, t8, l4, tl, dirs[md - 3]);
      for (int md = 3; md <= 8; md++) {
        bool av = (md == 3 || md == 7) ? ht : (md == 8 ? hl : (ht && hl));
        if (!av || !((allow >> md) & 1)) continue;
        uint32_t cst = satd4(src.y + by * 64 + bx * 4, 16, dirs[md - 3], 4) + bits(md);
        if (cst < best) { best = cst; bm = md; }
      }
      uint8_t pred[16];
      if (bm >= 3) memcpy(pred, dirs[bm - 3], 16);
      else pred4x4(bm, ht ? top : nullptr, hl ? left : nullptr, tl, pred);
      total += best;
      if (total >= budget) {
        for (int bb = 0; bb < 16; bb++) { int x, y; blk_xy(bb, x, y); intra4x4_modes[(mby * 4 + y) * g + mbx * 4 + x] = saved[bb]; }
        return false;
      }
      r.i4_modes[b] = (uint8_t)bm;
      intra4x4_modes[gy * g + gx] = (uint8_t)bm;
      int16_t d[16];
      for (int y = 0; y < 4; y++) for (int x = 0; x < 4; x++) d[y * 4 + x] = (int16_t)(src.y[by * 64 + bx * 4 + y * 16 + x] - pred[y * 4 + x]);
      int16_t c[16];
      fdct4(d, c);
      bool nz = false;
      for (int i = 0; i < 16; i++) {  // enc.rs:1705 quant_one
        int l = (int)(((uint32_t)iabs(c[i]) * quant.mf[i] + quant.bias) >> quant.shift);
        q4[b][i] = (int16_t)(c[i] < 0 ? -l : l);
        if (q4[b][i]) nz = true;
      }
      uint8_t rec[16];
      memcpy(rec, pred, 16);
      if (nz) {
        cbpl |= 1 << (b >> 2);
        int16_t dq[16];
        for (int i = 0; i < 16; i++) dq[i] = clamp_i16((int64_t)q4[b][i] * sc[i]);
        add_idct4(rec, 4, dq);
      }
      for (int y = 0; y < 4; y++) {
        memcpy(cur.y.ptr(px, py + y), rec + y * 4, 4);
        memcpy(recon + (by * 4 + y) * 16 + bx * 4, rec + y * 4, 4);
      }
    }
    return true;
  }

  // enc.rs:3311 code_intra (I slices)
  void code_intra(int mbx, int mby, const MbSrc& src, rg_mb_out& r) {
    uint32_t lambda = kLambda[cur_qp];
    uint32_t i16c; int i16m;
    analyse_i16(mbx, mby, src, i16c, i16m);
    if (i16c > 40 * lambda) {
      uint8_t recon[256]; int16_t q4[16][16]; int cbpl;
      const uint16_t* masks = form == 2 && hints ? hints[mby * mb_w + mbx].i4_mask : nullptr;
      if (analyse_i4(mbx, mby, src, i16c + lambda * 4, r, recon, q4, cbpl, masks)) {
        code_i4(mbx, mby, src, r, recon, q4, cbpl);
        return;
      }
    }
    code_i16(mbx, mby, src, i16m, r);
  }
  // enc.rs:3442 code_i4
  void code_i4(int mbx, int mby, const MbSrc& src, rg_mb_out& r, const uint8_t* recon, int16_t q4[16][16], int cbpl) {
    int m = mby * mb_w + mbx;
    uint8_t pu[64], pv[64];
    int cm = analyse_chroma(mbx, mby, src, pu, pv);
    int qpc = chroma_qp(cur_qp, 0);
    Chroma c;
    quant_chroma(src, pu, pv, qpc, true, c);
    int cbpc = chroma_cbp(c);
    fill_motion(mbx, mby, -1, 0, 0);
    r.mb_type = RG_MB_I4X4; r.chroma_mode = (uint8_t)cm; r.cbp = (uint8_t)(cbpl | (cbpc << 4));
    uint16_t nzm = 0;
    for (int b = 0; b < 16; b++) {
      zigzag16(q4[b], r.luma + b * 16);
      for (int i = 0; i < 16; i++) if (q4[b][i]) nzm |= 1 << b;
    }
    memcpy(r.chroma_dc, c.dc, sizeof c.dc);
    memcpy(r.chroma_ac, c.ac, sizeof c.ac);
    set_mb_state(m, true, cbpl, false, nzm);
    recon_chroma(pu, pv, c, cbpc, qpc);
    store_mb(mbx, mby, recon, pu, pv);
  }

  // enc.rs:3011 code_p_mb
  void code_p_mb(int mbx, int mby, const MbSrc& src, rg_mb_out& r) {
    int g = gstride(), m = mby * mb_w + mbx;
    int gx0 = mbx * 4, gy0 = mby * 4, x0 = mbx * 16, y0 = mby * 16;
    int q_ = cur_qp, qpc = chroma_qp(q_, 0);
    Bounds bd = mv_bounds(x0, y0);
    uint32_t lambda = kLambda[q_];
    int16_t mvp[2];
    mvp16(gx0, gy0, mvp);
    auto zero_nb = [&](int i) { return ref_grid[i] == 0 && mv_grid[2 * i] == 0 && mv_grid[2 * i + 1] == 0; };
    int16_t pskip[2] = {mvp[0], mvp[1]};
    if (gx0 == 0 || gy0 == 0 || zero_nb(gy0 * g + gx0 - 1) || zero_nb((gy0 - 1) * g + gx0)) { pskip[0] = 0; pskip[1] = 0; }
    uint8_t py[256], pu[64], pv[64];

    // 1. skip probe (enc.rs:2906 try_p_skip)
    if (in_bounds(bd, pskip[0], pskip[1])) {
      mc_luma16(x0, y0, pskip[0], pskip[1], py);
      uint32_t s = sad(src.y, 16, py, 16, 16, 16);
      if (s < sb_probe) {
        bool luma_zero = s <= sb_luma || ssd(src.y, 16, py, 16, 16) <= sb_luma_ssd;
        if (!luma_zero) luma_zero = probe_skip_luma(src, py, q_);
        if (luma_zero) {
          mc_chroma8(mbx, mby, pskip[0], pskip[1], pu, pv);
          auto plane_zero = [&](const uint8_t* s8, const uint8_t* p8) {
            return sad(s8, 8, p8, 8, 8, 8) <= sb_chroma || ssd(s8, 8, p8, 8, 8) <= sb_chroma_ssd;
          };
          bool chroma_zero = plane_zero(src.u, pu) && plane_zero(src.v, pv);
          if (!chroma_zero) chroma_zero = probe_skip_chroma(src, pu, pv, qpc);
          if (chroma_zero) {
            code_skip(mbx, mby, pskip, r);
            store_mb(mbx, mby, py, pu, pv);
            return;
          }
        }
      }
    }

    // 2. motion search
    int16_t cands[5][2];
    int n = 0;
    cands[n][0] = mvp[0]; cands[n][1] = mvp[1]; n++;
    cands[n][0] = 0; cands[n][1] = 0; n++;
    if (mbx > 0) { int i = gy0 * g + gx0 - 1; cands[n][0] = mv_grid[2 * i]; cands[n][1] = mv_grid[2 * i + 1]; n++; }
    if (mby > 0) { int i = (gy0 - 1) * g + gx0; cands[n][0] = mv_grid[2 * i]; cands[n][1] = mv_grid[2 * i + 1]; n++; }
    cands[n][0] = prev_mb_mv[2 * m]; cands[n][1] = prev_mb_mv[2 * m + 1]; n++;
    auto mv_cost = [&](int mx, int my) { return mvd_cost(mx - mvp[0], lambda) + mvd_cost(my - mvp[1], lambda); };
    auto cost_at = [&](int fx, int fy) {
      return sad(src.y, 16, refp.y.ptr(x0 + fx, y0 + fy), refp.y.stride, 16, 16) + mv_cost(fx * 4, fy * 4);
    };
    // enc.rs:1185 full_pel
    int imin[2] = {(bd.min[0] + 3) >> 2, (bd.min[1] + 3) >> 2}, imax[2] = {bd.max[0] >> 2, bd.max[1] >> 2};
    auto inside = [&](int x, int y) { return x >= imin[0] && x <= imax[0] && y >= imin[1] && y <= imax[1]; };
    int best[2] = {0, 0};
    uint32_t best_cost = UINT32_MAX;
    int seen[8][2];
    for (int k = 0; k < 8; k++) { seen[k][0] = INT32_MAX; seen[k][1] = INT32_MAX; }
    for (int k = 0; k < n; k++) {
      int mx = std::max(imin[0], std::min(imax[0], (cands[k][0] + 2) >> 2));
      int my = std::max(imin[1], std::min(imax[1], (cands[k][1] + 2) >> 2));
      bool dup = false;
      for (int j = 0; j < k; j++) if (seen[j][0] == mx && seen[j][1] == my) dup = true;
      if (dup) continue;
      seen[k][0] = mx; seen[k][1] = my;
      uint32_t c = cost_at(mx, my);
      if (c < best_cost) { best_cost = c; best[0] = mx; best[1] = my; }
    }
    for (int it = 0; it < 16; it++) {
      int pts[4][2] = {{best[0], best[1] - 1}, {best[0] - 1, best[1]}, {best[0] + 1, best[1]}, {best[0], best[1] + 1}};
      int moved = -1;
      for (int k = 0; k < 4; k++) {
        if (!inside(pts[k][0], pts[k][1])) continue;
        uint32_t c = cost_at(pts[k][0], pts[k][1]);
        if (c < best_cost) { best_cost = c; moved = k; }
      }
      if (moved < 0) break;
      best[0] = pts[moved][0]; best[1] = pts[moved][1];
    }
    int mv[2];
    uint32_t me_cost;
    int fmv[2] = {best[0] * 4, best[1] * 4};
    if (best_cost - mv_cost(fmv[0], fmv[1]) <= sb_luma) {
      mv[0] = fmv[0]; mv[1] = fmv[1]; me_cost = best_cost;
      mc_luma16(x0, y0, mv[0], mv[1], py);
    } else {
      // enc.rs:1283 sub_pel (window predictions equal h264_luma_mc, enc.rs:4030)
      int center[2] = {fmv[0], fmv[1]}, bq[2] = {fmv[0], fmv[1]};
      uint32_t bc = best_cost;
      const int steps[2] = {2, 1}, iters[2] = {1, 2};
      for (int si = 0; si < 2; si++) {
        int st = steps[si];
        for (int it = 0; it < iters[si]; it++) {
          int from[2] = {bq[0], bq[1]};
          int dd[4][2] = {{0, -st}, {-st, 0}, {st, 0}, {0, st}};
          for (int k = 0; k < 4; k++) {
            int cx = from[0] + dd[k][0], cy = from[1] + dd[k][1];
            if (iabs(cx - center[0]) > 3 || iabs(cy - center[1]) > 3 || !in_bounds(bd, cx, cy)) continue;
            uint8_t tmp[256];
            mc_luma16(x0, y0, cx, cy, tmp);
            uint32_t c = sad(src.y, 16, tmp, 16, 16, 16) + mv_cost(cx, cy);
            if (c < bc) { bc = c; bq[0] = cx; bq[1] = cy; }
          }
          if (bq[0] == from[0] && bq[1] == from[1]) break;
        }
      }
      mv[0] = bq[0]; mv[1] = bq[1]; me_cost = bc;
      mc_luma16(x0, y0, mv[0], mv[1], py);
    }
    (void)me_cost;

    // 3. intra 16x16 check
    uint32_t inter_satd = satd16(src.y, 16, py, 16);
    uint32_t inter_cost = inter_satd + lambda * (se_bits(mv[0] - mvp[0]) + se_bits(mv[1] - mvp[1]) + 1);
    if (inter_satd > 24 * lambda) {
      uint32_t i16c; int i16m;
      analyse_i16(mbx, mby, src, i16c, i16m);
      if (i16c + lambda * 8 < inter_cost) {
        code_i16(mbx, mby, src, i16m, r);
        return;
      }
    }

    // 4. P_L0_16x16 residual
    mc_chroma8(mbx, mby, mv[0], mv[1], pu, pv);
    int16_t q4[16][16];
    int cbp4 = quant_luma_inter(src.y, py, q_, q4);
    int cbpl = cbp4;
    bool use8 = false;
    int16_t q8[4][64];
    if (t8x8 && cabac && cbp4) {
      int cbp8 = quant_luma_8x8(src.y, py, q_, q8);
      int nnz4 = 0, nnz8 = 0;
      for (int b = 0; b < 16; b++) for (int i = 0; i < 16; i++) nnz4 += q4[b][i] != 0;
      for (int b = 0; b < 4; b++) for (int i = 0; i < 64; i++) nnz8 += q8[b][i] != 0;
      if (nnz8 <= nnz4) { use8 = true; cbpl = cbp8; }
    }
    Chroma c;
    quant_chroma(src, pu, pv, qpc, false, c);
    for (int p = 0; p < 2; p++) {
      bool anym = c.mask[p][0] | c.mask[p][1] | c.mask[p][2] | c.mask[p][3];
      if (anym && chroma_ac_score(c, p) < 7) {
        memset(c.ac[p], 0, sizeof c.ac[p]);
        memset(c.mask[p], 0, sizeof c.mask[p]);
        memset(c.raster[p], 0, sizeof c.raster[p]);
      }
    }
    int cbpc = chroma_cbp(c);
    if (cbpl == 0 && cbpc == 0 && mv[0] == pskip[0] && mv[1] == pskip[1]) {
      code_skip(mbx, mby, pskip, r);
      store_mb(mbx, mby, py, pu, pv);
      return;
    }
    // enc.rs:3196 code_inter
    r.mb_type = RG_MB_P_L0_16X16;
    r.mv[0] = (int16_t)mv[0]; r.mv[1] = (int16_t)mv[1];
    r.mvd[0] = (int16_t)(mv[0] - mvp[0]); r.mvd[1] = (int16_t)(mv[1] - mvp[1]);
    r.cbp = (uint8_t)(cbpl | (cbpc << 4));
    bool t8flag = use8 && cbpl != 0;
    r.transform_8x8 = t8flag;
    uint16_t nzm = 0;
    if (use8) {
      for (int b = 0; b < 4; b++) {
        for (int i = 0; i < 64; i++) r.luma[b * 64 + i] = q8[b][kZigzag8[i]];
        if (cbpl & (1 << b)) nzm |= 0xF << (4 * b);
      }
    } else {
      for (int b = 0; b < 16; b++) {
        zigzag16(q4[b], r.luma + b * 16);
        for (int i = 0; i < 16; i++) if (q4[b][i]) nzm |= 1 << b;
      }
    }
    memcpy(r.chroma_dc, c.dc, sizeof c.dc);
    memcpy(r.chroma_ac, c.ac, sizeof c.ac);
    set_mb_state(m, false, cbpl, t8flag, nzm);
    if (use8) {
      for (int b = 0; b < 4; b++)
        if (cbpl & (1 << b)) {
          int32_t d[64];
          dequant8(q8[b], q_, d);
          idct8_add(py + (b >> 1) * 128 + (b & 1) * 8, 16, d);
        }
    } else {
      int32_t sc[16];
      dequant4_scale(q_, sc);
      for (int b = 0; b < 16; b++)
        if (cbpl & (1 << (b >> 2))) {
          int16_t blk[16];
          memcpy(blk, q4[b], 32);
          dequant_block(blk, sc);
          int bx, by; blk_xy(b, bx, by);
          add_idct4(py + by * 64 + bx * 4, 16, blk);
        }
    }
    recon_chroma(pu, pv, c, cbpc, qpc);
    fill_motion(mbx, mby, 0, mv[0], mv[1]);
    store_mb(mbx, mby, py, pu, pv);
  }
  void code_skip(int mbx, int mby, const int16_t* mv, rg_mb_out& r) {
    int m = mby * mb_w + mbx;
    r.mb_type = RG_MB_P_SKIP;
    r.mv[0] = mv[0]; r.mv[1] = mv[1];
    fill_motion(mbx, mby, 0, mv[0], mv[1]);
    set_mb_state(m, false, 0, false, 0);
    mb_skip[m] = 1;
  }
  // enc.rs:2163 probe_skip_luma
  bool probe_skip_luma(const MbSrc& src, const uint8_t* py, int q_) const {
    int16_t c[16][16];
    dct_luma(src.y, py, c);
    Quant4 q = quant4(q_, false);
    uint32_t total = 0;
    for (int gi = 0; gi < 4; gi++) {
      int nz = 0;
      for (int k = 0; k < 4; k++) nz |= quant_block(c[gi * 4 + k], q);
      if (!nz) continue;
      if (nz & 2) return false;
      for (int k = 0; k < 4; k++) {
        int16_t zz[16]; zigzag16(c[gi * 4 + k], zz);
        total += decimate_score(zz, 16);
        if (total >= 6) return false;
      }
    }
    return true;
  }
  // enc.rs:2190 probe_skip_chroma
  bool probe_skip_chroma(const MbSrc& src, const uint8_t* pu, const uint8_t* pv, int qpc) const {
    Chroma c;
    quant_chroma(src, pu, pv, qpc, false, c);
    for (int p = 0; p < 2; p++) for (int b = 0; b < 4; b++) if (c.dc[p][b]) return false;
    return chroma_ac_score(c, 0) < 7 && chroma_ac_score(c, 1) < 7;
  }
  void skip_bounds(int q_) {
    int qpc = chroma_qp(q_, 0);
    Quant4 q = quant4(q_, false), qc = quant4(qpc, false);
    auto zsad = [](const Quant4& qq) {
      static const uint32_t W[4] = {1, 2, 1, 2};
      uint32_t room = (1u << qq.shift) - qq.bias - 1, mn = UINT32_MAX;
      for (int i = 0; i < 16; i++) mn = std::min(mn, room / (qq.mf[i] * W[i >> 2] * W[i & 3]));
      return mn;
    };
    auto zssd = [](const Quant4& qq) {
      static const uint32_t N[4] = {4, 10, 4, 10};
      uint32_t room = (1u << qq.shift) - qq.bias - 1, mn = UINT32_MAX;
      for (int i = 0; i < 16; i++) { uint32_t lim = room / qq.mf[i]; mn = std::min(mn, lim * lim / (N[i >> 2] * N[i & 3])); }
      return mn;
    };
    uint32_t dsh = 16 + qpc / 6;
    uint32_t droom = (1u << dsh) - (1u << dsh) / 3 - 1;
    uint32_t dc = droom / (uint32_t)kQuant4Mf[qpc % 6][0];
    sb_luma = zsad(q); sb_luma_ssd = zssd(q);
    sb_chroma = std::min(zsad(qc), dc);
    sb_chroma_ssd = std::min(zssd(qc), dc * dc / 64);
    sb_probe = 16 * (((1u << q.shift) - q.bias) / q.mf[0] + 1);
  }


  // ---- search forms: full search (form 1) and learned (form 2); no counterpart in the reference.
  // The same decisions as the GPU engine's search forms: the skip probe of the plain form, an
  // integer search over a window (quadrant SADs, nine partition parts, cost SAD + lambda * vector
  // bits against the 16x16 predictor, first minimum in raster order), quarter-sample refinement of
  // each part of every tried partition type (centre and 8 neighbours at distance 2, then 8 at
  // distance 1; cost SATD/2 + lambda * vector bits against the part's own H.264 8.4.1.3 predictor),
  // the type of least total cost (+ lambda * type bits, by default {1, 16, 16, 40}), then the plain
  // form's intra check, residual and late skip. Learned: +-2 around a centre chosen among seven
  // integer candidates (predictor plus the hinted offset, predictor, the hint's coarse vector when
  // it has one, left / top / top-right (else top-left) neighbour vectors, zero) by 16x16 SAD +
  // lambda * vector bits, first in that order on ties; re-centred on the 16x16 best while that lies
  // on the window's edge (`walk` times), then the full window; only the hinted types, refined by the
  // SAD diamonds of refine_part_sad_s; intra 4x4 blocks of IDR pictures restricted to their hinted
  // modes.
  int form = 0, search_range = 32, walk = 4;
  int type_bits[4] = {1, 16, 16, 40};   // bits charged per partition type (x lambda)
  const rg_mb_hint* hints = nullptr;    // learned form: this picture's hints
  std::vector<uint8_t> mb_split;        // per MB: quadrant vectors differ

  struct NbS { int ref, x, y; };
  NbS nb4s(int mbx, int mby, int bx, int by, const int own[4][2], int done) const {
    if (bx >= 0 && bx < 4 && by >= 0 && by < 4) {
      int q = (by >> 1) * 2 + (bx >> 1);
      if ((done >> q) & 1) return {0, own[q][0], own[q][1]};
      return {-2, 0, 0};
    }
    if ((bx == 4 && by >= 0) || by >= 4) return {-2, 0, 0};
    int g = gstride(), gx = mbx * 4 + bx, gy = mby * 4 + by;
    if (gx < 0 || gy < 0 || gx >= g) return {-2, 0, 0};
    int i = gy * g + gx;
    int ref = ref_grid[i];
    if (ref != 0) return {ref, 0, 0};
    return {0, mv_grid[2 * i], mv_grid[2 * i + 1]};
  }
  // H.264 8.4.1.3 (dir: 1 16x8 top, 2 16x8 bottom, 3 8x16 left, 4 8x16 right, 0 median)
  void mv_pred_s(int mbx, int mby, int bx, int by, int pw, int dir, const int own[4][2], int done, int mvp[2]) const {
    NbS A = nb4s(mbx, mby, bx - 1, by, own, done), B = nb4s(mbx, mby, bx, by - 1, own, done);
    NbS C = nb4s(mbx, mby, bx + pw, by - 1, own, done);
    if (C.ref == -2) C = nb4s(mbx, mby, bx - 1, by - 1, own, done);
    if (dir == 1 && B.ref == 0) { mvp[0] = B.x; mvp[1] = B.y; return; }
    if ((dir == 2 || dir == 3) && A.ref == 0) { mvp[0] = A.x; mvp[1] = A.y; return; }
    if (dir == 4 && C.ref == 0) { mvp[0] = C.x; mvp[1] = C.y; return; }
    if (B.ref == -2 && C.ref == -2 && A.ref != -2) { mvp[0] = A.x; mvp[1] = A.y; return; }
    int m = (A.ref == 0) + (B.ref == 0) + (C.ref == 0);
    if (m == 1) {
      const NbS& o = A.ref == 0 ? A : (B.ref == 0 ? B : C);
      mvp[0] = o.x; mvp[1] = o.y;
      return;
    }
    auto med = [](int x, int y, int z) { return std::min(std::max(x, y), std::max(std::min(x, y), z)); };
    mvp[0] = med(A.x, B.x, C.x);
    mvp[1] = med(A.y, B.y, C.y);
  }
  // integer search over [xlo, xhi] x [ylo, yhi]: best vector and cost of each of the nine parts
  void int_search_s(int x0, int y0, const MbSrc& src, int xlo, int xhi, int ylo, int yhi, const int mvp[2], uint32_t lambda,
                    int bx[9], int by[9]) const {
    uint32_t bc[9];
    for (int k = 0; k < 9; k++) { bc[k] = UINT32_MAX; bx[k] = xlo; by[k] = ylo; }
    for (int y = ylo; y <= yhi; y++)
      for (int x = xlo; x <= xhi; x++) {
        uint32_t q[4];
        for (int k = 0; k < 4; k++)
          q[k] = sad(src.y + (k >> 1) * 128 + (k & 1) * 8, 16, refp.y.ptr(x0 + x + (k & 1) * 8, y0 + y + (k >> 1) * 8),
                     refp.y.stride, 8, 8);
        uint32_t part[9] = {q[0] + q[1] + q[2] + q[3], q[0] + q[1], q[2] + q[3], q[0] + q[2], q[1] + q[3], q[0], q[1], q[2], q[3]};
        uint32_t mc = lambda * (se_bits(4 * x - mvp[0]) + se_bits(4 * y - mvp[1]));
        for (int k = 0; k < 9; k++)
          if (part[k] + mc < bc[k]) { bc[k] = part[k] + mc; bx[k] = x; by[k] = y; }
      }
  }
  // SATD cost of a part's prediction at vector (mx, my)
  uint32_t part_cost(int x0, int y0, const MbSrc& src, int px, int py, int pw, int ph, int mx, int my, const int mvp[2],
                     uint32_t lambda) const {
    uint8_t pred[256];
    luma_mc(refp.y.ptr(x0 + px + (mx >> 2), y0 + py + (my >> 2)), refp.y.stride, pw, ph, mx & 3, my & 3, pred, 16);
    uint32_t s = 0;
    for (int by = 0; by < ph; by += 4)
      for (int bx = 0; bx < pw; bx += 4) s += satd4_raw(src.y + (py + by) * 16 + px + bx, 16, pred + by * 16 + bx, 16);
    return (s >> 1) + lambda * (se_bits(mx - mvp[0]) + se_bits(my - mvp[1]));
  }
  uint32_t refine_part_s(int x0, int y0, const MbSrc& src, const Bounds& bd, int px, int py, int pw, int ph, int ix, int iy,
                         const int mvp[2], uint32_t lambda, int mv[2]) const {
    static const int st[8][2] = {{0, -2}, {-2, 0}, {2, 0}, {0, 2}, {-2, -2}, {2, -2}, {-2, 2}, {2, 2}};
    int cx = 4 * ix, cy = 4 * iy;
    uint32_t best = part_cost(x0, y0, src, px, py, pw, ph, cx, cy, mvp, lambda);
    for (int step = 0; step < 2; step++) {
      int fx = cx, fy = cy;
      for (int k = 0; k < 8; k++) {
        int vx = fx + (step == 0 ? st[k][0] : st[k][0] / 2), vy = fy + (step == 0 ? st[k][1] : st[k][1] / 2);
        if (!in_bounds(bd, vx, vy)) continue;
        uint32_t c = part_cost(x0, y0, src, px, py, pw, ph, vx, vy, mvp, lambda);
        if (c < best) { best = c; cx = vx; cy = vy; }
      }
    }
    mv[0] = cx; mv[1] = cy;
    return best;
  }
  // learned form: SAD diamonds (half-sample: up, left, right, down at distance 2, one step; then
  // quarter-sample at distance 1, up to two steps), cost SAD + lambda * vector bits, within 3
  // quarter samples of the integer start
  uint32_t part_sad_cost(int x0, int y0, const MbSrc& src, int px, int py, int pw, int ph, int mx, int my, const int mvp[2],
                         uint32_t lambda) const {
    uint8_t pred[256];
    luma_mc(refp.y.ptr(x0 + px + (mx >> 2), y0 + py + (my >> 2)), refp.y.stride, pw, ph, mx & 3, my & 3, pred, 16);
    return sad(src.y + py * 16 + px, 16, pred, 16, pw, ph) + lambda * (se_bits(mx - mvp[0]) + se_bits(my - mvp[1]));
  }
  uint32_t refine_part_sad_s(int x0, int y0, const MbSrc& src, const Bounds& bd, int px, int py, int pw, int ph, int ix,
                             int iy, const int mvp[2], uint32_t lambda, int mv[2]) const {
    int cx = 4 * ix, cy = 4 * iy;
    uint32_t best = part_sad_cost(x0, y0, src, px, py, pw, ph, cx, cy, mvp, lambda);
    for (int st = 2; st >= 1; st--)
      for (int it = 0; it < (st == 2 ? 1 : 2); it++) {
        int fx = cx, fy = cy;
        const int d[4][2] = {{0, -st}, {-st, 0}, {st, 0}, {0, st}};
        for (int k = 0; k < 4; k++) {
          int vx = fx + d[k][0], vy = fy + d[k][1];
          if (std::abs(vx - 4 * ix) > 3 || std::abs(vy - 4 * iy) > 3 || !in_bounds(bd, vx, vy)) continue;
          uint32_t c = part_sad_cost(x0, y0, src, px, py, pw, ph, vx, vy, mvp, lambda);
          if (c < best) { best = c; cx = vx; cy = vy; }
        }
        if (cx == fx && cy == fy) break;
      }
    mv[0] = cx; mv[1] = cy;
    return best;
  }
  void fill_motion_q(int mbx, int mby, const int qmv[4][2]) {
    int g = gstride();
    for (int y = 0; y < 4; y++)
      for (int x = 0; x < 4; x++) {
        int i = (mby * 4 + y) * g + mbx * 4 + x, q = (y >> 1) * 2 + (x >> 1);
        ref_grid[i] = 0;
        mv_grid[2 * i] = (int16_t)qmv[q][0];
        mv_grid[2 * i + 1] = (int16_t)qmv[q][1];
      }
    mb_split[mby * mb_w + mbx] = !(qmv[0][0] == qmv[1][0] && qmv[0][0] == qmv[2][0] && qmv[0][0] == qmv[3][0] &&
                                   qmv[0][1] == qmv[1][1] && qmv[0][1] == qmv[2][1] && qmv[0][1] == qmv[3][1]);
  }
  static void set_parts(rg_mb_out& r, int ptype, const int qmv[4][2], const int pmvd[4][2]) {
    for (int q = 0; q < 4; q++)
      for (int c = 0; c < 2; c++) { r.part_mv[q][c] = (int16_t)qmv[q][c]; r.part_mvd[q][c] = (int16_t)pmvd[q][c]; }
    r.part_type = (uint8_t)ptype;
  }

  void code_p_mb_search(int mbx, int mby, const MbSrc& src, rg_mb_out& r) {
    static const int parts[9][9] = {{0, 0, 16, 16, 0, 0, 4, 0, 0}, {0, 0, 16, 8, 0, 0, 4, 1, 1}, {0, 8, 16, 8, 0, 2, 4, 2, 2},
                                    {0, 0, 8, 16, 0, 0, 2, 3, 3}, {8, 0, 8, 16, 2, 0, 2, 4, 4}, {0, 0, 8, 8, 0, 0, 2, 0, 5},
                                    {8, 0, 8, 8, 2, 0, 2, 0, 6}, {0, 8, 8, 8, 0, 2, 2, 0, 7}, {8, 8, 8, 8, 2, 2, 2, 0, 8}};
    static const int first[4] = {0, 1, 3, 5}, nparts[4] = {1, 2, 2, 4};
    static const int quads[9] = {15, 3, 12, 5, 10, 1, 2, 4, 8};
    int m = mby * mb_w + mbx, x0 = mbx * 16, y0 = mby * 16;
    int q_ = cur_qp, qpc = chroma_qp(q_, 0);
    uint32_t lambda = kLambda[q_];
    Bounds bd = mv_bounds(x0, y0);
    int imin[2] = {(bd.min[0] + 3) >> 2, (bd.min[1] + 3) >> 2}, imax[2] = {bd.max[0] >> 2, bd.max[1] >> 2};
    const int none[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
    int mvp16[2];
    mv_pred_s(mbx, mby, 0, 0, 4, 0, none, 0, mvp16);
    int ps[2] = {mvp16[0], mvp16[1]};
    {
      NbS A = nb4s(mbx, mby, -1, 0, none, 0), B = nb4s(mbx, mby, 0, -1, none, 0);
      if (mbx == 0 || mby == 0 || (A.ref == 0 && A.x == 0 && A.y == 0) || (B.ref == 0 && B.x == 0 && B.y == 0)) ps[0] = ps[1] = 0;
    }
    uint8_t py[256], pu[64], pv[64];
    // 1. skip probe (enc.rs:2906 try_p_skip)
    if (in_bounds(bd, ps[0], ps[1])) {
      mc_luma16(x0, y0, ps[0], ps[1], py);
      uint32_t s0 = sad(src.y, 16, py, 16, 16, 16);
      if (s0 < sb_probe) {
        bool luma_zero = s0 <= sb_luma || ssd(src.y, 16, py, 16, 16) <= sb_luma_ssd;
        if (!luma_zero) luma_zero = probe_skip_luma(src, py, q_);
        if (luma_zero) {
          mc_chroma8(mbx, mby, ps[0], ps[1], pu, pv);
          auto plane_zero = [&](const uint8_t* s8, const uint8_t* p8) {
            return sad(s8, 8, p8, 8, 8, 8) <= sb_chroma || ssd(s8, 8, p8, 8, 8) <= sb_chroma_ssd;
          };
          bool chroma_zero = plane_zero(src.u, pu) && plane_zero(src.v, pv);
          if (!chroma_zero) chroma_zero = probe_skip_chroma(src, pu, pv, qpc);
          if (chroma_zero) {
            int16_t p16[2] = {(int16_t)ps[0], (int16_t)ps[1]};
            code_skip(mbx, mby, p16, r);
            store_mb(mbx, mby, py, pu, pv);
            int qmv[4][2] = {{ps[0], ps[1]}, {ps[0], ps[1]}, {ps[0], ps[1]}, {ps[0], ps[1]}};
            set_parts(r, 255, qmv, none);
            mb_split[m] = 0;
            return;
          }
        }
      }
    }
    // 2. integer search
    const rg_mb_hint* h = form == 2 && hints ? &hints[m] : nullptr;
    int R = search_range;
    int fc[2] = {std::min(std::max((mvp16[0] + 2) >> 2, imin[0]), imax[0]), std::min(std::max((mvp16[1] + 2) >> 2, imin[1]), imax[1])};
    int lo[2] = {std::max(fc[0] - R, imin[0]), std::max(fc[1] - R, imin[1])};
    int hi[2] = {std::min(fc[0] + R, imax[0]), std::min(fc[1] + R, imax[1])};
    int part_mask = 15;
    if (h) {
      NbS A = nb4s(mbx, mby, -1, 0, none, 0), B = nb4s(mbx, mby, 0, -1, none, 0), C = nb4s(mbx, mby, 4, -1, none, 0);
      if (C.ref == -2) C = nb4s(mbx, mby, -1, -1, none, 0);
      const int cv[7][2] = {{mvp16[0] + h->mv_off[0], mvp16[1] + h->mv_off[1]}, {mvp16[0], mvp16[1]},
                            {h->mv_coarse[0], h->mv_coarse[1]}, {A.x, A.y}, {B.x, B.y}, {C.x, C.y}, {0, 0}};
      const bool use[7] = {true, true, (h->flags & 1) != 0, A.ref == 0, B.ref == 0, C.ref == 0, true};
      int lc[2] = {0, 0};
      uint32_t best = UINT32_MAX;
      for (int k = 0; k < 7; k++) {
        if (!use[k]) continue;
        int v[2];
        for (int c = 0; c < 2; c++) v[c] = std::min(std::max((cv[k][c] + 2) >> 2, imin[c]), imax[c]);
        uint32_t cost = sad(src.y, 16, refp.y.ptr(x0 + v[0], y0 + v[1]), refp.y.stride, 16, 16) +
                        mvd_cost(4 * v[0] - mvp16[0], lambda) + mvd_cost(4 * v[1] - mvp16[1], lambda);
        if (cost < best) { best = cost; lc[0] = v[0]; lc[1] = v[1]; }
      }
      for (int c = 0; c < 2; c++) {
        lo[c] = std::max(lc[c] - 2, imin[c]);
        hi[c] = std::min(lc[c] + 2, imax[c]);
      }
      part_mask = h->part_mask & 15;
      if (!part_mask) part_mask = 1;
    }
    int ibx[9], iby[9];
    int_search_s(x0, y0, src, lo[0], hi[0], lo[1], hi[1], mvp16, lambda, ibx, iby);
    if (h) {
      auto on_edge = [&]() {
        return (ibx[0] == lo[0] && lo[0] > imin[0]) || (ibx[0] == hi[0] && hi[0] < imax[0]) ||
               (iby[0] == lo[1] && lo[1] > imin[1]) || (iby[0] == hi[1] && hi[1] < imax[1]);
      };
      bool edge = on_edge();
      for (int it = 0; edge && it < walk; it++) {  // centre the window on its best again
        int cc[2] = {ibx[0], iby[0]};
        for (int c = 0; c < 2; c++) { lo[c] = std::max(cc[c] - 2, imin[c]); hi[c] = std::min(cc[c] + 2, imax[c]); }
        int_search_s(x0, y0, src, lo[0], hi[0], lo[1], hi[1], mvp16, lambda, ibx, iby);
        edge = on_edge();
      }
      if (edge) {
        for (int c = 0; c < 2; c++) { lo[c] = std::max(fc[c] - R, imin[c]); hi[c] = std::min(fc[c] + R, imax[c]); }
        int_search_s(x0, y0, src, lo[0], hi[0], lo[1], hi[1], mvp16, lambda, ibx, iby);
      }
    }
    // 3-4. refinement and the partition type
    int best_t = -1;
    uint32_t best_j = UINT32_MAX;
    int bmv[4][2] = {}, bmvd[4][2] = {};
    for (int t = 0; t < 4; t++) {
      if (!((part_mask >> t) & 1)) continue;
      int own[4][2] = {}, done = 0, pm[4][2] = {}, pd[4][2] = {};
      uint32_t J = lambda * (uint32_t)type_bits[t];
      for (int k = 0; k < nparts[t]; k++) {
        const int* g = parts[first[t] + k];
        int mvp[2], mv[2];
        mv_pred_s(mbx, mby, g[4], g[5], g[6], g[7], own, done, mvp);
        J += h ? refine_part_sad_s(x0, y0, src, bd, g[0], g[1], g[2], g[3], ibx[g[8]], iby[g[8]], mvp, lambda, mv)
               : refine_part_s(x0, y0, src, bd, g[0], g[1], g[2], g[3], ibx[g[8]], iby[g[8]], mvp, lambda, mv);
        pm[k][0] = mv[0]; pm[k][1] = mv[1];
        pd[k][0] = mv[0] - mvp[0]; pd[k][1] = mv[1] - mvp[1];
        for (int q = 0; q < 4; q++)
          if ((quads[first[t] + k] >> q) & 1) { own[q][0] = mv[0]; own[q][1] = mv[1]; }
        done |= quads[first[t] + k];
      }
      if (J < best_j) {
        best_j = J; best_t = t;
        memcpy(bmv, pm, sizeof pm);
        memcpy(bmvd, pd, sizeof pd);
      }
    }
    int qmv[4][2];
    for (int k = 0; k < nparts[best_t]; k++) {
      const int* g = parts[first[best_t] + k];
      for (int q = 0; q < 4; q++)
        if ((quads[first[best_t] + k] >> q) & 1) { qmv[q][0] = bmv[k][0]; qmv[q][1] = bmv[k][1]; }
      luma_mc(refp.y.ptr(x0 + g[0] + (bmv[k][0] >> 2), y0 + g[1] + (bmv[k][1] >> 2)), refp.y.stride, g[2], g[3],
              bmv[k][0] & 3, bmv[k][1] & 3, py + g[1] * 16 + g[0], 16);
    }
    // 5. intra 16x16 check (the plain form's rule)
    uint32_t inter_satd = satd16(src.y, 16, py, 16);
    if (inter_satd > 24 * lambda) {
      uint32_t i16c; int i16m;
      analyse_i16(mbx, mby, src, i16c, i16m);
      if (i16c + lambda * 8 < best_j) {
        code_i16(mbx, mby, src, i16m, r);
        set_parts(r, best_t, none, none);
        mb_split[m] = 0;
        return;
      }
    }
    // chroma per quadrant vector, residual, late skip
    for (int q = 0; q < 4; q++) {
      uint8_t tu[64], tv[64];
      mc_chroma8(mbx, mby, qmv[q][0], qmv[q][1], tu, tv);
      int ox = (q & 1) * 4, oy = (q >> 1) * 4;
      for (int yy = 0; yy < 4; yy++)
        for (int xx = 0; xx < 4; xx++) {
          pu[(oy + yy) * 8 + ox + xx] = tu[(oy + yy) * 8 + ox + xx];
          pv[(oy + yy) * 8 + ox + xx] = tv[(oy + yy) * 8 + ox + xx];
        }
    }
    int16_t q4[16][16];
    int cbp4 = quant_luma_inter(src.y, py, q_, q4);
    int cbpl = cbp4;
    bool use8 = false;
    int16_t q8[4][64];
    if (t8x8 && cabac && cbp4) {
      int cbp8 = quant_luma_8x8(src.y, py, q_, q8);
      int nnz4 = 0, nnz8 = 0;
      for (int b = 0; b < 16; b++) for (int i = 0; i < 16; i++) nnz4 += q4[b][i] != 0;
      for (int b = 0; b < 4; b++) for (int i = 0; i < 64; i++) nnz8 += q8[b][i] != 0;
      if (nnz8 <= nnz4) { use8 = true; cbpl = cbp8; }
    }
    Chroma c;
    quant_chroma(src, pu, pv, qpc, false, c);
    for (int p = 0; p < 2; p++) {
      bool anym = c.mask[p][0] | c.mask[p][1] | c.mask[p][2] | c.mask[p][3];
      if (anym && chroma_ac_score(c, p) < 7) {
        memset(c.ac[p], 0, sizeof c.ac[p]);
        memset(c.mask[p], 0, sizeof c.mask[p]);
        memset(c.raster[p], 0, sizeof c.raster[p]);
      }
    }
    int cbpc = chroma_cbp(c);
    if (best_t == 0 && cbpl == 0 && cbpc == 0 && bmv[0][0] == ps[0] && bmv[0][1] == ps[1]) {
      int16_t p16[2] = {(int16_t)ps[0], (int16_t)ps[1]};
      code_skip(mbx, mby, p16, r);
      store_mb(mbx, mby, py, pu, pv);
      set_parts(r, best_t, qmv, none);
      mb_split[m] = 0;
      return;
    }
    static const uint8_t types[4] = {RG_MB_P_L0_16X16, RG_MB_P_L0_16X8, RG_MB_P_L0_8X16, RG_MB_P_8X8};
    r.mb_type = types[best_t];
    r.mv[0] = (int16_t)bmv[0][0]; r.mv[1] = (int16_t)bmv[0][1];
    r.mvd[0] = (int16_t)bmvd[0][0]; r.mvd[1] = (int16_t)bmvd[0][1];
    r.cbp = (uint8_t)(cbpl | (cbpc << 4));
    bool t8flag = use8 && cbpl != 0;
    r.transform_8x8 = t8flag;
    uint16_t nzm = 0;
    if (use8) {
      for (int b = 0; b < 4; b++) {
        for (int i = 0; i < 64; i++) r.luma[b * 64 + i] = q8[b][kZigzag8[i]];
        if (cbpl & (1 << b)) nzm |= 0xF << (4 * b);
      }
    } else {
      for (int b = 0; b < 16; b++) {
        zigzag16(q4[b], r.luma + b * 16);
        for (int i = 0; i < 16; i++) if (q4[b][i]) nzm |= 1 << b;
      }
    }
    memcpy(r.chroma_dc, c.dc, sizeof c.dc);
    memcpy(r.chroma_ac, c.ac, sizeof c.ac);
    set_mb_state(m, false, cbpl, t8flag, nzm);
    if (use8) {
      for (int b = 0; b < 4; b++)
        if (cbpl & (1 << b)) {
          int32_t d[64];
          dequant8(q8[b], q_, d);
          idct8_add(py + (b >> 1) * 128 + (b & 1) * 8, 16, d);
        }
    } else {
      int32_t sc[16];
      dequant4_scale(q_, sc);
      for (int b = 0; b < 16; b++)
        if (cbpl & (1 << (b >> 2))) {
          int16_t blk[16];
          memcpy(blk, q4[b], 32);
          dequant_block(blk, sc);
          int bx, by; blk_xy(b, bx, by);
          add_idct4(py + by * 64 + bx * 4, 16, blk);
        }
    }
    recon_chroma(pu, pv, c, cbpc, qpc);
    fill_motion_q(mbx, mby, qmv);
    store_mb(mbx, mby, py, pu, pv);
    set_parts(r, best_t, qmv, bmvd);
  }

  // enc.rs:2234 encode_frame_body (fixed QP, Balanced); returns Annex-B bytes (CAVLC only).
  std::vector<uint8_t> encode(const uint8_t* Y, const uint8_t* U, const uint8_t* V, int sy, int suv) {
    int n = mb_w * mb_h, n4 = n * 16;
    uint32_t gop_idx = frame_count % (uint32_t)std::max(keyint, 1);
    is_idr = (frame_count % (uint32_t)keyint == 0) || !has_ref;
    uint32_t idr_pic_id = frame_count / (uint32_t)std::max(keyint, 1);
    // EncState::prepare
    tc_nnz.assign(n4, 0);
    tc_cnnz[0].assign(n * 4, 0); tc_cnnz[1].assign(n * 4, 0);
    intra4x4_modes.assign(n4, 2);
    nz16.assign(n, 0);
    mb_intra.assign(n, 0); mb_cbp_luma.assign(n, 0); mb_t8.assign(n, 0); mb_qp.assign(n, (uint8_t)qp); mb_skip.assign(n, 0);
    mb_split.assign(n, 0);
    for (auto& r : recs) memset(&r, 0, sizeof r);
    cur_qp = qp;
    skip_run = 0;
    skip_bounds(qp);

    BitWriter w;
    // slice header (h264.rs:1071)
    w.ue(0);
    w.ue(is_idr ? 7 : 5);
    w.ue(0);
    w.put(gop_idx & 15, 4);
    if (is_idr) w.ue(idr_pic_id);
    w.put((gop_idx * 2) & 63, 6);
    if (!is_idr) { w.bit(false); w.bit(false); }
    if (is_idr) { w.bit(false); w.bit(false); } else w.bit(false);
    if (cabac && !is_idr) w.ue(0);
    w.se(0);
    w.ue(qp == 0 ? 1 : 0);
    if (qp != 0) { w.se(0); w.se(0); }
    if (cabac) {  // enc.rs:2347: cabac_alignment_one_bits, contexts for this slice
      if (w.bits() & 7) w.put((1u << (8 - (w.bits() & 7))) - 1, 8 - (int)(w.bits() & 7));
      cabac_prepare();
    }

    for (int mby = 0; mby < mb_h; mby++)
      for (int mbx = 0; mbx < mb_w; mbx++) {
        MbSrc src;
        load_src(Y, U, V, sy, suv, mbx, mby, src);
        rg_mb_out& r = recs[mby * mb_w + mbx];
        r.qp = (uint8_t)qp;
        if (form) {  // search forms: decisions and reconstruction only (no bitstream)
          r.part_type = 255;
          if (is_idr) code_intra(mbx, mby, src, r);
          else code_p_mb_search(mbx, mby, src, r);
          continue;
        }
        if (is_idr) code_intra(mbx, mby, src, r);
        else code_p_mb(mbx, mby, src, r);
        if (!cabac) {
          write_mb_cavlc(w, mbx, mby, r);
        } else {
          write_mb_cabac(mbx, mby, r);
          ce.terminate(mby == mb_h - 1 && mbx == mb_w - 1);  // end_of_slice_flag (enc.rs:2430)
        }
      }
    std::vector<uint8_t> rbsp;
    if (form) {
      rbsp.clear();
    } else if (cabac) {
      rbsp = w.finish();
      rbsp.insert(rbsp.end(), ce.out.begin(), ce.out.end());
    } else {
      if (!is_idr && skip_run > 0) w.ue(skip_run);
      w.trailing();
      rbsp = w.finish();
    }

    for (int p = 0; p < 3; p++) {
      const Plane& pl = p == 0 ? cur.y : (p == 1 ? cur.u : cur.v);
      recon_unfiltered[p].resize((size_t)pl.w * pl.h);
      for (int y = 0; y < pl.h; y++) memcpy(&recon_unfiltered[p][(size_t)y * pl.w], pl.ptr(0, y), pl.w);
    }
    if (qp != 0) deblock();
    cur.y.extend_borders(); cur.u.extend_borders(); cur.v.extend_borders();
    std::swap(cur, refp);
    has_ref = true;
    int g = gstride();
    for (int mby = 0; mby < mb_h; mby++)
      for (int mbx = 0; mbx < mb_w; mbx++) {
        int i = (mby * 4) * g + mbx * 4;
        prev_mb_mv[2 * (mby * mb_w + mbx)] = mv_grid[2 * i];
        prev_mb_mv[2 * (mby * mb_w + mbx) + 1] = mv_grid[2 * i + 1];
      }
    frame_count++;
    std::vector<uint8_t> out;
    if (form) return out;
    if (is_idr) {
      append_nal(out, 3, 7, sps_rbsp());
      append_nal(out, 3, 8, pps_rbsp());
    }
    append_nal(out, 3, is_idr ? 5 : 1, rbsp);
    return out;
  }
};

}  // namespace oracle

// ---------------------------------------------------------------------------------------------
// C API for the tests (ctypes).
extern "C" {

void* oracle_enc_create(int width, int height, int profile, int qp, int keyint, int fps_num, int fps_den) {
  if (width <= 0 || height <= 0 || keyint <= 0) return nullptr;
  auto* e = new oracle::Encoder();
  e->init(width, height, profile, qp, keyint, fps_num, fps_den);
  return e;
}
void oracle_enc_destroy(void* h) { delete (oracle::Encoder*)h; }

// Encodes one frame. Writes mb_w*mb_h records (if recs) and Annex-B bytes (Baseline only).
// Returns the number of bitstream bytes (or -needed if cap is too small); *is_idr set.
long oracle_enc_frame(void* h, const uint8_t* y, const uint8_t* u, const uint8_t* v, int sy, int suv,
                      rg_mb_out* recs, uint8_t* bits, long cap, int* is_idr) {
  auto* e = (oracle::Encoder*)h;
  std::vector<uint8_t> out = e->encode(y, u, v, sy, suv);
  oracle::g_pixel_ops.fetch_add(oracle::t_pixel_ops, std::memory_order_relaxed);
  oracle::t_pixel_ops = 0;
  if (is_idr) *is_idr = e->is_idr ? 1 : 0;
  if (recs) memcpy(recs, e->recs.data(), e->recs.size() * sizeof(rg_mb_out));
  if ((long)out.size() > cap) return -(long)out.size();
  if (bits && !out.empty()) memcpy(bits, out.data(), out.size());
  return (long)out.size();
}
// Copies the latest reconstruction at coded size: filtered (deblocked) or before deblocking.
void oracle_enc_recon(void* h, uint8_t* y, uint8_t* u, uint8_t* v, int filtered) {
  auto* e = (oracle::Encoder*)h;
  const oracle::Pic& p = e->refp;
  uint8_t* dst[3] = {y, u, v};
  const oracle::Plane* pl[3] = {&p.y, &p.u, &p.v};
  for (int k = 0; k < 3; k++) {
    if (!dst[k]) continue;
    if (filtered) {
      for (int r = 0; r < pl[k]->h; r++) memcpy(dst[k] + (size_t)r * pl[k]->w, pl[k]->ptr(0, r), pl[k]->w);
    } else {
      memcpy(dst[k], e->recon_unfiltered[k].data(), e->recon_unfiltered[k].size());
    }
  }
}
void oracle_mb_dims(void* h, int* mb_w, int* mb_h) {
  auto* e = (oracle::Encoder*)h;
  *mb_w = e->mb_w; *mb_h = e->mb_h;
}
int oracle_record_size(void) { return (int)sizeof(rg_mb_out); }
// Search forms (1 full search, 2 learned) with the integer search range; the learned form reads the
// hints set for the next frame (mb_w * mb_h records, host memory, kept until the next call).
void oracle_enc_set_form(void* h, int form, int search_range) {
  auto* e = (oracle::Encoder*)h;
  e->form = form;
  e->search_range = search_range;
}
void oracle_enc_set_hints(void* h, const rg_mb_hint* hints) { ((oracle::Encoder*)h)->hints = hints; }
// The search forms' decision constants (rg_set_search_tuning).
void oracle_enc_set_search_tuning(void* h, const int* type_bits, int walk) {
  auto* e = (oracle::Encoder*)h;
  for (int k = 0; k < 4; k++) e->type_bits[k] = type_bits[k];
  e->walk = walk;
}
// Pixel differences evaluated by the SAD / SSD / SATD of every frame encoded so far in this
// process (all threads); reset = 1 also sets the total back to 0.
unsigned long long oracle_pixel_ops(int reset) {
  return reset ? oracle::g_pixel_ops.exchange(0) : oracle::g_pixel_ops.load();
}

// Kernels behind the reference's own property tests (crates/ragdoll-codec/src/h264/enc.rs:4119
// transform_8x8_paths_match_the_reference, :4189 decimation_scores_follow_x264), exposed so the
// tests can restate them against this oracle.
// decimate_score (enc.rs:559) of n = 16 or 64 levels in zig-zag order.
unsigned oracle_decimate_score(const int16_t* zz, int n) { return oracle::decimate_score(zz, n == 64 ? 64 : 16); }
// quant_luma_8x8_inter (enc.rs:2041) of a 16x16 source / prediction pair (stride 16): raster levels
// of the four 8x8 blocks into q8 (4 x 64), returns cbp8; fine = the intra rounding (f = 2^s / 3).
int oracle_quant_luma_8x8(const uint8_t* src, const uint8_t* pred, int qp, int fine, int16_t* q8) {
  return oracle::Encoder::quant_luma_8x8(src, pred, qp, (int16_t(*)[64])q8, fine != 0);
}
// recon_8x8 (enc.rs:2020): dequantises 64 raster levels (dequantize_block8x8, h264.rs:1403) and adds
// their inverse transform (h264_idct8_add, h264_idct.rs:207) onto dst (stride).
void oracle_recon_8x8(uint8_t* dst, int stride, const int16_t* levels, int qp) {
  int32_t d[64];
  oracle::dequant8(levels, qp, d);
  oracle::idct8_add(dst, stride, d);
}

}  // extern "C"
