// B200 (sm_100a) macroblock engine: one warp analyses, reconstructs or deblocks one macroblock.
//
// A picture is processed as a 2:1 wavefront over anti-diagonals d = mb_x + 2 mb_y: every
// macroblock of diagonal d depends only on macroblocks of smaller diagonals (left, top, top-left
// and top-right neighbours: unfiltered reconstruction for intra edges, motion for the median
// predictor), so one launch per diagonal reproduces the reference's raster-order decisions
// exactly. Deblocking of diagonal d runs in the launch of analysis diagonal d + 3: by then every
// macroblock that reads its unfiltered pixels (right, below, below-left, below-right neighbours)
// has been analysed, and the two touch disjoint samples. Streams (independent GOPs) sit side by
// side in blockIdx.y.
//
// Arithmetic follows ragdoll's Balanced encoder (crates/ragdoll-codec/src/h264/enc.rs) and the
// scalar kernels it calls (crates/ragdoll-simd/src/*.rs); citations are given per function.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>
#include <vector>

#include "engine.h"
#include "h264_consts.h"

namespace rg {

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr uint32_t UMAX = 0xffffffffu;

__constant__ uint16_t c_lambda[52];
__constant__ uint8_t c_dec4[16];
__constant__ uint8_t c_dec8[64];
__constant__ uint8_t c_scan4[16];
__constant__ uint8_t c_scan8[64];
__constant__ uint16_t c_mf4[6][3];
__constant__ uint8_t c_dq4[6][3];
__constant__ uint16_t c_mf8[6][6];
__constant__ uint8_t c_dq8[6][6];
__constant__ uint8_t c_cqp[52];
__constant__ uint8_t c_alpha[52];
__constant__ uint8_t c_beta[52];
__constant__ uint8_t c_tc0[52][3];

// ---------------------------------------------------------------------------------------------
// Shared memory of one macroblock warp.
struct __align__(16) Smem {
  uint8_t src_y[256];
  uint8_t src_u[64];
  uint8_t src_v[64];
  uint8_t pred_y[256];
  uint8_t pred_u[64];
  uint8_t pred_v[64];
  uint8_t tmp_y[256];       // plane prediction / I4x4 reconstruction
  uint8_t win[23 * 24];     // integer samples of a half-sample window (rows -2.., cols -2..)
  // The half-sample planes live until the sub-pel search ends; the 8x8 transform's intermediates
  // are needed only after it (the residual), so they share the space.
  union {
    struct {
      uint8_t hph[18 * 20];  // b samples (horizontal half)
      uint8_t hpv[18 * 20];  // h samples (vertical half)
      uint8_t hpj[18 * 20];  // j samples (centre)
      int16_t hr[23 * 18];   // unrounded horizontal 6-tap sums
    };
    int32_t t8[256];         // 8x8 transform intermediates
  };
  int16_t coef[256];        // luma 4x4 levels: block b (decoding order) at [16 b], raster
  int16_t coef8[256];       // luma 8x8 levels: block b at [64 b], raster
  int16_t ccoef[128];       // chroma levels: block (plane * 4 + b) at [16 *], raster
  int16_t cdcraw[8];
  int16_t cdc[8];
  int16_t ldc[16];          // I16x16 DC levels, raster
  int16_t ldcr[16];         // I16x16 DC reconstruction, raster
  uint8_t top[24];          // luma row above the macroblock (x0 .. x0 + 23)
  uint8_t left[16];
  uint8_t ctop[2][8];
  uint8_t cleft[2][8];
  uint8_t i4m[16];          // Intra4x4PredMode of this macroblock (decoding order)
  uint8_t i4q[16];          // edge samples of the current 4x4 block (i4_edge_index)
};
static_assert(offsetof(Smem, coef) % 4 == 0 && offsetof(Smem, ccoef) % 4 == 0, "level arrays cleared by words");
static_assert(offsetof(rg_mb_out, luma) % 4 == 0 && offsetof(rg_mb_out, chroma_dc) % 4 == 0 &&
                  offsetof(rg_mb_out, chroma_ac) % 4 == 0 && sizeof(rg_mb_out) % 4 == 0,
              "record levels written by words");
static_assert(offsetof(Smem, pred_y) % 8 == 0 && offsetof(Smem, tmp_y) % 8 == 0, "16x16 predictions written 8 bytes per lane");

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ MbInfo ld_info(const MbInfo* p) {
  int4 v = *(const int4*)p;
  MbInfo m;
  *(int4*)&m = v;
  return m;
}
__device__ __forceinline__ uint32_t wsum(uint32_t v) { return __reduce_add_sync(FULL, v); }
__device__ __forceinline__ uint32_t wor(uint32_t v) { return __reduce_or_sync(FULL, v); }
__device__ __forceinline__ int clip255(int v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }
__device__ __forceinline__ int16_t clamp_i16(int v) { return (int16_t)(v < -32768 ? -32768 : (v > 32767 ? 32767 : v)); }

// Column and row of 4x4 block b in decoding order (enc.rs:522 blk_xy).
__device__ __forceinline__ int blk_x(int b) { return (b & 1) + ((b >> 1) & 2); }
__device__ __forceinline__ int blk_y(int b) { return ((b >> 1) & 1) + ((b >> 2) & 2); }
// Position class of raster coefficient i in a 4x4 / 8x8 block (h264.rs:1204, :1343).
__device__ __forceinline__ int pos4(int i) {
  int r = i >> 2, c = i & 3;
  if (((r | c) & 1) == 0) return 0;
  return ((r & c) & 1) ? 1 : 2;
}
__device__ __forceinline__ int pos8(int i) {
  int r = (i >> 3) & 3, c = i & 3;
  if (r == 0 && c == 0) return 0;
  if ((r & 1) && (c & 1)) return 1;
  if (r == 2 && c == 2) return 2;
  if ((r == 0 && (c & 1)) || ((r & 1) && c == 0)) return 3;
  if ((r == 0 && c == 2) || (r == 2 && c == 0)) return 4;
  return 5;
}
__device__ __forceinline__ int chroma_qp(int qp) { return c_cqp[qp < 0 ? 0 : (qp > 51 ? 51 : qp)]; }
// Bits of se(v) (enc.rs:546).
__device__ __forceinline__ uint32_t se_bits(int d) {
  uint32_t v = (uint32_t)(d < 0 ? -d : d) * 2u - (d > 0 ? 1u : 0u);
  return 2u * (32u - (uint32_t)__clz(v + 1u)) - 1u;
}
__device__ __forceinline__ uint32_t mvd_cost(int d, uint32_t lambda) {
  uint32_t c = lambda * se_bits(d);
  return (d >= -4096 && d <= 4096) ? (c & 0xFFFFu) : c;
}

// Reconstructed pictures and macroblock state are produced by other warps of the same launch in
// the pipelined mode. They are read with plain (weak, coherent-path) loads -- never the
// non-coherent read-only path -- and only after an ld.acquire that observed the producer's
// release, which the memory model makes sufficient for the loads to see the produced values.
// Plain loads also let the compiler issue independent loads back to back.
__device__ __forceinline__ uint32_t ldw32(const void* p) { return *(const uint32_t*)p; }
__device__ __forceinline__ uint8_t ldcg_u8(const uint8_t* p) { return *p; }
__device__ __forceinline__ uint32_t ldcg_u32(const uint8_t* p) { return ldw32(p); }
__device__ __forceinline__ uint2 ldg8(const uint8_t* p) {
  uintptr_t a = (uintptr_t)p;
  const uint32_t* b = (const uint32_t*)(a & ~(uintptr_t)3);
  uint32_t sh = (uint32_t)(a & 3) * 8u;
  uint32_t w0 = b[0], w1 = b[1], w2 = b[2];
  return make_uint2(__funnelshift_r(w0, w1, sh), __funnelshift_r(w1, w2, sh));
}
__device__ __forceinline__ uint32_t vsad8(uint2 a, uint2 b) { return __vsadu4(a.x, b.x) + __vsadu4(a.y, b.y); }

// ---------------------------------------------------------------------------------------------
// Per-lane transforms (crates/ragdoll-simd/src/fixed.rs:104,192,322; h264_idct.rs:225)
__device__ __forceinline__ void fdct4(const int* d, int* o) {
  int t[16];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    int s03 = d[r * 4] + d[r * 4 + 3], s12 = d[r * 4 + 1] + d[r * 4 + 2];
    int d03 = d[r * 4] - d[r * 4 + 3], d12 = d[r * 4 + 1] - d[r * 4 + 2];
    t[r * 4] = s03 + s12; t[r * 4 + 1] = 2 * d03 + d12; t[r * 4 + 2] = s03 - s12; t[r * 4 + 3] = d03 - 2 * d12;
  }
#pragma unroll
  for (int c = 0; c < 4; c++) {
    int s03 = t[c] + t[c + 12], s12 = t[c + 4] + t[c + 8], d03 = t[c] - t[c + 12], d12 = t[c + 4] - t[c + 8];
    o[c] = (int16_t)(s03 + s12); o[c + 4] = (int16_t)(2 * d03 + d12);
    o[c + 8] = (int16_t)(s03 - s12); o[c + 12] = (int16_t)(d03 - 2 * d12);
  }
}
__device__ __forceinline__ void idct4(const int* c, int* o) {
  int t[16];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    int e0 = c[r * 4] + c[r * 4 + 2], e1 = c[r * 4] - c[r * 4 + 2];
    int e2 = (c[r * 4 + 1] >> 1) - c[r * 4 + 3], e3 = c[r * 4 + 1] + (c[r * 4 + 3] >> 1);
    t[r * 4] = e0 + e3; t[r * 4 + 1] = e1 + e2; t[r * 4 + 2] = e1 - e2; t[r * 4 + 3] = e0 - e3;
  }
#pragma unroll
  for (int k = 0; k < 4; k++) {
    int e0 = t[k] + t[k + 8], e1 = t[k] - t[k + 8];
    int e2 = (t[k + 4] >> 1) - t[k + 12], e3 = t[k + 4] + (t[k + 12] >> 1);
    o[k] = (int16_t)((e0 + e3 + 32) >> 6); o[k + 4] = (int16_t)((e1 + e2 + 32) >> 6);
    o[k + 8] = (int16_t)((e1 - e2 + 32) >> 6); o[k + 12] = (int16_t)((e0 - e3 + 32) >> 6);
  }
}
// One row / column of the 8x8 forward transform (fixed.rs:392).
__device__ __forceinline__ void fdct8_1d(const int* a, int* o) {
  int a0 = a[0] + a[7], a1 = a[1] + a[6], a2 = a[2] + a[5], a3 = a[3] + a[4];
  int a4 = a[0] - a[7], a5 = a[1] - a[6], a6 = a[2] - a[5], a7 = a[3] - a[4];
  int b0 = a0 + a3, b1 = a1 + a2, b2 = a0 - a3, b3 = a1 - a2;
  int b4 = a5 + a6 + ((a4 >> 1) + a4), b5 = a4 - a7 - ((a6 >> 1) + a6);
  int b6 = a4 + a7 - ((a5 >> 1) + a5), b7 = a5 - a6 + ((a7 >> 1) + a7);
  o[0] = b0 + b1; o[1] = b4 + (b7 >> 2); o[2] = b2 + (b3 >> 1); o[3] = b5 + (b6 >> 2);
  o[4] = b0 - b1; o[5] = b6 - (b5 >> 2); o[6] = (b2 >> 1) - b3; o[7] = (b4 >> 2) - b7;
}
// The 1-D inverse 8x8 transform in wrapping 32-bit arithmetic (h264_idct.rs:225).
__device__ __forceinline__ void idct8_1d(const int* d, int* o) {
  unsigned a0 = (unsigned)d[0] + (unsigned)d[4];
  unsigned a1 = (unsigned)d[5] - (unsigned)d[3] - (unsigned)d[7] - (unsigned)(d[7] >> 1);
  unsigned a2 = (unsigned)d[0] - (unsigned)d[4];
  unsigned a3 = (unsigned)d[1] + (unsigned)d[7] - (unsigned)d[3] - (unsigned)(d[3] >> 1);
  unsigned a4 = (unsigned)(d[2] >> 1) - (unsigned)d[6];
  unsigned a5 = (unsigned)d[7] - (unsigned)d[1] + (unsigned)d[5] + (unsigned)(d[5] >> 1);
  unsigned a6 = (unsigned)d[2] + (unsigned)(d[6] >> 1);
  unsigned a7 = (unsigned)d[3] + (unsigned)d[5] + (unsigned)d[1] + (unsigned)(d[1] >> 1);
  unsigned b0 = a0 + a6, b1 = a1 + (unsigned)((int)a7 >> 2), b2 = a2 + a4, b3 = a3 + (unsigned)((int)a5 >> 2);
  unsigned b4 = a2 - a4, b5 = (unsigned)((int)a3 >> 2) - a5, b6 = a0 - a6, b7 = a7 - (unsigned)((int)a1 >> 2);
  o[0] = (int)(b0 + b7); o[1] = (int)(b2 + b5); o[2] = (int)(b4 + b3); o[3] = (int)(b6 + b1);
  o[4] = (int)(b6 - b1); o[5] = (int)(b4 - b3); o[6] = (int)(b2 - b5); o[7] = (int)(b0 - b7);
}
// SATD of a 4x4 block (metrics.rs:705, halved).
__device__ __noinline__ uint32_t satd4(const uint8_t* a, int sa, const uint8_t* b, int sb) {
  int t[4][4];
#pragma unroll
  for (int y = 0; y < 4; y++) {
    int d0 = a[y * sa] - b[y * sb], d1 = a[y * sa + 1] - b[y * sb + 1];
    int d2 = a[y * sa + 2] - b[y * sb + 2], d3 = a[y * sa + 3] - b[y * sb + 3];
    int s03 = d0 + d3, s12 = d1 + d2, d03 = d0 - d3, d12 = d1 - d2;
    t[y][0] = s03 + s12; t[y][1] = d03 + d12; t[y][2] = s03 - s12; t[y][3] = d03 - d12;
  }
  uint32_t s = 0;
#pragma unroll
  for (int x = 0; x < 4; x++) {
    int s03 = t[0][x] + t[3][x], s12 = t[1][x] + t[2][x], d03 = t[0][x] - t[3][x], d12 = t[1][x] - t[2][x];
    s += abs(s03 + s12) + abs(d03 + d12) + abs(s03 - s12) + abs(d03 - d12);
  }
  return s;  // caller halves the sum of the blocks
}

// One pass of the 4x4 forward core transform along the axis whose lanes are `step` apart in a
// 16-lane group (i = position along it): [1 1 1 1; 2 1 -1 -2; 1 -1 -1 1; 1 -2 2 -1].
__device__ __forceinline__ int fwd4_pass(int v, int step, int i) {
  int b = __shfl_xor_sync(FULL, v, 3 * step);
  int s = v + b, dd = v - b;
  int ps = __shfl_xor_sync(FULL, s, step), pd = __shfl_xor_sync(FULL, dd, step);
  return i == 0 ? s + ps : (i == 1 ? 2 * pd + dd : (i == 2 ? ps - s : 2 * pd - dd));
}
// One pass of the inverse core transform (fixed.rs:192): e0 = c0 + c2, e1 = c0 - c2,
// e2 = (c1 >> 1) - c3, e3 = c1 + (c3 >> 1); out = e0 + e3, e1 + e2, e1 - e2, e0 - e3.
__device__ __forceinline__ int inv4_pass(int v, int step, int i) {
  int b = __shfl_xor_sync(FULL, v, 2 * step);
  int ea, eb;
  if (i == 0) { ea = v + b; eb = v - b; }
  else if (i == 2) { ea = b + v; eb = b - v; }
  else if (i == 1) { ea = (v >> 1) - b; eb = v + (b >> 1); }
  else { ea = (b >> 1) - v; eb = b + (v >> 1); }
  int pa = __shfl_xor_sync(FULL, ea, step), pb = __shfl_xor_sync(FULL, eb, step);
  return i == 0 ? ea + pb : (i == 1 ? pb + ea : (i == 2 ? eb - pa : pa - eb));
}

// ---------------------------------------------------------------------------------------------
// Half-sample window (h264_enc.rs:747 hpel_window, :803 hpel_window_centre): integer origin
// (ox, oy); plane coordinate (r, c) is the sample at (ox + c, oy + r).
__device__ __noinline__ void stage_window(const uint8_t* ref, int stride, int ox, int oy, Smem& sm) {
  int lane = lane_id();
  // 23 rows x 6 words: five words per lane, all loads issued before the first use
  uint32_t lo[5], hi[5], sh[5];
#pragma unroll
  for (int r = 0; r < 5; r++) {
    int q = min(lane + 32 * r, 23 * 6 - 1);
    int k = q / 6, w = q - 6 * (q / 6);
    uintptr_t a = (uintptr_t)(ref + (long)(oy - 2 + k) * stride + (ox - 2) + 4 * w);
    const uint32_t* b = (const uint32_t*)(a & ~(uintptr_t)3);
    sh[r] = (uint32_t)(a & 3) * 8u;
    lo[r] = b[0];
    hi[r] = b[1];
  }
#pragma unroll
  for (int r = 0; r < 5; r++) {
    int q = lane + 32 * r;
    if (q < 23 * 6) {
      int k = q / 6, w = q - 6 * (q / 6);
      *(uint32_t*)&sm.win[k * 24 + 4 * w] = __funnelshift_r(lo[r], hi[r], sh[r]);
    }
  }
  __syncwarp();
}
// need: bit 0 b plane (h), bit 1 h plane (v), bit 2 j plane (c)
__device__ __noinline__ void build_hpel(Smem& sm, int need) {
  int lane = lane_id();
  if (need & 5) {
    for (int i = lane; i < 23 * 18; i += 32) {
      int k = i / 18, c = i - k * 18;
      const uint8_t* w = &sm.win[k * 24 + c];
      sm.hr[i] = (int16_t)(w[0] - 5 * w[1] + 20 * w[2] + 20 * w[3] - 5 * w[4] + w[5]);
    }
  }
  __syncwarp();
  for (int i = lane; i < 18 * 18; i += 32) {
    int r = i / 18, c = i - r * 18;
    if (need & 1) sm.hph[r * 20 + c] = (uint8_t)clip255((sm.hr[(r + 2) * 18 + c] + 16) >> 5);
    if (need & 2) {
      const uint8_t* w = &sm.win[r * 24 + c + 2];
      int v = w[0] - 5 * w[24] + 20 * w[48] + 20 * w[72] - 5 * w[96] + w[120];
      sm.hpv[r * 20 + c] = (uint8_t)clip255((v + 16) >> 5);
    }
    if (need & 4) {
      const int16_t* t = &sm.hr[r * 18 + c];
      int j = t[0] - 5 * t[18] + 20 * t[36] + 20 * t[54] - 5 * t[72] + t[90];
      sm.hpj[r * 20 + c] = (uint8_t)clip255((j + 512) >> 10);
    }
  }
  __syncwarp();
}
// Planes a vector with fractional part (fx, fy) reads (window_src, enc.rs:1395).
__device__ __forceinline__ int planes_needed(int fx, int fy) {
  if ((fx | fy) == 0) return 0;
  if (fy == 0) return 1;
  if (fx == 0) return 2;
  if (fx == 2 && fy == 2) return 4;
  if (fx == 2) return 5;
  if (fy == 2) return 6;
  return 3;
}
// Quarter-sample prediction of the 16x16 block whose integer position is (wx, wy) in window
// coordinates: one window plane, or the rounded average of two (window_src, enc.rs:1395; equal
// to h264_luma_mc_scalar, h264_mc.rs:148, by enc.rs:4030). Returns the two source rows' bases.
struct QSrc {
  const uint8_t* a;
  const uint8_t* b;
  int sa, sb, avg;
};
__device__ __noinline__ QSrc qpel_src(const Smem& sm, int wx, int wy, int fx, int fy) {
  const uint8_t* G = &sm.win[(wy + 2) * 24 + wx + 2];
  const uint8_t* B = &sm.hph[wy * 20 + wx];
  const uint8_t* V = &sm.hpv[wy * 20 + wx];
  const uint8_t* J = &sm.hpj[wy * 20 + wx];
  switch (fx | (fy << 2)) {
    case 0: return {G, G, 24, 24, 0};
    case 1: return {G, B, 24, 20, 1};
    case 2: return {B, B, 20, 20, 0};
    case 3: return {B, G + 1, 20, 24, 1};
    case 4: return {G, V, 24, 20, 1};
    case 5: return {B, V, 20, 20, 1};
    case 6: return {B, J, 20, 20, 1};
    case 7: return {B, V + 1, 20, 20, 1};
    case 8: return {V, V, 20, 20, 0};
    case 9: return {V, J, 20, 20, 1};
    case 10: return {J, J, 20, 20, 0};
    case 11: return {J, V + 1, 20, 20, 1};
    case 12: return {V, G + 24, 20, 24, 1};
    case 13: return {V, B + 20, 20, 20, 1};
    case 14: return {J, B + 20, 20, 20, 1};
    default: return {V + 1, B + 20, 20, 20, 1};
  }
}
// 8 bytes of shared memory at any alignment (rows of the window planes are 4-byte aligned).
__device__ __forceinline__ uint2 lds8(const uint8_t* p) {
  uintptr_t a = (uintptr_t)p;
  const uint32_t* b = (const uint32_t*)(a & ~(uintptr_t)3);
  uint32_t sh = (uint32_t)(a & 3) * 8u;
  uint32_t w0 = b[0], w1 = b[1], w2 = b[2];
  return make_uint2(__funnelshift_r(w0, w1, sh), __funnelshift_r(w1, w2, sh));
}
// This lane's 8 prediction samples (row lane/2, columns 8 (lane&1) ..) packed in two words.
__device__ __forceinline__ uint2 qpel8(const QSrc& q) {
  int lane = lane_id(), i = lane >> 1, j0 = (lane & 1) * 8;
  uint2 a = lds8(q.a + i * q.sa + j0);
  if (!q.avg) return a;
  uint2 b = lds8(q.b + i * q.sb + j0);
  return make_uint2(__vavgu4(a.x, b.x), __vavgu4(a.y, b.y));
}
// Cost of a full-pel position (mx, my): the warp's SAD of the 16x16 block (this lane's 8 source
// samples sv against its 8 reference samples r) plus lambda * bits of the vector difference to
// the predictor (enc.rs:1207 cost). Shared by the candidates and the diamond steps.
__device__ __noinline__ uint32_t fullpel_cost(uint2 sv, uint2 r, int mx, int my, int mvp0, int mvp1, uint32_t lambda) {
  return wsum(vsad8(sv, r)) + mvd_cost(mx * 4 - mvp0, lambda) + mvd_cost(my * 4 - mvp1, lambda);
}
// This lane's SAD against the quarter-sample prediction at window position (wx, wy), phase
// (fx, fy): shared by the candidates of the sub-pel search.
__device__ __noinline__ uint32_t qpel_sad(const Smem& sm, uint2 sv, int wx, int wy, int fx, int fy) {
  return vsad8(sv, qpel8(qpel_src(sm, wx, wy, fx, fy)));
}
__device__ __forceinline__ uint2 src8(const Smem& sm) {
  int lane = lane_id();
  return *(const uint2*)&sm.src_y[(lane >> 1) * 16 + (lane & 1) * 8];
}
// Prediction of the 16x16 block displaced by mv into pred_y (enc.rs:1058 mc_luma).
__device__ __noinline__ void mc_luma16(const uint8_t* ref, int stride, int x0, int y0, int mvx, int mvy, Smem& sm) {
  int ix = x0 + (mvx >> 2), iy = y0 + (mvy >> 2), fx = mvx & 3, fy = mvy & 3;
  int lane = lane_id();
  if ((fx | fy) == 0) {
    uint2 v = ldg8(ref + (long)(iy + (lane >> 1)) * stride + ix + (lane & 1) * 8);
    *(uint2*)&sm.pred_y[(lane >> 1) * 16 + (lane & 1) * 8] = v;
    __syncwarp();
    return;
  }
  stage_window(ref, stride, ix, iy, sm);
  build_hpel(sm, planes_needed(fx, fy));
  uint2 v = qpel8(qpel_src(sm, 0, 0, fx, fy));
  *(uint2*)&sm.pred_y[(lane >> 1) * 16 + (lane & 1) * 8] = v;
  __syncwarp();
}
// Chroma prediction of both planes (h264_enc.rs:1279 chroma_mc_8x8_x2_scalar; enc.rs:1082).
__device__ __noinline__ void mc_chroma8(const uint8_t* ru, const uint8_t* rv, int stride, int mbx, int mby, int mvx, int mvy, Smem& sm) {
  int lane = lane_id();
  int cx = mbx * 8 + (mvx >> 3), cy = mby * 8 + (mvy >> 3), fx = mvx & 7, fy = mvy & 7;
  int wa = (8 - fx) * (8 - fy), wb = fx * (8 - fy), wc = (8 - fx) * fy, wd = fx * fy;
  int plane = lane >> 4, idx = (lane & 15) * 4, r = idx >> 3, c0 = idx & 7;
  const uint8_t* src = (plane ? rv : ru) + (long)(cy + r) * stride + cx + c0;
  uint8_t* out = (plane ? sm.pred_v : sm.pred_u) + r * 8 + c0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    int a = ldcg_u8(src + k), b = ldcg_u8(src + k + 1), cc = ldcg_u8(src + stride + k), d = ldcg_u8(src + stride + k + 1);
    out[k] = (uint8_t)((wa * a + wb * b + wc * cc + wd * d + 32) >> 6);
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------------------------
// Quantisation helpers (enc.rs:1703-1779, h264_enc.rs:408)
__device__ __forceinline__ void quant4_params(int qp, bool intra, uint32_t& shift, uint32_t& bias) {
  shift = 15 + qp / 6;
  bias = (1u << shift) / (intra ? 3u : 6u);
}
__device__ __forceinline__ int quant_level(int c, uint32_t mf, uint32_t bias, uint32_t shift) {
  uint32_t a = (uint32_t)(c < 0 ? -c : c);
  uint64_t l = ((uint64_t)a * mf + bias) >> shift;
  if (l > 32767) l = 32767;
  return c < 0 ? -(int)l : (int)l;
}

// Zig-zag index of each raster position of a 4x4 block, 4 bits per position (inverse of the
// frame scan, Table 8-12).
constexpr unsigned long long kZigzagIndex4 = 0xfea9db83c7426510ull;

// Forward 4x4 core transform (fixed.rs:104, int16 output) and quantisation of `nblocks` 4x4
// residual blocks (src - pred): luma blocks in decoding order (chroma = false) or the eight chroma
// blocks, U then V (chroma = true). Lane = coefficient (raster p = lane & 15); half-warp h takes
// block 2 it + h, two blocks per step. Levels go to out[16 b + p]; the raw DC of each block to
// dc_raw[b] when given. Lane b then holds block b's: any level (among zig-zag indices >= first),
// any |level| > 1 (same), and the decimation score of its zig-zag levels from index `first`
// (enc.rs:559 decimate_score without its |level| > 1 rule; the caller applies it).
__device__ __noinline__ void quant4x4_blocks(Smem& sm, bool chroma, int nblocks, int first, int qp, uint32_t shift,
                                             uint32_t bias, int16_t* out, int16_t* dc_raw, int& my_nz, int& my_big,
                                             int& my_score) {
  int lane = lane_id(), p = lane & 15, h = lane >> 4, xl = p & 3, yl = p >> 2;
  int zi = (int)((kZigzagIndex4 >> (4 * p)) & 15);
  uint32_t mf = c_mf4[qp % 6][pos4(p)];
  bool counted = zi >= first;
  my_nz = my_big = my_score = 0;
#pragma unroll 1
  for (int it = 0; it < nblocks / 2; it++) {
    int b = 2 * it + h;
    const uint8_t *s, *pr;
    int stride;
    if (chroma) {
      int off = ((b & 3) >> 1) * 32 + (b & 1) * 4;
      s = ((b >> 2) ? sm.src_v : sm.src_u) + off;
      pr = ((b >> 2) ? sm.pred_v : sm.pred_u) + off;
      stride = 8;
    } else {
      int off = blk_y(b) * 64 + blk_x(b) * 4;
      s = sm.src_y + off;
      pr = sm.pred_y + off;
      stride = 16;
    }
    int d = (int)s[yl * stride + xl] - (int)pr[yl * stride + xl];
    int c = (int16_t)fwd4_pass(fwd4_pass(d, 1, xl), 4, yl);
    if (dc_raw && p == 0) dc_raw[b] = (int16_t)c;
    int l = quant_level(c, mf, bias, shift);
    out[b * 16 + p] = (int16_t)l;
    bool nz = l != 0 && counted;
    uint32_t nzm = __ballot_sync(FULL, nz);
    uint32_t bigm = __ballot_sync(FULL, nz && (l > 1 || l < -1));
    uint32_t zm = __reduce_or_sync(FULL, nz ? 1u << (zi + 16 * h) : 0u);
    uint32_t mine = (zm >> (16 * h)) & 0xffffu;
    uint32_t contrib = 0;
    if ((mine >> p) & 1u) {  // this lane as zig-zag index p: the run of zeros below it
      uint32_t below = mine & ((1u << p) - 1u);
      int prev = below ? 31 - __clz(below) : first - 1;
      int run = p - prev - 1;
      contrib = run == 0 ? 3u : (run <= 2 ? 2u : (run <= 5 ? 1u : 0u));
    }
    uint32_t sc = __reduce_add_sync(FULL, contrib << (16 * h));
    if (lane == 2 * it || lane == 2 * it + 1) {
      int k = lane & 1;
      my_nz = ((nzm >> (16 * k)) & 0xffffu) != 0;
      my_big = ((bigm >> (16 * k)) & 0xffffu) != 0;
      my_score = (int)((sc >> (16 * k)) & 0xffffu);
    }
  }
  __syncwarp();
}

// Luma 4x4 residual of pred_y, quantised (inter) and decimated into sm.coef
// (enc.rs:1810 quant_luma_4x4_inter). Returns cbp; lanes 0..15 report block lane's "any level".
__device__ __noinline__ int luma4x4_inter(int qp, Smem& sm, uint32_t* nz_lane_out) {
  int lane = lane_id();
  uint32_t shift, bias;
  quant4_params(qp, false, shift, bias);
  int my_nz, my_big, my_score;
  quant4x4_blocks(sm, false, 16, 0, qp, shift, bias, sm.coef, nullptr, my_nz, my_big, my_score);
  // per-8x8 aggregates (lanes 4g..4g+3)
  int g_nz = my_nz | __shfl_xor_sync(FULL, my_nz, 1);
  g_nz |= __shfl_xor_sync(FULL, g_nz, 2);
  int g_big = my_big | __shfl_xor_sync(FULL, my_big, 1);
  g_big |= __shfl_xor_sync(FULL, g_big, 2);
  uint32_t g_sc = my_score + __shfl_xor_sync(FULL, my_score, 1);
  g_sc += __shfl_xor_sync(FULL, g_sc, 2);
  int cbp = 0;
  uint32_t total = 0;
#pragma unroll
  for (int g = 0; g < 4; g++) {
    int nz = __shfl_sync(FULL, g_nz, 4 * g), big = __shfl_sync(FULL, g_big, 4 * g);
    uint32_t sc = __shfl_sync(FULL, g_sc, 4 * g);
    if (!nz) continue;
    if (big) { cbp |= 1 << g; total += 9; continue; }
    if (sc >= 4) cbp |= 1 << g;
    total += sc;
  }
  if (total < 6 && cbp) cbp = 0;
  // clear the levels of dropped 8x8 groups: word lane + 32 k of sm.coef lies in group k
#pragma unroll
  for (int k = 0; k < 4; k++)
    if (!((cbp >> k) & 1)) ((uint32_t*)sm.coef)[lane + 32 * k] = 0u;
  __syncwarp();
  if (nz_lane_out) *nz_lane_out = (lane < 16 && ((cbp >> (lane >> 2)) & 1)) ? (uint32_t)my_nz : 0u;
  return cbp;
}

// The 1-D forward 8x8 transform in place on p[0], p[stride], ..., p[7 * stride] (row and column
// passes share it).
__device__ __noinline__ void fdct8_inplace(int* p, int stride) {
  int a[8], o[8];
#pragma unroll
  for (int k = 0; k < 8; k++) a[k] = p[k * stride];
  fdct8_1d(a, o);
#pragma unroll
  for (int k = 0; k < 8; k++) p[k * stride] = o[k];
}

// Zig-zag index of (row y, column x) of an 8x8 block (frame scan, Table 8-13): diagonal s = x + y,
// walked up-right on even s and down-left on odd s.
__device__ __forceinline__ int zigzag8(int y, int x) {
  int s = x + y;
  if (s < 8) return s * (s + 1) / 2 + ((s & 1) ? y : x);
  return 64 - (16 - s) * (15 - s) / 2 + ((s & 1) ? 7 - x : 7 - y);
}

// Luma 8x8 residual of pred_y, quantised (inter) and decimated into sm.coef8
// (enc.rs:2041 quant_luma_8x8_inter). Lanes 8b..8b+7 own block b: a row each in the first pass,
// column q each in the second. The decimation score of a block comes from the bitmask of its
// nonzero zig-zag positions (run of zeros below each, weights 3 / 2 / 1 / 0 for runs of
// 0-3 / 4-11 / 12-23 / longer, enc.rs:559 with the 8x8 table). Returns cbp; *nnz8 = count.
__device__ __noinline__ int luma8x8_inter(int qp, Smem& sm, uint32_t* nnz8) {
  int lane = lane_id();
  int b = lane >> 3, q = lane & 7;
  int bx = (b & 1) * 8, by = (b >> 1) * 8;
  uint32_t shift = 16 + qp / 6, bias = (1u << shift) / 6u;
  // residual of row q, then the row pass and (after all rows) the column pass in place
#pragma unroll 1
  for (int x = 0; x < 8; x++) {
    int off = (by + q) * 16 + bx + x;
    sm.t8[b * 64 + q * 8 + x] = (int)sm.src_y[off] - (int)sm.pred_y[off];
  }
  fdct8_inplace(&sm.t8[b * 64 + q * 8], 1);
  __syncwarp();
  uint32_t mf6[6];
#pragma unroll
  for (int k = 0; k < 6; k++) mf6[k] = c_mf8[qp % 6][k];
  int any = 0, big = 0;
  unsigned long long zmask = 0;
  fdct8_inplace(&sm.t8[b * 64 + q], 8);  // column q; then quantisation row by row
#pragma unroll 1
  for (int y = 0; y < 8; y++) {
    int i = y * 8 + q, cls = pos8(i);
    uint32_t mf = cls == 0 ? mf6[0] : cls == 1 ? mf6[1] : cls == 2 ? mf6[2] : cls == 3 ? mf6[3] : cls == 4 ? mf6[4] : mf6[5];
    int l = quant_level((int16_t)sm.t8[b * 64 + i], mf, bias, shift);
    sm.coef8[b * 64 + i] = (int16_t)l;
    any |= l != 0;
    big |= l > 1 || l < -1;
    if (l) zmask |= 1ull << zigzag8(y, q);
  }
#pragma unroll
  for (int o = 1; o < 8; o <<= 1) {
    any |= __shfl_xor_sync(FULL, any, o);
    big |= __shfl_xor_sync(FULL, big, o);
    zmask |= __shfl_xor_sync(FULL, zmask, o);
  }
  // lane q scores zig-zag positions 8q .. 8q + 7
  uint32_t part = 0;
#pragma unroll 1
  for (int k = 0; k < 8; k++) {
    int z = 8 * q + k;
    if ((zmask >> z) & 1ull) {
      unsigned long long below = zmask & ((1ull << z) - 1ull);
      int run = z - (below ? 63 - __clzll((long long)below) : -1) - 1;
      part += run < 4 ? 3u : (run < 12 ? 2u : (run < 24 ? 1u : 0u));
    }
  }
#pragma unroll
  for (int o = 1; o < 8; o <<= 1) part += __shfl_xor_sync(FULL, part, o);
  uint32_t score = !any ? 0u : (big ? 9u : part);
  int cbp = 0;
  uint32_t total = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    uint32_t s = __shfl_sync(FULL, score, 8 * k);
    total += s;
    if (s >= 4) cbp |= 1 << k;
  }
  if (total < 6 && cbp) cbp = 0;
  uint32_t cnt = 0;
  if (!((cbp >> b) & 1)) {
#pragma unroll
    for (int y = 0; y < 8; y++) sm.coef8[b * 64 + y * 8 + q] = 0;
  } else {
    cnt = __popcll(zmask) * (q == 0);
  }
  __syncwarp();
  *nnz8 = wsum(cnt);
  return cbp;
}

// Chroma residual of pred_u/pred_v (enc.rs:1899 quant_chroma): lanes 0..7 own block
// (plane = lane / 4, b = lane % 4). Levels into sm.ccoef (raster), DC levels into sm.cdc.
// Outputs per plane: AC present and AC decimation score. Lanes 0..31 all return the values.
__device__ __noinline__ void chroma_quant(int qpc, bool intra, Smem& sm, uint32_t ac_any[2], uint32_t ac_score[2]) {
  int lane = lane_id();
  uint32_t shift, bias;
  quant4_params(qpc, intra, shift, bias);
  int ac, big, sc;
  quant4x4_blocks(sm, true, 8, 1, qpc, shift, bias, sm.ccoef, sm.cdcraw, ac, big, sc);
  uint32_t my_ac = lane < 8 ? (uint32_t)ac : 0u;
  uint32_t my_score = lane < 8 ? (big ? 9u : (uint32_t)sc) : 0u;  // decimate_score's |level| > 1 rule
  __syncwarp();
  // 2x2 DC transform + quantisation (enc.rs:1938 quant_chroma_dc; f = 2^qbits / 3 always)
  if (lane == 0 || lane == 4) {
    int d0 = sm.cdcraw[lane], d1 = sm.cdcraw[lane + 1], d2 = sm.cdcraw[lane + 2], d3 = sm.cdcraw[lane + 3];
    int had[4] = {d0 + d1 + d2 + d3, d0 - d1 + d2 - d3, d0 + d1 - d2 - d3, d0 - d1 - d2 + d3};
    int qbits = 16 + qpc / 6, mf = c_mf4[qpc % 6][0], f = (1 << qbits) / 3;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      int a = had[i] < 0 ? -had[i] : had[i];
      int l = (a * mf + f) >> qbits;
      sm.cdc[lane + i] = (int16_t)(had[i] < 0 ? -l : l);
    }
  }
  uint32_t pa = my_ac | __shfl_xor_sync(FULL, my_ac, 1);
  pa |= __shfl_xor_sync(FULL, pa, 2);
  uint32_t ps = my_score + __shfl_xor_sync(FULL, my_score, 1);
  ps += __shfl_xor_sync(FULL, ps, 2);
  ac_any[0] = __shfl_sync(FULL, pa, 0);
  ac_any[1] = __shfl_sync(FULL, pa, 4);
  ac_score[0] = __shfl_sync(FULL, ps, 0);
  ac_score[1] = __shfl_sync(FULL, ps, 4);
  __syncwarp();
}
__device__ __forceinline__ bool chroma_dc_any(const Smem& sm) {
  bool a = false;
#pragma unroll
  for (int i = 0; i < 8; i++) a |= sm.cdc[i] != 0;
  return a;
}

// Adds the dequantised chroma residual to pred_u / pred_v (enc.rs:1992 recon_chroma): the DC of
// each block from the 2x2 inverse (h264.rs:1674 dequantize_idct_chroma_dc2x2), its AC dequantised
// when cbpc == 2, then the inverse core transform. Lane = coefficient, two blocks per step.
__device__ __noinline__ void chroma_recon(int qpc, int cbpc, Smem& sm) {
  if (cbpc == 0) return;
  int lane = lane_id(), p = lane & 15, h = lane >> 4, xl = p & 3, yl = p >> 2;
  int qmul = (c_dq4[qpc % 6][0] * 16) << (qpc / 6 + 2);
  int dqs = (int)c_dq4[qpc % 6][pos4(p)] << (qpc / 6);
#pragma unroll 1
  for (int it = 0; it < 4; it++) {
    int b = 2 * it + h, pl = b >> 2, bb = b & 3;
    int a = sm.cdc[pl * 4], bv = sm.cdc[pl * 4 + 1], c = sm.cdc[pl * 4 + 2], d = sm.cdc[pl * 4 + 3];
    int e = a - bv, apb = a + bv, cmd = c - d, cpd = c + d;
    int dcv = bb == 0 ? apb + cpd : (bb == 1 ? e + cmd : (bb == 2 ? apb - cpd : e - cmd));
    int v = p == 0 ? (int)(int16_t)((dcv * qmul) >> 7)
                   : (cbpc >= 2 ? (int)clamp_i16((int)sm.ccoef[b * 16 + p] * dqs) : 0);
    int r = (int16_t)((inv4_pass(inv4_pass(v, 1, xl), 4, yl) + 32) >> 6);
    uint8_t* pr = (pl ? sm.pred_v : sm.pred_u) + (bb >> 1) * 32 + (bb & 1) * 4 + yl * 8 + xl;
    *pr = (uint8_t)clip255(*pr + r);
  }
  __syncwarp();
}

// Raster position of each 4x4 zig-zag index, 4 bits per index (frame scan, Table 8-12).
constexpr unsigned long long kScan4Packed = 0xfeb7adc963258410ull;

// The 1-D inverse 8x8 transform in place on p[0], p[stride], ..., p[7 * stride] (rows and columns
// of the 8x8 reconstruction share it).
__device__ __noinline__ void idct8_inplace(int* p, int stride) {
  int d[8], o[8];
#pragma unroll
  for (int k = 0; k < 8; k++) d[k] = p[k * stride];
  idct8_1d(d, o);
#pragma unroll
  for (int k = 0; k < 8; k++) p[k * stride] = o[k];
}

// Adds the dequantised 8x8 residual of the coded blocks of sm.coef8 to pred_y (enc.rs:2013
// recon_8x8: dequantize_block8x8, h264.rs:1403, then h264_idct8_add, h264_idct.rs:207).
// Lanes 8b..8b+7 own block b: row q, then column q.
__device__ __noinline__ void recon_luma8x8(Smem& sm, int qp, int cbp) {
  int lane = lane_id(), b = lane >> 3, q = lane & 7;
  bool coded = (cbp >> b) & 1;
  int qdiv = qp / 6, rem = qp % 6;
  int dq6[6];
#pragma unroll
  for (int k = 0; k < 6; k++) dq6[k] = c_dq8[rem][k];
  if (coded) {
#pragma unroll 1
    for (int x = 0; x < 8; x++) {
      int i = q * 8 + x, cls = pos8(i);
      int v = cls == 0 ? dq6[0] : cls == 1 ? dq6[1] : cls == 2 ? dq6[2] : cls == 3 ? dq6[3] : cls == 4 ? dq6[4] : dq6[5];
      int l = sm.coef8[b * 64 + i];
      int dv = qdiv >= 2 ? l * (v << (qdiv - 2)) : ((l * v + (1 << (1 - qdiv))) >> (2 - qdiv));
      sm.t8[b * 64 + i] = clamp_i16(dv);
    }
    idct8_inplace(&sm.t8[b * 64 + q * 8], 1);
  }
  __syncwarp();
  if (coded) {
    idct8_inplace(&sm.t8[b * 64 + q], 8);
    int bx = (b & 1) * 8, by = (b >> 1) * 8;
#pragma unroll 1
    for (int y = 0; y < 8; y++) {
      int off = (by + y) * 16 + bx + q;
      int v = (int)((unsigned)sm.t8[b * 64 + y * 8 + q] + 32u) >> 6;
      sm.pred_y[off] = (uint8_t)clip255((int)((unsigned)sm.pred_y[off] + (unsigned)v));
    }
  }
  __syncwarp();
}

// Adds the dequantised luma 4x4 residual of the coded 8x8 groups of sm.coef to pred_y
// (enc.rs:1978 recon_luma_4x4). Lane = coefficient, two blocks per step.
__device__ __noinline__ void recon_luma4x4(Smem& sm, int qp, int cbp) {
  int lane = lane_id(), p = lane & 15, h = lane >> 4, xl = p & 3, yl = p >> 2;
  int dqs = (int)c_dq4[qp % 6][pos4(p)] << (qp / 6);
#pragma unroll 1
  for (int it = 0; it < 8; it++) {
    int b = 2 * it + h;
    bool coded = (cbp >> (b >> 2)) & 1;
    int v = coded ? (int)clamp_i16((int)sm.coef[b * 16 + p] * dqs) : 0;
    int r = (int16_t)((inv4_pass(inv4_pass(v, 1, xl), 4, yl) + 32) >> 6);
    if (coded) {
      int o = (blk_y(b) * 4 + yl) * 16 + blk_x(b) * 4 + xl;
      sm.pred_y[o] = (uint8_t)clip255(sm.pred_y[o] + r);
    }
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------------------------
// Intra prediction (h264.rs:1715 predict_intra_16x16_scalar, :1967 chroma; enc.rs:1561,1586)
// Plane-mode parameters; called by the whole warp: lanes 0..7 take the terms of H
// ((q + 1) (top[8 + q] - top[6 - q])), lanes 8..15 those of V down the left column.
__device__ void plane16_params(const Smem& sm, bool ht, bool hl, int tl, int& pa, int& pb, int& pc) {
  int lane = lane_id(), q = lane & 7;
  int term = 0;
  if (lane < 16) {
    bool top = lane < 8, av = top ? ht : hl;
    const uint8_t* e = top ? sm.top : sm.left;
    int e8 = av ? e[8 + q] : 128, ep = q == 7 ? tl : (av ? e[6 - q] : 128);
    term = (q + 1) * (e8 - ep);
  }
  int H = (int)wsum(lane < 8 ? (uint32_t)term : 0u), V = (int)wsum(lane >= 8 ? (uint32_t)term : 0u);
  int t15 = ht ? sm.top[15] : 128, l15 = hl ? sm.left[15] : 128;
  pa = 16 * (t15 + l15);
  pb = (5 * H + 32) >> 6;
  pc = (5 * V + 32) >> 6;
}
// DC of the 16x16 prediction; called by the whole warp: lane q < 16 adds top[q], lane 16 + q
// left[q] (both sums below 2^16, one reduction).
__device__ __forceinline__ int dc16(const Smem& sm, bool ht, bool hl) {
  int lane = lane_id();
  uint32_t v = lane < 16 ? (ht ? (uint32_t)sm.top[lane] : 0u) : (hl ? (uint32_t)sm.left[lane - 16] << 16 : 0u);
  uint32_t both = wsum(v), st = both & 0xffffu, sl = both >> 16;
  if (ht && hl) return (int)((st + sl + 16) >> 5);
  if (ht) return (int)((st + 8) >> 4);
  if (hl) return (int)((sl + 8) >> 4);
  return 128;
}
__device__ __noinline__ void pred16_into(int mode, Smem& sm, uint8_t* dst, bool ht, bool hl, int tl) {
  int lane = lane_id();
  int y = lane >> 1, x0 = (lane & 1) * 8;
  uint8_t* o = dst + y * 16 + x0;  // this lane's 8 samples (8-byte aligned)
  if (mode == 3) {
    int pa, pb, pc;
    plane16_params(sm, ht, hl, tl, pa, pb, pc);
    uint32_t w[2] = {0u, 0u};
#pragma unroll
    for (int k = 0; k < 8; k++)
      w[k >> 2] |= (uint32_t)clip255((pa + pb * (x0 + k - 7) + pc * (y - 7) + 16) >> 5) << (8 * (k & 3));
    *(uint2*)o = make_uint2(w[0], w[1]);
  } else {
    uint2 v;
    if (mode == 0) {
      v = ht ? lds8(&sm.top[x0]) : make_uint2(0x80808080u, 0x80808080u);
    } else {
      uint32_t b = mode == 1 ? (hl ? sm.left[y] : 128u) : (uint32_t)dc16(sm, ht, hl);
      v = make_uint2(b * 0x01010101u, b * 0x01010101u);
    }
    *(uint2*)o = v;
  }
  __syncwarp();
}
// Intra 16x16 analysis (enc.rs:1637 analyse_i16_edges): SATD per mode; returns best mode.
__device__ __noinline__ int analyse_i16(Smem& sm, bool ht, bool hl, int tl, uint32_t* best_cost) {
  int lane = lane_id();
  int dc = dc16(sm, ht, hl);
  uint32_t sv = 0, sh = 0, sd = 0;
  if (lane < 16) {
    int bx = lane & 3, by = lane >> 2;
    // hadamard4x4_16x4_scalar of the source block, out[4 v + h]
    int rows[4][4];
#pragma unroll
    for (int y = 0; y < 4; y++) {
      const uint8_t* s = &sm.src_y[(by * 4 + y) * 16 + bx * 4];
      int s01 = s[0] + s[1], d01 = s[0] - s[1], s23 = s[2] + s[3], d23 = s[2] - s[3];
      rows[y][0] = s01 + s23; rows[y][1] = s01 - s23; rows[y][2] = d01 + d23; rows[y][3] = d01 - d23;
    }
    int tv[4], th[4];
    {
      const uint8_t* t = &sm.top[bx * 4];
      int e0 = ht ? t[0] : 0, e1 = ht ? t[1] : 0, e2 = ht ? t[2] : 0, e3 = ht ? t[3] : 0;
      int s01 = e0 + e1, d01 = e0 - e1, s23 = e2 + e3, d23 = e2 - e3;
      tv[0] = 4 * (s01 + s23); tv[1] = 4 * (s01 - s23); tv[2] = 4 * (d01 + d23); tv[3] = 4 * (d01 - d23);
      const uint8_t* l = &sm.left[by * 4];
      e0 = hl ? l[0] : 0; e1 = hl ? l[1] : 0; e2 = hl ? l[2] : 0; e3 = hl ? l[3] : 0;
      s01 = e0 + e1; d01 = e0 - e1; s23 = e2 + e3; d23 = e2 - e3;
      th[0] = 4 * (s01 + s23); th[1] = 4 * (s01 - s23); th[2] = 4 * (d01 + d23); th[3] = 4 * (d01 - d23);
    }
#pragma unroll
    for (int h = 0; h < 4; h++) {
      int c0 = rows[0][h], c1 = rows[1][h], c2 = rows[2][h], c3 = rows[3][h];
      int s01 = c0 + c1, d01 = c0 - c1, s23 = c2 + c3, d23 = c2 - c3;
      int col[4] = {s01 + s23, s01 - s23, d01 + d23, d01 - d23};
#pragma unroll
      for (int v = 0; v < 4; v++) {
        int c = col[v], k = 4 * v + h;
        int pv = v == 0 ? tv[h] : 0, ph = h == 0 ? th[v] : 0, pd = k == 0 ? 16 * dc : 0;
        sv += abs(c - pv); sh += abs(c - ph); sd += abs(c - pd);
      }
    }
  }
  sv = wsum(sv) >> 1; sh = wsum(sh) >> 1; sd = wsum(sd) >> 1;
  uint32_t best = sd;
  int mode = 2;
  if (ht && sv < best) { best = sv; mode = 0; }
  if (hl && sh < best) { best = sh; mode = 1; }
  if (ht && hl) {
    pred16_into(3, sm, sm.tmp_y, ht, hl, tl);
    uint32_t s = 0;
    if (lane < 16) {
      int bx = lane & 3, by = lane >> 2;
      s = satd4(&sm.src_y[by * 64 + bx * 4], 16, &sm.tmp_y[by * 64 + bx * 4], 16);
    }
    s = wsum(s) >> 1;
    if (s < best) { best = s; mode = 3; }
  }
  *best_cost = best;
  return mode;
}
// Chroma intra prediction sample of mode for plane p at (x, y).
__device__ __forceinline__ int predc_sample(int mode, const Smem& sm, int p, bool ht, bool hl, int tl, int x, int y,
                                            const int* dcv, int pa, int pb, int pc) {
  switch (mode) {
    case 0: return dcv[(y >> 2) * 2 + (x >> 2)];
    case 1: return hl ? sm.cleft[p][y] : 128;
    case 2: return ht ? sm.ctop[p][x] : 128;
    default: return clip255((pa + pb * (x - 3) + pc * (y - 3) + 16) >> 5);
  }
}
// DC and plane parameters of plane p's chroma prediction; called by the whole warp with p =
// lane / 16. In each half-warp lanes 0..7 hold top[0..7], lanes 8..15 left[0..7] (DC sums of four
// by two butterflies), then lanes 0..3 the terms of H, lanes 4..7 those of V.
__device__ void chroma_pred_params(const Smem& sm, int p, bool ht, bool hl, int tl, int* dcv, int& pa, int& pb, int& pc) {
  const uint8_t* t = sm.ctop[p];
  const uint8_t* l = sm.cleft[p];
  int lane = lane_id(), j = lane & 15, base = lane & 16;
  int e = j < 8 ? (ht ? t[j] : 0) : (hl ? l[j - 8] : 0);
  e += __shfl_xor_sync(FULL, e, 1);
  e += __shfl_xor_sync(FULL, e, 2);
  int st0 = __shfl_sync(FULL, e, base), st1 = __shfl_sync(FULL, e, base + 4);
  int sl0 = __shfl_sync(FULL, e, base + 8), sl1 = __shfl_sync(FULL, e, base + 12);
  if (ht && hl) {
    dcv[0] = (st0 + sl0 + 4) >> 3; dcv[1] = (st1 + 2) >> 2; dcv[2] = (sl1 + 2) >> 2; dcv[3] = (st1 + sl1 + 4) >> 3;
  } else if (ht) {
    dcv[0] = dcv[2] = (st0 + 2) >> 2; dcv[1] = dcv[3] = (st1 + 2) >> 2;
  } else if (hl) {
    dcv[0] = dcv[1] = (sl0 + 2) >> 2; dcv[2] = dcv[3] = (sl1 + 2) >> 2;
  } else {
    dcv[0] = dcv[1] = dcv[2] = dcv[3] = 128;
  }
  int q = j & 3;
  bool top = j < 4, av = top ? ht : hl;
  const uint8_t* ed = top ? t : l;
  int e4 = av ? ed[4 + q] : 128, ep = q == 3 ? tl : (av ? ed[2 - q] : 128);
  int term = j < 8 ? (q + 1) * (e4 - ep) : 0;
  term += __shfl_xor_sync(FULL, term, 1);
  term += __shfl_xor_sync(FULL, term, 2);
  int H = __shfl_sync(FULL, term, base), V = __shfl_sync(FULL, term, base + 4);
  pa = 16 * ((ht ? t[7] : 128) + (hl ? l[7] : 128));
  pb = (17 * H + 16) >> 5;
  pc = (17 * V + 16) >> 5;
}
// Intra chroma mode by SAD (enc.rs:1526 analyse_chroma_intra); best prediction into pred_u/v.
__device__ __noinline__ int analyse_chroma(Smem& sm, bool ht, bool hl, const int* ctl) {
  int lane = lane_id();
  int plane = lane >> 4, idx = (lane & 15) * 4, y = idx >> 3, x0 = idx & 7;
  int dcv[4], pa, pb, pc;
  chroma_pred_params(sm, plane, ht, hl, ctl[plane], dcv, pa, pb, pc);
  const uint8_t* s = (plane ? sm.src_v : sm.src_u) + y * 8 + x0;
  uint32_t best = UMAX;
  int bm = 0;
  for (int mode = 0; mode < 4; mode++) {
    bool ok = mode == 1 ? hl : (mode == 2 ? ht : (mode == 3 ? (ht && hl) : true));
    if (!ok) continue;
    uint32_t sad = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) sad += abs((int)s[k] - predc_sample(mode, sm, plane, ht, hl, ctl[plane], x0 + k, y, dcv, pa, pb, pc));
    uint32_t cost = wsum(sad) + (mode == 0 ? 0u : 8u);
    if (cost < best) { best = cost; bm = mode; }
  }
  uint8_t* out = (plane ? sm.pred_v : sm.pred_u) + y * 8 + x0;
#pragma unroll
  for (int k = 0; k < 4; k++) out[k] = (uint8_t)predc_sample(bm, sm, plane, ht, hl, ctl[plane], x0 + k, y, dcv, pa, pb, pc);
  __syncwarp();
  return bm;
}

// Intra 4x4 prediction of mode m (h264_dsp.rs:799 predict_intra_4x4_u8_scalar) into out[16].
// Intra 4x4 prediction (h264.rs:3223 predict_4x4, the nine modes of H.264 8.3.1.2) in closed
// form. The block's edge samples are gathered into Q[16]:
//   Q[0] = Q[1] = l3, Q[2] = l2, Q[3] = l1, Q[4] = l0, Q[5] = top-left, Q[6..13] = t0..t7,
//   Q[14] = t7, Q[15] = the DC value,
// so that every predicted sample of every mode is Q[i], avg2(Q[i], Q[i+1]) or avg3(Q[i], Q[i+1],
// Q[i+2]) with i a function of (mode, x, y) -- e.g. diagonal down-right is avg3 at 4 + x - y,
// horizontal-up at z = x + 2y is avg2 at 3 - z/2 (z even), avg3 at 2 - z/2 (z odd) and l3 past z = 5.
// Returns kind (0 copy, 1 avg2, 2 avg3) << 8 | i.
__host__ __device__ __forceinline__ int i4_tap(int m, int x, int y) {
  switch (m) {
    case 0: return 6 + x;
    case 1: return 4 - y;
    case 2: return 15;
    case 3: return 0x200 | (6 + x + y);
    case 4: return 0x200 | (4 + x - y);
    case 5: {
      int z = 2 * x - y;
      return z < 0 ? 0x200 | (5 + z) : ((z & 1) ? 0x200 | (4 + x - (y >> 1)) : 0x100 | (5 + x - (y >> 1)));
    }
    case 6: {
      int z = 2 * y - x;
      return z < 0 ? 0x200 | (3 - z) : ((z & 1) ? 0x200 | (3 - (z >> 1)) : 0x100 | (4 - (z >> 1)));
    }
    case 7: return ((y & 1) ? 0x200 : 0x100) | (6 + x + (y >> 1));
    default: {
      int z = x + 2 * y;
      return z > 5 ? 1 : ((z & 1) ? 0x200 | (2 - (z >> 1)) : 0x100 | (3 - (z >> 1)));
    }
  }
}
// The taps of every (mode, sample) for the nine-prediction loop: i | min(i + 1, 15) << 4 |
// min(i + 2, 15) << 8 | kind << 12, at [16 m + 4 y + x] (filled from i4_tap by upload_tables).
__device__ uint16_t g_i4tap[9 * 16];
// ---------------------------------------------------------------------------------------------
struct Ctx {
  const FrameParams* fp;
  const StreamDev* sd;
  int mbx, mby, mb;
};

// Loads the source macroblock, replicating the last row / column past the picture edges
// (enc.rs:400 MbSrc::load, h264.rs:3660 extract_mb_planes).
__device__ __noinline__ void load_source(const Ctx c, Smem& sm) {
  const FrameParams& fp = *c.fp;
  int lane = lane_id();
  int W = fp.width, H = fp.height, cw = (W + 1) >> 1, ch = (H + 1) >> 1;
  int y = min(c.mby * 16 + (lane >> 1), H - 1);
  const uint8_t* row = c.sd->src_y + (long)y * fp.src_stride_y;
  int x0 = c.mbx * 16 + (lane & 1) * 8;
#pragma unroll
  for (int k = 0; k < 8; k++) sm.src_y[(lane >> 1) * 16 + (lane & 1) * 8 + k] = __ldg(row + min(x0 + k, W - 1));
  int plane = lane >> 4, idx = (lane & 15) * 4, r = idx >> 3, c0 = idx & 7;
  int cy = min(c.mby * 8 + r, ch - 1);
  const uint8_t* crow = (plane ? c.sd->src_v : c.sd->src_u) + (long)cy * fp.src_stride_uv;
  uint8_t* dst = (plane ? sm.src_v : sm.src_u) + r * 8 + c0;
#pragma unroll
  for (int k = 0; k < 4; k++) dst[k] = __ldg(crow + min(c.mbx * 8 + c0 + k, cw - 1));
  __syncwarp();
}
// Intra edges from the unfiltered reconstruction of this picture (enc.rs:1459-1521).
__device__ __noinline__ void load_edges(const Ctx c, Smem& sm, bool want_topright, int& tl, int* ctl) {
  const FrameParams& fp = *c.fp;
  int lane = lane_id();
  const uint8_t* Y = c.sd->cur_y;
  int x0 = c.mbx * 16, y0 = c.mby * 16;
  bool ht = c.mby > 0, hl = c.mbx > 0;
  if (ht && lane < 24) {
    bool ok = lane < 16 || (want_topright && c.mbx + 1 < fp.mb_w);
    sm.top[lane] = ok ? ldcg_u8(Y + (long)(y0 - 1) * fp.stride_y + x0 + lane) : 0;
  }
  if (hl && lane < 16) sm.left[lane] = ldcg_u8(Y + (long)(y0 + lane) * fp.stride_y + x0 - 1);
  int cx0 = c.mbx * 8, cy0 = c.mby * 8;
  if (lane < 16) {
    int p = lane >> 3, k = lane & 7;
    const uint8_t* P = p ? c.sd->cur_v : c.sd->cur_u;
    if (ht) sm.ctop[p][k] = ldcg_u8(P + (long)(cy0 - 1) * fp.stride_c + cx0 + k);
    if (hl) sm.cleft[p][k] = ldcg_u8(P + (long)(cy0 + k) * fp.stride_c + cx0 - 1);
  }
  tl = (ht && hl) ? ldcg_u8(Y + (long)(y0 - 1) * fp.stride_y + x0 - 1) : 128;
  ctl[0] = (ht && hl) ? ldcg_u8(c.sd->cur_u + (long)(cy0 - 1) * fp.stride_c + cx0 - 1) : 128;
  ctl[1] = (ht && hl) ? ldcg_u8(c.sd->cur_v + (long)(cy0 - 1) * fp.stride_c + cx0 - 1) : 128;
  __syncwarp();
}

// Stores the reconstruction of pred_y/u/v (or tmp_y for luma) into the current picture.
__device__ __noinline__ void store_recon(const Ctx c, const uint8_t* ly, Smem& sm) {
  const FrameParams& fp = *c.fp;
  int lane = lane_id();
  int y = lane >> 1, x = (lane & 1) * 8;
  uint2 v = *(const uint2*)&ly[y * 16 + x];
  *(uint2*)(c.sd->cur_y + (long)(c.mby * 16 + y) * fp.stride_y + c.mbx * 16 + x) = v;
  if (c.sd->unf_y) {
    int cw = fp.mb_w * 16;
    *(uint2*)(c.sd->unf_y + (long)(c.mby * 16 + y) * cw + c.mbx * 16 + x) = v;
  }
  if (lane < 16) {
    int p = lane >> 3, r = lane & 7;
    uint2 cv = *(const uint2*)&(p ? sm.pred_v : sm.pred_u)[r * 8];
    uint8_t* P = p ? c.sd->cur_v : c.sd->cur_u;
    *(uint2*)(P + (long)(c.mby * 8 + r) * fp.stride_c + c.mbx * 8) = cv;
    uint8_t* U = p ? c.sd->unf_v : c.sd->unf_u;
    if (U) *(uint2*)(U + (long)(c.mby * 8 + r) * (fp.mb_w * 8) + c.mbx * 8) = cv;
  }
}

// Writes the chroma part of the record (chroma levels in zig-zag) and clears the rest.
// The chroma levels of the record, a word (two zig-zag levels) per lane and store: word w of the
// AC levels holds slots 2 (w & 7), 2 (w & 7) + 1 of block w / 8 (plane * 4 + block); slot 0 (the
// DC position) stays 0. Lanes 0..3 write the DC levels.
__device__ __noinline__ void record_chroma(rg_mb_out* rec, Smem& sm, int cbpc) {
  int lane = lane_id();
#pragma unroll 1
  for (int k = 0; k < 2; k++) {
    int w = lane + 32 * k, blk = w >> 3, i = (w & 7) * 2;
    int r0 = (int)((kScan4Packed >> (4 * i)) & 15), r1 = (int)((kScan4Packed >> (4 * i + 4)) & 15);
    int16_t v0 = (i && cbpc >= 2) ? sm.ccoef[blk * 16 + r0] : 0, v1 = cbpc >= 2 ? sm.ccoef[blk * 16 + r1] : 0;
    ((uint32_t*)rec->chroma_ac)[w] = (uint32_t)(uint16_t)v0 | ((uint32_t)(uint16_t)v1 << 16);
  }
  if (lane < 4) {
    int16_t d0 = cbpc >= 1 ? sm.cdc[2 * lane] : 0, d1 = cbpc >= 1 ? sm.cdc[2 * lane + 1] : 0;
    ((uint32_t*)rec->chroma_dc)[lane] = (uint32_t)(uint16_t)d0 | ((uint32_t)(uint16_t)d1 << 16);
  }
}
// The 4x4 luma levels of the record in zig-zag order, a word per lane and store: word w holds
// levels 2 (w & 7), 2 (w & 7) + 1 of block w / 8; lanes 8j..8j+7 of step k cover block 4k + j.
// Returns the blocks holding levels (bit b: block b).
__device__ __noinline__ uint16_t record_luma4x4(rg_mb_out* rec, const Smem& sm) {
  int lane = lane_id();
  uint32_t nz = 0;
#pragma unroll 1
  for (int k = 0; k < 4; k++) {
    int w = lane + 32 * k, b = w >> 3, i = (w & 7) * 2;
    int r0 = (int)((kScan4Packed >> (4 * i)) & 15), r1 = (int)((kScan4Packed >> (4 * i + 4)) & 15);
    int16_t v0 = sm.coef[b * 16 + r0], v1 = sm.coef[b * 16 + r1];
    ((uint32_t*)rec->luma)[w] = (uint32_t)(uint16_t)v0 | ((uint32_t)(uint16_t)v1 << 16);
    uint32_t bal = __ballot_sync(FULL, (v0 | v1) != 0);
#pragma unroll
    for (int j = 0; j < 4; j++)
      if ((bal >> (8 * j)) & 0xffu) nz |= 1u << (4 * k + j);
  }
  return (uint16_t)nz;
}
__device__ __noinline__ void record_header(rg_mb_out* rec, int type, int i16_mode, int cmode, int cbp, int t8, int qp, int mvx, int mvy,
                              int mvdx, int mvdy, uint16_t nz) {
  rec->mb_type = (uint8_t)type;
  rec->i16_mode = (uint8_t)i16_mode;
  rec->chroma_mode = (uint8_t)cmode;
  rec->cbp = (uint8_t)cbp;
  rec->transform_8x8 = (uint8_t)t8;
  rec->qp = (uint8_t)qp;
  rec->qp_delta = 0;
  rec->reserved0 = 0;
  rec->mv[0] = (int16_t)mvx;
  rec->mv[1] = (int16_t)mvy;
  rec->mvd[0] = (int16_t)mvdx;
  rec->mvd[1] = (int16_t)mvdy;
  rec->nz_mask = nz;
  rec->reserved1 = 0;
}
__device__ __noinline__ void write_info(const Ctx c, int flags, int cbpl, int mvx, int mvy, int ref, uint16_t nz, const uint8_t* i4m) {
  MbInfo inf;
  inf.mv[0] = (int16_t)mvx;
  inf.mv[1] = (int16_t)mvy;
  inf.ref = (int8_t)ref;
  inf.flags = (uint8_t)flags;
  inf.cbp_luma = (uint8_t)cbpl;
  inf.qp = (uint8_t)c.sd->qp;
  inf.nz16 = nz;
  inf.i4_bottom = 0;
  inf.i4_right = 0;
  for (int k = 0; k < 4; k++) {
    // bottom row blocks (x = k, y = 3) and right column blocks (x = 3, y = k), decoding order
    int bb = ((3 >> 1) << 3) | ((k >> 1) << 2) | ((3 & 1) << 1) | (k & 1);
    int br = ((k >> 1) << 3) | ((3 >> 1) << 2) | ((k & 1) << 1) | (3 & 1);
    inf.i4_bottom |= (uint16_t)((i4m ? i4m[bb] : 2) << (4 * k));
    inf.i4_right |= (uint16_t)((i4m ? i4m[br] : 2) << (4 * k));
  }
  inf.pad_ = 0;
  c.sd->info[c.mb] = inf;
}

// I16x16 coding and reconstruction (enc.rs:3587 code_i16) with prediction mode `mode`.
__device__ __noinline__ void code_i16(const Ctx c, Smem& sm, int mode, bool ht, bool hl, int tl, const int* ctl) {
  int lane = lane_id();
  int qp = c.sd->qp, qpc = c.sd->qpc;
  pred16_into(mode, sm, sm.pred_y, ht, hl, tl);
  int cmode = analyse_chroma(sm, ht, hl, ctl);
  uint32_t shift, bias;
  quant4_params(qp, true, shift, bias);
  uint32_t my_ac = 0, my_nz = 0;
  int lv[16];
  if (lane < 16) {
    int bx = blk_x(lane), by = blk_y(lane);
    int d[16], cc[16];
#pragma unroll
    for (int y = 0; y < 4; y++)
#pragma unroll
      for (int x = 0; x < 4; x++) {
        int o = (by * 4 + y) * 16 + bx * 4 + x;
        d[y * 4 + x] = (int)sm.src_y[o] - (int)sm.pred_y[o];
      }
    fdct4(d, cc);
    sm.ldc[by * 4 + bx] = (int16_t)cc[0];
#pragma unroll
    for (int i = 0; i < 16; i++) {
      lv[i] = quant_level(cc[i], c_mf4[qp % 6][pos4(i)], bias, shift);
      if (lv[i]) my_nz = 1;
    }
  }
  // a group with any level drops its DC slots; AC presence counts only slots 1..15
  uint32_t gnz = my_nz | __shfl_xor_sync(FULL, my_nz, 1);
  gnz |= __shfl_xor_sync(FULL, gnz, 2);
  if (lane < 16) {
    if (gnz) lv[0] = 0;
    else {
#pragma unroll
      for (int i = 0; i < 16; i++) lv[i] = 0;
    }
#pragma unroll
    for (int i = 1; i < 16; i++) if (lv[i]) my_ac = 1;
#pragma unroll
    for (int i = 0; i < 16; i++) sm.coef[lane * 16 + i] = (int16_t)lv[i];
  }
  __syncwarp();
  int cbpl = wor(my_ac) ? 15 : 0;
  // luma DC: Hadamard (>> 1) + quantisation (enc.rs:1960), then inverse (h264.rs:1645)
  if (lane == 0) {
    int t[16], had[16];
    for (int r = 0; r < 4; r++) {
      int b0 = sm.ldc[r * 4], b1 = sm.ldc[r * 4 + 1], b2 = sm.ldc[r * 4 + 2], b3 = sm.ldc[r * 4 + 3];
      int s03 = b0 + b3, s12 = b1 + b2, d03 = b0 - b3, d12 = b1 - b2;
      t[r * 4] = s03 + s12; t[r * 4 + 1] = d03 + d12; t[r * 4 + 2] = s03 - s12; t[r * 4 + 3] = d03 - d12;
    }
    for (int k = 0; k < 4; k++) {
      int s03 = t[k] + t[k + 12], s12 = t[k + 4] + t[k + 8], d03 = t[k] - t[k + 12], d12 = t[k + 4] - t[k + 8];
      had[k] = (int16_t)((s03 + s12) >> 1); had[k + 4] = (int16_t)((d03 + d12) >> 1);
      had[k + 8] = (int16_t)((s03 - s12) >> 1); had[k + 12] = (int16_t)((d03 - d12) >> 1);
    }
    int qbits = 16 + qp / 6, mf = c_mf4[qp % 6][0], f = (1 << qbits) / 3;
    int lvl[16];
    for (int i = 0; i < 16; i++) {
      int a = had[i] < 0 ? -had[i] : had[i];
      int l = (a * mf + f) >> qbits;
      lvl[i] = had[i] < 0 ? -l : l;
      sm.ldc[i] = (int16_t)lvl[i];
    }
    int qmul = (c_dq4[qp % 6][0] * 16) << (qp / 6 + 2);
    int tt[16];
    for (int i = 0; i < 4; i++) {
      int z0 = lvl[4 * i] + lvl[4 * i + 1], z1 = lvl[4 * i] - lvl[4 * i + 1];
      int z2 = lvl[4 * i + 2] - lvl[4 * i + 3], z3 = lvl[4 * i + 2] + lvl[4 * i + 3];
      tt[4 * i] = z0 + z3; tt[4 * i + 1] = z0 - z3; tt[4 * i + 2] = z1 - z2; tt[4 * i + 3] = z1 + z2;
    }
    for (int i = 0; i < 4; i++) {
      int z0 = tt[i] + tt[8 + i], z1 = tt[i] - tt[8 + i], z2 = tt[4 + i] - tt[12 + i], z3 = tt[4 + i] + tt[12 + i];
      sm.ldcr[i] = (int16_t)(((z0 + z3) * qmul + 128) >> 8);
      sm.ldcr[4 + i] = (int16_t)(((z1 + z2) * qmul + 128) >> 8);
      sm.ldcr[8 + i] = (int16_t)(((z1 - z2) * qmul + 128) >> 8);
      sm.ldcr[12 + i] = (int16_t)(((z0 - z3) * qmul + 128) >> 8);
    }
  }
  uint32_t ac_any[2], ac_sc[2];
  chroma_quant(qpc, true, sm, ac_any, ac_sc);
  int cbpc = (ac_any[0] | ac_any[1]) ? 2 : (chroma_dc_any(sm) ? 1 : 0);
  __syncwarp();
  // record
  rg_mb_out* rec = c.sd->rec + c.mb;
  uint16_t nzm = 0;
  if (lane < 16) {
#pragma unroll
    for (int i = 0; i < 16; i++) rec->luma[lane * 16 + i] = sm.coef[lane * 16 + c_scan4[i]];
    rec->luma_dc[lane] = sm.ldc[c_scan4[lane]];
    rec->i4_modes[lane] = 2;
  }
  nzm = (uint16_t)__ballot_sync(FULL, lane < 16 && cbpl && my_ac);
  record_chroma(rec, sm, cbpc);
  if (lane == 0) record_header(rec, RG_MB_I16X16, mode, cmode, cbpl | (cbpc << 4), 0, qp, 0, 0, 0, 0, nzm);
  // reconstruction
  if (lane < 16) {
    int bx = blk_x(lane), by = blk_y(lane);
    int blk[16], res[16];
#pragma unroll
    for (int i = 0; i < 16; i++) {
      int v = sm.coef[lane * 16 + i];
      blk[i] = cbpl ? clamp_i16(v * ((int)c_dq4[qp % 6][pos4(i)] << (qp / 6))) : v;
    }
    blk[0] = sm.ldcr[by * 4 + bx];
    idct4(blk, res);
#pragma unroll
    for (int y = 0; y < 4; y++)
#pragma unroll
      for (int x = 0; x < 4; x++) {
        int o = (by * 4 + y) * 16 + bx * 4 + x;
        sm.pred_y[o] = (uint8_t)clip255(sm.pred_y[o] + res[y * 4 + x]);
      }
  }
  __syncwarp();
  chroma_recon(qpc, cbpc, sm);
  store_recon(c, sm.pred_y, sm);
  if (lane == 0) write_info(c, kFlagIntra, cbpl, 0, 0, -1, nzm, nullptr);
}

// I4x4 analysis (enc.rs:3336 analyse_i4): sixteen blocks in decoding order, each choosing among
// the available modes by SATD + lambda * (1 if the predicted mode else 4), then quantising and
// reconstructing before the next block. Per block the warp gathers the edge samples (lane k ->
// Q[k]), builds all nine predictions (lane -> pixel, the two half-warps taking even / odd modes),
// costs the modes (lane -> mode), and transforms the chosen residual with shuffles (lane ->
// coefficient). Gives up (false) as soon as the running cost reaches `budget`.
// kMask: only the modes of masks[b] (bit m: Intra4x4PredMode m) that are available at block b are
// tried -- DC alone when none is (the learned form); the plain form tries every available mode.
template <bool kMask>
__device__ __noinline__ bool analyse_i4(const Ctx c, Smem& sm, uint32_t budget, bool ht_mb, bool hl_mb, int tl_mb, int* cbpl_out,
                                        const uint16_t* masks) {
  const FrameParams& fp = *c.fp;
  int lane = lane_id();
  int p = lane & 15, xl = p & 3, yl = p >> 2;
  int qp = c.sd->qp;
  uint32_t lambda = c_lambda[qp];
  uint32_t shift, bias;
  quant4_params(qp, true, shift, bias);
  uint32_t mf = c_mf4[qp % 6][pos4(p)];
  int dqs = (int)c_dq4[qp % 6][pos4(p)] << (qp / 6);
  uint32_t total = lambda * 24;
  int cbpl = 0;
  const MbInfo* info = c.sd->info;
  uint32_t lmodes = hl_mb ? ld_info(&info[c.mb - 1]).i4_right : 0x2222u;
  uint32_t tmodes = ht_mb ? ld_info(&info[c.mb - fp.mb_w]).i4_bottom : 0x2222u;
  // this lane's taps for its predictions (modes lane / 16 + 2 k, sample p): the same for every block
  uint32_t taps[5];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    int m = (lane >> 4) + 2 * k;
    taps[k] = m < 9 ? __ldg(&g_i4tap[m * 16 + p]) : 0u;
  }
  for (int b = 0; b < 16; b++) {
    int bx = blk_x(b), by = blk_y(b), px = bx * 4, py = by * 4;
    bool ht = by > 0 || ht_mb, hl = bx > 0 || hl_mb;
    bool tr = !(b == 3 || b == 7 || b == 11 || b == 13 || b == 15) && (b != 5 || c.mbx + 1 < fp.mb_w);
    // edge samples (unavailable ones 128; top-right replicated from t3 when unavailable)
    int q = 128;
    if (p <= 4) {
      int j = p <= 1 ? 3 : 4 - p;
      if (hl) q = bx > 0 ? sm.tmp_y[(py + j) * 16 + px - 1] : sm.left[py + j];
    } else if (p == 5) {
      if (ht && hl)
        q = (by > 0 && bx > 0) ? sm.tmp_y[(py - 1) * 16 + px - 1]
                               : (by > 0 ? sm.left[py - 1] : (bx > 0 ? sm.top[px - 1] : tl_mb));
    } else if (p <= 14) {
      int i = min(p - 6, 7);
      if (i >= 4 && !tr) i = 3;
      if (ht) q = by > 0 ? sm.tmp_y[(py - 1) * 16 + px + i] : sm.top[px + i];
    }
    uint32_t sums = wsum(lane < 16 ? ((p >= 6 && p <= 9) ? (uint32_t)q : 0u) + ((p >= 1 && p <= 4) ? (uint32_t)q << 16 : 0u) : 0u);
    int st = (int)(sums & 0xffff), sl = (int)(sums >> 16);
    int dc = ht && hl ? (st + sl + 4) >> 3 : (ht ? (st + 2) >> 2 : (hl ? (sl + 2) >> 2 : 128));
    if (lane < 16) sm.i4q[p] = (uint8_t)(p == 15 ? dc : q);
    // predicted mode (h264.rs:3283)
    int gx = c.mbx * 4 + bx, gy = c.mby * 4 + by;
    int pm;
    if (gx == 0 || gy == 0) pm = 2;
    else {
      int ml = bx > 0 ? sm.i4m[(((by >> 1) << 3) | (((bx - 1) >> 1) << 2) | ((by & 1) << 1) | ((bx - 1) & 1))]
                      : (int)((lmodes >> (4 * by)) & 15);
      int mt = by > 0 ? sm.i4m[((((by - 1) >> 1) << 3) | ((bx >> 1) << 2) | (((by - 1) & 1) << 1) | (bx & 1))]
                      : (int)((tmodes >> (4 * bx)) & 15);
      pm = min(ml, mt);
    }
    __syncwarp();
    // nine predictions and their SATDs: half-warp h takes modes h, h + 2, ... (k = 0..4), lane p
    // sample p; the 4x4 Hadamard of the difference (metrics.rs:705) by four shuffle butterflies,
    // both halves' sums of magnitudes in one reduction (each below 2^16). Every lane ends with
    // the same key, the least cost first and the lower mode on a tie.
    int srcp = sm.src_y[(py + yl) * 16 + px + xl];
    int pv[5];
    uint32_t key = UMAX;
    uint32_t allow = 0x1ffu;
    if constexpr (kMask) {
      uint32_t avail = 0x4u | (ht ? 0x89u : 0u) | (hl ? 0x102u : 0u) | (ht && hl ? 0x70u : 0u);
      allow = masks[b] & avail;
      if (!allow) allow = 0x4u;
    }
#pragma unroll
    for (int k = 0; k < 5; k++) {
      if constexpr (kMask) {
        if (!((allow >> (2 * k)) & 3u)) { pv[k] = 0; continue; }  // neither mode of this step is tried
      }
      uint32_t tp = taps[k], kind = tp >> 12;
      int a0 = sm.i4q[tp & 15], a1 = sm.i4q[(tp >> 4) & 15], a2 = sm.i4q[(tp >> 8) & 15];
      int v = kind == 0 ? a0 : (kind == 1 ? (a0 + a1 + 1) >> 1 : (a0 + 2 * a1 + a2 + 2) >> 2);
      pv[k] = v;
      int d = srcp - v;
#pragma unroll
      for (int b = 1; b < 16; b <<= 1) {
        int o = __shfl_xor_sync(FULL, d, b);
        d = (lane & b) ? o - d : d + o;
      }
      uint32_t sums = __reduce_add_sync(FULL, (uint32_t)(d < 0 ? -d : d) << (16 * (lane >> 4)));
#pragma unroll
      for (int h = 0; h < 2; h++) {
        int m = 2 * k + h;
        if (m > 8) continue;
        bool av = (m == 0 || m == 3 || m == 7) ? ht : ((m == 1 || m == 8) ? hl : (m == 2 ? true : (ht && hl)));
        if constexpr (kMask) av = av && ((allow >> m) & 1u);
        uint32_t cost = (((sums >> (16 * h)) & 0xffffu) >> 1) + lambda * (m == pm ? 1u : 4u);
        if (av) key = min(key, (cost << 4) | (uint32_t)m);
      }
    }
    int bm = (int)(key & 15);
    total += key >> 4;
    if (total >= budget) return false;
    if (lane == 0) sm.i4m[b] = (uint8_t)bm;
    // residual transform and quantisation, lane p -> coefficient p (raster); the chosen mode's
    // sample p is in lane 16 (bm & 1) + p
    int kb = bm >> 1, mine = pv[0];
#pragma unroll
    for (int k = 1; k < 5; k++)
      if (kb == k) mine = pv[k];
    int pred = __shfl_sync(FULL, mine, (bm & 1) * 16 + p);
    int acc = fwd4_pass(fwd4_pass(srcp - pred, 1, xl), 4, yl);
    acc = (int16_t)acc;
    uint32_t aa = (uint32_t)(acc < 0 ? -acc : acc);
    int l = (int)((aa * mf + bias) >> shift);
    int lvl = acc < 0 ? -l : l;
    if (lane < 16) sm.coef[b * 16 + p] = (int16_t)lvl;
    bool nz = __ballot_sync(FULL, lane < 16 && lvl != 0) != 0;
    if (nz) cbpl |= 1 << (b >> 2);
    // inverse transform (rows then columns) and reconstruction
    int rec = pred;
    if (nz) {
      int dq = clamp_i16(lvl * dqs);
      int r = (int16_t)((inv4_pass(inv4_pass(dq, 1, xl), 4, yl) + 32) >> 6);
      rec = clip255(pred + r);
    }
    if (lane < 16) sm.tmp_y[(py + yl) * 16 + px + xl] = (uint8_t)rec;
    __syncwarp();
  }
  *cbpl_out = cbpl;
  return true;
}

__device__ __noinline__ void code_i4(const Ctx c, Smem& sm, int cbpl, bool ht, bool hl, const int* ctl) {
  int lane = lane_id();
  int qpc = c.sd->qpc;
  int cmode = analyse_chroma(sm, ht, hl, ctl);
  uint32_t ac_any[2], ac_sc[2];
  chroma_quant(qpc, true, sm, ac_any, ac_sc);
  int cbpc = (ac_any[0] | ac_any[1]) ? 2 : (chroma_dc_any(sm) ? 1 : 0);
  rg_mb_out* rec = c.sd->rec + c.mb;
  uint16_t nzm = record_luma4x4(rec, sm);
  if (lane < 16) {
    rec->luma_dc[lane] = 0;
    rec->i4_modes[lane] = sm.i4m[lane];
  }
  record_chroma(rec, sm, cbpc);
  if (lane == 0) record_header(rec, RG_MB_I4X4, 0, cmode, cbpl | (cbpc << 4), 0, c.sd->qp, 0, 0, 0, 0, nzm);
  chroma_recon(qpc, cbpc, sm);
  store_recon(c, sm.tmp_y, sm);
  if (lane == 0) write_info(c, kFlagIntra, cbpl, 0, 0, -1, nzm, sm.i4m);
}

// One macroblock of an I slice (enc.rs:3311 code_intra).
__device__ __noinline__ void analyse_intra_mb(const Ctx c, Smem& sm) {
  int tl, ctl[2];
  load_edges(c, sm, true, tl, ctl);
  bool ht = c.mby > 0, hl = c.mbx > 0;
  uint32_t lambda = c_lambda[c.sd->qp];
  uint32_t i16c;
  int i16m = analyse_i16(sm, ht, hl, tl, &i16c);
  if (i16c > 40 * lambda) {
    int cbpl;
    if (analyse_i4<false>(c, sm, i16c + lambda * 4, ht, hl, tl, &cbpl, nullptr)) {
      code_i4(c, sm, cbpl, ht, hl, ctl);
      return;
    }
  }
  code_i16(c, sm, i16m, ht, hl, tl, ctl);
}

// Codes P_Skip with vector mv; prediction already in pred_y / pred_u / pred_v.
__device__ __noinline__ void code_skip(const Ctx c, Smem& sm, int mvx, int mvy) {
  int lane = lane_id();
  rg_mb_out* rec = c.sd->rec + c.mb;
  if (lane < 16) {
#pragma unroll
    for (int i = 0; i < 16; i++) rec->luma[lane * 16 + i] = 0;
    rec->luma_dc[lane] = 0;
    rec->i4_modes[lane] = 2;
  }
  if (lane < 8) {
#pragma unroll
    for (int i = 0; i < 16; i++) rec->chroma_ac[lane >> 2][lane & 3][i] = 0;
    rec->chroma_dc[lane >> 2][lane & 3] = 0;
  }
  if (lane == 0) {
    record_header(rec, RG_MB_P_SKIP, 0, 0, 0, 0, c.sd->qp, mvx, mvy, 0, 0, 0);
    write_info(c, kFlagSkip, 0, mvx, mvy, 0, 0, nullptr);
  }
  store_recon(c, sm.pred_y, sm);
}

// Probe of the skip residual (enc.rs:2163 probe_skip_luma): no level above 1 and a total
// decimation score below 6.
__device__ __noinline__ bool probe_skip_luma(int qp, Smem& sm) {
  int lane = lane_id();
  uint32_t shift, bias;
  quant4_params(qp, false, shift, bias);
  int nz, big, sc;  // levels go to sm.coef as scratch: a skipped macroblock records none
  quant4x4_blocks(sm, false, 16, 0, qp, shift, bias, sm.coef, nullptr, nz, big, sc);
  uint32_t b = wor(lane < 16 ? (uint32_t)big : 0u);
  uint32_t score = wsum(lane < 16 ? (uint32_t)sc : 0u);
  return !b && score < 6;
}

// ---------------------------------------------------------------------------------------------
// Pipelined mode synchronisation: monotonic progress counters, published with a release store
// after a fence, awaited with an acquire load. Every wait has a time limit; when it runs out
// the kernel records RG_ERR_TIMEOUT and all warps leave.
__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int atom_add_acq_rel(int* p, int v) {
  int old;
  asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ void st_release_sys(int* p, int v) {
  asm volatile("st.release.sys.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Waits until *p >= need. The first check and the final one are acquire loads by every lane;
// in between lane 0 polls with relaxed loads (which leave the SM's L1 alone) and sleeps 32 ns
// doubling to 512 ns. Returns the acquired value, or -1 on timeout (recorded in *error) or
// when another warp failed.
__device__ __noinline__ int wait_geq(const int* p, int need, int* error, unsigned long long timeout_ns) {
  int v = ld_acquire(p);
  if (__all_sync(FULL, v >= need)) return v;
  unsigned long long t0 = global_ns();
  unsigned int sleep = 32;
  while (true) {
    int r = 0;
    if (lane_id() == 0) r = ld_relaxed(p) >= need ? 1 : (ld_relaxed(error) ? 2 : 0);
    r = __shfl_sync(FULL, r, 0);
    if (r == 1) {
      v = ld_acquire(p);
      if (__all_sync(FULL, v >= need)) return v;
    }
    if (r == 2) return -1;
    unsigned long long dt = __shfl_sync(FULL, global_ns() - t0, 0);
    if (dt > timeout_ns) {
      if (lane_id() == 0) atomicCAS(error, 0, 1);
      return -1;
    }
    __nanosleep(sleep);
    sleep = min(sleep * 2, 512u);
  }
}
// wait_geq with the last acquired value of the counter kept in `seen`: no load when it already
// covers `need` (the acquire that returned it orders every later load of this warp).
__device__ __forceinline__ bool wait_seen(const int* p, int need, int& seen, int* error,
                                          unsigned long long timeout_ns) {
  if (seen >= need) return true;
  int v = wait_geq(p, need, error, timeout_ns);
  if (v < 0) return false;
  seen = v;
  return true;
}
// Makes this warp's global writes visible, then publishes v.
__device__ __forceinline__ void publish(int* p, int v) {
  __threadfence();
  __syncwarp();
  if (lane_id() == 0) st_release(p, v);
}
// What a P macroblock of the pipelined mode waits for in its reference picture.
struct PipeWait {
  const int* ana_prev;   // analysis progress per macroblock row of the reference picture
  const int* db_prev;    // deblocking progress per row of the reference picture (padding included)
  int* error;
  unsigned long long timeout_ns;
  int seen_ana;          // last acquired ana_prev[row of this segment]
  int db_row, seen_db;   // last acquired db_prev[db_row]
  int reach_y, reach_x;  // 1 + the largest reach waited for beyond zero motion, in macroblocks
  bool failed;
};

// One macroblock of a P slice (enc.rs:3011 code_p_mb). In the pipelined mode (pw != null) it
// first waits for the reference frame to be final over every sample its search can read; when
// a wait gives up it returns with pw->failed set and writes nothing.
__device__ __noinline__ void analyse_p_mb(const Ctx c, Smem& sm, PipeWait* pw) {
  const FrameParams& fp = *c.fp;
  const StreamDev& sd = *c.sd;
  int lane = lane_id();
  int mbx = c.mbx, mby = c.mby, mb_w = fp.mb_w;
  int x0 = mbx * 16, y0 = mby * 16;
  int qp = c.sd->qp;
  uint32_t lambda = c_lambda[qp];
  int cw = fp.mb_w * 16, chh = fp.mb_h * 16;
  // MvBounds (enc.rs:1105)
  int bmin0 = -4 * (x0 + 28), bmin1 = max(-4 * (y0 + 28), -2048);
  int bmax0 = 4 * (cw - 16 - x0 + 28), bmax1 = min(4 * (chh - 16 - y0 + 28), 2044);
  // neighbours (this picture)
  const MbInfo* info = sd.info;
  int lref = -2, tref = -2, dref = -2;
  int a0 = 0, a1 = 0, b0 = 0, b1 = 0, c0 = 0, c1 = 0;
  if (mbx > 0) { MbInfo n = ld_info(&info[c.mb - 1]); lref = n.ref; a0 = n.mv[0]; a1 = n.mv[1]; }
  if (mby > 0) { MbInfo n = ld_info(&info[c.mb - mb_w]); tref = n.ref; b0 = n.mv[0]; b1 = n.mv[1]; }
  if (mby > 0 && mbx + 1 < mb_w) { MbInfo n = ld_info(&info[c.mb - mb_w + 1]); dref = n.ref; c0 = n.mv[0]; c1 = n.mv[1]; }
  else if (mby > 0 && mbx > 0) { MbInfo n = ld_info(&info[c.mb - mb_w - 1]); dref = n.ref; c0 = n.mv[0]; c1 = n.mv[1]; }
  // pred_motion_partition (h264.rs:3577), 16x16, ref 0
  int mvp0, mvp1;
  {
    auto med = [](int x, int y, int z) { return min(max(x, y), max(min(x, y), z)); };
    int m = (lref == 0) + (tref == 0) + (dref == 0);
    if (m > 1) { mvp0 = med(a0, b0, c0); mvp1 = med(a1, b1, c1); }
    else if (m == 1) {
      if (lref == 0) { mvp0 = a0; mvp1 = a1; }
      else if (tref == 0) { mvp0 = b0; mvp1 = b1; }
      else { mvp0 = c0; mvp1 = c1; }
    } else if (tref == -2 && dref == -2 && lref != -2) { mvp0 = a0; mvp1 = a1; }
    else { mvp0 = med(a0, b0, c0); mvp1 = med(a1, b1, c1); }
  }
  int ps0 = mvp0, ps1 = mvp1;
  if (mbx == 0 || mby == 0 || (lref == 0 && a0 == 0 && a1 == 0) || (tref == 0 && b0 == 0 && b1 == 0)) { ps0 = 0; ps1 = 0; }
  load_source(c, sm);
  int qpc = c.sd->qpc;
  // co-located vector of the previous picture: a search candidate (enc.rs:3094)
  if (pw && !wait_seen(pw->ana_prev + mby, mbx + 1, pw->seen_ana, pw->error, pw->timeout_ns)) {
    pw->failed = true;
    return;
  }
  MbInfo prevmb = ld_info(&sd.prev_info[c.mb]);
  if (pw) {
    // The right- and bottom-most reference sample this macroblock can read: the full-pel
    // candidates, a diamond of at most 16 steps around the best, the half-sample window
    // (-3..+20) and 8-byte loads. Everything above and to the left of it (padding included) is
    // final once the macroblock holding it is.
    int cx[5] = {mvp0, 0, a0, b0, prevmb.mv[0]}, cy[5] = {mvp1, 0, a1, b1, prevmb.mv[1]};
    int hi0 = -(1 << 20), hi1 = -(1 << 20);
    int imn0 = (bmin0 + 3) >> 2, imn1 = (bmin1 + 3) >> 2, imx0 = bmax0 >> 2, imx1 = bmax1 >> 2;
    for (int k = 0; k < 5; k++) {
      hi0 = max(hi0, min(max((cx[k] + 2) >> 2, imn0), imx0));
      hi1 = max(hi1, min(max((cy[k] + 2) >> 2, imn1), imx1));
    }
    int xb = (x0 + hi0 + 44) >> 4, rb = (y0 + hi1 + 40) >> 4;
    int rr = min(max(rb, 0), fp.mb_h - 1), xx = min(max(xb, 0), fp.mb_w - 1);
    // rows above the last are final where the row below is deblocked; the last row where its
    // right neighbour is
    int row = rr < fp.mb_h - 1 ? rr + 1 : rr, need = rr < fp.mb_h - 1 ? xx + 1 : min(xx + 2, fp.mb_w);
    // zero motion reaches (mbx + 2, mby + 2); the host sizes the picture lag from the maximum
    pw->reach_y = max(pw->reach_y, max(rr - mby - 2, 0) + 1);
    pw->reach_x = max(pw->reach_x, max(xx - mbx - 2, 0) + 1);
    if (row != pw->db_row) {
      pw->db_row = row;
      pw->seen_db = 0;
    }
    if (!wait_seen(pw->db_prev + row, need, pw->seen_db, pw->error, pw->timeout_ns)) {
      pw->failed = true;
      return;
    }
  }

  // 1. skip probe (enc.rs:2906 try_p_skip)
  if (ps0 >= bmin0 && ps0 <= bmax0 && ps1 >= bmin1 && ps1 <= bmax1) {
    mc_luma16(sd.ref_y, fp.stride_y, x0, y0, ps0, ps1, sm);
    uint2 s = src8(sm), p = *(const uint2*)&sm.pred_y[(lane >> 1) * 16 + (lane & 1) * 8];
    uint32_t sad = wsum(vsad8(s, p));
    if (sad < c.sd->sb_probe) {
      bool lz = sad <= c.sd->sb_luma;
      if (!lz) {
        uint32_t ssd = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
          int d0 = (int)((s.x >> (8 * k)) & 255) - (int)((p.x >> (8 * k)) & 255);
          int d1 = (int)((s.y >> (8 * k)) & 255) - (int)((p.y >> (8 * k)) & 255);
          ssd += d0 * d0 + d1 * d1;
        }
        lz = wsum(ssd) <= c.sd->sb_luma_ssd;
      }
      if (!lz) lz = probe_skip_luma(qp, sm);
      if (lz) {
        mc_chroma8(sd.ref_u, sd.ref_v, fp.stride_c, mbx, mby, ps0, ps1, sm);
        // per plane SAD / SSD bounds (lanes 0..15 U, 16..31 V, 4 samples each)
        int plane = lane >> 4, idx = (lane & 15) * 4;
        const uint8_t* ss = (plane ? sm.src_v : sm.src_u) + idx;
        const uint8_t* pp = (plane ? sm.pred_v : sm.pred_u) + idx;
        uint32_t sadp = 0, ssdp = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) { int d = (int)ss[k] - (int)pp[k]; sadp += abs(d); ssdp += d * d; }
        uint32_t sad_u = wsum(plane == 0 ? sadp : 0), sad_v = wsum(plane == 1 ? sadp : 0);
        uint32_t ssd_u = wsum(plane == 0 ? ssdp : 0), ssd_v = wsum(plane == 1 ? ssdp : 0);
        bool zu = sad_u <= c.sd->sb_chroma || ssd_u <= c.sd->sb_chroma_ssd;
        bool zv = sad_v <= c.sd->sb_chroma || ssd_v <= c.sd->sb_chroma_ssd;
        bool cz = zu && zv;
        if (!cz) {
          uint32_t ac_any[2], ac_sc[2];
          chroma_quant(qpc, false, sm, ac_any, ac_sc);
          cz = !chroma_dc_any(sm) && ac_sc[0] < 7 && ac_sc[1] < 7;
        }
        if (cz) {
          code_skip(c, sm, ps0, ps1);
          return;
        }
      }
    }
  }

  // 2. motion search (enc.rs:3084-3117)
  const uint8_t* ref = sd.ref_y;
  int stride = fp.stride_y;
  // candidates in order: predictor, zero, left (if any), top (if any), co-located of the previous
  // picture -- five fixed slots, the left / top ones skipped when absent
  int imin0 = (bmin0 + 3) >> 2, imin1 = (bmin1 + 3) >> 2, imax0 = bmax0 >> 2, imax1 = bmax1 >> 2;
  uint2 sv = src8(sm);
  const uint8_t* base = ref + (long)(y0 + (lane >> 1)) * stride + x0 + (lane & 1) * 8;
  int best0 = 0, best1 = 0;
  uint32_t best_cost = UMAX;
  // clamped full-pel candidates, their samples loaded together, then costed in order (a
  // repeated position is skipped)
  int cmx[5], cmy[5];
  bool cval[5];
  uint2 cref[5];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    int vx = k == 0 ? mvp0 : k == 1 ? 0 : k == 2 ? a0 : k == 3 ? b0 : prevmb.mv[0];
    int vy = k == 0 ? mvp1 : k == 1 ? 0 : k == 2 ? a1 : k == 3 ? b1 : prevmb.mv[1];
    cval[k] = k == 2 ? mbx > 0 : (k == 3 ? mby > 0 : true);
    cmx[k] = min(max((vx + 2) >> 2, imin0), imax0);
    cmy[k] = min(max((vy + 2) >> 2, imin1), imax1);
    cref[k] = ldg8(base + (long)cmy[k] * stride + cmx[k]);
  }
#pragma unroll
  for (int k = 0; k < 5; k++) {
    bool use = cval[k];  // absent, or at the position of an earlier candidate: skipped
#pragma unroll
    for (int j = 0; j < k; j++) use &= !(cval[j] && cmx[j] == cmx[k] && cmy[j] == cmy[k]);
    if (!use) continue;  // uniform across the warp
    uint32_t cost = fullpel_cost(sv, cref[k], cmx[k], cmy[k], mvp0, mvp1, lambda);
    if (cost < best_cost) { best_cost = cost; best0 = cmx[k]; best1 = cmy[k]; }
  }
  // diamond (enc.rs:1207-1272): up, left, right, down around the best, first strict minimum
  // wins; each step's four loads are issued together
#pragma unroll 1
  for (int it = 0; it < 16; it++) {
    const uint8_t* cp = base + (long)best1 * stride + best0;
    uint2 r[4];
    bool in[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      int dx = k == 1 ? -1 : (k == 2 ? 1 : 0), dy = k == 0 ? -1 : (k == 3 ? 1 : 0);
      int px = best0 + dx, py = best1 + dy;
      in[k] = px >= imin0 && px <= imax0 && py >= imin1 && py <= imax1;
      r[k] = in[k] ? ldg8(cp + dy * stride + dx) : make_uint2(0u, 0u);
    }
    int nb0 = best0, nb1 = best1;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      int dx = k == 1 ? -1 : (k == 2 ? 1 : 0), dy = k == 0 ? -1 : (k == 3 ? 1 : 0);
      if (!in[k]) continue;  // uniform across the warp
      uint32_t cost = fullpel_cost(sv, r[k], best0 + dx, best1 + dy, mvp0, mvp1, lambda);
      if (cost < best_cost) {
        best_cost = cost;
        nb0 = best0 + dx;
        nb1 = best1 + dy;
      }
    }
    if (nb0 == best0 && nb1 == best1) break;
    best0 = nb0;
    best1 = nb1;
  }
  int mv0, mv1;
  {
    int fm0 = best0 * 4, fm1 = best1 * 4;
    uint32_t full_mvc = mvd_cost(fm0 - mvp0, lambda) + mvd_cost(fm1 - mvp1, lambda);
    if (best_cost - full_mvc <= c.sd->sb_luma) {
      mv0 = fm0; mv1 = fm1;
      uint2 v = ldg8(base + (long)best1 * stride + best0);
      *(uint2*)&sm.pred_y[(lane >> 1) * 16 + (lane & 1) * 8] = v;
      __syncwarp();
    } else {
      // sub-pel refinement over a half-sample window around the full-pel best (enc.rs:1283)
      int bxp = x0 + best0, byp = y0 + best1;
      stage_window(ref, stride, bxp - 1, byp - 1, sm);
      build_hpel(sm, 7);
      int q0 = fm0, q1 = fm1;
      uint32_t bc = best_cost;
#pragma unroll 1
      for (int si = 0; si < 2; si++) {
        int st = si == 0 ? 2 : 1, iters = si == 0 ? 1 : 2;
#pragma unroll 1
        for (int it = 0; it < iters; it++) {
          int f0 = q0, f1 = q1;
          int dd[4][2] = {{0, -st}, {-st, 0}, {st, 0}, {0, st}};
          uint32_t cc[4];
#pragma unroll
          for (int k = 0; k < 4; k++) {
            int cx = f0 + dd[k][0], cy = f1 + dd[k][1];
            bool ok = abs(cx - fm0) <= 3 && abs(cy - fm1) <= 3 && cx >= bmin0 && cx <= bmax0 && cy >= bmin1 && cy <= bmax1;
            uint32_t s = ok ? qpel_sad(sm, sv, (cx >> 2) - best0 + 1, (cy >> 2) - best1 + 1, cx & 3, cy & 3) : 0u;
            s = wsum(s);
            cc[k] = ok ? s + mvd_cost(cx - mvp0, lambda) + mvd_cost(cy - mvp1, lambda) : UMAX;
          }
#pragma unroll
          for (int k = 0; k < 4; k++)
            if (cc[k] < bc) { bc = cc[k]; q0 = f0 + dd[k][0]; q1 = f1 + dd[k][1]; }
          if (q0 == f0 && q1 == f1) break;
        }
      }
      mv0 = q0; mv1 = q1;
      uint2 v = qpel8(qpel_src(sm, (q0 >> 2) - best0 + 1, (q1 >> 2) - best1 + 1, q0 & 3, q1 & 3));
      *(uint2*)&sm.pred_y[(lane >> 1) * 16 + (lane & 1) * 8] = v;
      __syncwarp();
    }
  }

  // 3. intra 16x16 when the inter prediction is poor (enc.rs:3121-3156)
  uint32_t inter_satd = 0;
  if (lane < 16) {
    int bx = lane & 3, by = lane >> 2;
    inter_satd = satd4(&sm.src_y[by * 64 + bx * 4], 16, &sm.pred_y[by * 64 + bx * 4], 16);
  }
  inter_satd = wsum(inter_satd) >> 1;
  uint32_t inter_cost = inter_satd + lambda * (se_bits(mv0 - mvp0) + se_bits(mv1 - mvp1) + 1);
  if (inter_satd > 24 * lambda) {
    int tl, ctl[2];
    load_edges(c, sm, false, tl, ctl);
    bool ht = mby > 0, hl = mbx > 0;
    uint32_t i16c;
    int i16m = analyse_i16(sm, ht, hl, tl, &i16c);
    if (i16c + lambda * 8 < inter_cost) {
      code_i16(c, sm, i16m, ht, hl, tl, ctl);
      return;
    }
  }

  // 4. P_L0_16x16 residual (enc.rs:3158-3190)
  mc_chroma8(sd.ref_u, sd.ref_v, fp.stride_c, mbx, mby, mv0, mv1, sm);
  uint32_t nz_lane;
  int cbp4 = luma4x4_inter(qp, sm, &nz_lane);
  int cbpl = cbp4;
  bool use8 = false;
  if (fp.t8x8 && cbp4) {
    uint32_t nnz4 = 0;  // nonzero levels of the 4x4 coding: four words (eight levels) per lane
#pragma unroll
    for (int k = 0; k < 4; k++) {
      uint32_t w = ((const uint32_t*)sm.coef)[lane + 32 * k];
      nnz4 += ((w & 0xffffu) != 0) + ((w >> 16) != 0);
    }
    nnz4 = wsum(nnz4);
    uint32_t nnz8;
    int cbp8 = luma8x8_inter(qp, sm, &nnz8);
    if (nnz8 <= nnz4) { use8 = true; cbpl = cbp8; }
  }
  uint32_t ac_any[2], ac_sc[2];
  chroma_quant(qpc, false, sm, ac_any, ac_sc);
  // drop a plane's AC levels when nearly empty (enc.rs:2095)
  bool drop_u = ac_any[0] && ac_sc[0] < 7, drop_v = ac_any[1] && ac_sc[1] < 7;
  if (lane < 8) {
    bool d = (lane >> 2) ? drop_v : drop_u;
    if (d)
#pragma unroll
      for (int i = 0; i < 16; i++) sm.ccoef[lane * 16 + i] = 0;
  }
  __syncwarp();
  bool acu = ac_any[0] && !drop_u, acv = ac_any[1] && !drop_v;
  int cbpc = (acu || acv) ? 2 : (chroma_dc_any(sm) ? 1 : 0);
  if (cbpl == 0 && cbpc == 0 && mv0 == ps0 && mv1 == ps1) {
    code_skip(c, sm, mv0, mv1);
    return;
  }
  // code_inter (enc.rs:3196)
  rg_mb_out* rec = c.sd->rec + c.mb;
  bool t8flag = use8 && cbpl != 0;
  uint16_t nzm;
  if (use8) {
    int b = lane >> 3, q = lane & 7;  // column q of block b, each level to its zig-zag slot
#pragma unroll 1
    for (int y = 0; y < 8; y++) rec->luma[b * 64 + zigzag8(y, q)] = sm.coef8[b * 64 + y * 8 + q];
    nzm = 0;
    for (int k = 0; k < 4; k++) if ((cbpl >> k) & 1) nzm |= (uint16_t)(0xF << (4 * k));
  } else {
    nzm = record_luma4x4(rec, sm);
  }
  if (lane < 16) { rec->luma_dc[lane] = 0; rec->i4_modes[lane] = 2; }
  record_chroma(rec, sm, cbpc);
  if (lane == 0) {
    record_header(rec, RG_MB_P_L0_16X16, 0, 0, cbpl | (cbpc << 4), t8flag, qp, mv0, mv1, mv0 - mvp0, mv1 - mvp1, nzm);
    write_info(c, t8flag ? kFlagT8 : 0, cbpl, mv0, mv1, 0, nzm, nullptr);
  }
  // reconstruction
  if (use8) {
    recon_luma8x8(sm, qp, cbpl);
  } else if (cbpl) {
    recon_luma4x4(sm, qp, cbpl);
  }
  __syncwarp();
  chroma_recon(qpc, cbpc, sm);
  store_recon(c, sm.pred_y, sm);
  (void)nz_lane;
}

// ---------------------------------------------------------------------------------------------
// The full-search and learned forms' analysis (neither exists in the reference).
#include "search_form.cuh"

// ---------------------------------------------------------------------------------------------
// Deblocking of one macroblock (enc.rs:3776 deblock, h264_deblock.rs:71,187): vertical edges
// then horizontal ones, on a shared-memory tile with 4 samples of the left / top neighbours.
struct EdgeParams {
  int alpha, beta, tc0[4];
  bool strong, on;
};
__device__ __forceinline__ EdgeParams edge_params(int qp, const int* bs) {
  EdgeParams e;
  int ia = qp < 0 ? 0 : (qp > 51 ? 51 : qp);
  e.alpha = c_alpha[ia];
  e.beta = c_beta[ia];
  e.on = e.alpha != 0 && e.beta != 0;
  for (int k = 0; k < 4; k++) {
    int b = bs[k] > 4 ? 4 : bs[k];
    e.tc0[k] = b == 0 ? -1 : (b == 4 ? 0 : c_tc0[ia][b - 1]);
  }
  e.strong = bs[0] == 4;
  return e;
}
__device__ __forceinline__ void luma_line(uint8_t* o, int xs, const EdgeParams& e, int tc0) {
  if (!e.strong && tc0 < 0) return;
  int p0 = o[-xs], q0 = o[0], p1 = o[-2 * xs], q1 = o[xs];
  if (abs(p0 - q0) >= e.alpha || abs(p1 - p0) >= e.beta || abs(q1 - q0) >= e.beta) return;
  int p2 = o[-3 * xs], q2 = o[2 * xs];
  bool ap = abs(p2 - p0) < e.beta, aq = abs(q2 - q0) < e.beta;
  if (!e.strong) {
    int tc = tc0 + ap + aq;
    int d = min(max((((q0 - p0) << 2) + (p1 - q1) + 4) >> 3, -tc), tc);
    o[-xs] = (uint8_t)clip255(p0 + d);
    o[0] = (uint8_t)clip255(q0 - d);
    if (ap) o[-2 * xs] = (uint8_t)(p1 + min(max((p2 + ((p0 + q0 + 1) >> 1) - (p1 << 1)) >> 1, -tc0), tc0));
    if (aq) o[xs] = (uint8_t)(q1 + min(max((q2 + ((p0 + q0 + 1) >> 1) - (q1 << 1)) >> 1, -tc0), tc0));
  } else {
    int p3 = o[-4 * xs], q3 = o[3 * xs];
    bool small = abs(p0 - q0) < ((e.alpha >> 2) + 2);
    if (ap && small) {
      o[-xs] = (uint8_t)((p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3);
      o[-2 * xs] = (uint8_t)((p2 + p1 + p0 + q0 + 2) >> 2);
      o[-3 * xs] = (uint8_t)((2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3);
    } else {
      o[-xs] = (uint8_t)((2 * p1 + p0 + q1 + 2) >> 2);
    }
    if (aq && small) {
      o[0] = (uint8_t)((p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2 + 4) >> 3);
      o[xs] = (uint8_t)((p0 + q0 + q1 + q2 + 2) >> 2);
      o[2 * xs] = (uint8_t)((2 * q3 + 3 * q2 + q1 + q0 + p0 + 4) >> 3);
    } else {
      o[0] = (uint8_t)((2 * q1 + q0 + p1 + 2) >> 2);
    }
  }
}
__device__ __forceinline__ void chroma_line(uint8_t* o, int xs, const EdgeParams& e, int tc0) {
  if (!e.strong && tc0 < 0) return;
  int p1 = o[-2 * xs], p0 = o[-xs], q0 = o[0], q1 = o[xs];
  if (abs(p0 - q0) >= e.alpha || abs(p1 - p0) >= e.beta || abs(q1 - q0) >= e.beta) return;
  if (e.strong) {
    o[-xs] = (uint8_t)((2 * p1 + p0 + q1 + 2) >> 2);
    o[0] = (uint8_t)((2 * q1 + q0 + p1 + 2) >> 2);
  } else {
    int tc = tc0 + 1;
    int d = min(max((((q0 - p0) << 2) + (p1 - q1) + 4) >> 3, -tc), tc);
    o[-xs] = (uint8_t)clip255(p0 + d);
    o[0] = (uint8_t)clip255(q0 - d);
  }
}
__device__ __forceinline__ int nz_at(uint16_t nz, int bx, int by) {
  int b = ((by >> 1) << 3) | ((bx >> 1) << 2) | ((by & 1) << 1) | (bx & 1);
  return (nz >> b) & 1;
}
// Boundary strengths of edge e in direction dir (0 vertical); returns false to skip the edge.
// kMv4 (search forms): the motion term compares the quadrant vectors on either side of each
// 4-sample segment (qm: this macroblock's, pm4: the neighbour's across edge 0), so the internal
// edge between partitions gets strength 1 where their vectors differ by 4 quarter samples.
template <bool kMv4>
__device__ bool edge_bs(const MbInfo& q, const MbInfo* p, int dir, int e, int* bs, const MbMv4* qm, const MbMv4* pm4) {
  bool qi = q.flags & kFlagIntra;
  bool pi = p ? (p->flags & kFlagIntra) : qi;
  if (qi || pi) {
    for (int k = 0; k < 4; k++) bs[k] = e == 0 ? 4 : 3;
    return true;
  }
  int coded[4];
  for (int k = 0; k < 4; k++) {
    if (dir == 0) coded[k] = nz_at(q.nz16, e, k) | (e == 0 ? nz_at(p->nz16, 3, k) : nz_at(q.nz16, e - 1, k));
    else coded[k] = nz_at(q.nz16, k, e) | (e == 0 ? nz_at(p->nz16, k, 3) : nz_at(q.nz16, k, e - 1));
  }
  if constexpr (!kMv4) {
    bool motion = false;
    if (e == 0) motion = q.ref != p->ref || abs(q.mv[0] - p->mv[0]) >= 4 || abs(q.mv[1] - p->mv[1]) >= 4;
    if (!coded[0] && !coded[1] && !coded[2] && !coded[3] && !motion) return false;
    for (int k = 0; k < 4; k++) bs[k] = coded[k] ? 2 : (motion ? 1 : 0);
    return true;
  } else {
    bool any = false;
    for (int k = 0; k < 4; k++) {
      int qq = dir == 0 ? (k >> 1) * 2 + (e >> 1) : (e >> 1) * 2 + (k >> 1);
      int pq = e == 0 ? (dir == 0 ? (k >> 1) * 2 + 1 : 2 + (k >> 1))
                      : (dir == 0 ? (k >> 1) * 2 + ((e - 1) >> 1) : ((e - 1) >> 1) * 2 + (k >> 1));
      const MbMv4* pmm = e == 0 ? pm4 : qm;
      bool motion = (e == 0 && q.ref != p->ref) || abs(qm->mv[qq][0] - pmm->mv[pq][0]) >= 4 ||
                    abs(qm->mv[qq][1] - pmm->mv[pq][1]) >= 4;
      bs[k] = coded[k] ? 2 : (motion ? 1 : 0);
      any |= bs[k] != 0;
    }
    return any;
  }
}
// Whether a search-form macroblock's quadrants share one vector.
__device__ __forceinline__ bool one_vector(const MbMv4& m) {
  const uint32_t* w = (const uint32_t*)&m;
  return w[0] == w[1] && w[0] == w[2] && w[0] == w[3];
}

template <bool kMv4>
__device__ __noinline__ void deblock_mb(const FrameParams& fp, const StreamDev& sd, int mbx, int mby, Smem& sm) {
  int lane = lane_id();
  int m = mby * fp.mb_w + mbx;
  MbInfo q = ld_info(&sd.info[m]);
  MbInfo lf, tp;
  bool hasl = mbx > 0, hast = mby > 0;
  if (hasl) lf = ld_info(&sd.info[m - 1]);
  if (hast) tp = ld_info(&sd.info[m - fp.mb_w]);
  auto quiet = [](const MbInfo& i) { return !(i.flags & kFlagIntra) && i.cbp_luma == 0; };
  MbMv4 qm, lm, tm;
  bool split = false;
  if constexpr (kMv4) {
    qm = sd.mv4[m];
    if (hasl) lm = sd.mv4[m - 1];
    if (hast) tm = sd.mv4[m - fp.mb_w];
    split = !one_vector(qm);
    const uint32_t qv = *(const uint32_t*)&qm;
    if (quiet(q) && !split && (!hasl || (quiet(lf) && one_vector(lm) && *(const uint32_t*)&lm == qv)) &&
        (!hast || (quiet(tp) && one_vector(tm) && *(const uint32_t*)&tm == qv)))
      return;
  } else {
    if (quiet(q) && (!hasl || (quiet(lf) && lf.mv[0] == q.mv[0] && lf.mv[1] == q.mv[1])) &&
        (!hast || (quiet(tp) && tp.mv[0] == q.mv[0] && tp.mv[1] == q.mv[1])))
      return;
  }
  // tiles: luma 20x20 at (x0-4, y0-4) stride 20 in win; chroma 12x12 each in hph / hpv
  uint8_t* ty = sm.win;
  uint8_t* tc[2] = {sm.hph, sm.hpv};
  const int x0 = mbx * 16, y0 = mby * 16, cx0 = mbx * 8, cy0 = mby * 8;
  for (int w = lane; w < 100; w += 32) {  // 20 rows x 5 words
    int r = w / 5, k = w % 5;
    if ((r < 4 && !hast) || (k == 0 && !hasl)) continue;
    *(uint32_t*)&ty[r * 20 + 4 * k] = ldcg_u32(sd.cur_y + (long)(y0 - 4 + r) * fp.stride_y + x0 - 4 + 4 * k);
  }
  for (int w = lane; w < 72; w += 32) {  // 2 planes x 12 rows x 3 words
    int p = w / 36, rem = w % 36, r = rem / 3, k = rem % 3;
    if ((r < 4 && !hast) || (k == 0 && !hasl)) continue;
    const uint8_t* P = p ? sd.cur_v : sd.cur_u;
    *(uint32_t*)&tc[p][r * 12 + 4 * k] = ldcg_u32(P + (long)(cy0 - 4 + r) * fp.stride_c + cx0 - 4 + 4 * k);
  }
  __syncwarp();
  bool intra = q.flags & kFlagIntra;
  bool internal = intra || q.cbp_luma != 0 || split;
  bool skip_odd = q.flags & kFlagT8;
  int qpq = q.qp, qpcq = chroma_qp(qpq);
  for (int dir = 0; dir < 2; dir++) {
    for (int e = 0; e < 4; e++) {
      const MbInfo* pm;
      if (e == 0) {
        if (dir == 0 ? !hasl : !hast) continue;
        pm = dir == 0 ? &lf : &tp;
      } else {
        if (!internal || ((e & 1) && skip_odd)) continue;
        pm = nullptr;
      }
      int bs[4];
      if (!edge_bs<kMv4>(q, pm ? pm : &q, dir, e, bs, &qm, dir == 0 ? &lm : &tm)) continue;
      int qpl, qpc;
      if (!pm) { qpl = qpq; qpc = qpcq; }
      else { qpl = (qpq + pm->qp + 1) >> 1; qpc = (qpcq + chroma_qp(pm->qp) + 1) >> 1; }
      EdgeParams el = edge_params(qpl, bs);
      if (lane < 16 && el.on) {
        if (dir == 0) luma_line(&ty[(4 + lane) * 20 + 4 + e * 4], 1, el, el.tc0[lane >> 2]);
        else luma_line(&ty[(4 + e * 4) * 20 + 4 + lane], 20, el, el.tc0[lane >> 2]);
      }
      if (!(e & 1) && lane >= 16) {
        EdgeParams ec = edge_params(qpc, bs);
        if (ec.on) {
          int j = lane - 16, p = j >> 3, k = j & 7;
          if (dir == 0) chroma_line(&tc[p][(4 + k) * 12 + 4 + e * 2], 1, ec, ec.tc0[k >> 1]);
          else chroma_line(&tc[p][(4 + e * 2) * 12 + 4 + k], 12, ec, ec.tc0[k >> 1]);
        }
      }
      __syncwarp();
    }
  }
  // write back the samples this macroblock filters (rows 0..15 x cols -4..15, rows -4..-1 x cols 0..15)
  for (int w = lane; w < 100; w += 32) {
    int r = w / 5, k = w % 5;
    if (r < 4 && k == 0) continue;
    if ((r < 4 && !hast) || (k == 0 && !hasl)) continue;
    *(uint32_t*)(sd.cur_y + (long)(y0 - 4 + r) * fp.stride_y + x0 - 4 + 4 * k) = *(const uint32_t*)&ty[r * 20 + 4 * k];
  }
  for (int w = lane; w < 72; w += 32) {
    int p = w / 36, rem = w % 36, r = rem / 3, k = rem % 3;
    if (r < 4 && k == 0) continue;
    if ((r < 4 && !hast) || (k == 0 && !hasl)) continue;
    uint8_t* P = p ? sd.cur_v : sd.cur_u;
    *(uint32_t*)(P + (long)(cy0 - 4 + r) * fp.stride_c + cx0 - 4 + 4 * k) = *(const uint32_t*)&tc[p][r * 12 + 4 * k];
  }
}

// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ int diag_first(const FrameParams& fp, int d) {
  int a = d - fp.mb_w + 1;
  return a > 0 ? (a + 1) >> 1 : 0;
}
__device__ __forceinline__ int diag_len(const FrameParams& fp, int d) {
  if (d < 0) return 0;
  int lo = diag_first(fp, d), hi = min(fp.mb_h - 1, d >> 1);
  return hi >= lo ? hi - lo + 1 : 0;
}

struct NoSearchSmem {};
template <int kForm>
using FormSmem = typename std::conditional<kForm != 0, SearchSmem, NoSearchSmem>::type;

template <int kForm>
__global__ void __launch_bounds__(32) wavefront_step_kernel(const __grid_constant__ FrameParams fp, const StreamDev* __restrict__ streams, int step) {
  __shared__ Smem sm;
  __shared__ FormSmem<kForm> ss;
  const StreamDev& sd = streams[blockIdx.y];
  int na = diag_len(fp, step);
  int nd = fp.deblock ? diag_len(fp, step - 3) : 0;
  int k = blockIdx.x;
  if (k < na) {
    int mby = diag_first(fp, step) + k, mbx = step - 2 * mby;
    Ctx c{&fp, &sd, mbx, mby, mby * fp.mb_w + mbx};
    if (sd.kind == RG_FRAME_IDR) {
      load_source(c, sm);
      if constexpr (kForm != 0) analyse_intra_mb_search(c, sm);
      else analyse_intra_mb(c, sm);
    } else {
      if constexpr (kForm != 0) analyse_p_mb_search(c, sm, ss, nullptr);
      else analyse_p_mb(c, sm, nullptr);
    }
  } else if (k - na < nd) {
    int d = step - 3;
    int mby = diag_first(fp, d) + (k - na), mbx = d - 2 * mby;
    deblock_mb<kForm != 0>(fp, sd, mbx, mby, sm);
  }
  (void)ss;
}

// Border extension (enc.rs:165 extend_borders) of the padding that takes its values from
// macroblock (a, b), once that macroblock is final: the left / right padding of its rows when it
// is the first / last of its row, and the padding above / below its columns when it is in the
// first / last row -- corners included, which come from the corner macroblocks. Applied to every
// macroblock of the picture this writes every padding sample exactly once, so a picture's
// padding is complete wherever the macroblocks it copies are final. One warp, 4-byte stores.
__device__ __noinline__ void extend_mb(const FrameParams& fp, const StreamDev& sd, int a, int b) {
  int lane = lane_id();
  bool left = a == 0, right = a == fp.mb_w - 1, top = b == 0, bottom = b == fp.mb_h - 1;
  if (!(left || right || top || bottom)) return;
  for (int plane = 0; plane < 3; plane++) {
    uint8_t* P = plane == 0 ? sd.cur_y : (plane == 1 ? sd.cur_u : sd.cur_v);
    int bw = plane ? 8 : 16;
    int w = fp.mb_w * bw, h = fp.mb_h * bw;
    int pad = plane ? kPadC : kPadY, stride = plane ? fp.stride_c : fp.stride_y;
    int lw = pad / 4;
    // columns owned by this macroblock, in 4-byte words relative to the padded row start
    int c_lo = left ? 0 : (pad + a * bw) / 4;
    int c_hi = right ? stride / 4 : (pad + (a + 1) * bw) / 4;
    // rows owned: its own rows, plus the padding above / below the picture
    int r_lo = top ? -pad : b * bw, r_hi = bottom ? h + pad : (b + 1) * bw;
    int ncol = c_hi - c_lo, n = (r_hi - r_lo) * ncol;
    for (int i = lane; i < n; i += 32) {
      int yy = r_lo + i / ncol, cw = c_lo + i % ncol;
      int xw = cw * 4 - pad;  // first picture column of this word
      bool in_rows = yy >= 0 && yy < h;
      if (in_rows && cw >= lw && cw < lw + w / 4) continue;  // picture sample: no copy
      int sy = min(max(yy, 0), h - 1);
      const uint8_t* srow = P + (long)sy * stride;
      uint32_t v;
      if (xw < 0) v = ldcg_u8(srow) * 0x01010101u;
      else if (xw >= w) v = ldcg_u8(srow + w - 1) * 0x01010101u;
      else v = ldcg_u32(srow + xw);
      *(uint32_t*)(P + (long)yy * stride + xw) = v;
    }
  }
}

// Persistent pipelined mode: F pictures of every stream in one launch. The work is cut into
// segments of `seg` consecutive macroblocks of one row -- analysis segments and deblocking
// segments -- listed by the host in the order they are expected to become ready (pipeline_task_
// list) and handed out by an atomic ticket. A warp only holds one short segment, so the resident
// warps cover the work that is about to be ready rather than whole rows far from it, and every
// wait is normally for a segment of a smaller ticket. Picture f+1 of a stream starts as soon as
// the part of picture f its search can reach is deblocked and border-extended.
struct PipeParams {
  int* ticket;
  int* error;
  int* ana;    // analysed macroblocks per row, descriptor d's rows from ana + d.rows_base
  int* db;     // deblocked macroblocks per row (the same layout); a macroblock's deblocking also
               // extends the padding of the macroblocks it makes final
  const int2* tasks;  // {descriptor, row << 16 | first macroblock << 1 | deblock}
  int n_tasks;
  int qbeg[3], qend[3];  // queue q = tasks[qbeg[q], qend[q]): 0 analysis, 1 deblocking, 2 IDR analysis
  int deblock_sms;    // SMs whose warps take queue 1 first
  int intra_sms;      // the next SMs, whose warps take queue 2 first
  int role_by_sm;     // 0: by block index instead (a grid too small to reach every SM)
  int seg;
  unsigned long long timeout_ns;
  int* rows_done;     // [descriptor] rows of a picture fully analysed
  int* ready;         // [descriptor] in mapped host memory (or null): seq once a picture's records are final
  int seq;
  int* host_err;      // mapped host memory: the error word as the launch ends (no copy to wait for)
  int* reach;         // [2] 1 + the largest reach of a reference wait beyond zero motion (rows, columns)
  // compact records (cwords null: none): row r of the launch (rows like ana) has a slot of crow
  // words at cwords + r * crow in mapped host memory and its size in bytes (or -1) at cbytes[r]
  uint32_t* cwords;
  int crow;
  int* cbytes;
};
__device__ __forceinline__ unsigned sm_id() {
  unsigned r;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(r));
  return r;
}

// Counts a picture's fully analysed row; the warp completing its last row tells the host that the
// picture's records are final. Each row's records were ordered before its count by the release
// chain of the row's segments; the acq_rel count gathers all rows, and the system-scope release
// store orders them before the flag the host polls.
__device__ __noinline__ void picture_row_done(int* rows_done, int* ready, int seq, int H) {
  if (lane_id() == 0) {
    int before = atom_add_acq_rel(rows_done, 1);
    if (before == H - 1) st_release_sys(ready, seq);
  }
  __syncwarp();
}

static_assert(sizeof(rg_mb_out) == 4 * kRecordWords, "a record is kRecordWords words");
// Staging of compact records in the warp's shared memory (its Smem, which no task reads before
// writing it): kStageWords words, flushed to host memory in 16-byte stores.
constexpr int kStageWords = 512;
static_assert(sizeof(Smem) >= 4 * kStageWords, "the staging buffer fits the warp's shared memory");
static_assert(kStageWords >= 2 * (kCompactMaskWords + kRecordWords), "a flush leaves room for a whole record");

// Writes the first n (a multiple of 4) staged words to dst + at (16-byte aligned) while they fit
// the slot of cap words (a multiple of 4), then moves the rest (< 4 words) to the front.
__device__ __noinline__ void flush_stage(uint32_t* stage, int n, int rest, uint32_t* dst, long long at, int cap) {
  const int lane = lane_id();
  __syncwarp();
  const uint4* s4 = reinterpret_cast<const uint4*>(stage);
  uint4* d4 = reinterpret_cast<uint4*>(dst + at);
  for (int c = lane; c < n / 4; c += 32)
    if (at + 4 * c + 4 <= cap) d4[c] = s4[c];
  __syncwarp();
  uint32_t v = lane < rest ? stage[n + lane] : 0u;
  __syncwarp();
  if (lane < rest) stage[lane] = v;
  __syncwarp();
}

// Compact records of row y, written by the warp that deblocked the row's last segment (after it
// published its progress) into the row's own slot (no row waits for another). A record's compact form is kCompactMaskWords mask words (bit j of
// mask word i: record word 32 i + j is nonzero), then its nonzero words in increasing order:
// zero-filling rebuilds the record exactly. The row's records are final: the deblocking warp
// acquired the row's analysis progress up to its end; they are read through L2. The
// words are gathered in shared memory and leave in whole 16-byte stores (word-sized stores to
// host memory made the row ~10x slower). Words past the slot are not written, and the row's size
// is then -1 (the host copies the picture's full records instead). The size is written before the
// row is counted towards the picture's flag. (Scalar arguments: a reference to the kernel's
// parameters would copy them to local memory.)
__device__ __noinline__ void compact_row(const rg_mb_out* rec, uint32_t* dst, int cap, int* bytes, int Wm,
                                         uint32_t* stage) {
  const int lane = lane_id();
  long long done = 0;  // words flushed (a multiple of 4)
  int sp = 0;          // words staged
  const uint32_t* src = reinterpret_cast<const uint32_t*>(rec);
  const unsigned below = (1u << lane) - 1u;
  for (int m0 = 0; m0 < Wm; m0 += 4) {
    // four records in flight, then their words into the stage
    uint32_t w[4][kCompactMaskWords];
#pragma unroll
    for (int k = 0; k < 4; k++)
#pragma unroll
      for (int i = 0; i < kCompactMaskWords; i++) {
        const int j = lane + 32 * i;
        w[k][i] = (m0 + k < Wm && j < kRecordWords) ? __ldcg(src + (size_t)(m0 + k) * kRecordWords + j) : 0u;
      }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      if (m0 + k >= Wm) break;
      if (sp + kCompactMaskWords + kRecordWords > kStageWords) {
        const int n = sp & ~3;
        flush_stage(stage, n, sp - n, dst, done, cap);
        done += n;
        sp -= n;
      }
      uint32_t mask = 0;
      int at = sp + kCompactMaskWords;
#pragma unroll
      for (int i = 0; i < kCompactMaskWords; i++) {
        const unsigned b = __ballot_sync(FULL, w[k][i] != 0u);
        if (lane == i) mask = b;
        if (w[k][i] != 0u) stage[at + __popc(b & below)] = w[k][i];
        at += __popc(b);
      }
      if (lane < kCompactMaskWords) stage[sp + lane] = mask;
      sp = at;
    }
  }
  // the tail, padded to whole 16-byte stores (the padding stays inside the slot: cap is a
  // multiple of 4 and the row's words, when they fit, are at most cap)
  const long long total = done + sp;
  flush_stage(stage, (sp + 3) & ~3, 0, dst, done, cap);
  if (lane == 0) *bytes = total <= cap ? (int)(total * 4) : -1;
  // the row's words and size reach host memory before the row is counted towards the flag
  __threadfence_system();
  __syncwarp();
}

// At least 16 warps per SM: up to 128 registers a thread, so nothing spills (4.5 % faster than 20,
// which held it to 96 registers with spills).
template <int kForm>
__global__ void __launch_bounds__(32, 16) pipeline_kernel(const __grid_constant__ FrameGroups fg, const StreamDev* __restrict__ sds, PipeParams pp) {
  __shared__ Smem sm;
  __shared__ FormSmem<kForm> ss;
  const int lane = lane_id();
  // Warps on the first deblock_sms SMs take deblocking segments first, on the next intra_sms SMs
  // segments of IDR pictures (the critical path of a GOP), and the others the remaining analysis
  // (each SM then runs a smaller code footprint); a warp whose queue is empty takes from the next.
  int role = 0;
  if (pp.role_by_sm) {
    int id = (int)sm_id();
    role = id < pp.deblock_sms ? 1 : (id < pp.deblock_sms + pp.intra_sms ? 2 : 0);
  } else {
    int k = blockIdx.x % 9;
    role = k == 0 ? 1 : (k == 1 ? 2 : 0);
  }
  bool empty[3] = {pp.qbeg[0] >= pp.qend[0], pp.qbeg[1] >= pp.qend[1], pp.qbeg[2] >= pp.qend[2]};
  int reach_y = 0, reach_x = 0;  // this warp's, published once as it exits
  while (true) {
    int t = -1;
    if (lane == 0) {
      for (int k = 0; k < 3 && t < 0; k++) {
        int q = role + k >= 3 ? role + k - 3 : role + k;
        if (empty[q]) continue;
        int v = pp.qbeg[q] + atomicAdd(pp.ticket + (q ? q + 1 : 0), 1);
        if (v < pp.qend[q]) t = v; else empty[q] = true;
      }
    }
    t = __shfl_sync(FULL, t, 0);
    if (t < 0) break;
    if (__shfl_sync(FULL, lane == 0 ? ld_relaxed(pp.error) : 0, 0)) break;
    int2 task = __ldg(pp.tasks + t);
    int ps = task.x;
    const StreamDev& sd = sds[ps];
    const FrameParams& fp = fg.g[sd.group];  // the descriptor's picture size
    const int H = fp.mb_h, Wm = fp.mb_w;
    int y = task.y >> 16, x0 = (task.y >> 1) & 0x7fff, x1 = min(x0 + pp.seg, Wm);
    bool ana = (task.y & 1) == 0;
    int* ana_rows = pp.ana + sd.rows_base;
    int* db_rows = pp.db + sd.rows_base;
    bool failed = false;
    if (ana) {
      PipeWait pw;
      bool has_prev = sd.prev_ps >= 0 && sd.kind == RG_FRAME_P;
      if (has_prev) {
        const int pb = sds[sd.prev_ps].rows_base;
        pw.ana_prev = pp.ana + pb;
        pw.db_prev = pp.db + pb;
      }
      pw.error = pp.error;
      pw.timeout_ns = pp.timeout_ns;
      pw.seen_ana = 0;
      pw.db_row = -1;
      pw.seen_db = 0;
      pw.reach_y = reach_y;
      pw.reach_x = reach_x;
      pw.failed = false;
      int seen_own = 0, seen_up = 0;
      // the previous segment of this row, then per macroblock the row above two ahead
      if (x0 > 0 && !wait_seen(ana_rows + y, x0, seen_own, pp.error, pp.timeout_ns)) failed = true;
      for (int x = x0; x < x1 && !failed; x++) {
        if (y > 0 && !wait_seen(ana_rows + y - 1, min(x + 2, Wm), seen_up, pp.error, pp.timeout_ns)) {
          failed = true;
          break;
        }
        Ctx c{&fp, &sd, x, y, y * Wm + x};
        if (sd.kind == RG_FRAME_IDR) {
          load_source(c, sm);
          if constexpr (kForm != 0) analyse_intra_mb_search(c, sm);
          else analyse_intra_mb(c, sm);
        } else {
          if constexpr (kForm != 0) analyse_p_mb_search(c, sm, ss, has_prev ? &pw : nullptr);
          else analyse_p_mb(c, sm, has_prev ? &pw : nullptr);
          if (pw.failed) { failed = true; break; }
        }
        publish(ana_rows + y, x + 1);
      }
      // (with compact records, the row is counted once its deblocking warp has compacted it)
      int* const rdy = sd.ready ? sd.ready : (pp.ready ? pp.ready + ps : nullptr);
      if (!failed && x1 == Wm && rdy && !pp.cwords) picture_row_done(pp.rows_done + ps, rdy, pp.seq, H);
      reach_y = pw.reach_y;
      reach_x = pw.reach_x;
    } else {
      int seen_own = 0, seen_a0 = 0, seen_a1 = 0, seen_up = 0;
      if (x0 > 0 && !wait_seen(db_rows + y, x0, seen_own, pp.error, pp.timeout_ns)) failed = true;
      for (int x = x0; x < x1 && !failed; x++) {
        if (!wait_seen(ana_rows + y, min(x + 2, Wm), seen_a0, pp.error, pp.timeout_ns) ||
            (y + 1 < H && !wait_seen(ana_rows + y + 1, min(x + 1, Wm), seen_a1, pp.error, pp.timeout_ns)) ||
            (y > 0 && !wait_seen(db_rows + y - 1, min(x + 2, Wm), seen_up, pp.error, pp.timeout_ns))) {
          failed = true;
          break;
        }
        deblock_mb<kForm != 0>(fp, sd, x, y, sm);
        // Macroblock (x, y - 1) is final now: (x + 1, y - 1) was deblocked before this one. In
        // the last row, so is (x - 1, y), and the last macroblock is final after its own pass.
        __syncwarp();
        if (y >= 1) extend_mb(fp, sd, x, y - 1);
        if (y == H - 1) {
          if (x >= 1) extend_mb(fp, sd, x - 1, y);
          if (x == Wm - 1) extend_mb(fp, sd, x, y);
        }
        publish(db_rows + y, x + 1);
      }
      // Compact records of the row, by the warp that deblocked its last segment: on the deblocking
      // SMs and after the row's deblocking progress was published, so neither the analysis
      // wavefront nor the deblocking chain waits for it (done at the end of the row's analysis it
      // slowed the launch ~5 %). Its wait for the analysis of the row up to its end ordered every
      // record of the row before it.
      if (!failed && x1 == Wm && pp.cwords) {
        const long long r = (long long)sd.rows_base + y;
        compact_row(sd.rec + (size_t)y * Wm, pp.cwords + r * pp.crow, pp.crow, pp.cbytes + r, Wm,
                    reinterpret_cast<uint32_t*>(&sm));
        int* const rdy = sd.ready ? sd.ready : (pp.ready ? pp.ready + ps : nullptr);
        if (rdy) picture_row_done(pp.rows_done + ps, rdy, pp.seq, H);
      }
    }
    if (failed) break;
  }
  if (lane == 0 && reach_y) {
    atomicMax(pp.reach, reach_y);
    atomicMax(pp.reach + 1, reach_x);
  }
  (void)ss;
}

// The launch's error word (and the reach its reference waits saw) into mapped host memory, queued
// after the launch (a kernel, not a copy: a device-to-host copy waiting for a launch would stall
// later copies of the context).
__global__ void error_to_host_kernel(const int* error, const int* reach, int* host_err, int* host_reach) {
  if (host_reach) {
    host_reach[0] = reach[0];
    host_reach[1] = reach[1];
  }
  st_release_sys(host_err, *error);
}

// Border extension (enc.rs:165 extend_borders): every padding sample takes the value of the
// nearest picture sample. One thread per 16-byte chunk of a padded row.
__global__ void extend_borders_kernel(FrameParams fp, const StreamDev* __restrict__ streams) {
  const StreamDev& sd = streams[blockIdx.z / 3];
  int plane = blockIdx.z % 3;
  int w = plane ? fp.mb_w * 8 : fp.mb_w * 16, h = plane ? fp.mb_h * 8 : fp.mb_h * 16;
  int pad = plane ? kPadC : kPadY, stride = plane ? fp.stride_c : fp.stride_y;
  uint8_t* P = plane == 0 ? sd.cur_y : (plane == 1 ? sd.cur_u : sd.cur_v);
  int chunks = stride / 16;
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  int rows = h + 2 * pad;
  if (idx >= rows * chunks) return;
  int ry = idx / chunks, cx = (idx % chunks) * 16;  // padded coordinates
  int y = ry - pad;
  int xs = cx - pad;
  bool row_inside = y >= 0 && y < h;
  if (row_inside && xs >= 0 && xs + 16 <= w) return;  // all interior
  int sy = min(max(y, 0), h - 1);
  const uint8_t* srow = P + (long)sy * stride;
  uint8_t* drow = P + (long)y * stride;
  for (int k = 0; k < 16; k++) {
    int x = xs + k;
    if (row_inside && x >= 0 && x < w) continue;
    drow[x] = srow[min(max(x, 0), w - 1)];
  }
}

}  // namespace

void upload_tables() {
  using namespace tables;
  cudaMemcpyToSymbol(c_lambda, kLambda, sizeof(kLambda));
  cudaMemcpyToSymbol(c_dec4, kDecimate4, sizeof(kDecimate4));
  uint8_t d8[64] = {0};
  for (int i = 0; i < 24; i++) d8[i] = kDecimate8[i];
  cudaMemcpyToSymbol(c_dec8, d8, sizeof(d8));
  cudaMemcpyToSymbol(c_scan4, kScan4, sizeof(kScan4));
  cudaMemcpyToSymbol(c_scan8, kScan8, sizeof(kScan8));
  cudaMemcpyToSymbol(c_mf4, kMf4, sizeof(kMf4));
  cudaMemcpyToSymbol(c_dq4, kDq4, sizeof(kDq4));
  cudaMemcpyToSymbol(c_mf8, kMf8, sizeof(kMf8));
  cudaMemcpyToSymbol(c_dq8, kDq8, sizeof(kDq8));
  cudaMemcpyToSymbol(c_cqp, kChromaQp, sizeof(kChromaQp));
  cudaMemcpyToSymbol(c_alpha, kAlpha, sizeof(kAlpha));
  cudaMemcpyToSymbol(c_beta, kBeta, sizeof(kBeta));
  cudaMemcpyToSymbol(c_tc0, kTc0, sizeof(kTc0));
  uint16_t taps[9 * 16];
  for (int m = 0; m < 9; m++)
    for (int q = 0; q < 16; q++) {
      int t = i4_tap(m, q & 3, q >> 2), i = t & 0xff;
      taps[m * 16 + q] = (uint16_t)(i | (i + 1 < 15 ? i + 1 : 15) << 4 | (i + 2 < 15 ? i + 2 : 15) << 8 | (t >> 8) << 12);
    }
  cudaMemcpyToSymbol(g_i4tap, taps, sizeof(taps));
}

int wavefront_steps(const FrameParams& fp) {
  int diags = (fp.mb_w - 1) + 2 * (fp.mb_h - 1) + 1;
  return diags + (fp.deblock ? 3 : 0);
}

static int max_diag_len(const FrameParams& fp) {
  int best = 0;
  int diags = (fp.mb_w - 1) + 2 * (fp.mb_h - 1) + 1;
  for (int d = 0; d < diags; d++) {
    int a = d - fp.mb_w + 1;
    int lo = a > 0 ? (a + 1) >> 1 : 0, hi = fp.mb_h - 1 < (d >> 1) ? fp.mb_h - 1 : (d >> 1);
    if (hi - lo + 1 > best) best = hi - lo + 1;
  }
  return best;
}

void launch_wavefront_step(const FrameParams& fp, const StreamDev* d_streams, int step, cudaStream_t st, int form) {
  dim3 grid(2 * max_diag_len(fp), fp.n_streams);
  if (form) wavefront_step_kernel<1><<<grid, 32, 0, st>>>(fp, d_streams, step);
  else wavefront_step_kernel<0><<<grid, 32, 0, st>>>(fp, d_streams, step);
}

int pipeline_sms(int device) {
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return sms;
}

// Resident warps of the pipelined mode: sixteen per SM (fewer when they do not fit). More warps
// overlap more of each other's waits, until the SM's front end saturates and every macroblock on
// the critical path slows (measured on B200, 1080p 8 x 15 pictures, launch time: 7 per SM
// 62.9 ms, 8 61.0, 10 59.1, 12 57.4, 14 56.0, 16 55.8, 18 56.2, 20-21 56.3).
int pipeline_grid(int device, int form) {
  int per_sm = 0;
  if (form) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pipeline_kernel<1>, 32, 0);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pipeline_kernel<0>, 32, 0);
  return (per_sm < 16 ? per_sm : 16) * pipeline_sms(device);
}

// Work list of the pipelined mode, written to `tasks` (pipeline_task_count entries): every
// analysis and deblocking segment of every picture and stream, ordered by a key of the
// macroblock-time it can start -- a = max(seg, 2) per row, 1 per column, lag per picture:
//   analysis of row y from column x0:    a * y + x0 + lag * f
//   deblocking of row y from column x0:  a * (y + 1) + x0 + 1 + lag * f
// and, at equal keys, by picture, role (analysis first), stream and row. Every macroblock of a
// segment depends only on segments of a smaller key or of an equal key earlier in that order
// (the row above two macroblocks ahead lies in a segment of key <= a * (y - 1) + x0 + seg; the
// deblocking of (x, y) needs the analysis of (x + 1, y) and (x, y + 1) and the deblocking of
// (x + 1, y - 1)), so warps taking tickets in order never wait for an untaken segment of the same
// picture. The wait for the reference picture depends on the motion vectors: a search whose
// window reaches r macroblocks beyond the co-located ones (r = 0 for zero motion) waits for a
// smaller key when lag >= a * (4 + r) + seg + r + 3. lag <= 0 takes r = 4 (about 64 samples).
size_t pipeline_task_count(const FrameParams& fp, int frames, int seg) {
  size_t segs = (size_t)(fp.mb_w + seg - 1) / seg;
  return 2 * (size_t)frames * fp.n_streams * fp.mb_h * segs;
}

size_t pipeline_task_list(const FrameParams& fp, int frames, int lag, int seg, bool split, const int32_t* kinds,
                          int2* tasks, int qbeg[3], int qend[3], uint32_t* keys) {
  int S = fp.n_streams, H = fp.mb_h, W = fp.mb_w;
  int segs = (W + seg - 1) / seg, a = seg > 2 ? seg : 2;
  if (lag <= 0) lag = a * 8 + seg + 7;
  auto key = [&](int f, int role, int y, int k) {
    return (size_t)a * (y + role) + (size_t)k * seg + role + (size_t)lag * f;
  };
  // queue of a segment: deblocking (1) when split, analysis of an IDR picture (2) when kinds are
  // given, else 0; each queue occupies its own range of keys, so each is in key order
  auto queue = [&](int f, int s, int role) {
    if (role) return split ? 1 : 0;
    return kinds && kinds[f * S + s] == RG_FRAME_IDR ? 2 : 0;
  };
  size_t n_keys1 = key(frames - 1, 1, H - 1, segs - 1) + 1, n_keys = 3 * n_keys1;
  auto slot = [&](int f, int s, int role, int y, int k) { return key(f, role, y, k) + queue(f, s, role) * n_keys1; };
  std::vector<size_t> start(n_keys + 1, 0);
  for (int f = 0; f < frames; f++)
    for (int role = 0; role < 2; role++)
      for (int s = 0; s < S; s++)
        for (int y = 0; y < H; y++)
          for (int k = 0; k < segs; k++) start[slot(f, s, role, y, k) + 1]++;
  for (size_t i = 0; i < n_keys; i++) start[i + 1] += start[i];
  for (int q = 0; q < 3; q++) {
    qbeg[q] = (int)start[q * n_keys1];
    qend[q] = (int)start[(q + 1) * n_keys1];
  }
  // placed in (picture, role, stream, row, segment) order within a key: a stable counting sort
  for (int f = 0; f < frames; f++)
    for (int role = 0; role < 2; role++)
      for (int s = 0; s < S; s++)
        for (int y = 0; y < H; y++)
          for (int k = 0; k < segs; k++) {
            size_t at = start[slot(f, s, role, y, k)]++;
            tasks[at] = make_int2(f * S + s, (y << 16) | ((k * seg) << 1) | role);
            if (keys) keys[at] = (uint32_t)key(f, role, y, k);
          }
  return pipeline_task_count(fp, frames, seg);
}

void launch_pipeline(const FrameGroups& fg, const StreamDev* d_streams, int n_desc, int total_rows, int* counters,
                     const int2* d_tasks, size_t n_tasks, const int qbeg[3], const int qend[3], int deblock_sms,
                     int intra_sms, int sms, int seg, int grid, unsigned long long timeout_ns, int* ready, int seq,
                     int* host_err, int* host_reach, cudaStream_t st, int form, const CompactOut* co) {
  PipeParams pp;
  pp.ticket = counters;
  pp.error = counters + 1;
  pp.ana = counters + 4;
  pp.db = pp.ana + total_rows;
  pp.tasks = d_tasks;
  pp.n_tasks = (int)n_tasks;
  for (int q = 0; q < 3; q++) {
    pp.qbeg[q] = qbeg[q];
    pp.qend[q] = qend[q];
  }
  pp.deblock_sms = deblock_sms;
  pp.intra_sms = intra_sms;
  pp.role_by_sm = grid >= sms;
  pp.seg = seg;
  pp.timeout_ns = timeout_ns;
  pp.rows_done = pp.db + total_rows;
  pp.ready = ready;
  pp.seq = seq;
  pp.host_err = host_err;
  pp.reach = pp.rows_done + n_desc;
  pp.cwords = co ? co->words : nullptr;
  pp.crow = co ? co->row_words : 0;
  pp.cbytes = co ? co->row_bytes : nullptr;
  int g = grid < pp.n_tasks ? grid : pp.n_tasks;
  if (form) pipeline_kernel<1><<<g, 32, 0, st>>>(fg, d_streams, pp);
  else pipeline_kernel<0><<<g, 32, 0, st>>>(fg, d_streams, pp);
  if (host_err) error_to_host_kernel<<<1, 1, 0, st>>>(pp.error, pp.reach, host_err, host_reach);
}

void launch_error_to_host(const int* counters, int n_desc, int total_rows, int* host_err, int* host_reach,
                          cudaStream_t st) {
  const int* reach = counters + 4 + 2 * (size_t)total_rows + n_desc;
  error_to_host_kernel<<<1, 1, 0, st>>>(counters + 1, reach, host_err, host_reach);
}

size_t pipeline_counter_ints(int total_rows, int n_desc) { return 4 + 2 * (size_t)total_rows + n_desc + 2; }

size_t pipeline_counter_ints(const FrameParams& fp, int frames) {
  return pipeline_counter_ints(frames * fp.n_streams * fp.mb_h, frames * fp.n_streams);
}

void launch_extend_borders(const FrameParams& fp, const StreamDev* d_streams, cudaStream_t st) {
  int rows = fp.mb_h * 16 + 2 * kPadY;
  int chunks = fp.stride_y / 16;
  int threads = 256;
  dim3 grid((rows * chunks + threads - 1) / threads, 1, 3 * fp.n_streams);
  extend_borders_kernel<<<grid, threads, 0, st>>>(fp, d_streams);
}

}  // namespace rg
