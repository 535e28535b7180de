// The learned form's candidate network (no counterpart in the reference): a small CNN that reads
// each macroblock of a picture with a 4-sample border (24x24 luma of the picture, and the same
// window of the previous picture, as two channels) and predicts the partition types, the intra
// 4x4 modes and an offset of the integer search's centre that the learned analysis form tries.
//
//   x (2 x 24 x 24, (sample - 128) / 64)
//   conv 3x3 2 -> 32, ReLU (22 x 22); conv 3x3 32 -> 32, ReLU (20 x 20); conv 3x3 32 -> 32, ReLU (18 x 18)
//   g   = mean of the 18 x 18 map (32);   f_b = mean of 4x4 block b's 4 x 4 area of the map (32)
//   partition logits = Wp g + bp (4);  search offset = Wm g + bm (2, in units of 16 quarter samples)
//   intra 4x4 logits of block b = Wi f_b + bi (9)
//
// Inference (cnn_infer_kernel): BF16 implicit-GEMM convolutions on the 5th-generation tensor cores
// (tcgen05.mma, accumulators in tensor memory), two CTAs per SM, each a strip of two macroblocks
// per step: every activation map of the strip is stored with one row stride, so the 3x3 taps of a
// 128-position tile are the same K-major operand shifted by whole rows of 16 bytes, and each tap is
// one descriptor of the map -- no im2col copy. The epilogue adds the bias, applies the ReLU and
// stores the next layer's BF16 operand over its input; the heads run on the CUDA cores and write
// the hints. While one CTA's epilogue runs, the other's MMAs can.
// Training (cnn_train_*): the same network in f32 on the CUDA cores -- forward, the losses, the
// backward pass and Adam -- on per-macroblock crops.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/ragdoll_cuda.h"

namespace rg {
void set_last_error(const char* msg);
}

namespace {

constexpr int C = 32;
// parameter offsets (f32, the order of rg_net_params)
constexpr int kW1 = 0, kB1 = kW1 + C * 2 * 9, kW2 = kB1 + C, kB2 = kW2 + C * C * 9, kW3 = kB2 + C,
              kB3 = kW3 + C * C * 9, kWp = kB3 + C, kBp = kWp + 4 * C, kWm = kBp + 4, kBm = kWm + 2 * C,
              kWi = kBm + 2, kBi = kWi + 9 * C, kParams = kBi + 9;
constexpr int kLogits = 4 + 2 + 16 * 9;  // per macroblock: partition, offset, intra 4x4

__device__ __forceinline__ float pix_norm(uint8_t v) { return ((float)v - 128.0f) * (1.0f / 64.0f); }

// ---------------------------------------------------------------------------------------------
// Inference on the tensor cores. Two CTAs per SM, each a strip of two macroblocks at a time; one
// activation buffer per CTA holds every map of its strip in turn (the input in plane 0, then each
// layer's output over its input: a layer's epilogue starts once all its MMAs have completed).
constexpr int kStripMbs = 2;
constexpr int kThreads = 256;  // 8 warps; warps w and w + 4 share TMEM lanes 32 (w % 4)..
constexpr int kCtasPerSm = 2;
constexpr int kRow = 16 * kStripMbs + 8;  // row stride (positions) of every map of a strip: 40
constexpr int kTiles1 = (22 * kRow + 127) / 128, kTiles2 = (20 * kRow + 127) / 128, kTiles3 = (18 * kRow + 127) / 128;
constexpr int kTap = 2 * kRow + 2;  // reach of the last tap
constexpr int kPosBuf = ((kTiles1 * 128 + kTap > kTiles2 * 128 + kTap ? kTiles1 * 128 + kTap : kTiles2 * 128 + kTap) +
                         kThreads - 1) / kThreads * kThreads;  // positions of the buffer
static_assert(kPosBuf >= kTiles1 * 128 + kTap + 1 && kPosBuf >= kTiles3 * 128 + kTap,
              "tap reach (conv1's last pair one position further) and outputs fit the buffer");
static_assert(kPosBuf >= 24 * kRow, "the input map fits plane 0");
static_assert(kTiles1 * 32 <= 256, "accumulators of one layer fit the CTA's 256 tensor-memory columns");
static_assert(kStripMbs * 4 <= kThreads / 32, "pooling: a warp per (macroblock, 8-channel plane)");
// shared memory (bytes): the buffer (4 planes of 8 channels) | B operands | the rest
constexpr int kPlane = kPosBuf * 16;
constexpr int kOffBuf = 0, kOffB = kOffBuf + 4 * kPlane;
constexpr int kB1Mmas = 5, kBMmas = 18;  // conv1: taps paired; conv2/3: 9 taps x 2 channel halves
constexpr int kOffB2 = kOffB + kB1Mmas * 1024, kOffB3 = kOffB2 + kBMmas * 1024, kOffMisc = kOffB3 + kBMmas * 1024;
struct InferMisc {
  float bias[3][C];
  float head[kParams - kWp];   // Wp bp Wm bm Wi bi
  float pool[kStripMbs][17][C];  // per macroblock: the 18 x 18 mean, then the 16 block means
  uint64_t mbar;
  uint32_t tmem;
  int strip;
};
constexpr int kSmemInfer = kOffMisc + (int)sizeof(InferMisc);
static_assert(kSmemInfer <= 233472 / kCtasPerSm - 1024, "two CTAs' shared memory fit an SM");

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
// Shared-memory matrix descriptor, K-major without swizzle: 8-row core matrices of 16-byte rows,
// sbo between 8-row groups, lbo between the two 8-element halves of K (sm100 version 1).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}
// kind::f16 instruction descriptor: BF16 A and B (K-major), F32 accumulator, M = 128, N = 32.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(32 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void umma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// Waits for the mbarrier's phase `parity` to complete; false after ~4 M polls (the error path).
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity) {
  uint32_t a = smem_u32(mbar);
  for (int i = 0; i < (1 << 22); i++) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\tselp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
// 32 consecutive columns of this thread's lane (one accumulator tile).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,"
      "%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// The pictures one launch reads, and where the hints go.
struct InferJob {
  const uint8_t* cur;   // luma of the picture (display size)
  const uint8_t* prev;  // luma of the previous picture (the picture itself for an IDR picture)
  rg_mb_hint* hints;    // mb_w * mb_h hints
  float* logits;        // mb_w * mb_h * kLogits, or null
};
struct InferParams {
  const InferJob* jobs;
  int n_jobs, width, height, stride, mb_w, mb_h, strips_per_row;
  const __nv_bfloat16* bops;  // B operands of the three layers in their shared-memory layout
  const float* params;        // f32 parameters (biases and heads)
  int* counter;               // strip ticket
  int* error;                 // set when a wait on the tensor cores gives up
  int part_k, i4_k;           // hint policy: candidates kept at most,
  float part_margin, i4_margin;  // and only those within this logit margin of the best
};

// The candidates of n logits as a bit mask: the best, then the next ones in logit order (the lower
// index on ties) up to k in all, each only while its logit is at least the best's minus `margin`.
template <int N>
__device__ __forceinline__ uint32_t topk_mask(const float (&l)[N], int k, float margin) {
  uint32_t m = 0;
  float top = 0.0f;
#pragma unroll
  for (int r = 0; r < N; r++) {
    if (r >= k) break;
    int best = -1;
    float bv = 0.0f;
#pragma unroll
    for (int i = 0; i < N; i++)  // constant indices: the logits stay in registers
      if (!((m >> i) & 1) && (best < 0 || l[i] > bv)) {
        best = i;
        bv = l[i];
      }
    if (r == 0) top = bv;
    else if (bv < top - margin) break;
    m |= 1u << best;
  }
  return m;
}

__global__ void __launch_bounds__(kThreads, kCtasPerSm) cnn_infer_kernel(InferParams ip) {
  extern __shared__ __align__(1024) uint8_t smem[];
  InferMisc& ms = *reinterpret_cast<InferMisc*>(smem + kOffMisc);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint8_t* buf = smem + kOffBuf;
  // B operands, biases and heads once per CTA
  for (int i = tid; i < (kB1Mmas + 2 * kBMmas) * 1024 / 16; i += kThreads)
    ((uint4*)(smem + kOffB))[i] = ((const uint4*)ip.bops)[i];
  for (int i = tid; i < 3 * C; i += kThreads) ms.bias[i / C][i % C] = ip.params[(i / C == 0 ? kB1 : (i / C == 1 ? kB2 : kB3)) + i % C];
  for (int i = tid; i < kParams - kWp; i += kThreads) ms.head[i] = ip.params[kWp + i];
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&ms.mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(smem_u32(&ms.tmem)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = ms.tmem;
  const uint32_t sBuf = smem_u32(buf), sB1 = smem_u32(smem + kOffB), sB2 = smem_u32(smem + kOffB2),
                 sB3 = smem_u32(smem + kOffB3);
  uint32_t phase = 0;
  bool ok = true;
  const int total = ip.n_jobs * ip.mb_h * ip.strips_per_row;
  // The input map of a strip (plane 0 of the buffer): position r * kRow + c is sample (x0 - 4 + c,
  // y0 - 4 + r), clamped to the picture; 16 bytes each, the two channels and six zero channels. A
  // strip's bytes are loaded into registers while the previous strip's MMAs run.
  constexpr int kPer = kPosBuf / kThreads;
  uint8_t ca[kPer], pa[kPer];
  auto load_input = [&](int st) {
    const int job = st / (ip.mb_h * ip.strips_per_row), rem = st % (ip.mb_h * ip.strips_per_row);
    const int y0 = (rem / ip.strips_per_row) * 16 - 4, x0 = (rem % ip.strips_per_row) * kStripMbs * 16 - 4;
    const InferJob jb = ip.jobs[job];
#pragma unroll
    for (int k = 0; k < kPer; k++) {  // all of this thread's loads in flight together
      const int p = tid + kThreads * k;
      const int r = p / kRow, c = p - r * kRow;
      const int yy = min(max(y0 + r, 0), ip.height - 1), xx = min(max(x0 + c, 0), ip.width - 1);
      const size_t o = (size_t)yy * ip.stride + xx;
      ca[k] = p < 24 * kRow ? jb.cur[o] : 128;
      pa[k] = p < 24 * kRow ? jb.prev[o] : 128;
    }
  };
  if (tid == 0) ms.strip = atomicAdd(ip.counter, 1);
  __syncthreads();
  int strip = ms.strip;
  if (strip < total) load_input(strip);
  // shared-memory descriptors: conv1's five tap pairs on plane 0, the two channel halves of the
  // buffer for conv2 and conv3, the B operands; a tile / tap adds its offset in 16-byte units
  const uint64_t bufd0 = umma_desc(sBuf, kPlane, 128), bufd1 = umma_desc(sBuf + 2 * kPlane, kPlane, 128);
  const uint64_t b1d = umma_desc(sB1, 512, 128), b2d = umma_desc(sB2, 512, 128), b3d = umma_desc(sB3, 512, 128);
  while (strip < total && ok) {
    const int job = strip / (ip.mb_h * ip.strips_per_row), rem = strip % (ip.mb_h * ip.strips_per_row);
    const int mby = rem / ip.strips_per_row, mbx0 = (rem % ip.strips_per_row) * kStripMbs;
    const InferJob jb = ip.jobs[job];
#pragma unroll
    for (int k = 0; k < kPer; k++) {
      __nv_bfloat162 two = __floats2bfloat162_rn(pix_norm(ca[k]), pix_norm(pa[k]));
      ((uint4*)buf)[tid + kThreads * k] = make_uint4(*(uint32_t*)&two, 0u, 0u, 0u);
    }
    if (tid == 0) ms.strip = atomicAdd(ip.counter, 1);  // read after the first layer's barrier
    int next = total;
    for (int layer = 0; layer < 3; layer++) {
      fence_async_smem();
      fence_before_sync();
      __syncthreads();
      fence_after_sync();
      const int tiles = layer == 0 ? kTiles1 : (layer == 1 ? kTiles2 : kTiles3);
      if (tid == 0) {
        if (layer == 0) {
#pragma unroll 1
          for (int t = 0; t < tiles; t++)
#pragma unroll
            for (int k = 0; k < kB1Mmas; k++) {
              // taps 2k and 2k + 1 (tap 9: a zero-weight partner one position on) as the two
              // 8-element halves of K, LBO their distance
              const int ta = 2 * k, tb = 2 * k + 1;
              const int oa = (ta / 3) * kRow + ta % 3, ob = tb < 9 ? (tb / 3) * kRow + tb % 3 : oa + 1;
              const uint64_t a = umma_desc(sBuf + (uint32_t)((t * 128 + oa) * 16), (uint32_t)((ob - oa) * 16), 128);
              umma_bf16(tmem + (uint32_t)(t * 32), a, b1d + (uint64_t)(k * 64), k > 0);
            }
        } else {
          const uint64_t bd = layer == 1 ? b2d : b3d;
#pragma unroll 1
          for (int t = 0; t < tiles; t++) {
            const uint32_t d = tmem + (uint32_t)(t * 32);
#pragma unroll
            for (int tap = 0; tap < 9; tap++)
#pragma unroll
              for (int h = 0; h < 2; h++) {
                const uint64_t off = (uint64_t)(t * 128 + (tap / 3) * kRow + tap % 3);
                umma_bf16(d, (h ? bufd1 : bufd0) + off, bd + (uint64_t)((tap * 2 + h) * 64), tap > 0 || h > 0);
              }
          }
        }
        umma_commit(&ms.mbar);
      }
      if (layer == 0) {  // the next strip's bytes, in flight while the tensor cores work
        next = ms.strip;
        if (next < total) load_input(next);
      }
      // every thread polls the barrier; the outcome is made uniform before anyone acts on it
      ok = __syncthreads_and(mbar_wait(&ms.mbar, phase) ? 1 : 0) != 0;
      if (!ok && tid == 0) atomicExch(ip.error, 1);
      phase ^= 1;
      fence_after_sync();
      if (!ok) break;
      // epilogue over the layer's input (all its MMAs have completed): warp w reads rows 32 (w % 4)
      // .. + 31 of tiles w / 4, + 2, ..; bias, ReLU, BF16 into the buffer's four planes
      const int wl = warp & 3;
      for (int t = warp >> 2; t < tiles; t += 2) {
        float v[32];
        tmem_ld32(tmem + ((uint32_t)(wl * 32) << 16) + (uint32_t)(t * 32), v);
        const int p = t * 128 + wl * 32 + lane;
#pragma unroll
        for (int q = 0; q < 4; q++) {
          uint32_t w[4];
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const float a = fmaxf(v[8 * q + 2 * k] + ms.bias[layer][8 * q + 2 * k], 0.0f);
            const float b = fmaxf(v[8 * q + 2 * k + 1] + ms.bias[layer][8 * q + 2 * k + 1], 0.0f);
            __nv_bfloat162 two = __floats2bfloat162_rn(a, b);
            w[k] = *(uint32_t*)&two;
          }
          *(uint4*)(buf + q * kPlane + p * 16) = make_uint4(w[0], w[1], w[2], w[3]);
        }
      }
    }
    if (!ok) break;
    __syncthreads();  // conv3's map complete
    // pooling of the conv3 map (map column 16 j + i is sample x 16 (mbx0 + j) - 1 + i): warp w
    // takes macroblock j = w / 4 and 8-channel plane q = w % 4; lane l < 16 sums map column l + 1
    // down the 18 rows (16-byte reads), lanes 16 and 17 the border columns 0 and 17; block sums
    // over the four lanes of a block column, the 18 x 18 sum over the warp
    if (warp < kStripMbs * 4) {
      const int j = warp >> 2, q = warp & 3;
      const int col = lane < 16 ? lane + 1 : (lane == 16 ? 0 : 17);
      float tot[8], blk[4][8];
#pragma unroll
      for (int k = 0; k < 8; k++) {
        tot[k] = 0.0f;
#pragma unroll
        for (int b = 0; b < 4; b++) blk[b][k] = 0.0f;
      }
      if (lane < 18) {
        const uint8_t* colp = buf + q * kPlane + (16 * j + col) * 16;
#pragma unroll
        for (int r = 0; r < 18; r++) {
          const uint4 v = *(const uint4*)(colp + r * kRow * 16);
          const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const float2 f = __bfloat1622float2(*(const __nv_bfloat162*)&w[k]);
            tot[2 * k] += f.x;
            tot[2 * k + 1] += f.y;
            if (r >= 1 && r <= 16 && lane < 16) {
              blk[(r - 1) >> 2][2 * k] += f.x;
              blk[(r - 1) >> 2][2 * k + 1] += f.y;
            }
          }
        }
      }
#pragma unroll
      for (int k = 0; k < 8; k++) {
#pragma unroll
        for (int b = 0; b < 4; b++) {
          blk[b][k] += __shfl_xor_sync(0xffffffffu, blk[b][k], 1);
          blk[b][k] += __shfl_xor_sync(0xffffffffu, blk[b][k], 2);
        }
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) tot[k] += __shfl_xor_sync(0xffffffffu, tot[k], o);
      }
      if (lane < 16 && (lane & 3) == 0)
#pragma unroll
        for (int b = 0; b < 4; b++)
#pragma unroll
          for (int k = 0; k < 8; k++) ms.pool[j][1 + b * 4 + (lane >> 2)][8 * q + k] = blk[b][k] * (1.0f / 16.0f);
      if (lane == 0)
#pragma unroll
        for (int k = 0; k < 8; k++) ms.pool[j][0][8 * q + k] = tot[k] * (1.0f / 324.0f);
    }
    __syncthreads();
    // heads and hints: threads 0 .. 16 kStripMbs - 1 the intra 4x4 heads of (macroblock tid / 16,
    // block tid % 16), the next kStripMbs threads the partition and offset heads of their macroblock
    if (tid < 16 * kStripMbs + kStripMbs) {
      const bool blockhead = tid < 16 * kStripMbs;
      const int j = blockhead ? tid / 16 : tid - 16 * kStripMbs, mbx = mbx0 + j;
      if (mbx < ip.mb_w) {
        const float* H = ms.head;
        const int m = mby * ip.mb_w + mbx;
        float* lg = jb.logits ? jb.logits + (size_t)m * kLogits : nullptr;
        if (blockhead) {
          const int b = tid % 16;
          const float* f = ms.pool[j][1 + b];
          float li[9];
#pragma unroll
          for (int o = 0; o < 9; o++) {
            float s = H[kBi - kWp + o];
            for (int c = 0; c < C; c++) s += H[kWi - kWp + o * C + c] * f[c];
            li[o] = s;
          }
          // 4x4 block b in raster order; the hint holds decoding order
          const int bx = b & 3, by = b >> 2;
          const int dec = ((by >> 1) << 3) | ((bx >> 1) << 2) | ((by & 1) << 1) | (bx & 1);
          jb.hints[m].i4_mask[dec] = (uint16_t)topk_mask(li, ip.i4_k, ip.i4_margin);
          if (lg)
            for (int o = 0; o < 9; o++) lg[6 + b * 9 + o] = li[o];
        } else {
          const float* g = ms.pool[j][0];
          float lp[4], lm[2];
#pragma unroll
          for (int o = 0; o < 4; o++) {
            float s = H[kBp - kWp + o];
            for (int c = 0; c < C; c++) s += H[o * C + c] * g[c];
            lp[o] = s;
          }
          for (int o = 0; o < 2; o++) {
            float s = H[kBm - kWp + o];
            for (int c = 0; c < C; c++) s += H[kWm - kWp + o * C + c] * g[c];
            lm[o] = s;
          }
          rg_mb_hint& hh = jb.hints[m];
          hh.part_mask = (uint8_t)topk_mask(lp, ip.part_k, ip.part_margin);
          hh.flags = 0;  // the coarse motion pass, when on, follows
          hh.mv_coarse[0] = hh.mv_coarse[1] = 0;
          for (int o = 0; o < 2; o++) hh.mv_off[o] = (int8_t)max(-127, min(127, __float2int_rn(16.0f * lm[o])));
          if (lg) {
            for (int o = 0; o < 4; o++) lg[o] = lp[o];
            lg[4] = lm[0];
            lg[5] = lm[1];
          }
        }
      }
    }
    strip = next;
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(tmem));
}

// ---------------------------------------------------------------------------------------------
// Coarse motion (rg_net_set_coarse_range): a warp per macroblock, 8 per block. The decimated
// picture's sample (x, y) is the rounded mean of the four samples (2x + i, 2y + j), coordinates
// clamped to the picture; the macroblock's 8 x 8 decimated block is compared with the decimated
// previous picture at every displacement of +-r (SAD), the least (SAD, |dx| + |dy|, raster index)
// wins.
constexpr int kCoarseMaxR = 32;
constexpr int kCoarseRow = (8 + 2 * kCoarseMaxR + 3) / 4 * 4 + 4;  // window row stride (bytes)
constexpr int kCoarseWarps = 8;
struct CoarseParams {
  const InferJob* jobs;
  int n_jobs, width, height, stride, mb_w, mb_h, r;
};
__device__ __forceinline__ uint32_t dec_sample(const uint8_t* p, int stride, int w, int h, int x, int y) {
  const int x0 = min(max(2 * x, 0), w - 1), x1 = min(max(2 * x + 1, 0), w - 1);
  const int y0 = min(max(2 * y, 0), h - 1), y1 = min(max(2 * y + 1, 0), h - 1);
  const uint8_t* r0 = p + (size_t)y0 * stride;
  const uint8_t* r1 = p + (size_t)y1 * stride;
  return ((uint32_t)r0[x0] + r0[x1] + r1[x0] + r1[x1] + 2u) >> 2;
}
__device__ __forceinline__ uint32_t lds4_unaligned(const uint8_t* p) {
  const uintptr_t a = (uintptr_t)p;
  const uint32_t* b = (const uint32_t*)(a & ~(uintptr_t)3);
  return __funnelshift_r(b[0], b[1], (uint32_t)(a & 3) * 8u);
}
__global__ void __launch_bounds__(32 * kCoarseWarps) coarse_motion_kernel(CoarseParams cp) {
  __shared__ __align__(16) uint8_t win[kCoarseWarps][(8 + 2 * kCoarseMaxR) * kCoarseRow];
  __shared__ __align__(16) uint8_t blk[kCoarseWarps][64];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int per_pic = cp.mb_w * cp.mb_h;
  const long task = (long)blockIdx.x * kCoarseWarps + warp;
  if (task >= (long)cp.n_jobs * per_pic) return;
  const int job = (int)(task / per_pic), m = (int)(task % per_pic);
  const InferJob jb = cp.jobs[job];
  if (jb.cur == jb.prev) return;  // an IDR picture: no previous picture
  const int mbx = m % cp.mb_w, mby = m / cp.mb_w, R = cp.r, side = 8 + 2 * R;
  const int bx = 8 * mbx, by = 8 * mby;  // the block's decimated origin
  uint8_t* w = win[warp];
  for (int i = lane; i < side * side; i += 32) {
    const int y = i / side, x = i - y * side;
    w[y * kCoarseRow + x] = (uint8_t)dec_sample(jb.prev, cp.stride, cp.width, cp.height, bx - R + x, by - R + y);
  }
  for (int i = lane; i < 64; i += 32)
    blk[warp][i] = (uint8_t)dec_sample(jb.cur, cp.stride, cp.width, cp.height, bx + (i & 7), by + (i >> 3));
  __syncwarp();
  uint32_t b[16];
#pragma unroll
  for (int k = 0; k < 16; k++) b[k] = ((const uint32_t*)blk[warp])[k];
  const int n = (2 * R + 1) * (2 * R + 1);
  uint64_t best = ~0ull;
  for (int p = lane; p < n; p += 32) {
    const int dyi = p / (2 * R + 1), dxi = p - dyi * (2 * R + 1);
    const uint8_t* q = w + dyi * kCoarseRow + dxi;
    uint32_t sad = 0;
#pragma unroll
    for (int r = 0; r < 8; r++)
      sad = __vsadu4(lds4_unaligned(q + r * kCoarseRow), b[2 * r]) +
            __vsadu4(lds4_unaligned(q + r * kCoarseRow + 4), b[2 * r + 1]) + sad;
    const uint32_t dist = (uint32_t)(abs(dxi - R) + abs(dyi - R));
    best = min(best, ((uint64_t)sad << 32) | ((uint64_t)dist << 16) | (uint64_t)p);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) best = min(best, (uint64_t)__shfl_xor_sync(0xffffffffu, (unsigned long long)best, o));
  if (lane == 0) {
    const int p = (int)(best & 0xffffu), dyi = p / (2 * R + 1), dxi = p - dyi * (2 * R + 1);
    rg_mb_hint& h = jb.hints[m];
    h.mv_coarse[0] = (int16_t)(8 * (dxi - R));
    h.mv_coarse[1] = (int16_t)(8 * (dyi - R));
    h.flags |= 1;
  }
}

// ---------------------------------------------------------------------------------------------
// Training on the CUDA cores (f32), per-macroblock crops: 2 x 24 x 24 bytes per sample.
// Maps: A1 [N][32][22][22], A2 [N][32][20][20], A3 [N][32][18][18] (after the ReLU).
constexpr int kIn = 2 * 24 * 24, kA1 = C * 22 * 22, kA2 = C * 20 * 20, kA3 = C * 18 * 18;

// conv 3x3 valid of one sample per block: in [cin][hin][hin] (bytes normalised when u8 != null),
// out [32][hin-2][hin-2] = ReLU(W x + b).
__global__ void conv_fwd_kernel(const uint8_t* __restrict__ u8, const float* __restrict__ in, int cin, int hin,
                                const float* __restrict__ P, int woff, int boff, float* __restrict__ out) {
  extern __shared__ float4 sh4[];
  float* sh = (float*)sh4;
  float* w = sh;                       // [cin][9][32]
  float* x = sh + C * cin * 9;         // cin * hin * hin
  const int n = blockIdx.x, hout = hin - 2, npos = hout * hout, nin = cin * hin * hin;
  for (int i = threadIdx.x; i < nin; i += blockDim.x)
    x[i] = u8 ? pix_norm(u8[(size_t)n * nin + i]) : in[(size_t)n * nin + i];
  for (int i = threadIdx.x; i < C * cin * 9; i += blockDim.x) {
    const int o = i / (cin * 9), ci = (i / 9) % cin, t = i % 9;
    w[(ci * 9 + t) * C + o] = P[woff + i];
  }
  __syncthreads();
  for (int p = threadIdx.x; p < npos; p += blockDim.x) {
    const int y = p / hout, xx = p % hout;
    float acc[C];
#pragma unroll
    for (int o = 0; o < C; o++) acc[o] = P[boff + o];
    for (int ci = 0; ci < cin; ci++)
#pragma unroll
      for (int t = 0; t < 9; t++) {
        const float v = x[(ci * hin + y + t / 3) * hin + xx + t % 3];
        const float4* wv = (const float4*)&w[(ci * 9 + t) * C];
#pragma unroll
        for (int o4 = 0; o4 < C / 4; o4++) {
          const float4 q = wv[o4];
          acc[4 * o4] += q.x * v; acc[4 * o4 + 1] += q.y * v; acc[4 * o4 + 2] += q.z * v; acc[4 * o4 + 3] += q.w * v;
        }
      }
#pragma unroll
    for (int o = 0; o < C; o++) out[(size_t)n * C * npos + o * npos + p] = fmaxf(acc[o], 0.0f);
  }
}

// Heads, losses and their gradient (one block of 32 threads per sample): labels part [N] (-1 none),
// i4 [N][16] (raster 4x4 blocks, -1 none), mv [N][2] with mvv [N] (0 none); scale: 1 / the count of
// each loss's labels in the batch. Writes the logits (optional), the pooled features (feat [N][17][32]:
// the 18 x 18 mean, then the block means), the logit gradients (dlog [N][kLogits]) and dA3 (the
// gradient at the conv3 map, masked by its ReLU); the loss is added atomically.
__global__ void heads_kernel(const float* __restrict__ A3, const float* __restrict__ P, const int* __restrict__ part,
                             const int* __restrict__ i4, const float* __restrict__ mv, const int* __restrict__ mvv,
                             float sp, float si, float sm, float mv_weight, float* __restrict__ logits,
                             float* __restrict__ feat, float* __restrict__ dlog, float* __restrict__ dA3,
                             float* __restrict__ loss) {
  __shared__ float f[17][C], dg[C], df[16][C], dl[kLogits], lsum[17];
  const int n = blockIdx.x, c = threadIdx.x;
  const float* a = A3 + (size_t)n * kA3 + c * 324;
  float all = 0.0f, blk[16];
  for (int b = 0; b < 16; b++) blk[b] = 0.0f;
  for (int r = 0; r < 18; r++)
    for (int i = 0; i < 18; i++) {
      float x = a[r * 18 + i];
      all += x;
      if (r >= 1 && r <= 16 && i >= 1 && i <= 16) blk[((r - 1) >> 2) * 4 + ((i - 1) >> 2)] += x;
    }
  f[0][c] = all / 324.0f;
  for (int b = 0; b < 16; b++) f[1 + b][c] = blk[b] / 16.0f;
  __syncthreads();
  for (int k = 0; k < 17; k++) feat[((size_t)n * 17 + k) * C + c] = f[k][c];
  // thread 0: partition and offset; threads 1..16: block c - 1's intra 4x4 logits
  if (c <= 16) {
    float L = 0.0f;
    if (c == 0) {
      float lp[4], lm[2];
      for (int o = 0; o < 4; o++) {
        float s = P[kBp + o];
        for (int k = 0; k < C; k++) s += P[kWp + o * C + k] * f[0][k];
        lp[o] = s;
      }
      for (int o = 0; o < 2; o++) {
        float s = P[kBm + o];
        for (int k = 0; k < C; k++) s += P[kWm + o * C + k] * f[0][k];
        lm[o] = s;
      }
      for (int o = 0; o < 6; o++) dl[o] = 0.0f;
      if (part[n] >= 0) {
        float mx = fmaxf(fmaxf(lp[0], lp[1]), fmaxf(lp[2], lp[3])), se = 0.0f;
        for (int o = 0; o < 4; o++) se += expf(lp[o] - mx);
        for (int o = 0; o < 4; o++) dl[o] = sp * (expf(lp[o] - mx) / se - (o == part[n] ? 1.0f : 0.0f));
        L += sp * (logf(se) + mx - lp[part[n]]);
      }
      if (mvv[n]) {
        for (int o = 0; o < 2; o++) {  // Huber (delta 1) on the offset in units of 16 quarter samples
          float d = lm[o] - mv[2 * n + o];
          float ad = fabsf(d);
          L += sm * mv_weight * (ad <= 1.0f ? 0.5f * d * d : ad - 0.5f);
          dl[4 + o] = sm * mv_weight * (ad <= 1.0f ? d : (d > 0 ? 1.0f : -1.0f));
        }
      }
      if (logits) {
        for (int o = 0; o < 4; o++) logits[(size_t)n * kLogits + o] = lp[o];
        logits[(size_t)n * kLogits + 4] = lm[0];
        logits[(size_t)n * kLogits + 5] = lm[1];
      }
    } else {
      const int b = c - 1;
      float li[9];
      for (int o = 0; o < 9; o++) {
        float s = P[kBi + o];
        for (int k = 0; k < C; k++) s += P[kWi + o * C + k] * f[1 + b][k];
        li[o] = s;
        dl[6 + b * 9 + o] = 0.0f;
      }
      if (logits)
        for (int o = 0; o < 9; o++) logits[(size_t)n * kLogits + 6 + b * 9 + o] = li[o];
      const int lab = i4[n * 16 + b];
      if (lab >= 0) {
        float mx = li[0], se = 0.0f;
        for (int o = 1; o < 9; o++) mx = fmaxf(mx, li[o]);
        for (int o = 0; o < 9; o++) se += expf(li[o] - mx);
        for (int o = 0; o < 9; o++) dl[6 + b * 9 + o] = si * (expf(li[o] - mx) / se - (o == lab ? 1.0f : 0.0f));
        L += si * (logf(se) + mx - li[lab]);
      }
    }
    lsum[c] = L;
  }
  __syncthreads();
  if (c == 0) {
    float L = 0.0f;
    for (int k = 0; k < 17; k++) L += lsum[k];
    atomicAdd(loss, L);
  }
  for (int o = c; o < kLogits; o += C) dlog[(size_t)n * kLogits + o] = dl[o];
  // the gradient at the pooled features
  float dgc = 0.0f;
  for (int o = 0; o < 4; o++) dgc += P[kWp + o * C + c] * dl[o];
  for (int o = 0; o < 2; o++) dgc += P[kWm + o * C + c] * dl[4 + o];
  dg[c] = dgc;
  for (int b = 0; b < 16; b++) {
    float d = 0.0f;
    for (int o = 0; o < 9; o++) d += P[kWi + o * C + c] * dl[6 + b * 9 + o];
    df[b][c] = d;
  }
  __syncthreads();
  // dA3 = pooled gradients spread over the map, masked by the ReLU
  float* d = dA3 + (size_t)n * kA3 + c * 324;
  for (int r = 0; r < 18; r++)
    for (int i = 0; i < 18; i++) {
      float v = dg[c] / 324.0f;
      if (r >= 1 && r <= 16 && i >= 1 && i <= 16) v += df[((r - 1) >> 2) * 4 + ((i - 1) >> 2)][c] / 16.0f;
      d[r * 18 + i] = a[r * 18 + i] > 0.0f ? v : 0.0f;
    }
}

// Head parameter gradients: one block per parameter of the heads (kParams - kWp of them), a
// reduction over the samples (and the 16 blocks for the intra 4x4 head).
__global__ void head_grad_kernel(const float* __restrict__ feat, const float* __restrict__ dlog, int n,
                                 float* __restrict__ G) {
  __shared__ float red[256];
  const int e = blockIdx.x;  // index into the head parameters
  float s = 0.0f;
  for (int k = threadIdx.x; k < n * 16; k += blockDim.x) {
    const int i = k / 16, b = k % 16;
    const float* fi = feat + (size_t)i * 17 * C;
    const float* di = dlog + (size_t)i * kLogits;
    const int q = kWp + e;
    if (q < kBp) { if (b == 0) s += di[(q - kWp) / C] * fi[(q - kWp) % C]; }
    else if (q < kWm) { if (b == 0) s += di[q - kBp]; }
    else if (q < kBm) { if (b == 0) s += di[4 + (q - kWm) / C] * fi[(q - kWm) % C]; }
    else if (q < kWi) { if (b == 0) s += di[4 + q - kBm]; }
    else if (q < kBi) s += di[6 + b * 9 + (q - kWi) / C] * fi[(1 + b) * C + (q - kWi) % C];
    else s += di[6 + b * 9 + q - kBi];
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) G[kWp + e] = red[0];
}

// Gradient of a conv's input (one sample per block): din[ci][y][x] = sum over co, taps of
// dout[co][y - dy][x - dx] W[co][ci][dy][dx], masked by the ReLU of the input map (act > 0).
__global__ void conv_bwd_data_kernel(const float* __restrict__ dout, int hin, const float* __restrict__ P, int woff,
                                     const float* __restrict__ act, float* __restrict__ din) {
  extern __shared__ float4 sh4[];
  float* sh = (float*)sh4;
  const int n = blockIdx.x, hout = hin - 2, nout = C * hout * hout;
  float* w = sh;              // [9][co][ci]
  float* d = sh + C * C * 9;  // 32 * hout * hout
  for (int i = threadIdx.x; i < nout; i += blockDim.x) d[i] = dout[(size_t)n * nout + i];
  for (int i = threadIdx.x; i < C * C * 9; i += blockDim.x) {
    const int co = i / (C * 9), ci = (i / 9) % C, t = i % 9;
    w[(t * C + co) * C + ci] = P[woff + i];
  }
  __syncthreads();
  const int npos = hin * hin;
  for (int p = threadIdx.x; p < npos; p += blockDim.x) {
    const int y = p / hin, x = p % hin;
    float acc[C];
#pragma unroll
    for (int ci = 0; ci < C; ci++) acc[ci] = 0.0f;
    for (int t = 0; t < 9; t++) {
      const int oy = y - t / 3, ox = x - t % 3;
      if (oy < 0 || oy >= hout || ox < 0 || ox >= hout) continue;
      for (int co = 0; co < C; co++) {
        const float g = d[(co * hout + oy) * hout + ox];
        const float4* wv = (const float4*)&w[(t * C + co) * C];
#pragma unroll
        for (int c4 = 0; c4 < C / 4; c4++) {
          const float4 q = wv[c4];
          acc[4 * c4] += q.x * g; acc[4 * c4 + 1] += q.y * g; acc[4 * c4 + 2] += q.z * g; acc[4 * c4 + 3] += q.w * g;
        }
      }
    }
#pragma unroll
    for (int ci = 0; ci < C; ci++) {
      const size_t i = (size_t)n * C * npos + ci * npos + p;
      din[i] = act[i] > 0.0f ? acc[ci] : 0.0f;
    }
  }
}

// Gradient of a conv's weights and bias over a group of samples per block (atomic into G):
// dW[co][ci][t] = sum over samples, positions of dout[co][p] in[ci][p + t].
__global__ void conv_bwd_weight_kernel(const float* __restrict__ dout, const uint8_t* __restrict__ u8,
                                       const float* __restrict__ in, int cin, int hin, int n_samples, int per_block,
                                       int woff, int boff, float* __restrict__ G) {
  extern __shared__ float sh[];
  const int hout = hin - 2, nout = C * hout * hout, nin = cin * hin * hin, nw = C * cin * 9;
  float* d = sh;
  float* x = sh + nout;
  float acc[36];  // nw / blockDim.x entries per thread (blockDim.x = 256: up to 9216 / 256)
  const int per = (nw + blockDim.x - 1) / blockDim.x;
  for (int k = 0; k < 36; k++) acc[k] = 0.0f;
  float bacc = 0.0f;
  for (int s = 0; s < per_block; s++) {
    const int n = blockIdx.x * per_block + s;
    if (n >= n_samples) break;
    __syncthreads();
    for (int i = threadIdx.x; i < nout; i += blockDim.x) d[i] = dout[(size_t)n * nout + i];
    for (int i = threadIdx.x; i < nin; i += blockDim.x) x[i] = u8 ? pix_norm(u8[(size_t)n * nin + i]) : in[(size_t)n * nin + i];
    __syncthreads();
    for (int k = 0; k < per; k++) {
      const int e = threadIdx.x + k * blockDim.x;
      if (e >= nw) break;
      const int co = e / (cin * 9), ci = (e / 9) % cin, t = e % 9;
      const float* dp = d + co * hout * hout;
      const float* xp = x + ci * hin * hin + (t / 3) * hin + t % 3;
      float s2 = 0.0f;
      for (int y = 0; y < hout; y++)
        for (int xx = 0; xx < hout; xx++) s2 += dp[y * hout + xx] * xp[y * hin + xx];
      acc[k] += s2;
    }
    if (threadIdx.x < C) {
      const float* dp = d + threadIdx.x * hout * hout;
      for (int i = 0; i < hout * hout; i++) bacc += dp[i];
    }
  }
  for (int k = 0; k < per; k++) {
    const int e = threadIdx.x + k * blockDim.x;
    if (e < nw) atomicAdd(&G[woff + e], acc[k]);
  }
  if (threadIdx.x < C) atomicAdd(&G[boff + threadIdx.x], bacc);
}

__global__ void adam_kernel(float* P, const float* G, float* m, float* v, int n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = G[i];
  m[i] = b1 * m[i] + (1.0f - b1) * g;
  v[i] = b2 * v[i] + (1.0f - b2) * g * g;
  P[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
}

// Crops of the training set: sample k is macroblock (mbx, mby) of picture pics[k] (cur and prev
// luma, display size, stride), 2 x 24 x 24 bytes, coordinates clamped to the picture.
struct CropSrc {
  const uint8_t* cur;
  const uint8_t* prev;
  int mbx, mby;
};
__global__ void crops_kernel(const CropSrc* __restrict__ src, int n, int width, int height, int stride,
                             uint8_t* __restrict__ out) {
  const int k = blockIdx.x;
  if (k >= n) return;
  const CropSrc s = src[k];
  for (int i = threadIdx.x; i < kIn; i += blockDim.x) {
    const int ch = i / 576, r = (i % 576) / 24, c = i % 24;
    const int y = min(max(s.mby * 16 - 4 + r, 0), height - 1), x = min(max(s.mbx * 16 - 4 + c, 0), width - 1);
    out[(size_t)k * kIn + i] = (ch ? s.prev : s.cur)[(size_t)y * stride + x];
  }
}

}  // namespace

// ---------------------------------------------------------------------------------------------
struct rg_net {
  int device = 0;
  float* P = nullptr;      // parameters (f32)
  float* G = nullptr;      // gradients
  float* M = nullptr;      // Adam moments
  float* V = nullptr;
  int step = 0;
  __nv_bfloat16* bops = nullptr;  // inference B operands (from P)
  bool bops_stale = true;
  int* counter = nullptr;  // [0] strip ticket, [1] error word
  // training scratch
  float *a1 = nullptr, *a2 = nullptr, *a3 = nullptr, *d3 = nullptr, *d2 = nullptr, *d1 = nullptr, *loss = nullptr;
  float *feat = nullptr, *dlog = nullptr;
  int cap = 0;
  InferJob* jobs = nullptr;
  int jobs_cap = 0;
  int part_k = 3, i4_k = 3;  // hint policy (rg_net_set_hint_policy)
  float part_margin = INFINITY, i4_margin = INFINITY;
  int coarse_range = 32;      // rg_net_set_coarse_range
};

namespace {
int nfail(int code, const char* msg) {
  rg::set_last_error(msg);
  return code;
}
#define NCK(expr)                                                    \
  do {                                                               \
    cudaError_t e_ = (expr);                                         \
    if (e_ != cudaSuccess) return nfail(RG_ERR_CUDA, cudaGetErrorString(e_)); \
  } while (0)

// The B operands of the three layers in the shared-memory order the inference kernel loads: per
// MMA 1 KB -- two 8-element halves of K (512 bytes apart), 32 rows of N (output channels) of 16 bytes.
void pack_bops(const std::vector<float>& p, std::vector<__nv_bfloat16>& out) {
  out.assign((size_t)(kB1Mmas + 2 * kBMmas) * 512, __float2bfloat16(0.0f));
  auto put = [&](int mma, int n, int k, float v) { out[(size_t)mma * 512 + (k >> 3) * 256 + n * 8 + (k & 7)] = __float2bfloat16(v); };
  const int pairs[kB1Mmas][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {8, 9}};
  for (int m = 0; m < kB1Mmas; m++)
    for (int n = 0; n < C; n++)
      for (int h = 0; h < 2; h++) {
        int t = pairs[m][h];
        if (t > 8) continue;
        for (int ci = 0; ci < 2; ci++) put(m, n, 8 * h + ci, p[kW1 + (n * 2 + ci) * 9 + t]);
      }
  for (int layer = 0; layer < 2; layer++) {
    const int woff = layer == 0 ? kW2 : kW3, base = kB1Mmas + layer * kBMmas;
    for (int t = 0; t < 9; t++)
      for (int h = 0; h < 2; h++)
        for (int n = 0; n < C; n++)
          for (int k = 0; k < 16; k++) put(base + t * 2 + h, n, k, p[woff + (n * C + 16 * h + k) * 9 + t]);
  }
}
int ensure_bops(rg_net* net) {
  if (!net->bops_stale) return RG_OK;
  std::vector<float> p(kParams);
  NCK(cudaMemcpy(p.data(), net->P, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
  std::vector<__nv_bfloat16> b;
  pack_bops(p, b);
  NCK(cudaMemcpy(net->bops, b.data(), b.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
  net->bops_stale = false;
  return RG_OK;
}
int ensure_train(rg_net* net, int n) {
  if (n <= net->cap) return RG_OK;
  cudaFree(net->a1); cudaFree(net->a2); cudaFree(net->a3); cudaFree(net->d3); cudaFree(net->d2); cudaFree(net->d1);
  cudaFree(net->feat); cudaFree(net->dlog);
  size_t f = sizeof(float);
  if (cudaMalloc((void**)&net->feat, f * n * 17 * C) != cudaSuccess || cudaMalloc((void**)&net->dlog, f * n * kLogits) != cudaSuccess ||
      cudaMalloc((void**)&net->a1, f * n * kA1) != cudaSuccess || cudaMalloc((void**)&net->a2, f * n * kA2) != cudaSuccess ||
      cudaMalloc((void**)&net->a3, f * n * kA3) != cudaSuccess || cudaMalloc((void**)&net->d3, f * n * kA3) != cudaSuccess ||
      cudaMalloc((void**)&net->d2, f * n * kA2) != cudaSuccess || cudaMalloc((void**)&net->d1, f * n * kA1) != cudaSuccess) {
    net->cap = 0;
    return nfail(RG_ERR_OOM, "rg_net: training scratch allocation failed");
  }
  net->cap = n;
  return RG_OK;
}
}  // namespace

extern "C" {

int32_t rg_net_param_count(void) { return kParams; }

rg_net* rg_net_create(int32_t device, uint64_t seed) {
  if (cudaSetDevice(device) != cudaSuccess) { nfail(RG_ERR_CUDA, "rg_net_create: cudaSetDevice failed"); return nullptr; }
  auto* net = new rg_net();
  net->device = device;
  size_t pb = sizeof(float) * kParams;
  if (cudaMalloc((void**)&net->P, pb) != cudaSuccess || cudaMalloc((void**)&net->G, pb) != cudaSuccess ||
      cudaMalloc((void**)&net->M, pb) != cudaSuccess || cudaMalloc((void**)&net->V, pb) != cudaSuccess ||
      cudaMalloc((void**)&net->bops, (size_t)(kB1Mmas + 2 * kBMmas) * 1024) != cudaSuccess ||
      cudaMalloc((void**)&net->counter, 2 * sizeof(int)) != cudaSuccess ||
      cudaMalloc((void**)&net->loss, sizeof(float)) != cudaSuccess) {
    nfail(RG_ERR_OOM, "rg_net_create: allocation failed");
    rg_net_destroy(net);
    return nullptr;
  }
  // He-uniform initialisation from a 64-bit LCG (heads a tenth of that)
  std::vector<float> p(kParams, 0.0f);
  uint64_t s = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto uni = [&]() {
    s = s * 6364136223846793005ull + 1442695040888963407ull;
    return (float)((s >> 40) & 0xFFFFFF) / 16777216.0f * 2.0f - 1.0f;
  };
  auto fill = [&](int off, int n, float lim) { for (int i = 0; i < n; i++) p[off + i] = lim * uni(); };
  fill(kW1, C * 2 * 9, std::sqrt(6.0f / 18.0f));
  fill(kW2, C * C * 9, std::sqrt(6.0f / 288.0f));
  fill(kW3, C * C * 9, std::sqrt(6.0f / 288.0f));
  fill(kWp, 4 * C, 0.1f * std::sqrt(6.0f / 32.0f));
  fill(kWm, 2 * C, 0.1f * std::sqrt(6.0f / 32.0f));
  fill(kWi, 9 * C, 0.1f * std::sqrt(6.0f / 32.0f));
  if (rg_net_set_params(net, p.data(), kParams) != RG_OK) {
    rg_net_destroy(net);
    return nullptr;
  }
  return net;
}

void rg_net_destroy(rg_net* net) {
  if (!net) return;
  cudaFree(net->P); cudaFree(net->G); cudaFree(net->M); cudaFree(net->V); cudaFree(net->bops); cudaFree(net->counter);
  cudaFree(net->a1); cudaFree(net->a2); cudaFree(net->a3); cudaFree(net->d3); cudaFree(net->d2); cudaFree(net->d1);
  cudaFree(net->loss); cudaFree(net->jobs); cudaFree(net->feat); cudaFree(net->dlog);
  delete net;
}

int rg_net_set_params(rg_net* net, const float* params, int32_t count) {
  if (!net || !params || count != kParams) return nfail(RG_ERR_INVALID, "rg_net_set_params: bad arguments");
  NCK(cudaSetDevice(net->device));
  NCK(cudaMemcpy(net->P, params, sizeof(float) * kParams, cudaMemcpyHostToDevice));
  NCK(cudaMemset(net->M, 0, sizeof(float) * kParams));
  NCK(cudaMemset(net->V, 0, sizeof(float) * kParams));
  net->step = 0;
  net->bops_stale = true;
  return RG_OK;
}

int rg_net_get_params(const rg_net* net, float* params, int32_t count) {
  if (!net || !params || count != kParams) return nfail(RG_ERR_INVALID, "rg_net_get_params: bad arguments");
  NCK(cudaMemcpy(params, net->P, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
  return RG_OK;
}

int rg_net_crops(rg_net* net, const uint8_t* const* cur, const uint8_t* const* prev, const int32_t* mb_xy, int32_t n,
                 int32_t width, int32_t height, size_t stride, uint8_t* dev_out, void* stream) {
  if (!net || !cur || !prev || !mb_xy || !dev_out || n < 0) return nfail(RG_ERR_INVALID, "rg_net_crops: bad arguments");
  if (!n) return RG_OK;
  std::vector<CropSrc> h(n);
  for (int k = 0; k < n; k++) h[k] = CropSrc{cur[k], prev[k], mb_xy[2 * k], mb_xy[2 * k + 1]};
  CropSrc* d = nullptr;
  NCK(cudaMalloc((void**)&d, sizeof(CropSrc) * n));
  cudaStream_t st = (cudaStream_t)stream;
  NCK(cudaMemcpyAsync(d, h.data(), sizeof(CropSrc) * n, cudaMemcpyHostToDevice, st));
  crops_kernel<<<n, 256, 0, st>>>(d, n, width, height, (int)stride, dev_out);
  NCK(cudaGetLastError());
  NCK(cudaStreamSynchronize(st));
  cudaFree(d);
  return RG_OK;
}

int rg_net_forward_backward(rg_net* net, const uint8_t* dev_crops, int32_t n, const int32_t* dev_part,
                            const int32_t* dev_i4, const float* dev_mv, const int32_t* dev_mvv, float mv_weight,
                            float* dev_logits, float* loss_out, float* grads_out) {
  if (!net || !dev_crops || n < 1 || !dev_part || !dev_i4 || !dev_mv || !dev_mvv)
    return nfail(RG_ERR_INVALID, "rg_net_forward_backward: bad arguments");
  NCK(cudaSetDevice(net->device));
  int r = ensure_train(net, n);
  if (r) return r;
  // label counts normalise each loss (host copies of the small label arrays)
  std::vector<int32_t> part(n), i4((size_t)n * 16), mvv(n);
  NCK(cudaMemcpy(part.data(), dev_part, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
  NCK(cudaMemcpy(i4.data(), dev_i4, sizeof(int32_t) * n * 16, cudaMemcpyDeviceToHost));
  NCK(cudaMemcpy(mvv.data(), dev_mvv, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
  int np = 0, ni = 0, nm = 0;
  for (int k = 0; k < n; k++) { np += part[k] >= 0; nm += mvv[k] != 0; }
  for (size_t k = 0; k < i4.size(); k++) ni += i4[k] >= 0;
  const float sp = np ? 1.0f / np : 0.0f, si = ni ? 1.0f / ni : 0.0f, sm = nm ? 1.0f / nm : 0.0f;
  NCK(cudaMemset(net->G, 0, sizeof(float) * kParams));
  NCK(cudaMemset(net->loss, 0, sizeof(float)));
  const int th = 256;
  auto attr = [](const void* k, int bytes) { cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes); };
  const int s1 = (2 * 24 * 24 + C * 2 * 9) * 4, s2 = (C * 22 * 22 + C * C * 9) * 4, s3 = (C * 20 * 20 + C * C * 9) * 4;
  static_assert((C * 2 * 9) % 4 == 0, "input map after the weights stays 16-byte aligned");
  attr((const void*)conv_fwd_kernel, s2);
  conv_fwd_kernel<<<n, th, s1>>>(dev_crops, nullptr, 2, 24, net->P, kW1, kB1, net->a1);
  conv_fwd_kernel<<<n, th, s2>>>(nullptr, net->a1, C, 22, net->P, kW2, kB2, net->a2);
  conv_fwd_kernel<<<n, th, s3>>>(nullptr, net->a2, C, 20, net->P, kW3, kB3, net->a3);
  heads_kernel<<<n, C>>>(net->a3, net->P, dev_part, dev_i4, dev_mv, dev_mvv, sp, si, sm, mv_weight, dev_logits,
                         net->feat, net->dlog, net->d3, net->loss);
  head_grad_kernel<<<kParams - kWp, 256>>>(net->feat, net->dlog, n, net->G);
  const int sb3 = (C * 18 * 18 + C * C * 9) * 4, sb2 = (C * 20 * 20 + C * C * 9) * 4;
  attr((const void*)conv_bwd_data_kernel, sb2);
  conv_bwd_data_kernel<<<n, th, sb3>>>(net->d3, 20, net->P, kW3, net->a2, net->d2);
  conv_bwd_data_kernel<<<n, th, sb2>>>(net->d2, 22, net->P, kW2, net->a1, net->d1);
  const int per = 8, nb = (n + per - 1) / per;
  const int w3 = (C * 18 * 18 + C * 20 * 20) * 4, w2 = (C * 20 * 20 + C * 22 * 22) * 4, w1 = (C * 22 * 22 + 2 * 24 * 24) * 4;
  attr((const void*)conv_bwd_weight_kernel, w2);
  conv_bwd_weight_kernel<<<nb, th, w3>>>(net->d3, nullptr, net->a2, C, 20, n, per, kW3, kB3, net->G);
  conv_bwd_weight_kernel<<<nb, th, w2>>>(net->d2, nullptr, net->a1, C, 22, n, per, kW2, kB2, net->G);
  conv_bwd_weight_kernel<<<nb, th, w1>>>(net->d1, dev_crops, nullptr, 2, 24, n, per, kW1, kB1, net->G);
  NCK(cudaGetLastError());
  NCK(cudaDeviceSynchronize());
  if (loss_out) NCK(cudaMemcpy(loss_out, net->loss, sizeof(float), cudaMemcpyDeviceToHost));
  if (grads_out) NCK(cudaMemcpy(grads_out, net->G, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
  return RG_OK;
}

int rg_net_adam_step(rg_net* net, float lr) {
  if (!net || !(lr > 0.0f)) return nfail(RG_ERR_INVALID, "rg_net_adam_step: bad arguments");
  net->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - std::pow(b1, (float)net->step), c2 = 1.0f - std::pow(b2, (float)net->step);
  adam_kernel<<<(kParams + 255) / 256, 256>>>(net->P, net->G, net->M, net->V, kParams, lr, b1, b2, 1e-8f, c1, c2);
  NCK(cudaGetLastError());
  net->bops_stale = true;
  return RG_OK;
}

int rg_net_predict_hints(rg_net* net, const uint8_t* const* dev_cur, const uint8_t* const* dev_prev, int32_t n_pictures,
                         int32_t width, int32_t height, size_t stride, rg_mb_hint* const* dev_hints,
                         float* const* dev_logits, void* stream) {
  if (!net || !dev_cur || !dev_prev || !dev_hints || n_pictures < 1 || width < 1 || height < 1 || stride < (size_t)width)
    return nfail(RG_ERR_INVALID, "rg_net_predict_hints: bad arguments");
  NCK(cudaSetDevice(net->device));
  int r = ensure_bops(net);
  if (r) return r;
  if (n_pictures > net->jobs_cap) {
    cudaFree(net->jobs);
    if (cudaMalloc((void**)&net->jobs, sizeof(InferJob) * n_pictures) != cudaSuccess) {
      net->jobs_cap = 0;
      return nfail(RG_ERR_OOM, "rg_net_predict_hints: job list allocation failed");
    }
    net->jobs_cap = n_pictures;
  }
  std::vector<InferJob> h(n_pictures);
  for (int k = 0; k < n_pictures; k++)
    h[k] = InferJob{dev_cur[k], dev_prev[k], dev_hints[k], dev_logits ? dev_logits[k] : nullptr};
  cudaStream_t st = (cudaStream_t)stream;
  NCK(cudaMemcpyAsync(net->jobs, h.data(), sizeof(InferJob) * n_pictures, cudaMemcpyHostToDevice, st));
  NCK(cudaMemsetAsync(net->counter, 0, 2 * sizeof(int), st));
  InferParams ip;
  ip.jobs = net->jobs;
  ip.n_jobs = n_pictures;
  ip.width = width;
  ip.height = height;
  ip.stride = (int)stride;
  ip.mb_w = (width + 15) / 16;
  ip.mb_h = (height + 15) / 16;
  ip.strips_per_row = (ip.mb_w + kStripMbs - 1) / kStripMbs;
  ip.bops = net->bops;
  ip.params = net->P;
  ip.counter = net->counter;
  ip.error = net->counter + 1;
  ip.part_k = net->part_k;
  ip.i4_k = net->i4_k;
  ip.part_margin = net->part_margin;
  ip.i4_margin = net->i4_margin;
  NCK(cudaFuncSetAttribute(cnn_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemInfer));
  NCK(cudaFuncSetAttribute(cnn_infer_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, net->device);
  const int strips = n_pictures * ip.mb_h * ip.strips_per_row;
  const int ctas = kCtasPerSm * sms < strips ? kCtasPerSm * sms : strips;
  cnn_infer_kernel<<<ctas, kThreads, kSmemInfer, st>>>(ip);
  NCK(cudaGetLastError());
  if (net->coarse_range > 0) {
    CoarseParams cp{net->jobs, n_pictures, width, height, (int)stride, ip.mb_w, ip.mb_h, net->coarse_range / 2};
    const long tasks = (long)n_pictures * ip.mb_w * ip.mb_h;
    coarse_motion_kernel<<<(unsigned)((tasks + kCoarseWarps - 1) / kCoarseWarps), 32 * kCoarseWarps, 0, st>>>(cp);
    NCK(cudaGetLastError());
  }
  return RG_OK;
}

int rg_net_set_coarse_range(rg_net* net, int32_t range) {
  if (!net || range < 0 || range > 2 * kCoarseMaxR || (range & 1)) return nfail(RG_ERR_INVALID, "rg_net_set_coarse_range: bad arguments");
  net->coarse_range = range;
  return RG_OK;
}

int rg_net_set_hint_policy(rg_net* net, int32_t part_k, float part_margin, int32_t i4_k, float i4_margin) {
  if (!net || part_k < 1 || part_k > 4 || i4_k < 1 || i4_k > 9 || !(part_margin >= 0.0f) || !(i4_margin >= 0.0f))
    return nfail(RG_ERR_INVALID, "rg_net_set_hint_policy: bad arguments");
  net->part_k = part_k;
  net->part_margin = part_margin;
  net->i4_k = i4_k;
  net->i4_margin = i4_margin;
  return RG_OK;
}

int rg_net_check(rg_net* net, void* stream) {
  if (!net) return nfail(RG_ERR_INVALID, "rg_net_check: null network");
  int e[2] = {0, 0};
  NCK(cudaMemcpyAsync(e, net->counter, sizeof e, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  NCK(cudaStreamSynchronize((cudaStream_t)stream));
  if (e[1]) return nfail(RG_ERR_TIMEOUT, "rg_net_predict_hints: a wait on the tensor cores gave up");
  return RG_OK;
}

}  // extern "C"
