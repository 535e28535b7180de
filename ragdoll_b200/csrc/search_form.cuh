// Search forms of the macroblock engine (included by engine_kernels.cu inside its anonymous
// namespace; uses its helpers). Neither form exists in the reference: they are the exhaustive
// "full search" the learned form is trained on and judged against, and the learned form itself.
//
// P macroblock (analyse_p_mb_search):
//   1. the P_Skip probe of the plain form (enc.rs:2906 try_p_skip) with the skip vector of the
//      quadrant grid;
//   2. integer search: the SAD of each 8x8 quadrant at every integer vector of a window, and for
//      each of the nine partition parts (16x16; 16x8 top, bottom; 8x16 left, right; four 8x8) the
//      vector of least SAD + lambda * (bits(4 vx - mvp.x) + bits(4 vy - mvp.y)) against the 16x16
//      predictor, first in raster order on ties. Full search: the window is +-search_range around
//      the 16x16 predictor. Learned: +-2 around a centre chosen among seven integer candidates --
//      predictor plus the hinted offset, predictor, the hint's coarse vector (when it has one), the
//      left, top and top-right (top-left where that is absent) neighbours' vectors, zero -- by the
//      16x16 SAD + lambda * vector bits, first in that order on ties; while the 16x16 part's best lies on that window's edge (and not on
//      the vector bounds) the window is centred on it again, up to `walk` times, and then the full
//      window is searched;
//   3. for every partition type tried (all four; learned: the hinted ones), each part in coding
//      order from its integer best: half-sample step (centre, then 8 neighbours at distance 2,
//      quarter units) and quarter-sample step (8 neighbours at distance 1), costs (SATD >> 1) +
//      lambda * vector bits against the part's own predictor (H.264 8.4.1.3, directional for 16x8
//      and 8x16), least cost first in candidate order; learned: the SAD diamonds of
//      refine_part_sad instead;
//   4. the type of least total cost, the stream's type bits (per partition type) * lambda added,
//      first on ties;
//   5. intra 16x16 check, residual, late skip and reconstruction exactly as the plain form.
// IDR macroblock: the plain form's analysis; learned: intra 4x4 blocks try only their hinted modes
// (those of them available at the block, DC when none is).

constexpr int kBandRows = 8;               // integer vectors per band row
constexpr int kBandBytes = (kBandRows + 15) * (2 * kMaxSearchRange + 28);
constexpr int kLearnedRange = 2;           // learned form: integer window around the seed
constexpr int kCentreCands = 7;            // learned form: candidates of the window's centre


// A neighbouring 4x4 block for motion prediction: ref -2 not available, -1 intra, 0 inter.
struct NbMv {
  int ref, x, y;
};
// The neighbours of the current macroblock in the quadrant grid.
struct MbNb {
  int refA, refB, refC, refD;
  int a[2][2];   // left macroblock: quadrants 1 (rows 0-1) and 3 (rows 2-3)
  int b[2][2];   // top macroblock: quadrants 2 (columns 0-1) and 3 (columns 2-3)
  int cc[2];     // top-right macroblock: quadrant 2
  int d[2];      // top-left macroblock: quadrant 3
};
struct IntBest {
  int x[9], y[9];
  uint32_t c[9];
};
struct SearchSmem {
  uint8_t band[kBandBytes];
  IntBest ib;
  MbNb nb;
  int bmv[4][2], bmvd[4][2], own[4][2], pm[4][2], pd[4][2], qmv[4][2];
  int ccx[8], ccy[8];  // the learned form's centre candidates (ok: cok)
  bool cok[8];
};
__device__ __forceinline__ void ld_q(const MbMv4* m, int q, int* v) {
  uint32_t w = ((const uint32_t*)m)[q];
  v[0] = (int16_t)(w & 0xffffu);
  v[1] = (int16_t)(w >> 16);
}
__device__ __noinline__ MbNb load_nb(const Ctx c) {
  const StreamDev& sd = *c.sd;
  const int mb_w = c.fp->mb_w, mb = c.mb;
  MbNb n;
  n.refA = n.refB = n.refC = n.refD = -2;
  n.a[0][0] = n.a[0][1] = n.a[1][0] = n.a[1][1] = 0;
  n.b[0][0] = n.b[0][1] = n.b[1][0] = n.b[1][1] = 0;
  n.cc[0] = n.cc[1] = n.d[0] = n.d[1] = 0;
  if (c.mbx > 0) {
    n.refA = ld_info(&sd.info[mb - 1]).ref;
    if (n.refA == 0) { ld_q(&sd.mv4[mb - 1], 1, n.a[0]); ld_q(&sd.mv4[mb - 1], 3, n.a[1]); }
  }
  if (c.mby > 0) {
    n.refB = ld_info(&sd.info[mb - mb_w]).ref;
    if (n.refB == 0) { ld_q(&sd.mv4[mb - mb_w], 2, n.b[0]); ld_q(&sd.mv4[mb - mb_w], 3, n.b[1]); }
    if (c.mbx + 1 < mb_w) {
      n.refC = ld_info(&sd.info[mb - mb_w + 1]).ref;
      if (n.refC == 0) ld_q(&sd.mv4[mb - mb_w + 1], 2, n.cc);
    }
    if (c.mbx > 0) {
      n.refD = ld_info(&sd.info[mb - mb_w - 1]).ref;
      if (n.refD == 0) ld_q(&sd.mv4[mb - mb_w - 1], 3, n.d);
    }
  }
  return n;
}
// The 4x4 block at (bx, by) in 4x4 units relative to the macroblock (-1..4); own[q] / done bit q:
// this macroblock's quadrants already decided in the current partition type.
__device__ __forceinline__ NbMv nb4(const MbNb& n, int bx, int by, const int (*own)[2], int done) {
  if (bx >= 0 && bx < 4 && by >= 0 && by < 4) {
    int q = (by >> 1) * 2 + (bx >> 1);
    if ((done >> q) & 1) return {0, own[q][0], own[q][1]};
    return {-2, 0, 0};
  }
  if (bx == -1 && by == -1) return {n.refD, n.d[0], n.d[1]};
  if (bx == -1 && by >= 0 && by < 4) return {n.refA, n.a[by >> 1][0], n.a[by >> 1][1]};
  if (by == -1 && bx >= 0 && bx < 4) return {n.refB, n.b[bx >> 1][0], n.b[bx >> 1][1]};
  if (by == -1 && bx == 4) return {n.refC, n.cc[0], n.cc[1]};
  return {-2, 0, 0};  // right of or below the macroblock: not decoded yet
}
// Motion vector predictor of the partition whose top-left 4x4 block is (bx, by) and width pw (4x4
// units), H.264 8.4.1.3; dir 1 16x8 top, 2 16x8 bottom, 3 8x16 left, 4 8x16 right, 0 median only.
__device__ __noinline__ int2 mv_pred(const MbNb& n, int bx, int by, int pw, int dir, const int (*own)[2], int done) {
  NbMv A = nb4(n, bx - 1, by, own, done), B = nb4(n, bx, by - 1, own, done), C = nb4(n, bx + pw, by - 1, own, done);
  if (C.ref == -2) C = nb4(n, bx - 1, by - 1, own, done);
  if (dir == 1 && B.ref == 0) return make_int2(B.x, B.y);
  if ((dir == 2 || dir == 3) && A.ref == 0) return make_int2(A.x, A.y);
  if (dir == 4 && C.ref == 0) return make_int2(C.x, C.y);
  if (B.ref == -2 && C.ref == -2 && A.ref != -2) return make_int2(A.x, A.y);
  int m = (A.ref == 0) + (B.ref == 0) + (C.ref == 0);
  if (m == 1) {
    const NbMv& o = A.ref == 0 ? A : (B.ref == 0 ? B : C);
    return make_int2(o.x, o.y);
  }
  auto med = [](int x, int y, int z) { return min(max(x, y), max(min(x, y), z)); };
  return make_int2(med(A.x, B.x, C.x), med(A.y, B.y, C.y));
}
// A refined part: its cost and quarter-sample vector.
struct PartFit {
  uint32_t cost;
  int x, y;
};

struct Bounds {
  int min0, min1, max0, max1;  // quarter samples (MvBounds, enc.rs:1105)
};
__device__ __forceinline__ bool in_bounds(const Bounds& b, int x, int y) {
  return x >= b.min0 && x <= b.max0 && y >= b.min1 && y <= b.max1;
}
__device__ __forceinline__ uint32_t vec_cost(int dx, int dy, uint32_t lambda) {
  return lambda * (se_bits(dx) + se_bits(dy));
}

// ---------------------------------------------------------------------------------------------
// Integer search over [xlo, xhi] x [ylo, yhi]. Lanes take columns xlo + lane + 32 j; the reference
// rows of 8 vector rows (band) are staged in shared memory, and each lane slides its column's
// 16 x 16 comparison down the band, a reference row at a time against the source rows it pairs
// with. best_x / best_y / best_c: the nine parts' results (identical in every lane).
__device__ __forceinline__ uint32_t lds4u(const uint8_t* p) {
  uintptr_t a = (uintptr_t)p;
  const uint32_t* b = (const uint32_t*)(a & ~(uintptr_t)3);
  return __funnelshift_r(b[0], b[1], (uint32_t)(a & 3) * 8u);
}
// A window of at most 32 vectors (the learned form's): lane v takes vector v in raster order and
// sums its four quadrant SADs over the staged band; the same costs and ties as the wide search.
__device__ __noinline__ void int_search_small(const Ctx c, const Smem& sm, SearchSmem& ss, int xlo, int xhi, int ylo,
                                              int yhi, int mvp0, int mvp1, uint32_t lambda, IntBest& ib) {
  const int lane = lane_id();
  const int x0 = c.mbx * 16, y0 = c.mby * 16, stride = c.fp->stride_y;
  const uint8_t* ref = c.sd->ref_y;
  const int xs = (x0 + xlo) & ~3;
  const int bw = ((x0 + xhi + 20 - xs) + 3) & ~3;
  const int nwx = xhi - xlo + 1, nwy = yhi - ylo + 1, wpr = bw >> 2;
  __syncwarp();
  for (int w = lane; w < (nwy + 15) * wpr; w += 32) {
    const int r = w / wpr, k = w - r * wpr;
    ((uint32_t*)ss.band)[r * wpr + k] = ldw32(ref + (long)(y0 + ylo + r) * stride + xs + 4 * k);
  }
  __syncwarp();
  const bool act = lane < nwx * nwy;
  const int vx = act ? lane % nwx : 0, vy = act ? lane / nwx : 0;
  const int dx = xlo + vx, dy = ylo + vy;
  const uint8_t* rp = ss.band + vy * bw + (x0 + dx - xs);
  uint32_t q[4] = {0u, 0u, 0u, 0u};
#pragma unroll
  for (int r = 0; r < 16; r++) {
    const uint32_t* sp = (const uint32_t*)&sm.src_y[r * 16];
    const uint8_t* rr = rp + r * bw;
    const int h = (r >> 3) * 2;
    q[h] = __vsadu4(lds4u(rr), sp[0]) + __vsadu4(lds4u(rr + 4), sp[1]) + q[h];
    q[h + 1] = __vsadu4(lds4u(rr + 8), sp[2]) + __vsadu4(lds4u(rr + 12), sp[3]) + q[h + 1];
  }
  const uint32_t mc = lambda * se_bits(4 * dx - mvp0) + lambda * se_bits(4 * dy - mvp1);
  const uint32_t part[9] = {q[0] + q[1] + q[2] + q[3], q[0] + q[1], q[2] + q[3], q[0] + q[2], q[1] + q[3],
                            q[0], q[1], q[2], q[3]};
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const uint32_t cost = act ? part[k] + mc : UMAX;
    const uint32_t m = __reduce_min_sync(FULL, cost);
    const uint32_t i = __reduce_min_sync(FULL, act && cost == m ? (uint32_t)lane : 0xffffffffu);
    ib.c[k] = m;
    ib.x[k] = xlo + (int)(i % (uint32_t)nwx);
    ib.y[k] = ylo + (int)(i / (uint32_t)nwx);
  }
}

__device__ __noinline__ void int_search(const Ctx c, const Smem& sm, SearchSmem& ss, int xlo, int xhi, int ylo, int yhi,
                                        int mvp0, int mvp1, uint32_t lambda, IntBest& ib) {
  if ((xhi - xlo + 1) * (yhi - ylo + 1) <= 32) {
    int_search_small(c, sm, ss, xlo, xhi, ylo, yhi, mvp0, mvp1, lambda, ib);
    return;
  }
  const FrameParams& fp = *c.fp;
  const int lane = lane_id();
  const int x0 = c.mbx * 16, y0 = c.mby * 16, stride = fp.stride_y;
  const uint8_t* ref = c.sd->ref_y;
  const int xs = (x0 + xlo) & ~3;                        // picture column of band column 0
  const int bw = ((x0 + xhi + 20 - xs) + 3) & ~3;        // band row bytes
  const int nwx = xhi - xlo + 1;
  uint32_t bc[9];
  int bi[9];
#pragma unroll
  for (int k = 0; k < 9; k++) { bc[k] = UMAX; bi[k] = 0x7fffffff; }
  for (int dy0 = ylo; dy0 <= yhi; dy0 += kBandRows) {
    const int rows = min(kBandRows, yhi - dy0 + 1) + 15;
    // stage reference rows y0 + dy0 .. + rows - 1, columns xs .. xs + bw - 1 (4-byte loads)
    __syncwarp();
    const int wpr = bw >> 2;
    for (int w = lane; w < rows * wpr; w += 32) {
      int r = w / wpr, k = w - r * wpr;
      ((uint32_t*)ss.band)[r * wpr + k] = ldw32(ref + (long)(y0 + dy0 + r) * stride + xs + 4 * k);
    }
    __syncwarp();
    for (int j = 0; j * 32 < nwx; j++) {
      const int dx = xlo + lane + 32 * j;
      const bool act = lane + 32 * j < nwx;
      const int co = act ? x0 + dx - xs : 0;
      uint32_t top[kBandRows][2];
#pragma unroll
      for (int half = 0; half < 2; half++) {
        uint32_t s[8][4];
#pragma unroll
        for (int r = 0; r < 8; r++)
#pragma unroll
          for (int k = 0; k < 4; k++) s[r][k] = *(const uint32_t*)&sm.src_y[(half * 8 + r) * 16 + 4 * k];
        uint32_t acc[kBandRows][2];
#pragma unroll
        for (int d = 0; d < kBandRows; d++) acc[d][0] = acc[d][1] = 0;
#pragma unroll
        for (int i = 0; i < kBandRows + 7; i++) {
          // reference row half * 8 + i of the band pairs with source row r = i - d for d = 0..7
          const uint8_t* rp = ss.band + (half * 8 + i) * bw + co;
          uint32_t R0 = lds4u(rp), R1 = lds4u(rp + 4), R2 = lds4u(rp + 8), R3 = lds4u(rp + 12);
#pragma unroll
          for (int d = 0; d < kBandRows; d++) {
            const int r = i - d;
            if (r < 0 || r > 7) continue;
            acc[d][0] = __vsadu4(R0, s[r][0]) + __vsadu4(R1, s[r][1]) + acc[d][0];
            acc[d][1] = __vsadu4(R2, s[r][2]) + __vsadu4(R3, s[r][3]) + acc[d][1];
          }
        }
        if (half == 0) {
#pragma unroll
          for (int d = 0; d < kBandRows; d++) { top[d][0] = acc[d][0]; top[d][1] = acc[d][1]; }
        } else {
          const uint32_t cx = lambda * se_bits(4 * dx - mvp0);
#pragma unroll
          for (int d = 0; d < kBandRows; d++) {
            const int dy = dy0 + d;
            if (!act || dy > yhi) continue;
            const uint32_t mc = cx + lambda * se_bits(4 * dy - mvp1);
            const uint32_t q0 = top[d][0], q1 = top[d][1], q2 = acc[d][0], q3 = acc[d][1];
            const uint32_t part[9] = {q0 + q1 + q2 + q3, q0 + q1, q2 + q3, q0 + q2, q1 + q3, q0, q1, q2, q3};
            const int idx = (dy - ylo) * nwx + (dx - xlo);
#pragma unroll
            for (int k = 0; k < 9; k++) {
              const uint32_t cost = part[k] + mc;
              if (cost < bc[k] || (cost == bc[k] && idx < bi[k])) { bc[k] = cost; bi[k] = idx; }
            }
          }
        }
      }
    }
  }
  // first minimum in raster order across the warp
#pragma unroll
  for (int k = 0; k < 9; k++) {
    uint32_t m = __reduce_min_sync(FULL, bc[k]);
    uint32_t i = __reduce_min_sync(FULL, bc[k] == m ? (uint32_t)bi[k] : 0xffffffffu);
    ib.c[k] = m;
    ib.x[k] = xlo + (int)(i % (uint32_t)nwx);
    ib.y[k] = ylo + (int)(i / (uint32_t)nwx);
  }
}

// ---------------------------------------------------------------------------------------------
// Quarter-sample refinement of one part (px, py, pw, ph samples within the macroblock) from its
// integer best (bx, by) with predictor mvp. Candidates of one step are evaluated in parallel: slot
// = candidate * blocks + 4x4 block, each lane the SATD of one block's prediction (from the
// half-sample planes of a window around the integer best) against the source.
__device__ __forceinline__ uint32_t satd4_regs(const uint32_t* sa, const uint32_t* pa) {
  int t[4][4];
#pragma unroll
  for (int y = 0; y < 4; y++) {
    int d[4];
#pragma unroll
    for (int x = 0; x < 4; x++) d[x] = (int)((sa[y] >> (8 * x)) & 255) - (int)((pa[y] >> (8 * x)) & 255);
    int s03 = d[0] + d[3], s12 = d[1] + d[2], d03 = d[0] - d[3], d12 = d[1] - d[2];
    t[y][0] = s03 + s12; t[y][1] = d03 + d12; t[y][2] = s03 - s12; t[y][3] = d03 - d12;
  }
  uint32_t s = 0;
#pragma unroll
  for (int x = 0; x < 4; x++) {
    int s03 = t[0][x] + t[3][x], s12 = t[1][x] + t[2][x], d03 = t[0][x] - t[3][x], d12 = t[1][x] - t[2][x];
    s += abs(s03 + s12) + abs(d03 + d12) + abs(s03 - s12) + abs(d03 - d12);
  }
  return s;
}
// The 4x4 prediction at window position (wx, wy), phase (fx, fy): four packed rows.
__device__ __forceinline__ void qpel4(const Smem& sm, int wx, int wy, int fx, int fy, uint32_t* out) {
  QSrc q = qpel_src(sm, wx, wy, fx, fy);
#pragma unroll
  for (int r = 0; r < 4; r++) {
    uint32_t a = lds4u(q.a + r * q.sa);
    out[r] = q.avg ? __vavgu4(a, lds4u(q.b + r * q.sb)) : a;
  }
}
__device__ __constant__ int8_t c_hstep[8][2] = {{0, -2}, {-2, 0}, {2, 0}, {0, 2}, {-2, -2}, {2, -2}, {-2, 2}, {2, 2}};

// The half-sample planes in shared memory serve every part whose integer vector they were built
// around: a macroblock-level window (origin one sample above-left of the macroblock displaced by the
// vector) covers every 4x4 block of the macroblock at quarter-sample offsets -3..3.
struct WinState {
  int bx, by;  // integer vector of the planes held, or kNoWin
};
constexpr int kNoWin = 1 << 20;
__device__ __forceinline__ void ensure_window(const Ctx c, Smem& sm, WinState& ws, int bx, int by) {
  if (ws.bx == bx && ws.by == by) return;
  stage_window(c.sd->ref_y, c.fp->stride_y, c.mbx * 16 + bx - 1, c.mby * 16 + by - 1, sm);
  build_hpel(sm, 7);
  ws.bx = bx;
  ws.by = by;
}

__device__ __noinline__ PartFit refine_part(const Ctx c, Smem& sm, WinState& ws, int px, int py, int pw, int ph, int bx,
                                            int by, int2 mvp, uint32_t lambda, Bounds bd) {
  const int lane = lane_id();
  ensure_window(c, sm, ws, bx, by);
  const int bw4 = pw >> 2, nblk = bw4 * (ph >> 2);
  const int m0x = 4 * bx, m0y = 4 * by;
  int cx = m0x, cy = m0y;
  uint32_t best_key = UMAX;
  for (int step = 0; step < 2; step++) {
    const int ncand = step == 0 ? 9 : 8;
    const int sc = step == 0 ? 1 : 2;  // step 0: centre + distance 2; step 1: distance 1
    uint32_t key = step == 0 ? UMAX : best_key & ~15u;  // the current best keeps index 0
    for (int base = 0; base < ncand * nblk; base += 32) {
      const int slot = base + lane;
      const int cand = slot / nblk, blk = slot - cand * nblk;
      int vx = cx, vy = cy;
      if (cand < ncand) {
        if (step == 0 && cand > 0) { vx += c_hstep[cand - 1][0]; vy += c_hstep[cand - 1][1]; }
        if (step == 1) { vx += c_hstep[cand][0] / sc; vy += c_hstep[cand][1] / sc; }
      }
      const bool ok = cand < ncand && in_bounds(bd, vx, vy);
      uint32_t s = 0;
      if (ok) {
        const int ox = 4 * (blk % bw4), oy = 4 * (blk / bw4);
        uint32_t pa[4], sa[4];
        qpel4(sm, (vx >> 2) - bx + 1 + px + ox, (vy >> 2) - by + 1 + py + oy, vx & 3, vy & 3, pa);
#pragma unroll
        for (int r = 0; r < 4; r++) sa[r] = *(const uint32_t*)&sm.src_y[(py + oy + r) * 16 + px + ox];
        s = satd4_regs(sa, pa);
      }
      // sum over the candidate's blocks (consecutive lanes; nblk divides 32)
      for (int o = 1; o < nblk; o <<= 1) s += __shfl_xor_sync(FULL, s, o);
      uint32_t k = UMAX;
      if (ok && blk == 0) {
        uint32_t cost = (s >> 1) + vec_cost(vx - mvp.x, vy - mvp.y, lambda);
        k = (cost << 4) | (uint32_t)(step == 0 ? cand : cand + 1);
      }
      key = min(key, __reduce_min_sync(FULL, k));
    }
    // the winner's vector
    const int wi = (int)(key & 15u);
    if (step == 0) {
      if (wi > 0) { cx += c_hstep[wi - 1][0]; cy += c_hstep[wi - 1][1]; }
    } else if (wi > 0) {
      cx += c_hstep[wi - 1][0] / 2;
      cy += c_hstep[wi - 1][1] / 2;
    }
    best_key = (key & ~15u);
  }
  return PartFit{best_key >> 4, cx, cy};
}

// Learned form: refinement of one part from its integer best (bx, by) by SAD -- the half-sample
// diamond (up, left, right, down at distance 2, one step), then the quarter-sample diamond (the
// same at distance 1, up to two steps, each from the step's start), cost SAD + lambda * vector bits
// against the part's predictor, the first strict minimum in that order; lanes take the part's
// 4-sample words, one candidate at a time.
__device__ __noinline__ uint32_t part_sad(const Smem& sm, int px, int py, int pw, int ph, int bx, int by, int vx, int vy) {
  const int lane = lane_id();
  const QSrc q = qpel_src(sm, (vx >> 2) - bx + 1 + px, (vy >> 2) - by + 1 + py, vx & 3, vy & 3);
  const int wpr = pw >> 2, nw = wpr * ph;
  uint32_t s = 0;
  for (int w = lane; w < nw; w += 32) {
    const int r = w / wpr, x = (w - r * wpr) * 4;
    uint32_t a = lds4u(q.a + r * q.sa + x);
    if (q.avg) a = __vavgu4(a, lds4u(q.b + r * q.sb + x));
    s = __vsadu4(a, *(const uint32_t*)&sm.src_y[(py + r) * 16 + px + x]) + s;
  }
  return wsum(s);
}
__device__ __noinline__ PartFit refine_part_sad(const Ctx c, Smem& sm, WinState& ws, int px, int py, int pw, int ph,
                                                int bx, int by, int2 mvp, uint32_t lambda, Bounds bd) {
  ensure_window(c, sm, ws, bx, by);
  int cx = 4 * bx, cy = 4 * by;
  uint32_t best = part_sad(sm, px, py, pw, ph, bx, by, cx, cy) + vec_cost(cx - mvp.x, cy - mvp.y, lambda);
  for (int st = 2; st >= 1; st--) {
    for (int it = 0; it < (st == 2 ? 1 : 2); it++) {
      const int fx = cx, fy = cy;
      for (int k = 0; k < 4; k++) {
        const int vx = fx + (k == 1 ? -st : (k == 2 ? st : 0)), vy = fy + (k == 0 ? -st : (k == 3 ? st : 0));
        if (abs(vx - 4 * bx) > 3 || abs(vy - 4 * by) > 3 || !in_bounds(bd, vx, vy)) continue;  // uniform
        const uint32_t cost = part_sad(sm, px, py, pw, ph, bx, by, vx, vy) + vec_cost(vx - mvp.x, vy - mvp.y, lambda);
        if (cost < best) { best = cost; cx = vx; cy = vy; }
      }
      if (cx == fx && cy == fy) break;
    }
  }
  return PartFit{best, cx, cy};
}

// The luma prediction of a part at quarter-sample vector mv (within 3 quarter samples of 4 (bx, by),
// the integer vector its refinement started from) into pred_y.
__device__ __noinline__ void predict_part(const Ctx c, Smem& sm, WinState& ws, int px, int py, int pw, int ph, int bx,
                                          int by, int mvx, int mvy) {
  const int lane = lane_id();
  ensure_window(c, sm, ws, bx, by);
  QSrc q = qpel_src(sm, (mvx >> 2) - bx + 1 + px, (mvy >> 2) - by + 1 + py, mvx & 3, mvy & 3);
  for (int i = lane; i < pw * ph; i += 32) {
    const int r = i / pw, x = i - r * pw;
    int v = q.a[r * q.sa + x];
    if (q.avg) v = (v + q.b[r * q.sb + x] + 1) >> 1;
    sm.pred_y[(py + r) * 16 + px + x] = (uint8_t)v;
  }
  __syncwarp();
}
// Chroma prediction of both planes with each 8x8 luma quadrant's own vector (4x4 chroma blocks;
// the bilinear 1/8-sample filter of chroma_mc_8x8_x2, h264_enc.rs:1279, per sample).
__device__ __noinline__ void mc_chroma_q(const Ctx c, Smem& sm, const int (*qmv)[2]) {
  const FrameParams& fp = *c.fp;
  const StreamDev& sd = *c.sd;
  const int lane = lane_id();
  const int plane = lane >> 4, idx = (lane & 15) * 4, r = idx >> 3, c0 = idx & 7;
  const int q = (r >> 2) * 2 + (c0 >> 2);
  const int mvx = qmv[q][0], mvy = qmv[q][1];
  const int cx = c.mbx * 8 + c0 + (mvx >> 3), cy = c.mby * 8 + r + (mvy >> 3), fx = mvx & 7, fy = mvy & 7;
  const int wa = (8 - fx) * (8 - fy), wb = fx * (8 - fy), wc = (8 - fx) * fy, wd = fx * fy;
  const uint8_t* src = (plane ? sd.ref_v : sd.ref_u) + (long)cy * fp.stride_c + cx;
  uint8_t* out = (plane ? sm.pred_v : sm.pred_u) + r * 8 + c0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    int a = ldcg_u8(src + k), b = ldcg_u8(src + k + 1), cc = ldcg_u8(src + fp.stride_c + k), d = ldcg_u8(src + fp.stride_c + k + 1);
    out[k] = (uint8_t)((wa * a + wb * b + wc * cc + wd * d + 32) >> 6);
  }
  __syncwarp();
}

// Search-form side state of a coded macroblock: the record's partition fields and the quadrant
// vectors later macroblocks and the deblocking filter read (lane 0 writes).
__device__ __noinline__ void search_tail(const Ctx c, int ptype, const int (*qmv)[2], const int (*pmvd)[2]) {
  if (lane_id() != 0) return;
  rg_mb_out* rec = c.sd->rec + c.mb;
  MbMv4 m;
  for (int q = 0; q < 4; q++) {
    m.mv[q][0] = (int16_t)qmv[q][0];
    m.mv[q][1] = (int16_t)qmv[q][1];
    rec->part_mv[q][0] = (int16_t)qmv[q][0];
    rec->part_mv[q][1] = (int16_t)qmv[q][1];
    rec->part_mvd[q][0] = (int16_t)pmvd[q][0];
    rec->part_mvd[q][1] = (int16_t)pmvd[q][1];
  }
  rec->part_type = (uint8_t)ptype;
  rec->reserved2[0] = rec->reserved2[1] = rec->reserved2[2] = 0;
  c.sd->mv4[c.mb] = m;
}

// Reach of a search window for the pipelined mode's wait on the reference picture: every
// sample the integer search (band staging), the refinement windows and the final prediction can
// read lies above row (y0 + yhi + 28) and left of column (x0 + xhi + 36); everything above and
// to the left of the macroblock holding that sample is final once it is.
__device__ __noinline__ bool wait_window(const Ctx c, PipeWait* pw, int xhi, int yhi) {
  const FrameParams& fp = *c.fp;
  if (!pw) return true;
  const int x0 = c.mbx * 16, y0 = c.mby * 16;
  const int xb = (x0 + xhi + 36) >> 4, rb = (y0 + yhi + 28) >> 4;
  const int rr = min(max(rb, 0), fp.mb_h - 1), xx = min(max(xb, 0), fp.mb_w - 1);
  const int row = rr < fp.mb_h - 1 ? rr + 1 : rr, need = rr < fp.mb_h - 1 ? xx + 1 : min(xx + 2, fp.mb_w);
  pw->reach_y = max(pw->reach_y, max(rr - c.mby - 2, 0) + 1);
  pw->reach_x = max(pw->reach_x, max(xx - c.mbx - 2, 0) + 1);
  if (row != pw->db_row) {
    pw->db_row = row;
    pw->seen_db = 0;
  }
  if (!wait_seen(pw->db_prev + row, need, pw->seen_db, pw->error, pw->timeout_ns)) {
    pw->failed = true;
    return false;
  }
  return true;
}

// P_Skip probe of the plain form (enc.rs:2906 try_p_skip) at skip vector (ps0, ps1): true when the
// macroblock is coded as P_Skip (prediction left in pred_y / pred_u / pred_v).
__device__ __noinline__ bool skip_probe(const Ctx c, Smem& sm, int ps0, int ps1, const Bounds& bd) {
  const FrameParams& fp = *c.fp;
  const StreamDev& sd = *c.sd;
  const int lane = lane_id();
  if (!in_bounds(bd, ps0, ps1)) return false;
  mc_luma16(sd.ref_y, fp.stride_y, c.mbx * 16, c.mby * 16, ps0, ps1, sm);
  uint2 s = src8(sm), p = *(const uint2*)&sm.pred_y[(lane >> 1) * 16 + (lane & 1) * 8];
  uint32_t sad = wsum(vsad8(s, p));
  if (sad >= sd.sb_probe) return false;
  bool lz = sad <= sd.sb_luma;
  if (!lz) {
    uint32_t ssd = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      int d0 = (int)((s.x >> (8 * k)) & 255) - (int)((p.x >> (8 * k)) & 255);
      int d1 = (int)((s.y >> (8 * k)) & 255) - (int)((p.y >> (8 * k)) & 255);
      ssd += d0 * d0 + d1 * d1;
    }
    lz = wsum(ssd) <= sd.sb_luma_ssd;
  }
  if (!lz) lz = probe_skip_luma(sd.qp, sm);
  if (!lz) return false;
  mc_chroma8(sd.ref_u, sd.ref_v, fp.stride_c, c.mbx, c.mby, ps0, ps1, sm);
  int plane = lane >> 4, idx = (lane & 15) * 4;
  const uint8_t* ssrc = (plane ? sm.src_v : sm.src_u) + idx;
  const uint8_t* pp = (plane ? sm.pred_v : sm.pred_u) + idx;
  uint32_t sadp = 0, ssdp = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) { int d = (int)ssrc[k] - (int)pp[k]; sadp += abs(d); ssdp += d * d; }
  uint32_t sad_u = wsum(plane == 0 ? sadp : 0), sad_v = wsum(plane == 1 ? sadp : 0);
  uint32_t ssd_u = wsum(plane == 0 ? ssdp : 0), ssd_v = wsum(plane == 1 ? ssdp : 0);
  bool cz = (sad_u <= sd.sb_chroma || ssd_u <= sd.sb_chroma_ssd) && (sad_v <= sd.sb_chroma || ssd_v <= sd.sb_chroma_ssd);
  if (!cz) {
    uint32_t ac_any[2], ac_sc[2];
    chroma_quant(sd.qpc, false, sm, ac_any, ac_sc);
    cz = !chroma_dc_any(sm) && ac_sc[0] < 7 && ac_sc[1] < 7;
  }
  return cz;
}

// Learned form: the centre of the first +-2 window among n integer candidates (cx, cy; ok false:
// absent) -- the first of least 16x16 SAD + lambda * vector bits against the 16x16 predictor.
__device__ __noinline__ void learned_centre(const Ctx c, const Smem& sm, const int* cx, const int* cy, const bool* ok,
                                            int n, int mvp0, int mvp1, uint32_t lambda, int& bx, int& by) {
  const int lane = lane_id();
  const int stride = c.fp->stride_y;
  const uint8_t* base = c.sd->ref_y + (long)(c.mby * 16 + (lane >> 1)) * stride + c.mbx * 16 + (lane & 1) * 8;
  const uint2 sv = src8(sm);
  uint2 r[kCentreCands];
#pragma unroll
  for (int k = 0; k < kCentreCands; k++) r[k] = k < n && ok[k] ? ldg8(base + (long)cy[k] * stride + cx[k]) : make_uint2(0u, 0u);
  uint32_t best = UMAX;
  bx = cx[0];
  by = cy[0];
#pragma unroll
  for (int k = 0; k < kCentreCands; k++) {
    if (k >= n || !ok[k]) continue;  // uniform across the warp
    const uint32_t cost = fullpel_cost(sv, r[k], cx[k], cy[k], mvp0, mvp1, lambda);
    if (cost < best) { best = cost; bx = cx[k]; by = cy[k]; }
  }
}

// Partition geometry in coding order: {type, first part, parts}; part k: {px, py, pw, ph, bx, by,
// pw4, dir, integer-search index}.
__device__ __constant__ int8_t c_parts[9][9] = {
    {0, 0, 16, 16, 0, 0, 4, 0, 0},                                  // 16x16
    {0, 0, 16, 8, 0, 0, 4, 1, 1}, {0, 8, 16, 8, 0, 2, 4, 2, 2},      // 16x8
    {0, 0, 8, 16, 0, 0, 2, 3, 3}, {8, 0, 8, 16, 2, 0, 2, 4, 4},      // 8x16
    {0, 0, 8, 8, 0, 0, 2, 0, 5}, {8, 0, 8, 8, 2, 0, 2, 0, 6},        // 8x8
    {0, 8, 8, 8, 0, 2, 2, 0, 7}, {8, 8, 8, 8, 2, 2, 2, 0, 8}};
__device__ __constant__ int8_t c_type_first[4] = {0, 1, 3, 5};
__device__ __constant__ int8_t c_type_parts[4] = {1, 2, 2, 4};
// quadrants covered by part k (bit mask)
__device__ __constant__ uint8_t c_part_quads[9] = {15, 3, 12, 5, 10, 1, 2, 4, 8};

// One macroblock of a P slice in the search forms (see the head of this file).
__device__ __noinline__ void analyse_p_mb_search(const Ctx c, Smem& sm, SearchSmem& ss, PipeWait* pw) {
  const FrameParams& fp = *c.fp;
  const StreamDev& sd = *c.sd;
  const int lane = lane_id();
  const int mbx = c.mbx, mby = c.mby;
  const int x0 = mbx * 16, y0 = mby * 16;
  const int qp = sd.qp, qpc = sd.qpc;
  const uint32_t lambda = c_lambda[qp];
  const int cw = fp.mb_w * 16, chh = fp.mb_h * 16;
  Bounds bd;
  bd.min0 = -4 * (x0 + 28);
  bd.min1 = max(-4 * (y0 + 28), -2048);
  bd.max0 = 4 * (cw - 16 - x0 + 28);
  bd.max1 = min(4 * (chh - 16 - y0 + 28), 2044);
  const int imin0 = (bd.min0 + 3) >> 2, imin1 = (bd.min1 + 3) >> 2, imax0 = bd.max0 >> 2, imax1 = bd.max1 >> 2;
  // Warp-uniform state (every lane computes the same values) is held once per warp in shared memory
  // (SearchSmem) instead of once per lane on the stack; every lane writes the same value, and a
  // __syncwarp before each rewrite keeps a lane from overwriting what a slower lane still reads.
  MbNb& nb = ss.nb;
  __syncwarp();
  nb = load_nb(c);
  int none[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  const int2 p16 = mv_pred(nb, 0, 0, 4, 0, none, 0);
  const int mvp16[2] = {p16.x, p16.y};
  int ps0 = mvp16[0], ps1 = mvp16[1];
  {
    NbMv A = nb4(nb, -1, 0, none, 0), B = nb4(nb, 0, -1, none, 0);
    if (mbx == 0 || mby == 0 || (A.ref == 0 && A.x == 0 && A.y == 0) || (B.ref == 0 && B.x == 0 && B.y == 0)) {
      ps0 = 0;
      ps1 = 0;
    }
  }
  load_source(c, sm);
  const rg_mb_hint* hint = sd.hint ? sd.hint + c.mb : nullptr;
  // integer window: full search, or the learned seed's small window
  const int R = sd.search_range;
  int fcx = min(max((mvp16[0] + 2) >> 2, imin0), imax0), fcy = min(max((mvp16[1] + 2) >> 2, imin1), imax1);
  int xlo = max(fcx - R, imin0), xhi = min(fcx + R, imax0), ylo = max(fcy - R, imin1), yhi = min(fcy + R, imax1);
  int part_mask = 15;
  // learned: the candidates of the first window's centre (integer, clamped to the bounds)
  int* ccx = ss.ccx;  // warp-uniform, in shared memory
  int* ccy = ss.ccy;
  bool* cok = ss.cok;
  if (hint) {
    NbMv A = nb4(nb, -1, 0, none, 0), B = nb4(nb, 0, -1, none, 0), C = nb4(nb, 4, -1, none, 0);
    if (C.ref == -2) C = nb4(nb, -1, -1, none, 0);
    const int vx[kCentreCands] = {mvp16[0] + hint->mv_off[0], mvp16[0], hint->mv_coarse[0], A.x, B.x, C.x, 0};
    const int vy[kCentreCands] = {mvp16[1] + hint->mv_off[1], mvp16[1], hint->mv_coarse[1], A.y, B.y, C.y, 0};
    const bool use[kCentreCands] = {true, true, (hint->flags & 1) != 0, A.ref == 0, B.ref == 0, C.ref == 0, true};
    xhi = -(1 << 20);
    yhi = -(1 << 20);
#pragma unroll
    for (int k = 0; k < kCentreCands; k++) {
      ccx[k] = min(max((vx[k] + 2) >> 2, imin0), imax0);
      ccy[k] = min(max((vy[k] + 2) >> 2, imin1), imax1);
      cok[k] = use[k];
      if (use[k]) {
        xhi = max(xhi, min(ccx[k] + kLearnedRange, imax0));
        yhi = max(yhi, min(ccy[k] + kLearnedRange, imax1));
      }
    }
    part_mask = hint->part_mask & 15;
    if (!part_mask) part_mask = 1;
  }
  // the reference region of the skip probe and the search window (learned: every candidate's)
  if (!wait_window(c, pw, max(xhi, (max(ps0, 0) + 3) >> 2), max(yhi, (max(ps1, 0) + 3) >> 2))) return;
  const int off4[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  // 1. skip probe
  if (skip_probe(c, sm, ps0, ps1, bd)) {
    code_skip(c, sm, ps0, ps1);
    int q4[4][2] = {{ps0, ps1}, {ps0, ps1}, {ps0, ps1}, {ps0, ps1}};
    search_tail(c, 255, q4, off4);
    return;
  }
  // 2. integer search
  if (hint) {
    int lcx, lcy;
    learned_centre(c, sm, ccx, ccy, cok, kCentreCands, mvp16[0], mvp16[1], lambda, lcx, lcy);
    xlo = max(lcx - kLearnedRange, imin0);
    xhi = min(lcx + kLearnedRange, imax0);
    ylo = max(lcy - kLearnedRange, imin1);
    yhi = min(lcy + kLearnedRange, imax1);
  }
  IntBest& ib = ss.ib;  // warp-uniform: once per warp in shared memory
  int_search(c, sm, ss, xlo, xhi, ylo, yhi, mvp16[0], mvp16[1], lambda, ib);
  if (hint) {
    bool edge = (ib.x[0] == xlo && xlo > imin0) || (ib.x[0] == xhi && xhi < imax0) ||
                (ib.y[0] == ylo && ylo > imin1) || (ib.y[0] == yhi && yhi < imax1);
    for (int it = 0; edge && it < sd.walk; it++) {  // centre the window on its best again
      const int cx = ib.x[0], cy = ib.y[0];
      xlo = max(cx - kLearnedRange, imin0);
      xhi = min(cx + kLearnedRange, imax0);
      ylo = max(cy - kLearnedRange, imin1);
      yhi = min(cy + kLearnedRange, imax1);
      if (!wait_window(c, pw, xhi, yhi)) return;
      int_search(c, sm, ss, xlo, xhi, ylo, yhi, mvp16[0], mvp16[1], lambda, ib);
      edge = (ib.x[0] == xlo && xlo > imin0) || (ib.x[0] == xhi && xhi < imax0) ||
             (ib.y[0] == ylo && ylo > imin1) || (ib.y[0] == yhi && yhi < imax1);
    }
    if (edge) {  // the walk did not reach the minimum: full search
      xlo = max(fcx - R, imin0); xhi = min(fcx + R, imax0);
      ylo = max(fcy - R, imin1); yhi = min(fcy + R, imax1);
      if (!wait_window(c, pw, xhi, yhi)) return;
      int_search(c, sm, ss, xlo, xhi, ylo, yhi, mvp16[0], mvp16[1], lambda, ib);
    }
  }
  // 3-4. refinement of every tried type, the least total cost wins
  int best_t = -1;
  uint32_t best_j = UMAX;
  int (&bmv)[4][2] = ss.bmv;  // per part (coding order) of the best type (warp-uniform, shared)
  int (&bmvd)[4][2] = ss.bmvd;
  WinState ws{kNoWin, kNoWin};  // the skip probe's window is not a refinement window
  for (int t = 0; t < 4; t++) {
    if (!((part_mask >> t) & 1)) continue;
    int (&own)[4][2] = ss.own;
    __syncwarp();
    for (int q = 0; q < 4; q++) own[q][0] = own[q][1] = 0;
    int done = 0;
    uint32_t J = lambda * (uint32_t)sd.type_bits[t];
    int (&pm)[4][2] = ss.pm;
    int (&pd)[4][2] = ss.pd;
    const int first = c_type_first[t], np = c_type_parts[t];
    for (int k = 0; k < np; k++) {
      const int8_t* g = c_parts[first + k];
      const int2 mvp = mv_pred(nb, g[4], g[5], g[6], g[7], own, done);
      const PartFit fit = hint ? refine_part_sad(c, sm, ws, g[0], g[1], g[2], g[3], ib.x[g[8]], ib.y[g[8]], mvp, lambda, bd)
                               : refine_part(c, sm, ws, g[0], g[1], g[2], g[3], ib.x[g[8]], ib.y[g[8]], mvp, lambda, bd);
      const int mv[2] = {fit.x, fit.y};
      J += fit.cost;
      pm[k][0] = mv[0]; pm[k][1] = mv[1];
      pd[k][0] = mv[0] - mvp.x; pd[k][1] = mv[1] - mvp.y;
      const int qm = c_part_quads[first + k];
      for (int q = 0; q < 4; q++)
        if ((qm >> q) & 1) { own[q][0] = mv[0]; own[q][1] = mv[1]; }
      done |= qm;
    }
    if (J < best_j) {
      best_j = J;
      best_t = t;
      for (int k = 0; k < 4; k++) {
        bmv[k][0] = k < np ? pm[k][0] : 0; bmv[k][1] = k < np ? pm[k][1] : 0;
        bmvd[k][0] = k < np ? pd[k][0] : 0; bmvd[k][1] = k < np ? pd[k][1] : 0;
      }
    }
  }
  // quadrant vectors of the chosen type and its prediction
  int (&qmv)[4][2] = ss.qmv;
  __syncwarp();
  {
    const int first = c_type_first[best_t], np = c_type_parts[best_t];
    for (int k = 0; k < np; k++) {
      const int qm = c_part_quads[first + k];
      for (int q = 0; q < 4; q++)
        if ((qm >> q) & 1) { qmv[q][0] = bmv[k][0]; qmv[q][1] = bmv[k][1]; }
      const int8_t* g = c_parts[first + k];
      predict_part(c, sm, ws, g[0], g[1], g[2], g[3], ib.x[g[8]], ib.y[g[8]], bmv[k][0], bmv[k][1]);
    }
  }
  // 5. intra 16x16 when the inter prediction is poor (the plain form's rule, enc.rs:3121-3156)
  uint32_t inter_satd = 0;
  if (lane < 16) {
    int bx = lane & 3, by = lane >> 2;
    inter_satd = satd4(&sm.src_y[by * 64 + bx * 4], 16, &sm.pred_y[by * 64 + bx * 4], 16);
  }
  inter_satd = wsum(inter_satd) >> 1;
  if (inter_satd > 24 * lambda) {
    int tl, ctl[2];
    load_edges(c, sm, false, tl, ctl);
    bool ht = mby > 0, hl = mbx > 0;
    uint32_t i16c;
    int i16m = analyse_i16(sm, ht, hl, tl, &i16c);
    if (i16c + lambda * 8 < best_j) {
      code_i16(c, sm, i16m, ht, hl, tl, ctl);
      int z[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
      search_tail(c, best_t, z, z);
      return;
    }
  }
  // residual (enc.rs:3158-3190)
  mc_chroma_q(c, sm, qmv);
  uint32_t nz_lane;
  int cbp4 = luma4x4_inter(qp, sm, &nz_lane);
  int cbpl = cbp4;
  bool use8 = false;
  if (fp.t8x8 && cbp4) {
    uint32_t nnz4 = 0;
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
  if (best_t == 0 && cbpl == 0 && cbpc == 0 && bmv[0][0] == ps0 && bmv[0][1] == ps1) {
    code_skip(c, sm, ps0, ps1);
    search_tail(c, best_t, qmv, off4);
    return;
  }
  rg_mb_out* rec = sd.rec + c.mb;
  bool t8flag = use8 && cbpl != 0;
  uint16_t nzm;
  if (use8) {
    int b = lane >> 3, q = lane & 7;
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
    const int types[4] = {RG_MB_P_L0_16X16, RG_MB_P_L0_16X8, RG_MB_P_L0_8X16, RG_MB_P_8X8};
    record_header(rec, types[best_t], 0, 0, cbpl | (cbpc << 4), t8flag, qp, bmv[0][0], bmv[0][1], bmvd[0][0],
                  bmvd[0][1], nzm);
    write_info(c, t8flag ? kFlagT8 : 0, cbpl, bmv[0][0], bmv[0][1], 0, nzm, nullptr);
  }
  search_tail(c, best_t, qmv, bmvd);
  if (use8) recon_luma8x8(sm, qp, cbpl);
  else if (cbpl) recon_luma4x4(sm, qp, cbpl);
  __syncwarp();
  chroma_recon(qpc, cbpc, sm);
  store_recon(c, sm.pred_y, sm);
  (void)nz_lane;
}

// One macroblock of an I slice in the search forms: the plain analysis (enc.rs:3311 code_intra),
// intra 4x4 blocks restricted to the hinted modes in the learned form.
__device__ __noinline__ void analyse_intra_mb_search(const Ctx c, Smem& sm) {
  int tl, ctl[2];
  load_edges(c, sm, true, tl, ctl);
  bool ht = c.mby > 0, hl = c.mbx > 0;
  uint32_t lambda = c_lambda[c.sd->qp];
  uint32_t i16c;
  int i16m = analyse_i16(sm, ht, hl, tl, &i16c);
  const int z[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  if (i16c > 40 * lambda) {
    int cbpl;
    const uint16_t* masks = c.sd->hint ? c.sd->hint[c.mb].i4_mask : nullptr;
    bool ok = masks ? analyse_i4<true>(c, sm, i16c + lambda * 4, ht, hl, tl, &cbpl, masks)
                    : analyse_i4<false>(c, sm, i16c + lambda * 4, ht, hl, tl, &cbpl, nullptr);
    if (ok) {
      code_i4(c, sm, cbpl, ht, hl, ctl);
      search_tail(c, 255, z, z);
      return;
    }
  }
  code_i16(c, sm, i16m, ht, hl, tl, ctl);
  search_tail(c, 255, z, z);
}
