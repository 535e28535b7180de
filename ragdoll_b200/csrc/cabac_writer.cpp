// CABAC slice data from the engine's macroblock records (host code, no GPU): the serial half of
// encode_frame_body (crates/ragdoll-codec/src/h264/enc.rs:2346-2440) for Main and High profile
// slices of the Balanced preset -- mb_skip_flag, mb_type, transform_size_8x8_flag, intra
// prediction modes, mvd, coded_block_pattern, mb_qp_delta, the residual blocks of categories 0-5
// and end_of_slice_flag.
//
// The arithmetic coder follows the encoding process of ITU-T H.264 9.3.4 a byte at a time
// (carries resolved when the slice is done), and the context indices come from the
// derivations of 9.3.3.1.1 evaluated on a small per-macroblock summary (flags, coded block
// pattern, a 16-bit mask of the luma 4x4 blocks holding levels, 4-bit masks per chroma plane,
// |mvd|) kept for the row above and the macroblock to the left. The reference uses the same
// derivations (cabac.rs:562-1130, h264.rs:3293-3553); the bytes are equal for equal records.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#if defined(__AVX2__) && defined(__BMI2__)
#include <immintrin.h>
#endif

#include "bitstream.h"
#include "cabac_tables.h"

namespace rg {

namespace {

using cabac::kContexts;

// The arithmetic coder of ITU-T H.264 9.3.4.2-9.3.4.5, a byte at a time. `low` holds the code
// value's bits from the highest one not yet written (position `top`) down to the 10-bit window
// of the standard's codILow; a byte is split off once its 8 bits lie above the window. An
// addition to `low` may carry into bytes already split off: each byte is kept with the carry it
// received (up to 9 bits) and the carries are resolved, last byte first, when the slice is done.
// The first bit of the code value (the standard's firstBitFlag) is always 0 and never written.
// Context models are packed as pStateIdx << 1 | valMPS.
// The model after coding bin b with model m (pStateIdx << 1 | valMPS), at [2 m + b]: the
// transitions of 9.3.3.2.2 in one table.
struct ModelNext {
  uint8_t v[256];
  constexpr ModelNext() : v() {
    for (int m = 0; m < 128; m++)
      for (int b = 0; b < 2; b++) {
        int state = m >> 1, mps = m & 1;
        if (b != mps) {
          if (state == 0) mps ^= 1;
          state = cabac::kNextLps[state];
        } else if (state < 62) {
          state++;
        }
        v[2 * m + b] = (uint8_t)(state << 1 | mps);
      }
  }
};
constexpr ModelNext kModelNext{};

class Arith {
 public:
  explicit Arith(std::vector<uint8_t>& out) : out_(out) { pend_.reserve(1 << 16); }

  void decision(uint8_t& model, unsigned bin) {
    const unsigned m = model, state = m >> 1, lpsb = bin ^ (m & 1u);
    const uint32_t lps = cabac::kRangeLps[state][(range_ >> 6) & 3];
    const uint32_t rmps = range_ - lps;
    // the least probable symbol adds the MPS sub-range to low and keeps the LPS sub-range
    low_ += lpsb ? rmps : 0u;
    range_ = lpsb ? lps : rmps;
    model = kModelNext.v[2 * m + bin];
    const int shift = __builtin_clz(range_) - 23;  // range_ < 512: doubles it to 256..511
    range_ <<= shift;
    low_ <<= shift;
    top_ += shift;
    split();
  }
  void bypass(unsigned bin) {
    low_ <<= 1;
    if (bin) low_ += range_;
    top_++;
    split();
  }
  // end_of_slice_flag; 1 flushes the coder (9.3.4.5): the rest of the code value down to bit 8
  // of the window, then rbsp_stop_one_bit, zeros to the byte boundary, and the carries resolved.
  void terminate(unsigned bin) {
    range_ -= 2;
    if (!bin) {
      if (range_ < 256) {
        range_ <<= 1;
        low_ <<= 1;
        top_++;
        split();
      }
      return;
    }
    low_ += range_;
    low_ <<= 7;  // range 2 renormalised
    top_ += 7;
    split();
    uint32_t v = (low_ >> 8) << 1 | 1u;  // bits top_..8, the stop bit; a carry above them
    int n = top_ - 6;
    const int pad = (8 - n % 8) % 8;
    v <<= pad;
    n += pad;
    for (; n > 0; n -= 8) {
      pend_.push_back((uint16_t)(v >> (n - 8)));
      v &= (1u << (n - 8)) - 1;
    }
    size_t at = out_.size();
    out_.resize(at + pend_.size());
    unsigned carry = 0;
    for (size_t i = pend_.size(); i-- > 0;) {
      const unsigned b = pend_[i] + carry;
      out_[at + i] = (uint8_t)b;
      carry = b >> 8;
    }
  }

 private:
  void split() {
    if (top_ >= 17) {  // bits top_..top_-7 are above the window
      pend_.push_back((uint16_t)(low_ >> (top_ - 7)));
      low_ &= (1u << (top_ - 7)) - 1;
      top_ -= 8;
    }
  }

  std::vector<uint8_t>& out_;
  std::vector<uint16_t> pend_;
  uint32_t low_ = 0, range_ = 510;
  int top_ = 8;
};

// What later macroblocks read of a coded one.
struct MbSummary {
  bool avail = false, skip = false, intra = false, i16 = false, t8 = false, chroma_pred = false;
  bool dc = false;              // Intra16x16 DC levels present
  uint8_t cbpl = 0, cbpc = 0;
  uint8_t cdc = 0;              // bit p: chroma DC levels present in plane p
  uint16_t luma = 0;            // bit 4 * y + x: luma 4x4 block (x, y) holds levels (8x8: the whole 8x8)
  uint8_t chroma[2] = {0, 0};   // bit 2 * y + x: chroma AC block (x, y) holds levels
  uint16_t amvd[4][2] = {};     // |mvd| per 8x8 quadrant (raster) and component
};

// Context index offsets (Table 9-34) and the coded_block_flag / residual offsets per category.
constexpr int kSkipP = 11, kMbTypeI = 3, kMbTypeP = 14, kMbTypePIntra = 17, kSubMbTypeP = 21, kMvdX = 40, kMvdY = 47;
constexpr int kQpDelta = 60, kChromaPred = 64, kPrevI4 = 68, kRemI4 = 69, kCbpLuma = 73, kCbpChroma = 77;
constexpr int kTransform8x8 = 399;
constexpr int kCbf[5] = {85, 89, 93, 97, 101};
constexpr int kSig[6] = {105, 120, 134, 149, 152, 402};
constexpr int kLast[6] = {166, 181, 195, 210, 213, 417};
constexpr int kAbs[6] = {227, 237, 247, 257, 266, 426};

// 4x4 block b (decoding order) -> x, y inside the macroblock.
inline int blk_x(int b) { return (b & 1) | ((b >> 1) & 2); }
inline int blk_y(int b) { return ((b >> 1) & 1) | ((b >> 2) & 2); }

// Bit i set where level i of c[0..n) (n <= 64) is not 0.
inline uint64_t nonzero_mask(const int16_t* c, int n) {
  uint64_t m = 0;
  int i = 0;
#if defined(__AVX2__) && defined(__BMI2__)
  const __m256i zero = _mm256_setzero_si256();
  for (; i + 16 <= n; i += 16) {
    const __m256i v = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(c + i));
    const uint32_t eq = (uint32_t)_mm256_movemask_epi8(_mm256_cmpeq_epi16(v, zero));  // 2 bits per level
    m |= (uint64_t)(_pext_u32(~eq, 0x55555555u)) << i;
  }
#endif
  for (; i < n; i++) m |= (uint64_t)(c[i] != 0) << i;
  return m;
}

class SliceCoder {
 public:
  SliceCoder(int mb_w, int mb_h, int qp, bool idr, bool t8x8, std::vector<uint8_t>& out)
      : mb_w_(mb_w), mb_h_(mb_h), idr_(idr), t8x8_(t8x8), ar_(out), above_(mb_w), modes_(mb_w * 4) {
    const int table = idr ? 0 : 1;  // cabac_init_idc 0
    for (int i = 0; i < kContexts; i++) {
      const cabac::MN mn = cabac::kInit[table][i];
      int pre = ((mn.m * std::min(qp, 51)) >> 4) + mn.n;
      pre = std::min(126, std::max(1, pre));
      ctx_[i] = pre <= 63 ? (uint8_t)((63 - pre) << 1) : (uint8_t)((pre - 64) << 1 | 1);
    }
  }

  int code(RecordReader& recs) {
    for (int y = 0; y < mb_h_; y++) {
      left_ = MbSummary();
      std::fill(left_modes_, left_modes_ + 4, 2);
      for (int x = 0; x < mb_w_; x++) {
        const rg_mb_out* rp = recs.next();
        if (!rp) return -1;
        const rg_mb_out& r = *rp;
        const MbSummary& top = above_[x];
        MbSummary cur;
        int rc = macroblock(r, x, y, top, cur);
        if (rc) return rc;
        ar_.terminate(x == mb_w_ - 1 && y == mb_h_ - 1);
        cur.avail = true;
        above_[x] = cur;
        left_ = cur;
      }
    }
    return 0;
  }

 private:
  void bin(int ctx, unsigned b) { ar_.decision(ctx_[ctx], b); }

  // mb_type of an I slice (Table 9-36 binarisation) or the intra suffix of a P slice.
  void intra_type(unsigned t, const MbSummary& top) {
    if (idr_) {
      bin(kMbTypeI + (left_.avail && left_.i16) + (top.avail && top.i16), t != 0);
    } else {
      bin(kMbTypeP, 1);
      bin(kMbTypePIntra, t != 0);
    }
    if (t == 0) return;
    ar_.terminate(0);
    const unsigned k = t - 1, mode = k & 3, cbpc = (k >> 2) % 3, cbpl = k >= 12;
    const int c = idr_ ? kMbTypeI : kMbTypePIntra;
    // bins after the terminate: luma cbp, chroma cbp != 0, [chroma cbp == 2], two mode bits
    const int luma_ctx = idr_ ? c + 3 : c + 1, chroma_ctx = idr_ ? c + 4 : c + 2;
    const int chroma2_ctx = idr_ ? c + 5 : c + 2, mode_hi = idr_ ? c + 6 : c + 3, mode_lo = idr_ ? c + 7 : c + 3;
    bin(luma_ctx, cbpl);
    bin(chroma_ctx, cbpc != 0);
    if (cbpc) bin(chroma2_ctx, cbpc == 2);
    bin(mode_hi, mode >> 1);
    bin(mode_lo, mode & 1);
  }

  void chroma_pred(unsigned mode, const MbSummary& top) {
    bin(kChromaPred + (left_.avail && left_.chroma_pred) + (top.avail && top.chroma_pred), mode != 0);
    if (!mode) return;
    bin(kChromaPred + 3, mode != 1);
    if (mode != 1) bin(kChromaPred + 3, mode == 3);
  }

  void qp_delta(int d) {
    bin(kQpDelta + prev_qp_delta_, d != 0);
    prev_qp_delta_ = d != 0;
    if (!d) return;
    const unsigned code = d > 0 ? 2u * (unsigned)d - 1u : 2u * (unsigned)(-d);
    // unary, the first of the remaining bins at ctx 62, the rest at 63
    for (unsigned k = 1; k < code; k++) bin(k == 1 ? kQpDelta + 2 : kQpDelta + 3, 1);
    bin(code == 1 ? kQpDelta + 2 : kQpDelta + 3, 0);
  }

  // UEG3 with signed suffix, uCoff 9 (9.3.2.3); ctxIdxInc of the prefix bins 0, 3, 4, 5, 6, 6, ...
  void mvd(int base, unsigned neighbours, int v) {
    const unsigned a = (unsigned)std::abs(v);
    bin(base + (neighbours < 3 ? 0 : (neighbours <= 32 ? 1 : 2)), a != 0);
    if (!a) return;
    const unsigned prefix = std::min(a, 9u);
    for (unsigned k = 1; k < prefix; k++) bin(base + 2 + (int)std::min(k, 4u), 1);
    if (a < 9) {
      bin(base + 2 + (int)std::min(a, 4u), 0);
    } else {
      exp_golomb(a - 9, 3);
    }
    ar_.bypass(v < 0);
  }

  // |mvd| component c of the 4x4 block (bx, by) relative to the current macroblock (-1: the left /
  // top neighbour's): 0 when not available, skipped or intra (9.3.3.1.1.7).
  unsigned amvd_at(const MbSummary& cur, const MbSummary& top, int bx, int by, int c) const {
    if (bx < 0) return left_.avail ? left_.amvd[(by >> 1) * 2 + 1][c] : 0u;
    if (by < 0) return top.avail ? top.amvd[2 + (bx >> 1)][c] : 0u;
    return cur.amvd[(by >> 1) * 2 + (bx >> 1)][c];
  }

  void exp_golomb(unsigned v, unsigned k) {
    while (v >= (1u << k)) {
      ar_.bypass(1);
      v -= 1u << k;
      k++;
    }
    ar_.bypass(0);
    while (k--) ar_.bypass((v >> k) & 1u);
  }

  // One residual block in scan order (9.3.2.3 / 9.3.3.1.3); cat 5 has no coded_block_flag.
  // Returns whether it holds levels.
  bool block(int cat, int cbf_inc, const int16_t* c, int n) {
    const uint64_t nz = nonzero_mask(c, n);
    if (cat < 5) {
      bin(kCbf[cat] + cbf_inc, nz != 0);
      if (!nz) return false;
    }
    const int last = nz ? 63 - __builtin_clzll(nz) : 0;
    for (int i = 0; i <= std::min(last, n - 2); i++) {
      const int sig = cat == 5 ? cabac::kSig8x8[i] : i, lst = cat == 5 ? cabac::kLast8x8[i] : i;
      const unsigned s = (unsigned)(nz >> i) & 1u;
      bin(kSig[cat] + sig, s);
      if (s) bin(kLast[cat] + lst, i == last);
    }
    const int lvl = kAbs[cat], gt_cap = cat == 3 ? 3 : 4;
    int ones = 0, bigger = 0;
    for (uint64_t left = nz; left; left &= ~(1ull << (63 - __builtin_clzll(left)))) {
      const int i = 63 - __builtin_clzll(left);
      const unsigned m1 = (unsigned)std::abs(c[i]) - 1;
      bin(lvl + (bigger ? 0 : std::min(1 + ones, 4)), m1 != 0);
      if (!m1) {
        ones++;
      } else {
        const int ctx = lvl + 5 + std::min(bigger, gt_cap);
        for (unsigned k = 1; k < std::min(m1, 14u); k++) bin(ctx, 1);
        if (m1 < 14) bin(ctx, 0);
        else exp_golomb(m1 - 14, 0);
        bigger++;
      }
      ar_.bypass(c[i] < 0);
    }
    return true;
  }

  // coded_block_flag condition of a neighbouring luma 4x4 block at (x, y), x or y -1 = outside.
  int luma_cond(const MbSummary& cur, const MbSummary& top, int x, int y, bool intra) const {
    if (x < 0) return left_.avail ? (left_.luma >> (4 * y + 3)) & 1 : intra;
    if (y < 0) return top.avail ? (top.luma >> (12 + x)) & 1 : intra;
    return (cur.luma >> (4 * y + x)) & 1;
  }
  int chroma_cond(const MbSummary& cur, const MbSummary& top, int p, int x, int y, bool intra) const {
    if (x < 0) return left_.avail ? (left_.chroma[p] >> (2 * y + 1)) & 1 : intra;
    if (y < 0) return top.avail ? (top.chroma[p] >> (2 + x)) & 1 : intra;
    return (cur.chroma[p] >> (2 * y + x)) & 1;
  }

  void cbp(const MbSummary& top, unsigned cbpl, unsigned cbpc) {
    for (int b8 = 0; b8 < 4; b8++) {
      const int x = b8 & 1, y = b8 >> 1;
      // condTerm: the neighbouring 8x8 block exists and has no coded luma
      const int a = x ? !((cbpl >> (b8 - 1)) & 1) : (left_.avail && !((left_.cbpl >> (b8 + 1)) & 1));
      const int b = y ? !((cbpl >> (b8 - 2)) & 1) : (top.avail && !((top.cbpl >> (b8 + 2)) & 1));
      bin(kCbpLuma + a + 2 * b, (cbpl >> b8) & 1);
    }
    const unsigned lc = left_.avail ? left_.cbpc : 0, tc = top.avail ? top.cbpc : 0;
    bin(kCbpChroma + (lc != 0) + 2 * (tc != 0), cbpc != 0);
    if (cbpc) bin(kCbpChroma + 4 + (lc == 2) + 2 * (tc == 2), cbpc == 2);
  }

  void chroma_residual(const rg_mb_out& r, const MbSummary& top, MbSummary& cur, bool intra) {
    if (cur.cbpc >= 1)
      for (int p = 0; p < 2; p++) {
        const int a = left_.avail ? (left_.cdc >> p) & 1 : intra, b = top.avail ? (top.cdc >> p) & 1 : intra;
        if (block(3, a + 2 * b, r.chroma_dc[p], 4)) cur.cdc |= (uint8_t)(1 << p);
      }
    if (cur.cbpc >= 2)
      for (int p = 0; p < 2; p++)
        for (int k = 0; k < 4; k++) {
          const int x = k & 1, y = k >> 1;
          const int a = chroma_cond(cur, top, p, x - 1, y, intra), b = chroma_cond(cur, top, p, x, y - 1, intra);
          if (block(4, a + 2 * b, r.chroma_ac[p][k] + 1, 15)) cur.chroma[p] |= (uint8_t)(1 << (2 * y + x));
        }
  }

  // coded_block_pattern, transform flag, mb_qp_delta and residual of P_L0_16x16 and I_NxN.
  void residual(const rg_mb_out& r, const MbSummary& top, MbSummary& cur, bool intra) {
    cbp(top, cur.cbpl, cur.cbpc);
    if (!cur.cbpl && !cur.cbpc) {
      prev_qp_delta_ = false;
      return;
    }
    if (t8x8_ && cur.cbpl && !intra) bin(kTransform8x8 + (left_.avail && left_.t8) + (top.avail && top.t8), cur.t8);
    qp_delta(r.qp_delta);
    if (cur.t8) {
      for (int b8 = 0; b8 < 4; b8++)
        if ((cur.cbpl >> b8) & 1) {
          block(5, 0, r.luma + 64 * b8, 64);
          const int x = (b8 & 1) * 2, y = (b8 >> 1) * 2;
          cur.luma |= (uint16_t)(0x33u << (4 * y + x));
        }
    } else {
      for (int b = 0; b < 16; b++) {
        if (!((cur.cbpl >> (b >> 2)) & 1)) continue;
        const int x = blk_x(b), y = blk_y(b);
        const int a = luma_cond(cur, top, x - 1, y, intra), c = luma_cond(cur, top, x, y - 1, intra);
        if (block(2, a + 2 * c, r.luma + 16 * b, 16)) cur.luma |= (uint16_t)(1u << (4 * y + x));
      }
    }
    chroma_residual(r, top, cur, intra);
  }

  int macroblock(const rg_mb_out& r, int x, int y, const MbSummary& top, MbSummary& cur) {
    if (r.cbp > 47) return -1;
    const int skip_inc = (left_.avail && !left_.skip) + (top.avail && !top.skip);
    int* mode_row = &modes_[x * 4];
    if (r.mb_type == RG_MB_P_SKIP) {
      if (idr_) return -1;
      bin(kSkipP + skip_inc, 1);
      cur.skip = true;
      prev_qp_delta_ = false;
      std::fill(left_modes_, left_modes_ + 4, 2);
      std::fill(mode_row, mode_row + 4, 2);
      return 0;
    }
    if (!idr_) bin(kSkipP + skip_inc, 0);
    cur.cbpl = r.cbp & 15;
    cur.cbpc = r.cbp >> 4;
    if (r.mb_type == RG_MB_P_L0_16X16 || (r.mb_type >= RG_MB_P_L0_16X8 && r.mb_type <= RG_MB_P_8X8)) {
      if (idr_) return -1;
      cur.t8 = r.transform_8x8 && cur.cbpl;
      // mb_type (Table 9-37 binarisation; bin 2 at ctxIdx 16 after a 0, 17 after a 1):
      // P_L0_16x16 000, P_L0_L0_16x8 011, P_L0_L0_8x16 010, P_8x8 001
      const int t = r.mb_type == RG_MB_P_L0_16X16 ? 0 : r.mb_type - RG_MB_P_L0_16X8 + 1;
      static const uint8_t kBins[4][2] = {{0, 0}, {1, 1}, {1, 0}, {0, 1}};
      bin(kMbType, 0);
      bin(kMbType + 1, kBins[t][0]);
      bin(kMbType + 2 + kBins[t][0], kBins[t][1]);
      if (t == 3)
        for (int k = 0; k < 4; k++) bin(kSubMbTypeP, 1);  // sub_mb_type P_L0_8x8: "1"
      // partitions in coding order: top-left 4x4 block and the quadrants each covers
      static const int8_t kParts[4][4][3] = {{{0, 0, 15}},
                                             {{0, 0, 3}, {0, 2, 12}},
                                             {{0, 0, 5}, {2, 0, 10}},
                                             {{0, 0, 1}, {2, 0, 2}, {0, 2, 4}, {2, 2, 8}}};
      static const int kNum[4] = {1, 2, 2, 4};
      for (int k = 0; k < kNum[t]; k++) {
        const int bx = kParts[t][k][0], by = kParts[t][k][1], qm = kParts[t][k][2];
        for (int c = 0; c < 2; c++) {
          const int v = t == 0 ? r.mvd[c] : r.part_mvd[k][c];
          const unsigned sum = amvd_at(cur, top, bx - 1, by, c) + amvd_at(cur, top, bx, by - 1, c);
          mvd(c ? kMvdY : kMvdX, sum, v);
          const uint16_t a = (uint16_t)std::min(std::abs(v), 65535);
          for (int q = 0; q < 4; q++)
            if ((qm >> q) & 1) cur.amvd[q][c] = a;
        }
      }
      residual(r, top, cur, false);
      std::fill(left_modes_, left_modes_ + 4, 2);
      std::fill(mode_row, mode_row + 4, 2);
      return 0;
    }
    cur.intra = true;
    cur.chroma_pred = r.chroma_mode != 0;
    if (r.mb_type == RG_MB_I4X4) {
      intra_type(0, top);
      if (t8x8_) bin(kTransform8x8 + (left_.avail && left_.t8) + (top.avail && top.t8), 0);
      int mb_modes[16];
      for (int b = 0; b < 16; b++) {
        const int bx = blk_x(b), by = blk_y(b);
        // Intra4x4PredMode of the neighbours: 2 (DC) outside the picture or in a non-I4x4
        // macroblock; the prediction is DC when either neighbour is outside the picture.
        const bool have_a = bx > 0 || x > 0, have_b = by > 0 || y > 0;
        int pred = 2;
        if (have_a && have_b) {
          const int ma = bx > 0 ? mb_modes[by * 4 + bx - 1] : left_modes_[by];
          const int mb = by > 0 ? mb_modes[(by - 1) * 4 + bx] : mode_row[bx];
          pred = std::min(ma, mb);
        }
        const int m = r.i4_modes[b];
        if (m > 8) return -1;
        mb_modes[by * 4 + bx] = m;
        bin(kPrevI4, m == pred);
        if (m != pred) {
          const int rem = m < pred ? m : m - 1;
          for (int k = 0; k < 3; k++) bin(kRemI4, (rem >> k) & 1);
        }
      }
      for (int k = 0; k < 4; k++) {
        left_modes_[k] = mb_modes[k * 4 + 3];
        mode_row[k] = mb_modes[12 + k];
      }
      chroma_pred(r.chroma_mode, top);
      residual(r, top, cur, true);
      return 0;
    }
    if (r.mb_type != RG_MB_I16X16) return -1;
    cur.i16 = true;
    std::fill(left_modes_, left_modes_ + 4, 2);
    std::fill(mode_row, mode_row + 4, 2);
    intra_type(1 + r.i16_mode + 4 * cur.cbpc + (cur.cbpl ? 12 : 0), top);
    chroma_pred(r.chroma_mode, top);
    qp_delta(r.qp_delta);
    const int a = left_.avail ? left_.dc : 1, b = top.avail ? top.dc : 1;
    cur.dc = block(0, a + 2 * b, r.luma_dc, 16);
    if (cur.cbpl)
      for (int k = 0; k < 16; k++) {
        const int bx = blk_x(k), by = blk_y(k);
        const int ca = luma_cond(cur, top, bx - 1, by, true), cb = luma_cond(cur, top, bx, by - 1, true);
        if (block(1, ca + 2 * cb, r.luma + 16 * k + 1, 15)) cur.luma |= (uint16_t)(1u << (4 * by + bx));
      }
    chroma_residual(r, top, cur, true);
    return 0;
  }

  static constexpr int kMbType = kMbTypeP;

  int mb_w_, mb_h_;
  bool idr_, t8x8_;
  Arith ar_;
  uint8_t ctx_[kContexts];
  std::vector<MbSummary> above_;
  MbSummary left_;
  std::vector<int> modes_;   // Intra4x4PredMode of the bottom 4x4 row of the macroblocks above
  int left_modes_[4] = {2, 2, 2, 2};
  bool prev_qp_delta_ = false;
};

}  // namespace

// Appends the CABAC slice data of one picture (after the byte-aligned slice header) to out;
// ends with the flushed coder and the alignment to a byte. Returns 0, or -1 for a record that
// no Balanced slice holds.
int cabac_slice_data(int mb_w, int mb_h, int qp, bool idr, bool transform_8x8, RecordReader& recs,
                     std::vector<uint8_t>& out) {
  SliceCoder coder(mb_w, mb_h, qp, idr, transform_8x8, out);
  return coder.code(recs);
}

}  // namespace rg
