// Host-side bitstream pieces shared by the writer, the CABAC slice coder and the encoder.
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/ragdoll_cuda.h"

namespace rg {

void set_last_error(const char* msg);

// The records of one picture as the writers read them, one at a time in raster order: dense
// (rg_mb_out[n]) or compact -- per record RG_COMPACT_MASK_WORDS mask words (bit j of word i: the
// record's 32-bit word 32 i + j is nonzero) and then its nonzero words in increasing order, as
// rg_analyse_gops_fetch_compact hands them out; a compact record is rebuilt by zero-filling.
class RecordReader {
 public:
  explicit RecordReader(const rg_mb_out* dense) : dense_(dense) {}
  RecordReader(const void* compact, size_t bytes)
      : at_(static_cast<const uint32_t*>(compact)), end_(static_cast<const uint32_t*>(compact) + bytes / 4) {}
  // The next record, or null when a compact stream ends early or is malformed.
  const rg_mb_out* next() {
    if (dense_) return dense_++;
    if (end_ - at_ < RG_COMPACT_MASK_WORDS) return nullptr;
    const uint32_t* mask = at_;
    at_ += RG_COMPACT_MASK_WORDS;
    if (mask[RG_COMPACT_MASK_WORDS - 1] >> (kWords - 32 * (RG_COMPACT_MASK_WORDS - 1))) return nullptr;
    uint32_t* w = reinterpret_cast<uint32_t*>(&scratch_);
    for (int i = 0; i < kWords; i++) w[i] = 0;
    for (int i = 0; i < RG_COMPACT_MASK_WORDS; i++)
      for (uint32_t m = mask[i]; m; m &= m - 1) {
        if (at_ == end_) return nullptr;
        w[32 * i + __builtin_ctz(m)] = *at_++;
      }
    return &scratch_;
  }
  // Whether a compact stream was read to its end exactly.
  bool done() const { return dense_ || at_ == end_; }

 private:
  static constexpr int kWords = (int)(sizeof(rg_mb_out) / 4);
  const rg_mb_out* dense_ = nullptr;
  const uint32_t* at_ = nullptr;
  const uint32_t* end_ = nullptr;
  rg_mb_out scratch_;
};
static_assert(sizeof(rg_mb_out) % 4 == 0 && sizeof(rg_mb_out) / 4 <= 32 * RG_COMPACT_MASK_WORDS,
              "a record's words fit its mask");

// CABAC slice data of one picture, appended to out after the byte-aligned slice header
// (cabac_writer.cpp). 0, or -1 for a record no Balanced slice holds.
int cabac_slice_data(int mb_w, int mb_h, int qp, bool idr, bool transform_8x8, RecordReader& recs,
                     std::vector<uint8_t>& out);

// The access unit of one picture with explicit frame counters (cavlc_writer.cpp); the writer
// supplies configuration and scratch only. 0 or a negative RG_ERR_* code.
int writer_access_unit(rg_writer* w, RecordReader& records, bool idr, uint32_t since_idr, uint32_t idr_id, int qp,
                       std::vector<uint8_t>& au);
inline int writer_access_unit(rg_writer* w, const rg_mb_out* records, bool idr, uint32_t since_idr, uint32_t idr_id,
                              int qp, std::vector<uint8_t>& au) {
  RecordReader rd(records);
  return writer_access_unit(w, rd, idr, since_idr, idr_id, qp, au);
}

}  // namespace rg
