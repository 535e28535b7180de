// Host side of the compact record form (rg_records_compact / rg_records_expand): per record,
// RG_COMPACT_MASK_WORDS mask words of its nonzero 32-bit words, then those words in order. The
// pipelined launch writes the same form on the device (engine_kernels.cu compact_row).
#include <cstring>

#include "bitstream.h"

namespace {
constexpr int kWords = (int)(sizeof(rg_mb_out) / 4);

int rfail(int code, const char* msg) {
  rg::set_last_error(msg);
  return code;
}
}  // namespace

extern "C" {

int64_t rg_records_compact(const rg_mb_out* records, int32_t n, void* out, size_t cap) {
  if (!records || !out || n < 0) return rfail(RG_ERR_INVALID, "rg_records_compact: null argument or negative count");
  uint32_t* o = static_cast<uint32_t*>(out);
  const size_t cap_words = cap / 4;
  size_t at = 0;
  for (int32_t r = 0; r < n; r++) {
    uint32_t w[kWords];
    memcpy(w, records + r, sizeof(rg_mb_out));
    uint32_t mask[RG_COMPACT_MASK_WORDS] = {0};
    size_t nz = 0;
    for (int k = 0; k < kWords; k++)
      if (w[k]) {
        mask[k / 32] |= 1u << (k % 32);
        nz++;
      }
    if (at + RG_COMPACT_MASK_WORDS + nz > cap_words) return rfail(RG_ERR_INVALID, "rg_records_compact: buffer too small");
    for (int i = 0; i < RG_COMPACT_MASK_WORDS; i++) o[at++] = mask[i];
    for (int k = 0; k < kWords; k++)
      if (w[k]) o[at++] = w[k];
  }
  return (int64_t)(at * 4);
}

int rg_records_expand(const void* compact, size_t bytes, int32_t n, rg_mb_out* out) {
  if (!compact || !out || n < 0) return rfail(RG_ERR_INVALID, "rg_records_expand: null argument or negative count");
  if (bytes % 4) return rfail(RG_ERR_INVALID, "rg_records_expand: not whole words");
  rg::RecordReader rd(compact, bytes);
  for (int32_t r = 0; r < n; r++) {
    const rg_mb_out* rec = rd.next();
    if (!rec) return rfail(RG_ERR_INVALID, "rg_records_expand: the stream ends early or is malformed");
    out[r] = *rec;
  }
  if (!rd.done()) return rfail(RG_ERR_INVALID, "rg_records_expand: the stream holds more than n records");
  return RG_OK;
}

}  // extern "C"
