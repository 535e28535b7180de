// Host-side bitstream pieces shared by the writer, the CABAC slice coder and the encoder.
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/ragdoll_cuda.h"

namespace rg {

void set_last_error(const char* msg);

// CABAC slice data of one picture, appended to out after the byte-aligned slice header
// (cabac_writer.cpp). 0, or -1 for a record no Balanced slice holds.
int cabac_slice_data(int mb_w, int mb_h, int qp, bool idr, bool transform_8x8, const rg_mb_out* recs,
                     std::vector<uint8_t>& out);

// The access unit of one picture with explicit frame counters (cavlc_writer.cpp); the writer
// supplies configuration and scratch only. 0 or a negative RG_ERR_* code.
int writer_access_unit(rg_writer* w, const rg_mb_out* records, bool idr, uint32_t since_idr, uint32_t idr_id,
                       int qp, std::vector<uint8_t>& au);

}  // namespace rg
