// Host-side bitstream writer: turns the per-macroblock records of the engine into the Annex-B
// access units of ragdoll's Balanced encoder (the serial half of encode_frame_body,
// crates/ragdoll-codec/src/h264/enc.rs:2234): SPS / PPS of h264.rs:556-660 and 806-832 for the
// Baseline, Main and High profiles, the slice header, and the NAL packing with emulation
// prevention of h264.rs:189. Baseline slices are CAVLC, written here (skip runs and macroblock
// layer of enc.rs:989-1054 / 3260-3285 / 3540-3577 / 3736-3750, residual blocks of h264.rs:2215
// encode_cavlc_block); Main and High slices are CABAC, written by cabac_writer.cpp after the
// cabac_alignment_one_bits. One writer per stream (GOP); no CUDA.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/ragdoll_cuda.h"
#include "cavlc_tables.h"

#include "bitstream.h"

namespace {

int wfail(int code, const char* fmt, ...) {
  char buf[256];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  rg::set_last_error(buf);
  return code;
}

// MSB-first bit sink of one RBSP.
class Rbsp {
 public:
  void put(uint32_t v, int n) {
    for (int i = n - 1; i >= 0; i--) {
      cur_ = (uint8_t)((cur_ << 1) | (i < 32 ? (v >> i) & 1u : 0u));
      if (++fill_ == 8) {
        bytes_.push_back(cur_);
        cur_ = 0;
        fill_ = 0;
      }
    }
  }
  void put(const rg::cavlc::Vlc& c) { put(c.code, c.len); }
  void flag(bool b) { put(b ? 1u : 0u, 1); }
  // Exp-Golomb ue(v): M leading zeros, then the M+1 bits of v + 1.
  void ue(uint32_t v) {
    uint64_t x = (uint64_t)v + 1;
    int m = 63 - __builtin_clzll(x);
    put(0, m);
    if (m >= 32) {
      put((uint32_t)(x >> 32), m + 1 - 32);
      put((uint32_t)x, 32);
    } else {
      put((uint32_t)x, m + 1);
    }
  }
  void se(int32_t v) { ue(v > 0 ? 2u * (uint32_t)v - 1u : 2u * (uint32_t)(-(int64_t)v)); }
  // cabac_alignment_one_bit up to the byte boundary; the bytes so far.
  std::vector<uint8_t>& align_ones() {
    while (fill_) put(1, 1);
    return bytes_;
  }
  // rbsp_trailing_bits: a stop bit, then zeros to the byte boundary.
  const std::vector<uint8_t>& close() {
    put(1, 1);
    while (fill_) put(0, 1);
    return bytes_;
  }

 private:
  std::vector<uint8_t> bytes_;
  uint8_t cur_ = 0;
  int fill_ = 0;
};

// NAL unit with a 4-byte start code; an emulation-prevention byte goes before any byte <= 3
// that follows two zero bytes.
void emit_nal(std::vector<uint8_t>& out, int nal_ref_idc, int nal_type, const std::vector<uint8_t>& rbsp) {
  const uint8_t head[5] = {0, 0, 0, 1, (uint8_t)((nal_ref_idc << 5) | nal_type)};
  out.insert(out.end(), head, head + 5);
  int zeros = 0;
  for (uint8_t b : rbsp) {
    if (zeros >= 2 && b <= 3) {
      out.push_back(3);
      zeros = 0;
    }
    out.push_back(b);
    zeros = b ? 0 : zeros + 1;
  }
}

// One residual block (coefficients in zig-zag order, n = 4, 15 or 16); nc < 0 selects the chroma
// DC tables. Returns TotalCoeff.
int residual_block(Rbsp& w, const int16_t* zz, int n, int nc) {
  using namespace rg::cavlc;
  // nonzero levels from the highest frequency down, with the zeros below each one
  int level[16], zeros_below[16], total = 0;
  int last = n - 1;
  while (last >= 0 && zz[last] == 0) last--;
  for (int i = last; i >= 0; i--) {
    if (zz[i] == 0) continue;
    int z = 0;
    for (int j = i - 1; j >= 0 && zz[j] == 0; j--) z++;
    level[total] = zz[i];
    zeros_below[total] = z;
    total++;
  }
  int ones = 0;  // trailing +-1 levels, at most 3
  while (ones < total && ones < 3 && (level[ones] == 1 || level[ones] == -1)) ones++;
  if (nc < 0) w.put(kChromaDcToken[total][ones]);
  else w.put(kCoeffToken[nc < 2 ? 0 : (nc < 4 ? 1 : (nc < 8 ? 2 : 3))][total][ones]);
  if (total == 0) return 0;
  for (int k = 0; k < ones; k++) w.flag(level[k] < 0);
  int suffix_len = (total > 10 && ones < 3) ? 1 : 0;
  for (int k = ones; k < total; k++) {
    int a = level[k] < 0 ? -level[k] : level[k];
    uint32_t code = 2u * (uint32_t)a - (level[k] < 0 ? 1u : 2u);
    if (k == ones && ones < 3) code -= 2;  // the first level after fewer than 3 trailing ones is > 1
    if (suffix_len == 0) {
      if (code < 14) {
        w.put(1, code + 1);                 // level_prefix = code
      } else if (code < 30) {
        w.put(1, 15);                       // level_prefix 14, 4-bit suffix
        w.put(code - 14, 4);
      } else {
        w.put(1, 16);                       // level_prefix 15, 12-bit suffix
        w.put((code - 30) & 0xFFF, 12);
      }
    } else if (code < (15u << suffix_len)) {
      w.put(1, (int)(code >> suffix_len) + 1);
      w.put(code & ((1u << suffix_len) - 1), suffix_len);
    } else {
      w.put(1, 16);
      w.put((code - (15u << suffix_len)) & 0xFFF, 12);
    }
    if (suffix_len == 0) suffix_len = 1;
    if (a > (3 << (suffix_len - 1)) && suffix_len < 6) suffix_len++;
  }
  int zeros_left = 0;
  for (int k = 0; k < total; k++) zeros_left += zeros_below[k];
  if (total < n) w.put(nc < 0 ? kChromaDcTotalZeros[total - 1][zeros_left] : kTotalZeros[total - 1][zeros_left]);
  for (int k = 0; k + 1 < total && zeros_left > 0; k++) {
    w.put(kRunBefore[std::min(zeros_left, 7) - 1][zeros_below[k]]);
    zeros_left -= zeros_below[k];
  }
  return total;
}

inline int count_nonzero(const int16_t* v, int n) {
  int c = 0;
  for (int i = 0; i < n; i++) c += v[i] != 0;
  return c;
}

// Position of 4x4 block b (decoding order) inside its macroblock.
inline int bx4(int b) { return (b & 1) | ((b >> 1) & 2); }
inline int by4(int b) { return ((b >> 1) & 1) | ((b >> 2) & 2); }

}  // namespace

struct rg_writer {
  int width = 0, height = 0, qp = 26, fps_num = 30, fps_den = 1;
  int profile = RG_PROFILE_BASELINE;  // Main / High: CABAC; High: 8x8 transform
  int mb_w = 0, mb_h = 0;
  uint32_t since_idr = 0;  // pictures since the last IDR (frame_num, POC)
  uint32_t idrs = 0;       // IDR pictures written (idr_pic_id)
  bool have_idr = false;
  // per picture: TotalCoeff per luma 4x4 block, per chroma AC block, Intra4x4PredMode per 4x4
  std::vector<uint8_t> nnz, cnnz[2], mode4;

  std::vector<uint8_t> sps() const {
    Rbsp w;
    // profile_idc and constraint flags (h264.rs:247): Constrained Baseline 66 / set0+set1,
    // Main 77 / set1, High 100
    const int idc = profile == RG_PROFILE_BASELINE ? 66 : (profile == RG_PROFILE_MAIN ? 77 : 100);
    w.put(idc, 8);
    w.put(profile == RG_PROFILE_BASELINE ? 0xC0 : (profile == RG_PROFILE_MAIN ? 0x40 : 0x00), 8);
    w.put(40, 8);    // level_idc 4.0
    w.ue(0);         // seq_parameter_set_id
    if (idc == 100) {
      w.ue(1);       // chroma_format_idc 4:2:0
      w.ue(0);       // bit_depth_luma_minus8
      w.ue(0);       // bit_depth_chroma_minus8
      w.flag(false); // qpprime_y_zero_transform_bypass_flag
      w.flag(false); // seq_scaling_matrix_present_flag
    }
    w.ue(0);         // log2_max_frame_num_minus4
    w.ue(0);         // pic_order_cnt_type
    w.ue(2);         // log2_max_pic_order_cnt_lsb_minus4
    w.ue(2);         // max_num_ref_frames
    w.flag(false);   // gaps_in_frame_num_value_allowed_flag
    w.ue(mb_w - 1);
    w.ue(mb_h - 1);
    w.flag(true);    // frame_mbs_only_flag
    w.flag(true);    // direct_8x8_inference_flag
    int crop_r = (mb_w * 16 - width) / 2, crop_b = (mb_h * 16 - height) / 2;
    w.flag(crop_r || crop_b);
    if (crop_r || crop_b) {
      w.ue(0);
      w.ue(crop_r);
      w.ue(0);
      w.ue(crop_b);
    }
    w.flag(true);                   // vui_parameters_present_flag
    w.flag(true);                   // aspect_ratio_info_present_flag
    w.put(1, 8);                    //   square samples
    w.flag(false);                  // overscan_info_present_flag
    w.flag(true);                   // video_signal_type_present_flag
    w.put(5, 3);                    //   video_format: unspecified
    w.flag(false);                  //   video_full_range_flag
    w.flag(true);                   //   colour_description_present_flag
    w.put(1, 8);                    //   BT.709 primaries,
    w.put(1, 8);                    //   transfer,
    w.put(1, 8);                    //   matrix
    w.flag(false);                  // chroma_loc_info_present_flag
    w.flag(true);                   // timing_info_present_flag
    w.put((uint32_t)fps_den, 32);   //   num_units_in_tick
    w.put((uint32_t)fps_num * 2, 32);  // time_scale
    w.flag(true);                   //   fixed_frame_rate_flag
    w.flag(false);                  // nal_hrd_parameters_present_flag
    w.flag(false);                  // vcl_hrd_parameters_present_flag
    w.flag(false);                  // pic_struct_present_flag
    w.flag(false);                  // bitstream_restriction_flag
    return w.close();
  }
  std::vector<uint8_t> pps(int qp) const {
    Rbsp w;
    w.ue(0);         // pic_parameter_set_id
    w.ue(0);         // seq_parameter_set_id
    w.flag(profile != RG_PROFILE_BASELINE);  // entropy_coding_mode_flag: CABAC beyond Baseline
    w.flag(false);   // bottom_field_pic_order_in_frame_present_flag
    w.ue(0);         // num_slice_groups_minus1
    w.ue(0);         // num_ref_idx_l0_default_active_minus1
    w.ue(0);         // num_ref_idx_l1_default_active_minus1
    w.flag(false);   // weighted_pred_flag
    w.put(0, 2);     // weighted_bipred_idc
    w.se(qp - 26);   // pic_init_qp_minus26
    w.se(0);         // pic_init_qs_minus26
    w.se(0);         // chroma_qp_index_offset
    w.flag(true);    // deblocking_filter_control_present_flag
    w.flag(false);   // constrained_intra_pred_flag
    w.flag(false);   // redundant_pic_cnt_present_flag
    if (profile == RG_PROFILE_HIGH) {
      w.flag(true);  // transform_8x8_mode_flag
      w.flag(false); // pic_scaling_matrix_present_flag
      w.se(0);       // second_chroma_qp_index_offset
    }
    return w.close();
  }

  int nc_at(const std::vector<uint8_t>& grid, int gw, int gx, int gy) const {
    bool a = gx > 0, b = gy > 0;
    int na = a ? grid[gy * gw + gx - 1] : 0, nb = b ? grid[(gy - 1) * gw + gx] : 0;
    return a && b ? (na + nb + 1) >> 1 : (a ? na : nb);
  }
  void luma_4x4_blocks(Rbsp& w, int mbx, int mby, const rg_mb_out& r, bool ac_only, bool all_coded) {
    int gw = mb_w * 4;
    for (int b = 0; b < 16; b++) {
      int gx = mbx * 4 + bx4(b), gy = mby * 4 + by4(b);
      bool coded = all_coded || ((r.cbp >> (b >> 2)) & 1);
      if (!coded) {
        nnz[gy * gw + gx] = 0;
        continue;
      }
      const int16_t* c = r.luma + b * 16 + (ac_only ? 1 : 0);
      int nc = nc_at(nnz, gw, gx, gy);
      residual_block(w, c, ac_only ? 15 : 16, nc);
      nnz[gy * gw + gx] = (uint8_t)count_nonzero(c, ac_only ? 15 : 16);
    }
  }
  void chroma_blocks(Rbsp& w, int mbx, int mby, const rg_mb_out& r) {
    int cbpc = r.cbp >> 4, gw = mb_w * 2;
    if (cbpc == 0) return;
    for (int p = 0; p < 2; p++) residual_block(w, r.chroma_dc[p], 4, -1);
    if (cbpc < 2) return;
    for (int p = 0; p < 2; p++)
      for (int b = 0; b < 4; b++) {
        int gx = mbx * 2 + (b & 1), gy = mby * 2 + (b >> 1);
        residual_block(w, r.chroma_ac[p][b] + 1, 15, nc_at(cnnz[p], gw, gx, gy));
        cnnz[p][gy * gw + gx] = (uint8_t)count_nonzero(r.chroma_ac[p][b] + 1, 15);
      }
  }
  int mb_layer(Rbsp& w, int mbx, int mby, const rg_mb_out& r, bool idr, uint32_t& skip_run) {
    using namespace rg::cavlc;
    if (r.mb_type == RG_MB_P_SKIP) {
      if (idr) return wfail(RG_ERR_INVALID, "rg_writer_picture: P_Skip in an IDR picture at mb (%d,%d)", mbx, mby);
      skip_run++;
      return RG_OK;
    }
    if (!idr) {
      w.ue(skip_run);
      skip_run = 0;
    }
    if (r.cbp > 47) return wfail(RG_ERR_INVALID, "rg_writer_picture: cbp %d at mb (%d,%d)", r.cbp, mbx, mby);
    int intra_base = idr ? 0 : 5;  // I macroblock types follow the five P types in a P slice
    switch (r.mb_type) {
      case RG_MB_P_L0_16X16:
        if (idr) return wfail(RG_ERR_INVALID, "rg_writer_picture: inter macroblock in an IDR picture");
        w.ue(0);  // P_L0_16x16, one reference picture: no ref_idx
        w.se(r.mvd[0]);
        w.se(r.mvd[1]);
        w.ue(kInterCbpCode[r.cbp]);
        if (r.cbp) {
          w.se(r.qp_delta);
          luma_4x4_blocks(w, mbx, mby, r, false, false);
          chroma_blocks(w, mbx, mby, r);
        }
        return RG_OK;
      case RG_MB_I16X16: {
        int cbpl = r.cbp & 15, cbpc = r.cbp >> 4;
        w.ue(intra_base + 1 + r.i16_mode + 4 * cbpc + (cbpl ? 12 : 0));
        w.ue(r.chroma_mode);
        w.se(r.qp_delta);
        int gw = mb_w * 4;
        residual_block(w, r.luma_dc, 16, nc_at(nnz, gw, mbx * 4, mby * 4));
        if (cbpl) luma_4x4_blocks(w, mbx, mby, r, true, true);
        chroma_blocks(w, mbx, mby, r);
        return RG_OK;
      }
      case RG_MB_I4X4: {
        int gw = mb_w * 4;
        w.ue(intra_base);
        for (int b = 0; b < 16; b++) {
          int gx = mbx * 4 + bx4(b), gy = mby * 4 + by4(b);
          int pred = (gx == 0 || gy == 0) ? 2 : std::min(mode4[gy * gw + gx - 1], mode4[(gy - 1) * gw + gx]);
          int m = r.i4_modes[b];
          if (m > 8) return wfail(RG_ERR_INVALID, "rg_writer_picture: intra 4x4 mode %d", m);
          if (m == pred) {
            w.flag(true);
          } else {
            w.flag(false);
            w.put(m < pred ? m : m - 1, 3);
          }
          mode4[gy * gw + gx] = (uint8_t)m;
        }
        w.ue(r.chroma_mode);
        w.ue(kIntraCbpCode[r.cbp]);
        if (r.cbp) {
          w.se(r.qp_delta);
          luma_4x4_blocks(w, mbx, mby, r, false, false);
          chroma_blocks(w, mbx, mby, r);
        }
        return RG_OK;
      }
      default:
        return wfail(RG_ERR_INVALID, "rg_writer_picture: macroblock type %d at (%d,%d)", r.mb_type, mbx, mby);
    }
  }
};

namespace rg {

// The access unit of one picture (SPS and PPS first for an IDR) with explicit frame_num / POC
// (pictures since the IDR), idr_pic_id and QP; uses the writer's configuration and scratch only, so
// writers of the same configuration can write pictures of one stream on several threads.
int writer_access_unit(rg_writer* w, RecordReader& records, bool idr, uint32_t since_idr, uint32_t idr_id, int qp,
                       std::vector<uint8_t>& au) {
  int n4 = w->mb_w * w->mb_h * 16;
  w->nnz.assign(n4, 0);
  w->cnnz[0].assign(w->mb_w * w->mb_h * 4, 0);
  w->cnnz[1].assign(w->mb_w * w->mb_h * 4, 0);
  w->mode4.assign(n4, 2);

  Rbsp s;
  s.ue(0);                          // first_mb_in_slice
  s.ue(idr ? 7 : 5);                // slice_type: I or P, all slices of the picture alike
  s.ue(0);                          // pic_parameter_set_id
  s.put(since_idr & 15, 4);         // frame_num
  if (idr) s.ue(idr_id);            // idr_pic_id
  s.put((since_idr * 2) & 63, 6);   // pic_order_cnt_lsb
  if (!idr) {
    s.flag(false);                  // num_ref_idx_active_override_flag
    s.flag(false);                  // ref_pic_list_modification_flag_l0
  }
  if (idr) {
    s.flag(false);                  // no_output_of_prior_pics_flag
    s.flag(false);                  // long_term_reference_flag
  } else {
    s.flag(false);                  // adaptive_ref_pic_marking_mode_flag
  }
  const bool cabac = w->profile != RG_PROFILE_BASELINE;
  if (cabac && !idr) s.ue(0);       // cabac_init_idc
  s.se(0);                          // slice_qp_delta
  s.ue(0);                          // disable_deblocking_filter_idc (QP >= 1)
  s.se(0);                          // slice_alpha_c0_offset_div2
  s.se(0);                          // slice_beta_offset_div2
  const std::vector<uint8_t>* rbsp;
  if (cabac) {
    std::vector<uint8_t>& bytes = s.align_ones();
    if (rg::cabac_slice_data(w->mb_w, w->mb_h, qp, idr, w->profile == RG_PROFILE_HIGH, records, bytes))
      return wfail(RG_ERR_INVALID, "rg_writer_picture: a record no %s slice holds", idr ? "IDR" : "P");
    rbsp = &bytes;
  } else {
    uint32_t skip_run = 0;
    for (int mby = 0; mby < w->mb_h; mby++)
      for (int mbx = 0; mbx < w->mb_w; mbx++) {
        const rg_mb_out* rec = records.next();
        if (!rec) return wfail(RG_ERR_INVALID, "rg_writer_picture: compact records end before mb (%d,%d)", mbx, mby);
        int r = w->mb_layer(s, mbx, mby, *rec, idr, skip_run);
        if (r) return r;
      }
    if (!idr && skip_run) s.ue(skip_run);
    rbsp = &s.close();
  }
  if (!records.done()) return wfail(RG_ERR_INVALID, "rg_writer_picture: compact records longer than the picture");
  au.clear();
  if (idr) {
    emit_nal(au, 3, 7, w->sps());
    emit_nal(au, 3, 8, w->pps(qp));
  }
  emit_nal(au, 3, idr ? 5 : 1, *rbsp);
  return 0;
}

}  // namespace rg

extern "C" {

rg_writer* rg_writer_create(const rg_config* cfg, int32_t fps_num, int32_t fps_den) {
  if (!cfg) {
    wfail(RG_ERR_INVALID, "rg_writer_create: null config");
    return nullptr;
  }
  if (cfg->profile != RG_PROFILE_BASELINE && cfg->profile != RG_PROFILE_MAIN && cfg->profile != RG_PROFILE_HIGH) {
    wfail(RG_ERR_INVALID, "rg_writer_create: profile %d", cfg->profile);
    return nullptr;
  }
  if (cfg->width < 1 || cfg->height < 1 || cfg->width > 8192 || cfg->height > 8192 || cfg->qp < 1 || cfg->qp > 51 ||
      fps_num < 1 || fps_den < 1) {
    wfail(RG_ERR_INVALID, "rg_writer_create: size %dx%d, qp %d, rate %d/%d", cfg->width, cfg->height, cfg->qp, fps_num,
          fps_den);
    return nullptr;
  }
  rg_writer* w = new rg_writer;
  w->width = cfg->width;
  w->height = cfg->height;
  w->qp = cfg->qp;
  w->profile = cfg->profile;
  w->fps_num = fps_num;
  w->fps_den = fps_den;
  w->mb_w = (cfg->width + 15) / 16;
  w->mb_h = (cfg->height + 15) / 16;
  return w;
}

void rg_writer_destroy(rg_writer* w) { delete w; }

size_t rg_writer_bound(const rg_writer* w) {
  if (!w) return 0;
  // 384 levels per macroblock at up to 32 bits each, plus the macroblock header, headers and
  // emulation prevention (one byte in three at worst)
  size_t per_mb = 384 * 4 + 64;
  return ((size_t)w->mb_w * w->mb_h * per_mb + 512) * 3 / 2;
}

static int64_t writer_picture(rg_writer* w, rg::RecordReader& records, int32_t kind, uint8_t* out, size_t cap) {
  if (kind != RG_FRAME_IDR && kind != RG_FRAME_P) return wfail(RG_ERR_INVALID, "rg_writer_picture: kind %d", kind);
  if (kind == RG_FRAME_P && !w->have_idr) return wfail(RG_ERR_STATE, "rg_writer_picture: P picture before an IDR");
  bool idr = kind == RG_FRAME_IDR;
  if (idr) w->since_idr = 0;
  std::vector<uint8_t> au;
  int r = rg::writer_access_unit(w, records, idr, w->since_idr, w->idrs, w->qp, au);
  if (r) return r;
  if (au.size() > cap)
    return wfail(RG_ERR_INVALID, "rg_writer_picture: access unit of %zu bytes exceeds the %zu-byte buffer", au.size(), cap);
  memcpy(out, au.data(), au.size());
  if (idr) {
    w->idrs++;
    w->have_idr = true;
  }
  w->since_idr++;
  return (int64_t)au.size();
}

int64_t rg_writer_picture(rg_writer* w, const rg_mb_out* records, int32_t kind, uint8_t* out, size_t cap) {
  if (!w || !records || !out) return wfail(RG_ERR_INVALID, "rg_writer_picture: null argument");
  rg::RecordReader rd(records);
  return writer_picture(w, rd, kind, out, cap);
}

int64_t rg_writer_picture_compact(rg_writer* w, const void* compact, size_t bytes, int32_t kind, uint8_t* out,
                                  size_t cap) {
  if (!w || !compact || !out) return wfail(RG_ERR_INVALID, "rg_writer_picture_compact: null argument");
  if (bytes % 4) return wfail(RG_ERR_INVALID, "rg_writer_picture_compact: %zu bytes, not whole words", bytes);
  rg::RecordReader rd(compact, bytes);
  return writer_picture(w, rd, kind, out, cap);
}

}  // extern "C"
