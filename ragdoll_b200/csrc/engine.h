// Internal layout shared by the engine kernels (engine_kernels.cu) and the C-ABI (rg_api.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/ragdoll_cuda.h"

namespace rg {

// Padding of the reconstructed planes. Motion compensation of a vector within the Balanced
// search bounds (MV_MARGIN = 28 samples past the edge, enc.rs:61) plus the 6-tap reach stays
// within 48 luma / 16 chroma samples; 64 / 32 keep every row 64-byte aligned.
constexpr int kPadY = 64;
constexpr int kPadC = 32;
constexpr int kMaxStreams = 1024;

// Per-macroblock state read by later macroblocks of the same picture (motion prediction,
// intra mode prediction) and by the deblocking filter; 16 bytes, one per macroblock.
struct __align__(16) MbInfo {
  int16_t mv[2];      // quarter-sample vector (0 for intra)
  int8_t ref;         // 0 inter / skip, -1 intra
  uint8_t flags;      // bit 0 intra, bit 1 skip, bit 2 transform 8x8 with levels
  uint8_t cbp_luma;   // coded_block_pattern luma bits
  uint8_t qp;         // QP_Y
  uint16_t nz16;      // 4x4 luma blocks holding levels (decoding-order bit)
  uint16_t i4_bottom;  // Intra4x4PredMode of the bottom row, 4 bits per x = 0..3 (2 if not I4x4)
  uint16_t i4_right;   // of the right column, 4 bits per y = 0..3
  uint16_t pad_;
};
static_assert(sizeof(MbInfo) == 16, "MbInfo layout");

constexpr uint8_t kFlagIntra = 1, kFlagSkip = 2, kFlagT8 = 4;

// Quadrant vectors of a macroblock of the search forms (raster: top-left, top-right, bottom-left,
// bottom-right), read by later macroblocks' predictors and by the deblocking filter.
struct __align__(16) MbMv4 {
  int16_t mv[4][2];
};

// Integer search range limit of the search forms (samples).
constexpr int kMaxSearchRange = 64;

// Device view of one stream for one picture.
struct StreamDev {
  const uint8_t* src_y;   // source planes (display size, any stride)
  const uint8_t* src_u;
  const uint8_t* src_v;
  uint8_t* cur_y;         // reconstruction being built: pointer to sample (0, 0) of the padded plane
  uint8_t* cur_u;
  uint8_t* cur_v;
  const uint8_t* ref_y;   // previous (deblocked, border-extended) reconstruction
  const uint8_t* ref_u;
  const uint8_t* ref_v;
  MbInfo* info;           // this picture's macroblock state
  const MbInfo* prev_info;  // previous picture's (co-located candidate vectors)
  rg_mb_out* rec;         // decision records (raster order)
  uint8_t* unf_y;         // optional copy of the reconstruction before deblocking (coded size)
  uint8_t* unf_u;
  uint8_t* unf_v;
  int32_t kind;           // RG_FRAME_IDR or RG_FRAME_P
  int32_t qp, qpc;        // the stream's QP and chroma QP
  // SkipBounds (enc.rs:2104) of the stream's QP
  uint32_t sb_luma, sb_luma_ssd, sb_chroma, sb_chroma_ssd, sb_probe;
  // pipelined launches: the descriptor's size group (its FrameParams), the offset of its rows in the
  // launch's row counters, and the descriptor of the previous picture of its stream (-1: none)
  int32_t group, rows_base, prev_ps;
  // search forms only (null / 0 in the plain form)
  MbMv4* mv4;              // this picture's quadrant vectors
  const rg_mb_hint* hint;  // learned form: this picture's hints (null: full search)
  int32_t search_range;    // integer search range of the full search (samples)
  int32_t walk;            // learned form: re-centrings of the seed's window before the full search
  uint16_t type_bits[4];   // search forms: bits charged per partition type (x lambda)
  uint16_t pad3_[4];
  // pipelined launches: this picture's ready flag in mapped host memory (null: the launch's
  // ready array at the descriptor's index, if any)
  int32_t* ready;
};

// Frame-constant parameters of one wavefront (all streams share the size; qp / qpc / sb_* are the
// context's default QP -- the kernels read each stream's own from its StreamDev). A pipelined launch
// takes up to kMaxGroups of them, one per picture size among its streams.
struct FrameParams {
  int32_t width, height;      // display size
  int32_t mb_w, mb_h;
  int32_t src_stride_y, src_stride_uv;
  int32_t stride_y, stride_c; // padded reconstruction strides
  int32_t qp, qpc;
  int32_t t8x8;               // High profile: 8x8 transform decision (needs CABAC too)
  int32_t deblock;            // disable_deblocking_filter_idc == 0
  // SkipBounds (enc.rs:2104) of qp
  uint32_t sb_luma, sb_luma_ssd, sb_chroma, sb_chroma_ssd, sb_probe;
  int32_t n_streams;
};

// Host launchers (engine_kernels.cu).
// form: 0 the plain (Balanced) analysis, 1 the search forms (full search; learned where a stream's
// descriptor carries hints).
void launch_wavefront_step(const FrameParams& fp, const StreamDev* d_streams, int step, cudaStream_t st, int form = 0);
void launch_extend_borders(const FrameParams& fp, const StreamDev* d_streams, cudaStream_t st);
int wavefront_steps(const FrameParams& fp);
// Pipelined mode: d_streams holds frames x n_streams descriptors (picture-major); counters is
// pipeline_counter_ints() zeroed ints; counters[1] is non-zero after a failed wait. ready (device
// address of mapped host memory, or null): frames x n_streams ints, each set to seq once that
// picture's records are final. host_err: mapped host int receiving the launch's error word (zero
// it before the launch). host_reach (mapped host, or null): two ints receiving 1 + the largest
// reach, in macroblock rows and columns beyond zero motion, of the launch's waits for a reference
// picture (0: no such wait); the work order never waits for an untaken segment when
// lag >= max(seg, 2) * (4 + rows) + seg + columns + 3.
constexpr int kMaxGroups = 8;
struct FrameGroups {
  FrameParams g[kMaxGroups];
  int32_t n;
};
int pipeline_grid(int device, int form = 0);
int pipeline_sms(int device);
size_t pipeline_counter_ints(const FrameParams& fp, int frames);
// Work list: every analysis / deblocking segment of `seg` macroblocks, in expected-ready order
// with `lag` macroblock-times between consecutive pictures of a stream.
size_t pipeline_task_count(const FrameParams& fp, int frames, int seg);
// Queues: 0 analysis, 1 deblocking (split), 2 analysis of IDR pictures (kinds != null; [f][s]).
constexpr int kPipeQueues = 3;
// keys (or null): each task's key, ascending within each queue.
size_t pipeline_task_list(const FrameParams& fp, int frames, int lag, int seg, bool split, const int32_t* kinds,
                          int2* tasks, int qbeg[3], int qend[3], uint32_t* keys = nullptr);
// One launch over n_desc descriptors of up to kMaxGroups picture sizes (descriptor d: group
// d.group, rows d.rows_base .. + its mb_h in the row counters, total_rows in all). host_err null:
// no error hand-off kernel (launch_error_to_host queues one per caller instead).
// Compact records (co != null): the warp deblocking a row's last segment also writes that row's
// records, word-sparse (kCompactMaskWords mask words per record, then its nonzero words in order),
// into the row's slot (row r of the launch, counted as the row counters are: row_words words at
// words + r * row_words) and the row's size in bytes, or -1 when it did not fit, into
// row_bytes[r] -- both before the picture's ready flag.
constexpr int kRecordWords = 222;      // sizeof(rg_mb_out) / 4
constexpr int kCompactMaskWords = 7;   // ceil(kRecordWords / 32)
struct CompactOut {
  uint32_t* words;   // device address of mapped host memory
  int row_words;     // words per row slot
  int* row_bytes;    // device address of mapped host memory: [row]
};
void launch_pipeline(const FrameGroups& fg, const StreamDev* d_streams, int n_desc, int total_rows, int* counters,
                     const int2* d_tasks, size_t n_tasks, const int qbeg[3], const int qend[3], int deblock_sms,
                     int intra_sms, int sms, int seg, int grid, unsigned long long timeout_ns, int* ready, int seq,
                     int* host_err, int* host_reach, cudaStream_t st, int form = 0, const CompactOut* co = nullptr);
void launch_error_to_host(const int* counters, int n_desc, int total_rows, int* host_err, int* host_reach,
                          cudaStream_t st);
size_t pipeline_counter_ints(int total_rows, int n_desc);
void upload_tables();

}  // namespace rg
