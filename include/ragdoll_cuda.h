/*
 * ragdoll_cuda.h -- C ABI of the B200 (sm_100a) macroblock analysis / reconstruction engine.
 *
 * The engine performs the data-parallel half of ragdoll's Balanced H.264 encoder on the GPU:
 * per-macroblock P_Skip probe, diamond + quarter-pel motion search, intra 16x16 / 4x4 analysis,
 * 4x4 / 8x8 transform, quantisation, decimation, dequantisation, reconstruction, the in-loop
 * deblocking filter and SSIM / MS-SSIM of the reconstruction. Entropy coding (CAVLC / CABAC),
 * slice headers and NAL packing stay on the host, driven by the per-macroblock records below.
 *
 * Reference boundary replaced (oddurs/ragdoll):
 *   H264Encoder::new / with_profile / with_rate_control   crates/ragdoll-codec/src/h264.rs:3032-3135
 *   H264Encoder::encode_frame                              crates/ragdoll-codec/src/h264.rs:3153
 *   MB raster loop of encode_frame_body                    crates/ragdoll-codec/src/h264/enc.rs:2382-2434
 *   EncState::deblock + extend_borders                     crates/ragdoll-codec/src/h264/enc.rs:3776, :165
 *   ssim_plane_u8 / ms_ssim_plane_u8                       crates/ragdoll-pix/src/metrics.rs:55, :154
 *   GopRingEncoder::encode_wave (GOP batching)             crates/ragdoll-pipeline/src/lib.rs:543
 *
 * Conventions: every entry point returns 0 on success or a negative RG_ERR_* code, and
 * rg_last_error() describes the most recent failure of the calling thread. A context is used by
 * one host thread at a time. Pointers are plain host pointers unless a name says "device".
 */
#ifndef RAGDOLL_CUDA_H
#define RAGDOLL_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes ------------------------------------------------------------------------- */
#define RG_OK 0
#define RG_ERR_INVALID (-1)     /* bad argument or dimension (RagdollError::InvalidArgument)  */
#define RG_ERR_OOM (-2)         /* device allocation failed                                    */
#define RG_ERR_CUDA (-3)        /* CUDA runtime error                                          */
#define RG_ERR_TIMEOUT (-4)     /* a device wait gave up (bounded spin)                         */
#define RG_ERR_UNSUPPORTED (-5) /* configuration outside the GPU form (RagdollError::Unsupported)*/
#define RG_ERR_STATE (-6)       /* call out of order (e.g. P frame before any IDR)              */

/* ---- configuration ----------------------------------------------------------------------- */
/* Profile ids follow H264Profile (crates/ragdoll-codec/src/h264.rs:30). */
#define RG_PROFILE_BASELINE 0
#define RG_PROFILE_MAIN 1
#define RG_PROFILE_HIGH 2

/* Frame kinds (PicKind, crates/ragdoll-codec/src/h264/enc.rs:447). */
#define RG_FRAME_IDR 0
#define RG_FRAME_P 1

typedef struct rg_config {
    int32_t width;       /* display width in luma samples (1..8192)                          */
    int32_t height;      /* display height (1..8192)                                          */
    int32_t profile;     /* RG_PROFILE_*; Main/High enable CABAC-side decisions, High the 8x8 */
    int32_t qp;          /* fixed QP 1..51 (RateControlMode::FixedQp)                          */
    int32_t num_streams; /* independent streams / GOPs analysed together (>= 1)                */
    int32_t device;      /* CUDA device ordinal                                                */
    int32_t max_frames;  /* pictures per stream in one rg_analyse_gops call (0 or 1: one)       */
} rg_config;

/* ---- per-macroblock decision record ------------------------------------------------------ */
#define RG_MB_P_SKIP 0
#define RG_MB_P_L0_16X16 1
#define RG_MB_I16X16 2
#define RG_MB_I4X4 3
/* Partitioned inter macroblocks, coded only by the search forms (rg_set_analysis_form): two 16x8
 * or 8x16 partitions, or four 8x8 sub-macroblocks (P_8x8, every sub_mb_type P_L0_8x8). Their
 * vectors are part_mv / part_mvd below. */
#define RG_MB_P_L0_16X8 4
#define RG_MB_P_L0_8X16 5
#define RG_MB_P_8X8 6

/*
 * One macroblock's decisions and levels, everything the entropy coder reads
 * (code_inter / code_i16 / code_i4 / code_skip, enc.rs:2874-3772). Levels are stored in coding
 * (zig-zag) order so the host coder scans nothing.
 */
typedef struct rg_mb_out {
    uint8_t mb_type;       /* RG_MB_*                                                          */
    uint8_t i16_mode;      /* Intra16x16PredMode (0 V, 1 H, 2 DC, 3 plane)                      */
    uint8_t chroma_mode;   /* intra_chroma_pred_mode (0 DC, 1 H, 2 V, 3 plane)                  */
    uint8_t cbp;           /* coded_block_pattern: luma bits 0-3 | chroma (0..2) << 4           */
    uint8_t transform_8x8; /* transform_size_8x8_flag of an inter MB                            */
    uint8_t qp;            /* QP_Y of the macroblock                                            */
    int8_t qp_delta;       /* mb_qp_delta (0 under fixed QP)                                    */
    uint8_t reserved0;
    int16_t mv[2];         /* motion vector, quarter samples (P_Skip: the skip vector)          */
    int16_t mvd[2];        /* mv - mvp                                                          */
    uint8_t i4_modes[16];  /* Intra4x4PredMode per 4x4 block, decoding order                     */
    uint16_t nz_mask;      /* bit b: luma 4x4 block b (decoding order) holds levels            */
    uint16_t reserved1;
    int16_t luma[256];     /* 16 blocks x 16 zig-zag levels, or (8x8) 4 blocks x 64 zig-zag     */
    int16_t luma_dc[16];   /* Intra16x16 DC levels, zig-zag                                     */
    int16_t chroma_dc[2][4];
    int16_t chroma_ac[2][4][16]; /* zig-zag; slot 0 (the DC position) is unused              */
    /* Written by the search forms only (zero in the plain form): the vector of each 8x8 quadrant
     * (raster order: top-left, top-right, bottom-left, bottom-right), the vector differences of
     * the partitions in coding order (16x8: top, bottom; 8x16: left, right; 8x8: the four
     * sub-macroblocks; one for 16x16), and the partition type the search found cheapest before
     * the skip and intra decisions (0 16x16, 1 16x8, 2 8x16, 3 8x8; 255 when not searched) --
     * the label the learned form's network is trained on. */
    int16_t part_mv[4][2];
    int16_t part_mvd[4][2];
    uint8_t part_type;
    uint8_t reserved2[3];
} rg_mb_out;

/* Quality of a reconstruction against its source (QualityReport, crates/ragdoll-pix/src/metrics.rs:13;
 * evaluate_frame_quality :328): SSIM per plane and (4Y + U + V) / 6, 5-scale MS-SSIM of luma, PSNR
 * per plane, over all samples (psnr_avg) and 6:1:1 weighted, SSIM in dB, VMAF-Lite of luma. */
typedef struct rg_quality {
    double ssim_y, ssim_u, ssim_v, ssim_avg, ms_ssim;
    double psnr_y, psnr_u, psnr_v;
    double psnr_avg, psnr_yuv_611, ssim_db, vmaf_lite;
} rg_quality;

typedef struct rg_ctx rg_ctx;

/* Last error message of the calling thread ("" when none). */
const char* rg_last_error(void);

/* Version string of the library build. */
const char* rg_version(void);

/*
 * Creates a context: device buffers for cfg->num_streams streams of one size, each holding its
 * reference picture and motion state (replaces H264Encoder::new + with_profile +
 * with_rate_control(FixedQp), h264.rs:3032-3135). Returns NULL on failure (see rg_last_error).
 */
rg_ctx* rg_create(const rg_config* cfg);

/* Frees every device and host resource of the context. NULL is allowed. */
void rg_destroy(rg_ctx* ctx);

/* Coded (macroblock-aligned) size in macroblocks. */
int rg_mb_dims(const rg_ctx* ctx, int32_t* mb_w, int32_t* mb_h);

/*
 * Sets the fixed QP (1..51) of one stream; the others keep theirs (cfg.qp by default). Streams of
 * different QPs share every launch. Pictures queued before the call keep the QP they were queued
 * with. A stream's bitstream has one QP (the writer's, in its PPS), so set it before the stream's
 * first picture or at an IDR with a writer of the new QP. No counterpart in the reference (one
 * H264Encoder per stream, each with its own rate control).
 */
int rg_set_stream_qp(rg_ctx* ctx, int32_t stream, int32_t qp);

/*
 * Analyses, reconstructs and deblocks one frame of one stream from host planes (replaces
 * encode_frame_body's macroblock loop, deblock and border extension, enc.rs:2382-2503).
 * kind: RG_FRAME_IDR or RG_FRAME_P (a P frame needs an earlier frame of the stream).
 * out: mb_w * mb_h records in raster order (may be NULL to skip the copy). In a context of
 * several streams only `stream` is analysed (its own wavefront launches); the others stay put.
 */
int rg_analyse_frame(rg_ctx* ctx, int32_t stream, const uint8_t* y, const uint8_t* u,
                     const uint8_t* v, size_t stride_y, size_t stride_uv, int32_t kind,
                     rg_mb_out* out);

/*
 * Batched form of rg_analyse_frame: the next frame of every stream, all analysed in one
 * macroblock wavefront (one launch per anti-diagonal step, streams side by side). planes holds
 * 3 * num_streams host pointers (y, u, v per stream); kinds one RG_FRAME_* per stream; out
 * num_streams * mb_w * mb_h records (stream-major) or NULL.
 */
int rg_analyse_batch(rg_ctx* ctx, const uint8_t* const* planes, size_t stride_y,
                     size_t stride_uv, const int32_t* kinds, rg_mb_out* out);

/*
 * Same as rg_analyse_batch with the source planes already resident on the device:
 * dev_planes holds 3 * num_streams device pointers with the given strides. Records stay on the
 * device (rg_copy_records fetches them). Asynchronous on the context's stream; rg_sync waits.
 */
int rg_analyse_batch_device(rg_ctx* ctx, const uint8_t* const* dev_planes, size_t stride_y,
                            size_t stride_uv, const int32_t* kinds);

/*
 * Pipelined form: `frames` consecutive pictures of every stream (frames <= cfg.max_frames) in
 * one persistent launch (the frame loop of GopRingEncoder::encode_wave's workers,
 * crates/ragdoll-pipeline/src/lib.rs:580-597, for all GOPs at once). Picture f+1 of a stream
 * starts as soon as the region of picture f its motion search can reach is final, so the
 * pictures of a GOP overlap. dev_planes: frames * num_streams * 3 device pointers, picture-major
 * ([f][s][y,u,v]); kinds: frames * num_streams RG_FRAME_* values ([f][s]). Records of picture f,
 * stream s land at record index (f * num_streams + s) * mb_w * mb_h (rg_copy_records_gops).
 * Asynchronous; rg_sync reports RG_ERR_TIMEOUT if a device wait gave up.
 */
int rg_analyse_gops_device(rg_ctx* ctx, const uint8_t* const* dev_planes, size_t stride_y,
                           size_t stride_uv, const int32_t* kinds, int32_t frames);

/*
 * rg_analyse_gops_device for n contexts of different picture sizes (1..8 contexts on one device,
 * all in the plain form or all in the full-search form) in ONE persistent launch: the work lists
 * of the contexts (each with its own lag) merged in key order, so macroblocks of every size share
 * the SMs; the segment length, SM roles and wait limit of the context with the most macroblocks
 * (rg_set_pipeline_tuning), the largest grid of any. dev_planes[i], stride_y[i], stride_uv[i],
 * kinds[i]: context i's arguments as rg_analyse_gops_device takes them; `frames` pictures of every
 * stream of every context. Queued on ctxs[0]'s stream; each context's later calls wait for it,
 * and each context resolves its part as its own pending call (a wait that gave up re-runs that
 * context's pictures on the per-diagonal path). The batched transcode of many independent
 * streams of several sizes (the pipeline's parallel_gop_map over encoders,
 * crates/ragdoll-pipeline/src/lib.rs:110-157) as one launch; no single counterpart in the reference.
 * The launch's stream work (descriptor copy, counter reset, the persistent launch, the error
 * hand-offs) is a CUDA graph captured once per launch shape and replayed by later calls of that
 * shape.
 */
int rg_analyse_gops_group(rg_ctx* const* ctxs, int32_t n, const uint8_t* const* const* dev_planes,
                          const size_t* stride_y, const size_t* stride_uv, const int32_t* const* kinds,
                          int32_t frames);
/*
 * rg_analyse_gops_async for n contexts in one group launch (as rg_analyse_gops_group): each
 * context's host sources (planes[i], strides of its own size) are copied into its staging, the one
 * launch analyses every context's pictures, and each context's records are copied into outs[i]
 * (frames * its num_streams * its macroblocks, picture-major). rg_analyse_gops_wait(ctxs[i],
 * outs[i]) waits for context i's records (re-running its pictures if a wait of the launch gave up).
 * The batched transcode's waves of many streams of several sizes, one launch per wave.
 */
int rg_analyse_gops_group_async(rg_ctx* const* ctxs, int32_t n, const uint8_t* const* const* planes,
                                const size_t* stride_y, const size_t* stride_uv, const int32_t* const* kinds,
                                int32_t frames, rg_mb_out* const* outs);
/* rg_analyse_gops_group_async without the copy of all records at the end, as
 * rg_analyse_gops_stream: rg_analyse_gops_fetch(ctxs[i], outs[i], picture) copies each of context
 * i's pictures as the launch flags it final, and rg_analyse_gops_wait(ctxs[i], outs[i]) ends it. */
int rg_analyse_gops_group_stream(rg_ctx* const* ctxs, int32_t n, const uint8_t* const* const* planes,
                                 const size_t* stride_y, const size_t* stride_uv, const int32_t* const* kinds,
                                 int32_t frames, rg_mb_out* const* outs);
/* Group calls led by ctx (ctxs[0]) so far: graphs captured and graph launches. */
int rg_group_graph_counts(const rg_ctx* ctx, int64_t* captures, int64_t* launches);

/* Host-buffer form of rg_analyse_gops_device; out receives frames * num_streams * mb_w * mb_h
 * records (or NULL). */
int rg_analyse_gops(rg_ctx* ctx, const uint8_t* const* planes, size_t stride_y, size_t stride_uv,
                    const int32_t* kinds, int32_t frames, rg_mb_out* out);

/* Copies the records of the last `frames` pictures of an rg_analyse_gops / _device call. */
int rg_copy_records_gops(rg_ctx* ctx, int32_t frames, rg_mb_out* out);

/*
 * Asynchronous host-buffer form of rg_analyse_gops, for a caller that encodes batch after batch
 * (GopRingEncoder::encode_wave, crates/ragdoll-pipeline/src/lib.rs:543, one wave per call): the
 * call queues the copy of the sources in, the launch, and the copy of the records out into `out`
 * (frames * num_streams * mb_w * mb_h records, picture-major) and returns. The copy in of one call
 * overlaps the launch of the previous call and its copy out the launch of the next, when `planes`
 * and `out` are in pinned host memory (cudaHostAlloc). The sources may be reused, and `out` read,
 * after rg_sync. Two calls' staging are kept on the device (allocated by the first call). A call
 * whose device wait gave up is re-run on the per-diagonal path before the next call starts (or in
 * rg_sync) and its records copied again, so results are always exact.
 */
int rg_analyse_gops_async(rg_ctx* ctx, const uint8_t* const* planes, size_t stride_y, size_t stride_uv,
                          const int32_t* kinds, int32_t frames, rg_mb_out* out);

/* Waits until the records of the rg_analyse_gops_async call that copies into `out` are in host
 * memory and final (for the latest call: everything queued, as rg_sync; for the one before it:
 * its copy out only, so the latest call's launch keeps running). No counterpart in the reference. */
int rg_analyse_gops_wait(rg_ctx* ctx, const rg_mb_out* out);

/*
 * rg_analyse_gops_async without the copy of all records at the end: the launch flags each picture
 * (index f * num_streams + s) in mapped host memory once its records are final, and
 * rg_analyse_gops_fetch copies that picture's records into out -- while the launch still runs.
 * rg_analyse_gops_wait(ctx, out) then waits for the launch; if one of its waits gave up, it re-runs
 * the call and copies every record into out. Fetch every picture of a call before the call two
 * calls later is queued. No counterpart in the reference.
 */
int rg_analyse_gops_stream(rg_ctx* ctx, const uint8_t* const* planes, size_t stride_y, size_t stride_uv,
                           const int32_t* kinds, int32_t frames, rg_mb_out* out);
/* 1: the picture's records are copied into out; 0: not final yet; 2: the launch ended without
 * finishing it (call rg_analyse_gops_wait); negative RG_ERR_*. Safe to call from several host threads
 * at once (for different pictures) while the context's own thread is not in another call. */
int rg_analyse_gops_fetch(rg_ctx* ctx, rg_mb_out* out, int32_t picture);

/*
 * Compact records. A picture's records in compact form are, per macroblock in raster order,
 * RG_COMPACT_MASK_WORDS 32-bit mask words -- bit j of mask word i set when the record's 32-bit
 * word 32 i + j (of the sizeof(rg_mb_out) / 4 = 222) is nonzero -- followed by those nonzero words
 * in increasing order; zero-filling the rest rebuilds the record exactly. Most of a record is zero
 * levels, so the form is ~10x smaller than the records.
 *
 * rg_set_record_compaction(ctx, words_per_mb > 0) makes the launches of rg_analyse_gops_stream
 * also write each picture's compact records, row by row as its analysis completes, straight into
 * mapped host memory of the context (each macroblock row into its own slot of words_per_mb words
 * per macroblock, packed together by the first fetch; a picture with a row that does not fit is
 * handed out as full records instead). 0 turns it off (the default). Not while calls are in
 * flight. No counterpart in the reference (its records never leave the CPU).
 */
#define RG_COMPACT_MASK_WORDS 7
int rg_set_record_compaction(rg_ctx* ctx, int32_t words_per_mb);
/*
 * rg_analyse_gops_fetch of a call made with compaction on: 1 with *data / *bytes the picture's
 * compact records in the context's mapped memory (valid until the call two calls later is
 * queued), or, when a row did not fit its slot, *data NULL and the full records copied into
 * out + picture * mb_w * mb_h; 0, 2 and errors as rg_analyse_gops_fetch.
 */
int rg_analyse_gops_fetch_compact(rg_ctx* ctx, rg_mb_out* out, int32_t picture, const void** data, size_t* bytes);
/* Host helpers of the compact form: n records into out (returns the bytes written, or
 * RG_ERR_INVALID when cap is too small), and back (RG_ERR_INVALID for a stream that is not n
 * compact records exactly). */
int64_t rg_records_compact(const rg_mb_out* records, int32_t n, void* out, size_t cap);
int rg_records_expand(const void* compact, size_t bytes, int32_t n, rg_mb_out* out);

/* Tuning of the pipelined mode (rg_set_pipeline_tuning); 0 in any field selects the default. */
typedef struct rg_pipeline_tuning {
    int32_t lag;          /* macroblock-times between consecutive pictures in the work order    */
    int32_t seg;          /* macroblocks per work segment                                         */
    int32_t grid;         /* resident warps                                                       */
    int32_t timeout_ms;   /* limit of one device wait                                             */
    int32_t deblock_sms;  /* SMs taking deblocking segments first (-1: no deblocking queue)       */
    int32_t intra_sms;    /* next SMs taking IDR-picture analysis first (-1: no such queue)       */
} rg_pipeline_tuning;

/*
 * Tuning / test hook of the pipelined mode (tuning NULL: all defaults): lag = macroblock-times between consecutive pictures
 * of a stream in the work order (1..4096; 0 = derived from the searches: max(seg, 2) * (4 + ry)
 * + seg + rx + 3, which orders every wait of a search reaching up to ry macroblock rows and rx
 * columns beyond zero motion after the work it waits for; ry = rx = 4 until the context's
 * launches have shown their reach, raised as soon as a launch reaches further, lowered after two
 * launches in a row that both reached less; larger is safer for long motion, smaller favours newer
 * pictures), seg = macroblocks per
 * work segment (1..mb_w, 0 = 1), grid = resident warps (0 = sixteen per SM, fewer if they do not
 * fit), timeout_ms = limit of one device wait (0 = 2000), deblock_sms = SMs whose warps take
 * deblocking segments first from a queue of their own (0 = one SM in five, -1 = one mixed queue
 * for all warps), intra_sms = the next SMs, whose warps take the analysis of IDR pictures first
 * from a queue of their own (0 = one SM in seven, -1 = none). A wait that runs out makes the launch stop and rg_sync re-run the
 * call on the per-diagonal path, which has no waits. No counterpart in the reference (its GOP
 * threads have no device schedule).
 */
int rg_set_pipeline_tuning(rg_ctx* ctx, const rg_pipeline_tuning* tuning);

/* The picture lag the next pipelined launch of the context uses (the set one, or the one derived
 * from the reach of its searches); negative RG_ERR_* on a null context. No counterpart in the
 * reference. */
int32_t rg_pipeline_lag(const rg_ctx* ctx);

/* ---- analysis forms ------------------------------------------------------------------------ */
/*
 * Two forms beside the plain one (the Balanced preset, byte-identical to the reference), neither
 * of which exists in the reference; both need CABAC (Main / High profile):
 *
 * RG_FORM_FULLSEARCH: P macroblocks search every integer vector within +-search_range samples of
 *   the 16x16 predictor (the sum of absolute differences of each 8x8 quadrant at every position,
 *   plus lambda times the vector bits), refine the best vector of every partition of the four
 *   partition types (16x16, 16x8, 8x16, 8x8) to quarter samples by SATD with each partition's own
 *   predictor, and code the type of least cost. Intra and the residual follow the plain form.
 * RG_FORM_LEARNED: the same decisions restricted by a per-macroblock hint (rg_mb_hint, from the
 *   candidate network of rg_net_predict_hints): the integer search covers +-2 samples around a
 *   centre chosen among integer candidates (the predictor plus the hinted offset, the predictor,
 *   the hint's coarse vector, the left / top / top-right neighbours' vectors, zero) by 16x16 SAD
 *   plus vector bits, re-centred on its best up to `walk` times while that lies on the window's
 *   edge, then the full +-search_range search; only the hinted partition types are refined (by
 *   SAD: a half-sample diamond step, then up to two quarter-sample diamond steps), and intra 4x4
 *   blocks of IDR pictures try only their hinted prediction modes.
 */
#define RG_FORM_PLAIN 0
#define RG_FORM_FULLSEARCH 1
#define RG_FORM_LEARNED 2

/* Per-macroblock hint of the learned form (raster order, one per macroblock of a picture). */
typedef struct rg_mb_hint {
    uint8_t part_mask;      /* bit t: partition type t is tried (t as rg_mb_out.part_type)       */
    uint8_t flags;          /* bit 0: mv_coarse holds a vector                                   */
    int8_t mv_off[2];       /* offset of the integer search's centre from the 16x16 predictor,
                               quarter samples                                                   */
    uint16_t i4_mask[16];   /* bit m: Intra4x4PredMode m is tried for 4x4 block b (decoding order) */
    int16_t mv_coarse[2];   /* coarse motion against the previous picture's source (quarter samples;
                               rg_net_predict_hints, see rg_net_set_coarse_range)                */
} rg_mb_hint;

/* ---- the learned form's candidate network (no counterpart in the reference) ----------------- */
/*
 * A small CNN over each macroblock and a 4-sample border (24 x 24 luma of the picture and of the
 * previous picture): three 3x3 convolutions of 32 channels with ReLU, then heads over the 18 x 18
 * map's mean (4 partition-type logits, a 2-component offset of the integer search's centre in units
 * of 16 quarter samples) and over each 4x4 block's mean (9 intra 4x4 mode logits). Inference runs
 * in BF16 on the tensor cores; training in f32 on the CUDA cores. Parameters are rg_net_param_count()
 * floats: conv weights [32][in][3][3] and biases of the three layers, then the partition head
 * [4][32] + 4, the offset head [2][32] + 2 and the intra head [9][32] + 9.
 */
typedef struct rg_net rg_net;
int32_t rg_net_param_count(void);
/* A network on `device` with parameters drawn from `seed` (He-uniform). NULL on failure. */
rg_net* rg_net_create(int32_t device, uint64_t seed);
void rg_net_destroy(rg_net* net);
int rg_net_set_params(rg_net* net, const float* params, int32_t count);
int rg_net_get_params(const rg_net* net, float* params, int32_t count);
/*
 * Hints of n_pictures pictures on the device: dev_cur[k] / dev_prev[k] the luma planes (display
 * size width x height, row stride `stride`; prev = cur for an IDR picture), dev_hints[k] receives
 * mb_w * mb_h rg_mb_hint (the candidate partition types and intra 4x4 modes of each block that
 * rg_net_set_hint_policy keeps, the rounded offset), dev_logits[k] (or dev_logits NULL) mb_w * mb_h * 150 floats (partition
 * 4, offset 2, intra 4x4 9 per block in raster order). Asynchronous on `stream`; rg_net_check
 * reports a wait on the tensor cores that gave up.
 */
int rg_net_predict_hints(rg_net* net, const uint8_t* const* dev_cur, const uint8_t* const* dev_prev, int32_t n_pictures,
                         int32_t width, int32_t height, size_t stride, rg_mb_hint* const* dev_hints,
                         float* const* dev_logits, void* stream);
int rg_net_check(rg_net* net, void* stream);
/*
 * Which candidates rg_net_predict_hints keeps: per macroblock the partition type of the largest
 * logit, then the next ones in logit order up to part_k types in all (1..4), each only while its
 * logit is at least the largest minus part_margin (>= 0; INFINITY: no margin); per intra 4x4 block
 * the same with i4_k (1..9) and i4_margin. Default: 3, INFINITY, 3, INFINITY (the top three).
 */
int rg_net_set_hint_policy(rg_net* net, int32_t part_k, float part_margin, int32_t i4_k, float i4_margin);
/*
 * Coarse motion of rg_net_predict_hints (range 0: off, the hints' flags bit 0 clear; else an even
 * 2..64, default 32): per macroblock of a picture whose previous picture differs from it, the
 * vector of least SAD of the 2:1 decimated macroblock (2x2 means, rounded) against the decimated
 * previous picture (coordinates clamped to the picture) over +-range/2 decimated samples, ties to
 * the least |x| + |y| and then the first in raster order; written as twice that vector in
 * mv_coarse (quarter samples) with flags bit 0 set.
 */
int rg_net_set_coarse_range(rg_net* net, int32_t range);
/* Training crops: sample k is macroblock (mb_xy[2k], mb_xy[2k+1]) of the luma planes cur[k] /
 * prev[k] (device, display size): 2 x 24 x 24 bytes each into dev_out. */
int rg_net_crops(rg_net* net, const uint8_t* const* cur, const uint8_t* const* prev, const int32_t* mb_xy, int32_t n,
                 int32_t width, int32_t height, size_t stride, uint8_t* dev_out, void* stream);
/*
 * One forward and backward pass over n crops (device arrays): labels dev_part [n] (partition type,
 * -1 none), dev_i4 [n][16] (intra 4x4 mode of each raster 4x4 block, -1 none), dev_mv [n][2] (the
 * offset target in units of 16 quarter samples) with dev_mvv [n] (0: none). Loss = mean
 * cross-entropy of the partition labels + mean cross-entropy of the block labels + mv_weight * mean
 * Huber loss of the offsets. dev_logits (n * 150 floats), loss_out and grads_out (host, the
 * parameters' layout) may be NULL. The gradients stay for rg_net_adam_step.
 */
int rg_net_forward_backward(rg_net* net, const uint8_t* dev_crops, int32_t n, const int32_t* dev_part,
                            const int32_t* dev_i4, const float* dev_mv, const int32_t* dev_mvv, float mv_weight,
                            float* dev_logits, float* loss_out, float* grads_out);
/* Adam (beta 0.9 / 0.999) step of the last gradients with learning rate lr. */
int rg_net_adam_step(rg_net* net, float lr);

/*
 * Selects the analysis form of the context's next calls (RG_FORM_*) and the integer search range
 * of the search forms (1..128 samples; ignored by the plain form). The learned form needs hints
 * for every analysed picture (rg_set_hints). Returns RG_ERR_UNSUPPORTED for a search form in a
 * Baseline (CAVLC) context. No counterpart in the reference.
 */
int rg_set_analysis_form(rg_ctx* ctx, int32_t form, int32_t search_range);

/*
 * Decision constants of the search forms (test and tuning hook): the bits charged per partition
 * type (16x16, 16x8, 8x16, 8x8; type_bits NULL: the defaults), times lambda, and the learned form's
 * re-centrings of its +-2 window before the full search (`walk`, 0..64). No counterpart in the
 * reference.
 */
int rg_set_search_tuning(rg_ctx* ctx, const int32_t* type_bits, int32_t walk);

/*
 * Device hints of the learned form for the next pipelined or batched call: dev_hints[f * S + s] is
 * the device address of picture f of stream s's mb_w * mb_h rg_mb_hint records (the order of the
 * call's planes). They must stay valid until the call is resolved. No counterpart in the reference.
 */
int rg_set_hints(rg_ctx* ctx, const rg_mb_hint* const* dev_hints, int32_t count);

/*
 * The network the learned form predicts its hints with (NULL: none): a pipelined call
 * (rg_analyse_gops*) without rg_set_hints first runs `net` on its own sources -- each picture's luma
 * with the previous picture's of the same call (the picture itself for an IDR picture and for the
 * call's first picture) -- on the context's stream, into hint buffers of the context. The network
 * must outlive its use. No counterpart in the reference.
 */
int rg_set_hint_net(rg_ctx* ctx, rg_net* net);

/* Waits for queued device work of the context. */
int rg_sync(rg_ctx* ctx);

/* Copies the records of the last analysed frame of every stream to host memory. */
int rg_copy_records(rg_ctx* ctx, rg_mb_out* out);

/*
 * Copies the deblocked reconstruction (display size) of the last frame of `stream` into host
 * planes (VideoFrame layout: luma width x height, chroma ceil(w/2) x ceil(h/2)).
 */
int rg_get_recon(rg_ctx* ctx, int32_t stream, uint8_t* y, uint8_t* u, uint8_t* v,
                 size_t stride_y, size_t stride_uv);

/*
 * Copies the reconstruction before deblocking (coded size, luma mb_w*16 x mb_h*16) of the last
 * frame of `stream`; used by the parity tests of the deblocking filter.
 */
int rg_get_recon_unfiltered(rg_ctx* ctx, int32_t stream, uint8_t* y, uint8_t* u, uint8_t* v);

/*
 * Deblocked reconstruction of the last frame of `stream` at coded size (luma mb_w*16 x
 * mb_h*16, chroma half that, tightly packed): the reference picture the next P frame predicts
 * from, as EncState::refp holds it after deblock (enc.rs:2470-2490).
 */
int rg_get_recon_coded(rg_ctx* ctx, int32_t stream, uint8_t* y, uint8_t* u, uint8_t* v);

/*
 * Keeps a device copy of every reconstruction before deblocking so that
 * rg_get_recon_unfiltered can return it (a test hook of this library; costs one extra store per
 * macroblock while enabled).
 */
int rg_keep_unfiltered(rg_ctx* ctx, int32_t enable);

/* The context's CUDA stream (cudaStream_t) for callers that time or order work around it. */
void* rg_cuda_stream(rg_ctx* ctx);

/*
 * SSIM of Y/U/V, their (4Y+U+V)/6 average, 5-scale luma MS-SSIM and PSNR of the last
 * reconstruction of `stream` against the given source planes (evaluate_frame_quality,
 * crates/ragdoll-pix/src/metrics.rs:328), computed on the device.
 */
int rg_quality_frame(rg_ctx* ctx, int32_t stream, const uint8_t* y, const uint8_t* u,
                     const uint8_t* v, size_t stride_y, size_t stride_uv, rg_quality* q);

/* rg_quality_frame with the previous source frame's luma (stride_prev), for VMAF-Lite's motion
 * term (evaluate_frame_quality's prev_reference); prev_y NULL is rg_quality_frame. */
int rg_quality_frame_prev(rg_ctx* ctx, int32_t stream, const uint8_t* y, const uint8_t* u,
                          const uint8_t* v, size_t stride_y, size_t stride_uv, const uint8_t* prev_y,
                          size_t stride_prev, rg_quality* q);

/* VMAF-Lite (crates/ragdoll-pix/src/metrics.rs:218 vmaf_lite_plane_u8) of host planes on `device`:
 * ref against dist, prev the previous reference plane or NULL. Result in *score (0..100). */
int rg_vmaf_lite_plane(int32_t device, const uint8_t* ref, size_t stride_ref, const uint8_t* dist,
                       size_t stride_dist, int32_t width, int32_t height, const uint8_t* prev,
                       size_t stride_prev, double* score);

/*
 * Stand-alone plane metrics on host planes (ssim_plane_u8 / ms_ssim_plane_u8,
 * crates/ragdoll-pix/src/metrics.rs:55, :154), computed on device `device`.
 */
int rg_ssim_plane(int32_t device, const uint8_t* a, size_t stride_a, const uint8_t* b,
                  size_t stride_b, int32_t width, int32_t height, double* ssim, double* ms_ssim);

/*
 * SSIM and (if ms_ssim) 5-scale MS-SSIM of n plane pairs of one size already on the device --
 * e.g. every reconstructed picture of a job against its source -- in shared launches: one 2x2
 * decimation launch per pyramid level for all pairs, then one SSIM launch over every pair and
 * level, then one for the row totals. Same arithmetic as rg_ssim_plane. dev_a[i] / dev_b[i]: device
 * planes with the given strides; ssim / ms_ssim: host arrays of n doubles (either may be NULL).
 * Synchronous on cuda_stream (NULL: legacy default stream); allocates its working memory.
 */
int rg_ssim_batch_device(int32_t device, const uint8_t* const* dev_a, const uint8_t* const* dev_b, int32_t n,
                         int32_t width, int32_t height, size_t stride_a, size_t stride_b, double* ssim, double* ms_ssim,
                         void* cuda_stream);

/*
 * Allocation-free SSIM / MS-SSIM of two planes already on the device. No counterpart in the
 * reference: it exists for callers that may not call cudaMalloc / cudaFree when they measure --
 * a frame loop whose device memory is all reserved by another allocator (a framework's caching
 * pool), or a latency-critical loop where an allocation would synchronise the device and stall
 * its other streams. SSIM is bit-identical to rg_ssim_plane's (same f32 row order); MS-SSIM is
 * combined on the device (pow / fmin / fmax there, std::pow on the host in rg_ssim_plane) and
 * agrees with rg_ssim_plane's within 1e-6.
 *
 * dev_a / dev_b: device planes (8-bit, given strides); dev_out: caller-owned device memory for two
 * doubles, written as {SSIM, MS-SSIM}; cuda_stream: the cudaStream_t to run on (NULL = legacy
 * default stream). Asynchronous: the results are ready when the stream reaches them.
 *
 * The working memory is one fixed __device__ array of the library (about 1.4 MB per GPU that
 * loads it, held until the process exits), so planes are limited to width and height in 8..4096
 * and at most 1920 x 1088 samples; larger ones get RG_ERR_INVALID (use rg_ssim_plane). Every call
 * on a device shares that array: calls that overlap on the GPU (other streams, other threads)
 * race and must be serialised by the caller. The first call on each device looks the array up
 * (cudaGetSymbolAddress) with that device current and keeps the address for the life of the
 * process; make that first call before any stream capture begins. Resetting a device
 * (cudaDeviceReset, or any teardown of its primary context) after that first call is not
 * supported: the kept address and the kernel's shared-memory attribute would be stale.
 */
int rg_ssim_plane_device_noalloc(const uint8_t* dev_a, size_t stride_a, const uint8_t* dev_b,
                                 size_t stride_b, int32_t width, int32_t height, double* dev_out,
                                 void* cuda_stream);

/*
 * Diagnostic: the work list of the pipelined mode for a shape (host code, no GPU), as the
 * kernel receives it -- per segment {picture * streams + stream, row << 16 | first macroblock
 * << 1 | deblocking} -- and each queue's range [queues[2q], queues[2q+1]) (queues: analysis,
 * deblocking, IDR-picture analysis; kinds[f * streams + s] or NULL). lag 0 = the default.
 * Returns the number of segments. Used by the tests that check the order never makes a
 * wait depend on a segment that no warp can take. No counterpart in the reference.
 */
int64_t rg_pipeline_work_list(int32_t mb_w, int32_t mb_h, int32_t streams, int32_t frames, int32_t lag, int32_t seg,
                              int32_t split, const int32_t* kinds, int32_t* tasks, int64_t cap, int32_t* queues);

/* ---- CAVLC bitstream writer (host) ------------------------------------------------------ */
/*
 * The serial half of encode_frame_body (crates/ragdoll-codec/src/h264/enc.rs:2234) for the
 * Baseline profile: turns one picture's records into its Annex-B access unit -- SPS and PPS
 * before an IDR (h264.rs:556-660, 806-832), the slice header (h264.rs:1071), skip runs and the
 * macroblock layer (enc.rs:989-1054, 3260-3285, 3540-3577, 3736-3750), CAVLC residual blocks
 * (h264.rs:2215 encode_cavlc_block) and NAL packing with emulation prevention (h264.rs:189).
 * Host code only; one writer per stream, usable from one thread each. Main / High use CABAC:
 * rg_writer_create returns NULL (RG_ERR_UNSUPPORTED) for them.
 */
typedef struct rg_writer rg_writer;
rg_writer* rg_writer_create(const rg_config* cfg, int32_t fps_num, int32_t fps_den);
void rg_writer_destroy(rg_writer* writer);
/* A buffer size that always holds one access unit of this writer. */
size_t rg_writer_bound(const rg_writer* writer);
/* Writes the access unit of one picture (records: mb_w * mb_h, raster order; kind RG_FRAME_*)
 * into out; returns its size in bytes, or a negative RG_ERR_* (the buffer too small included). */
int64_t rg_writer_picture(rg_writer* writer, const rg_mb_out* records, int32_t kind, uint8_t* out, size_t cap);
/* rg_writer_picture from the picture's compact records (rg_analyse_gops_fetch_compact). */
int64_t rg_writer_picture_compact(rg_writer* writer, const void* compact, size_t bytes, int32_t kind, uint8_t* out,
                                  size_t cap);

/* ---- Encoder (host + GPU) ---------------------------------------------------------------- */
/*
 * H264Encoder (crates/ragdoll-codec/src/h264.rs:2996) with the macroblock loop on the GPU: the
 * engine analyses, reconstructs and deblocks each picture and the host writes its access unit
 * (rg_writer_* coding: CAVLC for Baseline, CABAC for Main / High). Stream s is an independent
 * encoder (GOP); its picture k is an IDR picture when k % keyint == 0 (enc.rs:2245). threads <= 0:
 * one per host core.
 */
typedef struct rg_encoder rg_encoder;
rg_encoder* rg_encoder_create(const rg_config* cfg, int32_t fps_num, int32_t fps_den, int32_t keyint, int32_t threads);
void rg_encoder_destroy(rg_encoder* enc);
int32_t rg_encoder_threads(const rg_encoder* enc);
/* The engine context the encoder analyses with, for rg_set_pipeline_tuning (owned by the
 * encoder). No counterpart in the reference. */
rg_ctx* rg_encoder_context(rg_encoder* enc);
/* The fixed QP (1..51) of one stream, before its first picture (default cfg.qp): streams of
 * different QPs are analysed in the same launches and written with their own PPS. */
int rg_encoder_set_stream_qp(rg_encoder* enc, int32_t stream, int32_t qp);
/* H264Encoder::encode_frame (h264.rs:3153) for one stream: the Annex-B access unit of the next
 * picture into out; returns its size or a negative RG_ERR_*. Not while waves are in flight. */
int64_t rg_encode_frame(rg_encoder* enc, int32_t stream, const uint8_t* y, const uint8_t* u, const uint8_t* v,
                        size_t stride_y, size_t stride_uv, uint8_t* out, size_t cap);
/*
 * One wave of GopRingEncoder::encode_wave (crates/ragdoll-pipeline/src/lib.rs:543): the next
 * `frames` pictures of every stream (planes: frames * num_streams * 3 host pointers, [f][s][y,u,v];
 * frames <= cfg.max_frames) are queued for the GPU and the call returns. At most two waves are in
 * flight: while the host writes one (rg_encoder_collect) the GPU analyses the next. The sources
 * may be reused after the wave is collected; pinned sources copy fastest.
 */
int rg_encoder_submit(rg_encoder* enc, const uint8_t* const* planes, size_t stride_y, size_t stride_uv, int32_t frames);
/*
 * rg_encoder_submit for n encoders of different picture sizes at once (1..8 encoders on one
 * device, all in the plain form or all in the full-search form): every stream of every encoder is
 * analysed by ONE persistent launch (rg_analyse_gops_group_async; a CUDA graph per launch shape),
 * and each encoder's wave is then collected on its own (rg_encoder_collect, from any thread),
 * its pictures written as the launch finishes them. planes[i], stride_y[i], stride_uv[i]: encoder i's
 * arguments as rg_encoder_submit takes them. The batched transcode of many streams of mixed size.
 */
int rg_encoder_submit_group(rg_encoder* const* encs, int32_t n, const uint8_t* const* const* planes,
                            const size_t* stride_y, const size_t* stride_uv, int32_t frames);
/*
 * The access units of the oldest wave, written on the pool's threads: concatenated picture-major
 * ([f][s]) into out, sizes[f * num_streams + s] their sizes; returns the total. With out NULL only
 * the sizes and the total are returned and the wave stays to be collected.
 */
int64_t rg_encoder_collect(rg_encoder* enc, uint8_t* out, size_t cap, int64_t* sizes);
/*
 * Starts a new GOP on every stream with the next submitted picture, as the pipeline's fresh
 * H264Encoder per chunk does (GopRingEncoder::encode_wave, crates/ragdoll-pipeline/src/lib.rs:580-585):
 * the streams' picture counters restart, so that picture is an IDR picture with idr_pic_id 0 and
 * frame_num / POC from 0. Waves already submitted keep their counters.
 */
int rg_encoder_new_gops(rg_encoder* enc);
/* The analysis form of the encoder's next waves (rg_set_analysis_form on its context); the learned
 * form with its candidate network `net` (rg_set_hint_net), which must outlive its use. Not while
 * waves are in flight. No counterpart in the reference. */
int rg_encoder_set_form(rg_encoder* enc, int32_t form, int32_t search_range, rg_net* net);
/*
 * Per-picture latency of the wave collected last, [f * num_streams + s]: milliseconds from its
 * rg_encoder_submit to its access unit being written (up to n values into ms); returns the
 * wave's picture count (0 before the first collect). Telemetry of this library; no counterpart
 * in the reference.
 */
int32_t rg_encoder_latencies(const rg_encoder* enc, double* ms, int32_t n);
/* Bytes of records the wave collected last brought to the host: full records, or with
 * rg_set_record_compaction on rg_encoder_context (off by default: on a PCIe host whose copy engine
 * hides the full records' copy behind the launch, the launch's compaction costs more than it
 * saves) compact records plus the full records of pictures handed out without them. */
int64_t rg_encoder_record_bytes(const rg_encoder* enc);

/* ---- Containers (host) ------------------------------------------------------------------ */
/*
 * The muxers `ragdoll transcode` writes its H.264 output with: fast-start MP4
 * (crates/ragdoll-format/src/mp4.rs:1668 Mp4Muxer, :1746 finish) and Matroska
 * (crates/ragdoll-format/src/mkv.rs:840 MkvMuxer, :906 finish), one H.264 video track.
 * Access units go in as Annex-B (what rg_writer_picture returns); SPS and PPS move into the avcC
 * record (crates/ragdoll-format/src/mpegts.rs:273 build_avcc_from_sps_pps) and samples are
 * 4-byte length-prefixed (mpegts.rs:123 h264_annex_b_to_avcc_au). Given the same access units,
 * frame rate and size, the output is the reference's file byte for byte. Host code only.
 */
#define RG_CONTAINER_MP4 0
#define RG_CONTAINER_MKV 1

typedef struct rg_mux rg_mux;
/* fps_num / fps_den: the frame rate (pictures are evenly spaced on a 90 kHz clock). */
rg_mux* rg_mux_create(int32_t container, int32_t width, int32_t height, int32_t fps_num, int32_t fps_den);
void rg_mux_destroy(rg_mux* mux);
/* Adds one access unit in decoding order. The first must be an IDR picture carrying SPS and PPS;
 * parameter sets that change later are RG_ERR_UNSUPPORTED. */
int rg_mux_write(rg_mux* mux, const uint8_t* access_unit, size_t size);
/* The whole file: returns its size; with out non-NULL also writes it (cap must hold it).
 * May be called more than once (a size query first). */
int64_t rg_mux_finish(rg_mux* mux, uint8_t* out, size_t cap);

/*
 * Demuxers of the same two containers (mp4.rs:186 Mp4Demuxer, mkv.rs MkvDemuxer), for the first
 * H.264 video track, back to Annex-B access units (SPS and PPS in front of every IDR picture,
 * as the writer emits them). The data is copied at open. Laced Matroska blocks and files
 * without an H.264 track are RG_ERR_UNSUPPORTED.
 */
typedef struct rg_stream_info {
  int32_t container;      /* RG_CONTAINER_* */
  int32_t width, height;  /* from the sample entry / track entry */
  int32_t fps_num, fps_den;
  int32_t profile_idc;    /* from the SPS */
  int64_t access_units;
  int64_t keyframes;      /* access units holding an IDR slice */
} rg_stream_info;

typedef struct rg_demux rg_demux;
rg_demux* rg_demux_open(const uint8_t* data, size_t size);
void rg_demux_destroy(rg_demux* demux);
int rg_demux_info(const rg_demux* demux, rg_stream_info* info);
/* Access unit `index` as Annex-B: returns its size; with out non-NULL also writes it. */
int64_t rg_demux_access_unit(const rg_demux* demux, int64_t index, uint8_t* out, size_t cap);

#ifdef __cplusplus
}
#endif

#endif /* RAGDOLL_CUDA_H */
