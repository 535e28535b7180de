// C ABI of the engine (include/ragdoll_cuda.h): contexts, batched wavefront launches, host <->
// device copies, reconstruction and quality read-back.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <array>
#include <atomic>
#include <vector>

#include "engine.h"
#include "h264_consts.h"
#include "ssim_kernels.h"

using namespace rg;

namespace {

thread_local std::string g_last_error;

constexpr int kDefaultLag = 0;   // pipelined work order: 0 = derived from the reach of the searches
constexpr int kDefaultSeg = 1;
// Search forms: bits charged per partition type (16x16, 16x8, 8x16, 8x8), times lambda, and the
// learned form's window re-centrings before it falls back to the full search. On 1080p High, 4 GOPs
// x 15, QP 22-34, the full search's BD-rate against the plain form was -6.5 % with {1, 3, 3, 7} and
// -8.5 % with these bits; with the coarse-motion candidate the learned form's rate no longer depends
// on the walk (-27.2 % at 0, -26.9 % at 2 and 64) while its speed does (760, 1008, 1105 frames/s).
constexpr uint16_t kDefaultTypeBits[4] = {1, 16, 16, 40};
constexpr int kDefaultWalk = 4;
// Deblocking SMs: one in five takes the deblocking queue first (30 of 148). Measured on B200 with
// 16 warps per SM, 1080p 8 x 15 launch: 25 SMs 52.3-53.2 ms, 30 51.4-52.3, 35-40 52.6-52.8
// (at 7 warps per SM, before the IDR path got faster: 16 SMs 1326 frames/s, 20-30 1394-1417).
int default_deblock_sms(int sms) { return sms >= 5 ? (sms + 4) / 5 : 0; }
// The analysis of IDR pictures heads every GOP (each P picture trails it): the next one SM in
// seven takes it first (21 of 148; with 30 deblocking SMs: 20 IDR SMs 51.6 ms, 30 51.8, 49 52.3;
// at 7 warps per SM one in three was best). Those warps continue with P pictures once the IDR
// queue is empty.
int default_intra_sms(int sms) { return sms >= 7 ? sms / 7 : 0; }

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define CK(expr)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (expr);                                                              \
    if (e_ != cudaSuccess) return fail(RG_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
  } while (0)

struct Quant4Host {
  uint32_t mf[16], bias, shift;
};
int pos4h(int i) {
  int r = i >> 2, c = i & 3;
  if (((r | c) & 1) == 0) return 0;
  return ((r & c) & 1) ? 1 : 2;
}
Quant4Host quant4h(int qp, bool intra) {
  Quant4Host q;
  q.shift = 15 + qp / 6;
  for (int i = 0; i < 16; i++) q.mf[i] = tables::kMf4[qp % 6][pos4h(i)];
  q.bias = (1u << q.shift) / (intra ? 3u : 6u);
  return q;
}

// SkipBounds::new (enc.rs:2135) for the inter quantiser at qp / qpc.
void skip_bounds(int qp, int qpc, FrameParams& fp) {
  Quant4Host q = quant4h(qp, false), qc = quant4h(qpc, false);
  auto zsad = [](const Quant4Host& qq) {
    static const uint32_t W[4] = {1, 2, 1, 2};
    uint32_t room = (1u << qq.shift) - qq.bias - 1, mn = 0xffffffffu;
    for (int i = 0; i < 16; i++) mn = std::min(mn, room / (qq.mf[i] * W[i >> 2] * W[i & 3]));
    return mn;
  };
  auto zssd = [](const Quant4Host& qq) {
    static const uint32_t N[4] = {4, 10, 4, 10};
    uint32_t room = (1u << qq.shift) - qq.bias - 1, mn = 0xffffffffu;
    for (int i = 0; i < 16; i++) {
      uint32_t lim = room / qq.mf[i];
      mn = std::min(mn, lim * lim / (N[i >> 2] * N[i & 3]));
    }
    return mn;
  };
  uint32_t dsh = 16 + qpc / 6;
  uint32_t droom = (1u << dsh) - (1u << dsh) / 3 - 1;
  uint32_t dc = droom / tables::kMf4[qpc % 6][0];
  fp.sb_luma = zsad(q);
  fp.sb_luma_ssd = zssd(q);
  fp.sb_chroma = std::min(zsad(qc), dc);
  fp.sb_chroma_ssd = std::min(zssd(qc), dc * dc / 64);
  fp.sb_probe = 16 * (((1u << q.shift) - q.bias) / q.mf[0] + 1);
}

// The per-stream QP fields of a StreamDev at qp.
struct StreamQp {
  int32_t qp, qpc;
  uint32_t sb_luma, sb_luma_ssd, sb_chroma, sb_chroma_ssd, sb_probe;
};
StreamQp stream_qp(int qp) {
  FrameParams t{};
  int qpc = tables::kChromaQp[qp];
  skip_bounds(qp, qpc, t);
  return {qp, qpc, t.sb_luma, t.sb_luma_ssd, t.sb_chroma, t.sb_chroma_ssd, t.sb_probe};
}
void apply_qp(StreamDev& d, const StreamQp& q) {
  d.qp = q.qp;
  d.qpc = q.qpc;
  d.sb_luma = q.sb_luma;
  d.sb_luma_ssd = q.sb_luma_ssd;
  d.sb_chroma = q.sb_chroma;
  d.sb_chroma_ssd = q.sb_chroma_ssd;
  d.sb_probe = q.sb_probe;
}

}  // namespace

namespace rg {
// Records msg as the calling thread's rg_last_error() (used by entry points in other files).
void set_last_error(const char* msg) { g_last_error = msg; }
}  // namespace rg

struct rg_ctx {
  rg_config cfg{};
  FrameParams fp{};
  int S = 0, n_mb = 0;
  int rows_y = 0, rows_c = 0;      // padded rows
  size_t pic_y = 0, pic_c = 0;     // bytes of one padded plane
  cudaStream_t stream = nullptr;
  uint8_t* pics = nullptr;         // [S][2][Y U V]
  MbInfo* infos = nullptr;         // [S][2][n_mb]
  rg_mb_out* recs = nullptr;       // [S][n_mb]
  uint8_t* srcs = nullptr;         // [S][Y U V] compact display-size staging
  uint8_t* unf = nullptr;          // [S][Y U V] coded-size copies before deblocking
  bool keep_unfiltered = false;
  StreamDev* d_streams[2] = {nullptr, nullptr};  // [max_frames][S] descriptors each
  StreamDev* h_streams[2] = {nullptr, nullptr};  // pinned
  cudaEvent_t slot_done[2] = {nullptr, nullptr};
  int slot = 0;
  int max_frames = 1, nslots = 2;  // pictures per pipelined call; picture ring per stream
  int* counters = nullptr;         // pipelined-mode progress counters
  size_t n_counters = 0;
  int* h_err = nullptr;            // mapped host memory: each pending launch's error word
  int* d_err = nullptr;            // the same, as the device sees it
  int grid = 0;
  int lag = kDefaultLag;           // macroblock-times between pictures of a stream in the work order
  // Reach of the searches the lag is derived from when lag is 0 (macroblock rows / columns beyond
  // zero motion): 4 until launches show otherwise; lowered only after kReachLowRuns launches that
  // all reached less (a new work list costs ~10 ms of host time at 1080p x 120 pictures).
  int reach_y = 4, reach_x = 4;
  int reach_low = 0, low_y = 0, low_x = 0;
  int seg = kDefaultSeg;           // macroblocks per work segment
  unsigned long long timeout_ns = 2000000000ull;  // limit of one device wait
  int deblock_sms = 0;             // SMs preferring deblocking segments (0 = one mixed queue)
  int intra_sms = 0;               // SMs preferring IDR-picture analysis (0 = no such queue)
  int sms = 0;
  int2* d_tasks = nullptr;         // work list of the pipelined mode
  size_t tasks_cap = 0, n_tasks = 0;
  int qbeg[3] = {0, 0, 0}, qend[3] = {0, 0, 0};
  int tasks_frames = -1, tasks_lag = -1, tasks_seg = -1, tasks_split = -1;  // what d_tasks holds
  std::vector<int32_t> tasks_kinds;
  std::vector<int2> h_tasks;
  // the pending pipelined call, kept to re-run it on the per-diagonal path after a failed wait
  // Pipelined calls queued and not yet resolved (at most two, oldest first): what a re-run needs.
  struct Pending {
    std::vector<const uint8_t*> planes;  // device planes, [f][s][y,u,v]
    std::vector<int32_t> kinds;
    std::vector<int> start;              // frames analysed per stream before the call
    int frames = 0;
    size_t sy = 0, suv = 0;
    rg_mb_out* rec = nullptr;            // device records
    rg_mb_out* out = nullptr;            // host copy queued by an asynchronous call, or null
    size_t out_bytes = 0;
    int* h_err = nullptr;                // mapped host: the launch's error word
    int* h_reach = nullptr;              // mapped host: 1 + the reach its reference waits saw [2]
    cudaEvent_t done = nullptr;          // after the launch
    std::vector<const rg_mb_hint*> hints;  // learned form: [f][s] (empty otherwise)
  };
  Pending pend[2];
  int pend_head = 0, pend_count = 0;
  // asynchronous host-buffer calls (rg_analyse_gops_async): two slots of source staging and
  // records, a copy-in and a copy-out stream; allocated on the first such call
  uint8_t* a_srcs[2] = {nullptr, nullptr};
  rg_mb_out* a_recs[2] = {nullptr, nullptr};
  cudaStream_t a_in = nullptr, a_out = nullptr;
  cudaEvent_t a_in_done[2] = {nullptr, nullptr}, a_kern_done[2] = {nullptr, nullptr};
  cudaEvent_t a_out_done[2] = {nullptr, nullptr};
  rg_mb_out* a_out_ptr[2] = {nullptr, nullptr};  // host buffer each slot's call copies into
  // rg_analyse_gops_group: as the leader, the launch's descriptors, counters and merged work list;
  // as any member, an event that orders the leader's launch after this context's earlier work
  StreamDev* g_dstreams = nullptr;
  StreamDev* g_hstreams = nullptr;  // pinned
  size_t g_streams_cap = 0;
  int* g_counters = nullptr;
  size_t g_counters_cap = 0;
  int2* g_dtasks = nullptr;
  size_t g_tasks_cap = 0, g_ntasks = 0;
  std::vector<int2> g_htasks;
  std::vector<int64_t> g_shape;
  int g_qbeg[3] = {0, 0, 0}, g_qend[3] = {0, 0, 0};
  cudaEvent_t g_done = nullptr, g_order = nullptr;
  // the launch's stream work as CUDA graphs, one per launch shape (two kept: calls alternate
  // between two error words), replayed while the shape holds
  struct GroupGraph {
    std::vector<int64_t> key;
    cudaGraphExec_t exec = nullptr;
  };
  GroupGraph g_graphs[2];
  int g_graph_next = 0;
  int64_t g_graph_captures = 0, g_graph_launches = 0;
  int* h_ready[2] = {nullptr, nullptr};  // mapped host memory: per picture, the launch seq once final
  int* d_ready[2] = {nullptr, nullptr};  // the same, as the device sees it
  int a_seq[2] = {0, 0}, a_frames[2] = {0, 0};
  // compact records of rg_analyse_gops_stream (rg_set_record_compaction): per slot, mapped host
  // memory of c_row words per macroblock row, each row's compact size, and per picture the bytes
  // of its compact records once the host packed its rows together (-1 not yet, -2 did not fit)
  int compact_words = 0;           // words per macroblock of a slot; 0: off
  uint32_t* h_cwords[2] = {nullptr, nullptr};
  uint32_t* d_cwords[2] = {nullptr, nullptr};
  int* h_cbytes[2] = {nullptr, nullptr};
  int* d_cbytes[2] = {nullptr, nullptr};
  int c_row[2] = {0, 0};           // words per row slot of each slot's buffers
  std::vector<int64_t> c_packed[2];
  bool a_compact[2] = {false, false};  // the slot's call writes compact records
  int launch_seq = 0;
  int a_slot = 0;
  int form = RG_FORM_PLAIN;        // analysis form (rg_set_analysis_form)
  int search_range = 32;           // integer search range of the search forms
  int walk = kDefaultWalk;         // learned form: re-centrings of the seed's window
  uint16_t type_bits[4] = {kDefaultTypeBits[0], kDefaultTypeBits[1], kDefaultTypeBits[2], kDefaultTypeBits[3]};
  MbMv4* mv4s = nullptr;           // [S][nslots][n_mb] quadrant vectors (search forms; on first use)
  std::vector<const rg_mb_hint*> hints;  // learned form: the next call's hints (rg_set_hints)
  rg_net* net = nullptr;           // learned form: the network that predicts a call's hints itself
  rg_mb_hint* d_hints = nullptr;   // [2][max_frames][S][n_mb] hints the context predicted (two calls)
  int hint_slot = 0;
  std::vector<int> frames;         // frames analysed per stream
  std::vector<StreamQp> qps;       // QP of each stream (rg_set_stream_qp; default cfg.qp)
  // metrics scratch
  float* m_rows = nullptr;
  double* m_out = nullptr;
  unsigned long long* m_sse = nullptr;
  uint8_t* m_pyr = nullptr;
  SsimJob* m_jobs = nullptr;
  DecimateJob* m_djobs = nullptr;
  uint8_t* m_src = nullptr;

  uint8_t* pic_plane(int s, int slot_, int plane) const {
    size_t per_pic = pic_y + 2 * pic_c;
    uint8_t* base = pics + ((size_t)s * nslots + slot_) * per_pic;
    if (plane == 0) return base + (size_t)kPadY * fp.stride_y + kPadY;
    return base + pic_y + (plane - 1) * pic_c + (size_t)kPadC * fp.stride_c + kPadC;
  }
  size_t src_bytes() const {
    int cw = (cfg.width + 1) / 2, ch = (cfg.height + 1) / 2;
    return (size_t)cfg.width * cfg.height + 2 * (size_t)cw * ch;
  }
  size_t unf_bytes() const { return (size_t)fp.mb_w * fp.mb_h * 384; }
};

extern "C" {

const char* rg_last_error(void) { return g_last_error.c_str(); }

const char* rg_version(void) { return "ragdoll_b200 0.1 (sm_100a)"; }

rg_ctx* rg_create(const rg_config* cfg) {
  if (!cfg) { fail(RG_ERR_INVALID, "rg_create: null config"); return nullptr; }
  if (cfg->width < 1 || cfg->height < 1 || cfg->width > 8192 || cfg->height > 8192) {
    fail(RG_ERR_INVALID, "rg_create: size %dx%d outside 1..8192", cfg->width, cfg->height);
    return nullptr;
  }
  if (cfg->qp < 1 || cfg->qp > 51) {
    fail(RG_ERR_UNSUPPORTED, "rg_create: qp %d outside 1..51 (QP 0 codes I_PCM)", cfg->qp);
    return nullptr;
  }
  if (cfg->profile < RG_PROFILE_BASELINE || cfg->profile > RG_PROFILE_HIGH) {
    fail(RG_ERR_INVALID, "rg_create: profile %d", cfg->profile);
    return nullptr;
  }
  if (cfg->num_streams < 1 || cfg->num_streams > kMaxStreams) {
    fail(RG_ERR_INVALID, "rg_create: num_streams %d outside 1..%d", cfg->num_streams, kMaxStreams);
    return nullptr;
  }
  if (cudaSetDevice(cfg->device) != cudaSuccess) {
    fail(RG_ERR_CUDA, "rg_create: cudaSetDevice(%d) failed", cfg->device);
    return nullptr;
  }
  auto* c = new rg_ctx();
  c->cfg = *cfg;
  c->S = cfg->num_streams;
  FrameParams& fp = c->fp;
  fp.width = cfg->width;
  fp.height = cfg->height;
  fp.mb_w = (cfg->width + 15) / 16;
  fp.mb_h = (cfg->height + 15) / 16;
  fp.stride_y = ((fp.mb_w * 16 + 2 * kPadY) + 63) & ~63;
  fp.stride_c = ((fp.mb_w * 8 + 2 * kPadC) + 63) & ~63;
  fp.src_stride_y = cfg->width;
  fp.src_stride_uv = (cfg->width + 1) / 2;
  fp.qp = cfg->qp;
  fp.qpc = tables::kChromaQp[cfg->qp];
  fp.t8x8 = cfg->profile == RG_PROFILE_HIGH;
  fp.deblock = 1;
  fp.n_streams = c->S;
  skip_bounds(fp.qp, fp.qpc, fp);
  c->n_mb = fp.mb_w * fp.mb_h;
  c->rows_y = fp.mb_h * 16 + 2 * kPadY;
  c->rows_c = fp.mb_h * 8 + 2 * kPadC;
  c->pic_y = (size_t)fp.stride_y * c->rows_y;
  c->pic_c = (size_t)fp.stride_c * c->rows_c;
  c->frames.assign(c->S, 0);
  c->qps.assign(c->S, stream_qp(cfg->qp));
  c->max_frames = cfg->max_frames > 1 ? cfg->max_frames : 1;
  if (c->max_frames > 64) {
    fail(RG_ERR_INVALID, "rg_create: max_frames %d outside 0..64", cfg->max_frames);
    delete c;
    return nullptr;
  }
  c->nslots = c->max_frames + 1;
  c->n_counters = pipeline_counter_ints(fp, c->max_frames);
  bool ok = true;
  auto alloc = [&](void** p, size_t n) {
    if (!ok) return;
    if (cudaMalloc(p, n) != cudaSuccess) { ok = false; return; }
    cudaMemset(*p, 0, n);
  };
  alloc((void**)&c->pics, (c->pic_y + 2 * c->pic_c) * c->nslots * c->S);
  alloc((void**)&c->infos, sizeof(MbInfo) * c->n_mb * c->nslots * c->S);
  alloc((void**)&c->recs, sizeof(rg_mb_out) * c->n_mb * c->S * c->max_frames);
  alloc((void**)&c->srcs, c->src_bytes() * c->S * c->max_frames);
  alloc((void**)&c->d_streams[0], sizeof(StreamDev) * c->S * c->max_frames);
  alloc((void**)&c->d_streams[1], sizeof(StreamDev) * c->S * c->max_frames);
  alloc((void**)&c->counters, sizeof(int) * c->n_counters);
  c->tasks_cap = pipeline_task_count(fp, c->max_frames, c->seg);
  alloc((void**)&c->d_tasks, sizeof(int2) * c->tasks_cap);
  if (!ok) {
    fail(RG_ERR_OOM, "rg_create: device allocation failed");
    rg_destroy(c);
    return nullptr;
  }
  if (cudaMallocHost((void**)&c->h_streams[0], sizeof(StreamDev) * c->S * c->max_frames) != cudaSuccess ||
      cudaMallocHost((void**)&c->h_streams[1], sizeof(StreamDev) * c->S * c->max_frames) != cudaSuccess ||
      cudaHostAlloc((void**)&c->h_err, 6 * sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer((void**)&c->d_err, c->h_err, 0) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->pend[0].done, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->pend[1].done, cudaEventDisableTiming) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->slot_done[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->slot_done[1], cudaEventDisableTiming) != cudaSuccess) {
    fail(RG_ERR_CUDA, "rg_create: stream / pinned buffer setup failed");
    rg_destroy(c);
    return nullptr;
  }
  for (int k = 0; k < 6; k++) c->h_err[k] = 0;
  c->pend[0].h_err = c->h_err;
  c->pend[1].h_err = c->h_err + 1;
  c->pend[0].h_reach = c->h_err + 2;
  c->pend[1].h_reach = c->h_err + 4;
  c->grid = pipeline_grid(cfg->device);
  c->sms = pipeline_sms(cfg->device);
  c->deblock_sms = default_deblock_sms(c->sms);
  c->intra_sms = default_intra_sms(c->sms);
  upload_tables();
  if (cudaDeviceSynchronize() != cudaSuccess) {
    fail(RG_ERR_CUDA, "rg_create: %s", cudaGetErrorString(cudaGetLastError()));
    rg_destroy(c);
    return nullptr;
  }
  return c;
}

void rg_destroy(rg_ctx* c) {
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->pics);
  cudaFree(c->infos);
  cudaFree(c->mv4s);
  cudaFree(c->d_hints);
  cudaFree(c->recs);
  cudaFree(c->srcs);
  cudaFree(c->unf);
  cudaFree(c->d_streams[0]);
  cudaFree(c->d_streams[1]);
  cudaFree(c->m_rows);
  cudaFree(c->m_out);
  cudaFree(c->m_sse);
  cudaFree(c->m_pyr);
  cudaFree(c->m_jobs);
  cudaFree(c->m_djobs);
  cudaFree(c->m_src);
  cudaFree(c->counters);
  cudaFree(c->d_tasks);
  cudaFree(c->g_dstreams);
  cudaFree(c->g_counters);
  cudaFree(c->g_dtasks);
  if (c->g_hstreams) cudaFreeHost(c->g_hstreams);
  if (c->g_done) cudaEventDestroy(c->g_done);
  for (auto& g : c->g_graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (c->g_order) cudaEventDestroy(c->g_order);
  if (c->a_in) cudaStreamSynchronize(c->a_in);
  if (c->a_out) cudaStreamSynchronize(c->a_out);
  for (int i = 0; i < 2; i++) {
    cudaFree(c->a_srcs[i]);
    cudaFree(c->a_recs[i]);
    if (c->h_ready[i]) cudaFreeHost(c->h_ready[i]);
    if (c->h_cwords[i]) cudaFreeHost(c->h_cwords[i]);
    if (c->h_cbytes[i]) cudaFreeHost(c->h_cbytes[i]);
    for (cudaEvent_t e : {c->a_in_done[i], c->a_kern_done[i], c->a_out_done[i]})
      if (e) cudaEventDestroy(e);
  }
  if (c->a_in) cudaStreamDestroy(c->a_in);
  if (c->a_out) cudaStreamDestroy(c->a_out);
  if (c->h_err) cudaFreeHost(c->h_err);
  for (auto& p : c->pend)
    if (p.done) cudaEventDestroy(p.done);
  if (c->h_streams[0]) cudaFreeHost(c->h_streams[0]);
  if (c->h_streams[1]) cudaFreeHost(c->h_streams[1]);
  for (auto& e : c->slot_done) if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int rg_mb_dims(const rg_ctx* c, int32_t* mb_w, int32_t* mb_h) {
  if (!c || !mb_w || !mb_h) return fail(RG_ERR_INVALID, "rg_mb_dims: null argument");
  *mb_w = c->fp.mb_w;
  *mb_h = c->fp.mb_h;
  return RG_OK;
}

// Test hook: keep a copy of every reconstruction before deblocking (rg_get_recon_unfiltered).
int rg_keep_unfiltered(rg_ctx* c, int32_t enable) {
  if (!c) return fail(RG_ERR_INVALID, "rg_keep_unfiltered: null context");
  if (enable && !c->unf) {
    if (cudaMalloc((void**)&c->unf, c->unf_bytes() * c->S) != cudaSuccess)
      return fail(RG_ERR_OOM, "rg_keep_unfiltered: allocation failed");
  }
  c->keep_unfiltered = enable != 0;
  return RG_OK;
}

void* rg_cuda_stream(rg_ctx* c) { return c ? (void*)c->stream : nullptr; }

static int enqueue_wavefront(rg_ctx* c, const uint8_t* const* dev_planes, size_t stride_y, size_t stride_uv,
                             const int32_t* kinds, rg_mb_out* rec_base, int only = -1,
                             const rg_mb_hint* const* hints = nullptr);
static int take_hints(rg_ctx* c, int count, const char* who, std::vector<const rg_mb_hint*>& out);
static int async_copy_in(rg_ctx* c, int slot, const uint8_t* const* planes, size_t stride_y, size_t stride_uv,
                         int32_t frames, std::vector<const uint8_t*>& dev, const char* who);
static int resolve_pending(rg_ctx* c, bool wait_out);
static int resolve_oldest(rg_ctx* c);
static int auto_lag(const rg_ctx* c);

int rg_analyse_batch_device(rg_ctx* c, const uint8_t* const* dev_planes, size_t stride_y, size_t stride_uv,
                            const int32_t* kinds) {
  if (!c) return fail(RG_ERR_INVALID, "rg_analyse_batch_device: null context");
  int r = resolve_pending(c, false);
  if (r) return r;
  std::vector<const rg_mb_hint*> hv;
  r = take_hints(c, c->S, "rg_analyse_batch_device", hv);
  if (r) return r;
  return enqueue_wavefront(c, dev_planes, stride_y, stride_uv, kinds, nullptr, -1, hv.empty() ? nullptr : hv.data());
}

// The learned form's hints for a call of `count` pictures (rg_set_hints before the call); none for
// the other forms.
static int take_hints(rg_ctx* c, int count, const char* who, std::vector<const rg_mb_hint*>& out) {
  out.clear();
  if (c->form != RG_FORM_LEARNED) {
    c->hints.clear();
    return RG_OK;
  }
  if ((int)c->hints.size() != count)
    return fail(RG_ERR_STATE, "%s: the learned form needs %d hint arrays (rg_set_hints), %d set", who, count,
                (int)c->hints.size());
  for (int i = 0; i < count; i++)
    if (!c->hints[i]) return fail(RG_ERR_INVALID, "%s: null hint array %d", who, i);
  out.swap(c->hints);
  c->hints.clear();
  return RG_OK;
}

// One picture of every stream (or of stream `only`), one launch per anti-diagonal step; records
// at rec_base (default: the first picture's records). dev_planes and kinds hold one entry per
// stream launched.
static int enqueue_wavefront(rg_ctx* c, const uint8_t* const* dev_planes, size_t stride_y, size_t stride_uv,
                             const int32_t* kinds, rg_mb_out* rec_base, int only, const rg_mb_hint* const* hints) {
  if (!c || !dev_planes || !kinds) return fail(RG_ERR_INVALID, "rg_analyse_batch_device: null argument");
  if (stride_y < (size_t)c->cfg.width || stride_uv < (size_t)(c->cfg.width + 1) / 2)
    return fail(RG_ERR_INVALID, "rg_analyse_batch_device: stride too small");
  const int n = only >= 0 ? 1 : c->S;
  for (int i = 0; i < n; i++) {
    int s = only >= 0 ? only : i;
    if (kinds[i] != RG_FRAME_IDR && kinds[i] != RG_FRAME_P)
      return fail(RG_ERR_INVALID, "rg_analyse_batch_device: stream %d kind %d", s, kinds[i]);
    if (kinds[i] == RG_FRAME_P && c->frames[s] == 0)
      return fail(RG_ERR_STATE, "rg_analyse_batch_device: stream %d P frame without a reference", s);
    if (!dev_planes[3 * i] || !dev_planes[3 * i + 1] || !dev_planes[3 * i + 2])
      return fail(RG_ERR_INVALID, "rg_analyse_batch_device: stream %d null plane", s);
  }
  int slot = c->slot;
  c->slot ^= 1;
  CK(cudaEventSynchronize(c->slot_done[slot]));  // the pinned descriptor slot is free again
  StreamDev* h = c->h_streams[slot];
  size_t unf = c->unf_bytes();
  for (int i = 0; i < n; i++) {
    int s = only >= 0 ? only : i;
    int par = c->frames[s] % c->nslots, prv = (c->frames[s] + c->nslots - 1) % c->nslots;
    StreamDev& d = h[i];
    d.src_y = dev_planes[3 * i];
    d.src_u = dev_planes[3 * i + 1];
    d.src_v = dev_planes[3 * i + 2];
    d.cur_y = c->pic_plane(s, par, 0);
    d.cur_u = c->pic_plane(s, par, 1);
    d.cur_v = c->pic_plane(s, par, 2);
    d.ref_y = c->pic_plane(s, prv, 0);
    d.ref_u = c->pic_plane(s, prv, 1);
    d.ref_v = c->pic_plane(s, prv, 2);
    d.info = c->infos + ((size_t)s * c->nslots + par) * c->n_mb;
    d.prev_info = c->infos + ((size_t)s * c->nslots + prv) * c->n_mb;
    d.rec = (rec_base ? rec_base : c->recs) + (size_t)s * c->n_mb;
    if (c->keep_unfiltered) {
      uint8_t* u = c->unf + unf * s;
      d.unf_y = u;
      d.unf_u = u + (size_t)c->fp.mb_w * c->fp.mb_h * 256;
      d.unf_v = d.unf_u + (size_t)c->fp.mb_w * c->fp.mb_h * 64;
    } else {
      d.unf_y = d.unf_u = d.unf_v = nullptr;
    }
    d.kind = kinds[i];
    apply_qp(d, c->qps[s]);
    d.group = 0;
    d.rows_base = 0;
    d.prev_ps = -1;
    d.mv4 = c->mv4s ? c->mv4s + ((size_t)s * c->nslots + par) * c->n_mb : nullptr;
    d.hint = hints ? hints[i] : nullptr;
    d.search_range = c->search_range;
    d.walk = c->walk;
    for (int k = 0; k < 4; k++) { d.type_bits[k] = c->type_bits[k]; d.pad3_[k] = 0; }
    d.ready = nullptr;
  }
  FrameParams fp = c->fp;
  fp.src_stride_y = (int)stride_y;
  fp.src_stride_uv = (int)stride_uv;
  fp.n_streams = n;
  CK(cudaMemcpyAsync(c->d_streams[slot], h, sizeof(StreamDev) * n, cudaMemcpyHostToDevice, c->stream));
  CK(cudaEventRecord(c->slot_done[slot], c->stream));
  int steps = wavefront_steps(fp);
  for (int t = 0; t < steps; t++) launch_wavefront_step(fp, c->d_streams[slot], t, c->stream, c->form != RG_FORM_PLAIN);
  launch_extend_borders(fp, c->d_streams[slot], c->stream);
  CK(cudaGetLastError());
  for (int i = 0; i < n; i++) c->frames[only >= 0 ? only : i]++;
  return RG_OK;
}

// One persistent launch for `frames` pictures of every stream; records at rec_base. The previous
// pipelined call is resolved first (waited for, and re-run on the per-diagonal path if one of its
// waits gave up), so a call never starts from the pictures of a failed one. (Queueing it behind
// the previous launch without waiting measured slower end to end: the host's writing of the
// previous wave then runs during that wave's own launch and slows it.) ready / seq: per-picture
// flags in mapped host memory (rg_analyse_gops_stream), or null.
// Descriptor of picture f of stream s of a pipelined call (records at rec_base, [f][s]); in a launch
// of several contexts, this context's descriptors start at desc_base, its row counters at
// rows_base, and its picture size is group `group`.
static void gop_desc(const rg_ctx* c, StreamDev& d, int f, int s, const uint8_t* const* dev_planes,
                     const int32_t* kinds, rg_mb_out* rec_base, const rg_mb_hint* hint, int group, int desc_base,
                     int rows_base, int* ready = nullptr) {
  const int S = c->S, g = c->frames[s] + f;
  const int cur = g % c->nslots, prv = (g + c->nslots - 1) % c->nslots;
  d.src_y = dev_planes[(f * S + s) * 3];
  d.src_u = dev_planes[(f * S + s) * 3 + 1];
  d.src_v = dev_planes[(f * S + s) * 3 + 2];
  d.cur_y = c->pic_plane(s, cur, 0);
  d.cur_u = c->pic_plane(s, cur, 1);
  d.cur_v = c->pic_plane(s, cur, 2);
  d.ref_y = c->pic_plane(s, prv, 0);
  d.ref_u = c->pic_plane(s, prv, 1);
  d.ref_v = c->pic_plane(s, prv, 2);
  d.info = c->infos + ((size_t)s * c->nslots + cur) * c->n_mb;
  d.prev_info = c->infos + ((size_t)s * c->nslots + prv) * c->n_mb;
  d.rec = rec_base + ((size_t)f * S + s) * c->n_mb;
  d.unf_y = d.unf_u = d.unf_v = nullptr;
  d.kind = kinds[f * S + s];
  apply_qp(d, c->qps[s]);
  d.group = group;
  d.rows_base = rows_base + (f * S + s) * c->fp.mb_h;
  d.prev_ps = f > 0 ? desc_base + (f - 1) * S + s : -1;
  d.mv4 = c->mv4s ? c->mv4s + ((size_t)s * c->nslots + cur) * c->n_mb : nullptr;
  d.hint = hint;
  d.search_range = c->search_range;
  d.walk = c->walk;
  for (int k = 0; k < 4; k++) { d.type_bits[k] = c->type_bits[k]; d.pad3_[k] = 0; }
  d.ready = ready ? ready + f * S + s : nullptr;
}

static int enqueue_gops(rg_ctx* c, const uint8_t* const* dev_planes, size_t stride_y, size_t stride_uv,
                        const int32_t* kinds, int32_t frames, rg_mb_out* rec_base, int* ready = nullptr, int seq = 0,
                        bool resolved = false, const CompactOut* co = nullptr) {
  if (!c || !dev_planes || !kinds) return fail(RG_ERR_INVALID, "rg_analyse_gops_device: null argument");
  if (frames < 1 || frames > c->max_frames)
    return fail(RG_ERR_INVALID, "rg_analyse_gops_device: frames %d outside 1..%d (rg_config.max_frames)", frames,
                c->max_frames);
  if (stride_y < (size_t)c->cfg.width || stride_uv < (size_t)(c->cfg.width + 1) / 2)
    return fail(RG_ERR_INVALID, "rg_analyse_gops_device: stride too small");
  int S = c->S;
  if (!resolved) {
    int r = resolve_pending(c, false);
    if (r) return r;
  }
  for (int f = 0; f < frames; f++)
    for (int s = 0; s < S; s++) {
      int k = kinds[f * S + s];
      if (k != RG_FRAME_IDR && k != RG_FRAME_P)
        return fail(RG_ERR_INVALID, "rg_analyse_gops_device: picture %d stream %d kind %d", f, s, k);
      if (k == RG_FRAME_P && f == 0 && c->frames[s] == 0)
        return fail(RG_ERR_STATE, "rg_analyse_gops_device: stream %d starts with a P picture without a reference", s);
      for (int p = 0; p < 3; p++)
        if (!dev_planes[(f * S + s) * 3 + p])
          return fail(RG_ERR_INVALID, "rg_analyse_gops_device: picture %d stream %d null plane", f, s);
    }
  std::vector<const rg_mb_hint*> hv;
  if (c->form == RG_FORM_LEARNED && c->net && c->hints.empty()) {
    // the network reads each picture's luma and the previous picture's of the same call (the picture
    // itself for the first one and for IDR pictures)
    rg_mb_hint* base = c->d_hints + (size_t)c->hint_slot * c->max_frames * S * c->n_mb;
    c->hint_slot ^= 1;
    std::vector<const uint8_t*> cur((size_t)frames * S), prev((size_t)frames * S);
    std::vector<rg_mb_hint*> dst((size_t)frames * S);
    for (int f = 0; f < frames; f++)
      for (int s = 0; s < S; s++) {
        const size_t i = (size_t)f * S + s;
        cur[i] = dev_planes[i * 3];
        prev[i] = (f > 0 && kinds[i] == RG_FRAME_P) ? dev_planes[(i - S) * 3] : cur[i];
        dst[i] = base + i * c->n_mb;
      }
    int r = rg_net_predict_hints(c->net, cur.data(), prev.data(), frames * S, c->cfg.width, c->cfg.height, stride_y,
                                 dst.data(), nullptr, c->stream);
    if (r) return r;
    hv.assign(dst.begin(), dst.end());
  } else {
    int r = take_hints(c, frames * S, "rg_analyse_gops_device", hv);
    if (r) return r;
  }
  int slot = c->slot;
  c->slot ^= 1;
  CK(cudaEventSynchronize(c->slot_done[slot]));
  StreamDev* h = c->h_streams[slot];
  for (int f = 0; f < frames; f++)
    for (int s = 0; s < S; s++)
      gop_desc(c, h[f * S + s], f, s, dev_planes, kinds, rec_base, hv.empty() ? nullptr : hv[f * S + s], 0, 0, 0);
  FrameParams fp = c->fp;
  fp.src_stride_y = (int)stride_y;
  fp.src_stride_uv = (int)stride_uv;
  CK(cudaMemcpyAsync(c->d_streams[slot], h, sizeof(StreamDev) * S * frames, cudaMemcpyHostToDevice, c->stream));
  CK(cudaEventRecord(c->slot_done[slot], c->stream));
  CK(cudaMemsetAsync(c->counters, 0, sizeof(int) * pipeline_counter_ints(c->fp, frames), c->stream));
  int split = c->deblock_sms > 0 && c->grid >= 2 ? 1 : 0;
  // IDR pictures get their own queue when SMs are set aside for them
  std::vector<int32_t> kinds_key;
  if (c->intra_sms > 0 && c->grid >= 3) kinds_key.assign(kinds, kinds + (size_t)frames * S);
  const int lag = c->lag > 0 ? c->lag : auto_lag(c);
  if (frames != c->tasks_frames || lag != c->tasks_lag || c->seg != c->tasks_seg || split != c->tasks_split ||
      kinds_key != c->tasks_kinds) {
    // rebuilt only when the call's shape, its picture kinds or the tuning change; the copy is
    // stream-ordered after any launch still reading the old list
    c->h_tasks.resize(pipeline_task_count(fp, frames, c->seg));
    c->n_tasks = pipeline_task_list(fp, frames, lag, c->seg, split != 0,
                                    kinds_key.empty() ? nullptr : kinds_key.data(), c->h_tasks.data(), c->qbeg, c->qend);
    c->tasks_kinds = kinds_key;
    CK(cudaMemcpyAsync(c->d_tasks, c->h_tasks.data(), sizeof(int2) * c->n_tasks, cudaMemcpyHostToDevice, c->stream));
    c->tasks_frames = frames;
    c->tasks_lag = lag;
    c->tasks_seg = c->seg;
    c->tasks_split = split;
  }
  // The launch writes its error word into mapped host memory itself: a device-to-host copy queued
  // behind the launch would hold up, until the launch ends, every later device-to-host copy of the
  // context (the copy engine takes them in order), such as a picture fetched while it runs.
  int pslot = (c->pend_head + c->pend_count) & 1;
  rg_ctx::Pending& p = c->pend[pslot];
  *(volatile int*)p.h_err = 0;  // the launch that used this word before was resolved
  FrameGroups fg{};
  fg.g[0] = fp;
  fg.n = 1;
  launch_pipeline(fg, c->d_streams[slot], frames * S, frames * S * fp.mb_h, c->counters, c->d_tasks, c->n_tasks, c->qbeg,
                  c->qend, c->deblock_sms, c->intra_sms, c->sms, c->seg, c->grid, c->timeout_ns, ready, seq,
                  c->d_err + pslot, c->d_err + 2 + 2 * pslot, c->stream, c->form != RG_FORM_PLAIN, co);
  CK(cudaGetLastError());
  CK(cudaEventRecord(p.done, c->stream));
  p.planes.assign(dev_planes, dev_planes + (size_t)frames * S * 3);
  p.kinds.assign(kinds, kinds + (size_t)frames * S);
  p.start = c->frames;
  p.frames = frames;
  p.sy = stride_y;
  p.suv = stride_uv;
  p.rec = rec_base;
  p.out = nullptr;
  p.out_bytes = 0;
  p.hints = hv;
  c->pend_count++;
  for (int s = 0; s < S; s++) c->frames[s] += frames;
  return RG_OK;
}

int rg_analyse_gops_device(rg_ctx* c, const uint8_t* const* dev_planes, size_t stride_y, size_t stride_uv,
                           const int32_t* kinds, int32_t frames) {
  if (!c) return fail(RG_ERR_INVALID, "rg_analyse_gops_device: null context");
  return enqueue_gops(c, dev_planes, stride_y, stride_uv, kinds, frames, c->recs);
}

// ---- several contexts, one persistent launch ----------------------------------------------------
// The leader (ctxs[0]) keeps the launch's descriptors, counters and merged work list.
// The group launch (rg_analyse_gops_group): each context's records at rec_bases[i] (null: its own
// records buffer); resolved: the caller already resolved every context's earlier calls.
// readies (or null): per context the device address of its per-picture ready flags, set to seq
// as each picture's records are final.
static int group_launch(rg_ctx* const* ctxs, int32_t n, const uint8_t* const* const* dev_planes,
                        const size_t* stride_y, const size_t* stride_uv, const int32_t* const* kinds, int32_t frames,
                        rg_mb_out* const* rec_bases, bool resolved, const char* who, int* const* readies = nullptr,
                        int seq = 0) {
  if (!ctxs || !dev_planes || !stride_y || !stride_uv || !kinds || n < 1 || n > kMaxGroups)
    return fail(RG_ERR_INVALID, "%s: null argument or %d contexts (1..%d)", who, n, kMaxGroups);
  rg_ctx* L = ctxs[0];
  for (int i = 0; i < n; i++) {
    rg_ctx* c = ctxs[i];
    if (!c || !dev_planes[i] || !kinds[i]) return fail(RG_ERR_INVALID, "%s: null context or argument %d", who, i);
    for (int j = 0; j < i; j++)
      if (ctxs[j] == c) return fail(RG_ERR_INVALID, "%s: context %d given twice", who, i);
    if (c->cfg.device != L->cfg.device) return fail(RG_ERR_INVALID, "%s: contexts on different devices", who);
    if ((c->form != RG_FORM_PLAIN) != (L->form != RG_FORM_PLAIN) || c->form == RG_FORM_LEARNED)
      return fail(RG_ERR_UNSUPPORTED, "%s: the contexts must all be plain or all full search", who);
    if (frames < 1 || frames > c->max_frames)
      return fail(RG_ERR_INVALID, "%s: frames %d outside 1..%d of context %d", who, frames, c->max_frames, i);
    if (stride_y[i] < (size_t)c->cfg.width || stride_uv[i] < (size_t)(c->cfg.width + 1) / 2)
      return fail(RG_ERR_INVALID, "%s: stride too small (context %d)", who, i);
  }
  for (int i = 0; i < n; i++) {
    rg_ctx* c = ctxs[i];
    int r = resolved ? RG_OK : resolve_pending(c, false);
    if (r) return r;
    for (int f = 0; f < frames; f++)
      for (int s = 0; s < c->S; s++) {
        const int k = kinds[i][f * c->S + s];
        if (k != RG_FRAME_IDR && k != RG_FRAME_P)
          return fail(RG_ERR_INVALID, "%s: context %d picture %d stream %d kind %d", who, i, f, s, k);
        if (k == RG_FRAME_P && f == 0 && c->frames[s] == 0)
          return fail(RG_ERR_STATE, "%s: context %d stream %d starts with a P picture", who, i, s);
        for (int p = 0; p < 3; p++)
          if (!dev_planes[i][(f * c->S + s) * 3 + p])
            return fail(RG_ERR_INVALID, "%s: context %d picture %d stream %d null plane", who, i, f, s);
      }
    c->hints.clear();
  }
  CK(cudaSetDevice(L->cfg.device));
  // descriptors and rows of every context, one after the other, the contexts with more macroblocks
  // first whatever the argument order (64 streams of four sizes: 263 ms against 364 ms with the
  // smallest size's descriptors first)
  std::vector<int> lay(n);
  for (int i = 0; i < n; i++) lay[i] = i;
  std::stable_sort(lay.begin(), lay.end(), [&](int x, int y) {
    return (long)ctxs[x]->n_mb * ctxs[x]->S > (long)ctxs[y]->n_mb * ctxs[y]->S;
  });
  std::vector<int> desc_base(n, 0), rows_base(n, 0);
  int n_desc = 0, total_rows = 0;
  for (int i : lay) {
    desc_base[i] = n_desc;
    rows_base[i] = total_rows;
    n_desc += frames * ctxs[i]->S;
    total_rows += frames * ctxs[i]->S * ctxs[i]->fp.mb_h;
  }
  if ((size_t)n_desc > L->g_streams_cap) {
    if (L->g_done) CK(cudaEventSynchronize(L->g_done));
    cudaFree(L->g_dstreams);
    if (L->g_hstreams) cudaFreeHost(L->g_hstreams);
    L->g_dstreams = nullptr;
    L->g_hstreams = nullptr;
    L->g_streams_cap = 0;
    if (cudaMalloc((void**)&L->g_dstreams, sizeof(StreamDev) * n_desc) != cudaSuccess ||
        cudaHostAlloc((void**)&L->g_hstreams, sizeof(StreamDev) * n_desc, cudaHostAllocDefault) != cudaSuccess)
      return fail(RG_ERR_OOM, "%s: %d descriptors", who, n_desc);
    L->g_streams_cap = n_desc;
  }
  const size_t n_counters = pipeline_counter_ints(total_rows, n_desc);
  if (n_counters > L->g_counters_cap) {
    if (L->g_done) CK(cudaEventSynchronize(L->g_done));
    cudaFree(L->g_counters);
    L->g_counters = nullptr;
    if (cudaMalloc((void**)&L->g_counters, sizeof(int) * n_counters) != cudaSuccess)
      return fail(RG_ERR_OOM, "%s: %zu counters", who, n_counters);
    L->g_counters_cap = n_counters;
  }
  if (!L->g_done) CK(cudaEventCreateWithFlags(&L->g_done, cudaEventDisableTiming));
  CK(cudaEventSynchronize(L->g_done));  // the pinned descriptors of the last group call were copied
  FrameGroups fg{};
  fg.n = n;
  for (int i = 0; i < n; i++) {
    rg_ctx* c = ctxs[i];
    fg.g[i] = c->fp;
    fg.g[i].src_stride_y = (int)stride_y[i];
    fg.g[i].src_stride_uv = (int)stride_uv[i];
    for (int f = 0; f < frames; f++)
      for (int s = 0; s < c->S; s++)
        gop_desc(c, L->g_hstreams[desc_base[i] + f * c->S + s], f, s, dev_planes[i], kinds[i],
                 rec_bases && rec_bases[i] ? rec_bases[i] : c->recs, nullptr, i, desc_base[i], rows_base[i],
                 readies ? readies[i] : nullptr);
  }
  // launch shape: the segment length and SM roles of the context with the most macroblocks (its
  // tuning suits the bulk of the work), the largest grid of any
  const rg_ctx* T = L;
  int grid = 0;
  for (int i = 0; i < n; i++) {
    const rg_ctx* c = ctxs[i];
    if ((long)c->n_mb * c->S > (long)T->n_mb * T->S) T = c;
    grid = std::max(grid, c->grid);
  }
  // work list: each context's own (that segment length, each context's lag), merged by key queue
  // by queue; rebuilt only when the shape, the lags or the picture kinds change
  const int seg = T->seg, a = seg > 2 ? seg : 2;
  const int split = T->deblock_sms > 0 && grid >= 2 ? 1 : 0;
  const bool intra_q = T->intra_sms > 0 && grid >= 3;
  std::vector<int64_t> shape = {frames, seg, split, intra_q ? 1 : 0, n, grid};
  for (int i = 0; i < n; i++) {
    rg_ctx* c = ctxs[i];
    const int lag = c->lag > 0 ? c->lag : a * (4 + c->reach_y) + seg + c->reach_x + 3;
    shape.insert(shape.end(), {c->cfg.width, c->cfg.height, c->S, lag});
    if (intra_q) shape.insert(shape.end(), kinds[i], kinds[i] + (size_t)frames * c->S);
  }
  if (shape != L->g_shape) {
    std::vector<std::vector<int2>> lists(n);
    std::vector<std::vector<uint32_t>> keys(n);
    std::vector<std::array<int, 3>> qb(n), qe(n);
    size_t total = 0;
    for (int i = 0; i < n; i++) {
      rg_ctx* c = ctxs[i];
      const int lag = c->lag > 0 ? c->lag : a * (4 + c->reach_y) + seg + c->reach_x + 3;
      FrameParams fp = c->fp;
      lists[i].resize(pipeline_task_count(fp, frames, seg));
      keys[i].resize(lists[i].size());
      std::vector<int32_t> kk;
      if (intra_q) kk.assign(kinds[i], kinds[i] + (size_t)frames * c->S);
      pipeline_task_list(fp, frames, lag, seg, split != 0, intra_q ? kk.data() : nullptr, lists[i].data(), qb[i].data(),
                         qe[i].data(), keys[i].data());
      total += lists[i].size();
    }
    L->g_htasks.resize(total);
    // on equal keys the context with more macroblocks first: its pictures are the longest chains
    // (64 streams of four sizes, 30 pictures each: 263 ms against 364 ms with the smallest first)
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
      return (long)ctxs[x]->n_mb * ctxs[x]->S > (long)ctxs[y]->n_mb * ctxs[y]->S;
    });
    size_t at = 0;
    for (int q = 0; q < kPipeQueues; q++) {
      L->g_qbeg[q] = (int)at;
      std::vector<int> pos(n);
      for (int i = 0; i < n; i++) pos[i] = qb[i][q];
      while (true) {  // the least key first
        int best = -1;
        for (int i : order)
          if (pos[i] < qe[i][q] && (best < 0 || keys[i][pos[i]] < keys[best][pos[best]])) best = i;
        if (best < 0) break;
        int2 t = lists[best][pos[best]++];
        t.x += desc_base[best];
        L->g_htasks[at++] = t;
      }
      L->g_qend[q] = (int)at;
    }
    if (total > L->g_tasks_cap) {
      CK(cudaStreamSynchronize(L->stream));
      cudaFree(L->g_dtasks);
      L->g_dtasks = nullptr;
      L->g_tasks_cap = 0;
      if (cudaMalloc((void**)&L->g_dtasks, sizeof(int2) * total) != cudaSuccess)
        return fail(RG_ERR_OOM, "%s: %zu tasks", who, total);
      L->g_tasks_cap = total;
    }
    CK(cudaMemcpyAsync(L->g_dtasks, L->g_htasks.data(), sizeof(int2) * total, cudaMemcpyHostToDevice, L->stream));
    L->g_ntasks = total;
    L->g_shape = shape;
  }
  // the launch runs on the leader's stream after every context's earlier work
  for (int i = 1; i < n; i++) {
    rg_ctx* c = ctxs[i];
    if (!c->g_order) CK(cudaEventCreateWithFlags(&c->g_order, cudaEventDisableTiming));
    CK(cudaEventRecord(c->g_order, c->stream));
    CK(cudaStreamWaitEvent(L->stream, c->g_order, 0));
  }
  std::vector<int> pslot(n);
  for (int i = 0; i < n; i++) {
    rg_ctx* c = ctxs[i];
    pslot[i] = (c->pend_head + c->pend_count) & 1;
    *(volatile int*)c->pend[pslot[i]].h_err = 0;
  }
  // The stream work of the launch -- the descriptors' copy, the counters' reset, the persistent
  // launch and, per context, the hand-off of the launch's error word and reach (every context
  // holds the launch as its own pending call, resolved and if a wait gave up re-run picture by
  // picture by the context itself) -- as a CUDA graph, captured for each launch shape and replayed
  // while it holds (the descriptors' contents change per call; the copy reads them as it runs).
  std::vector<int64_t> key = L->g_shape;
  key.insert(key.end(), {n_desc, total_rows, (int64_t)n_counters, (int64_t)L->g_ntasks, T->deblock_sms,
                         T->intra_sms, L->sms, (int64_t)T->timeout_ns, (int64_t)(uintptr_t)L->g_dstreams,
                         (int64_t)(uintptr_t)L->g_hstreams, (int64_t)(uintptr_t)L->g_counters,
                         (int64_t)(uintptr_t)L->g_dtasks, L->form, seq});
  for (int i = 0; i < n; i++)
    key.insert(key.end(), {(int64_t)stride_y[i], (int64_t)stride_uv[i], (int64_t)(uintptr_t)(ctxs[i]->d_err + pslot[i])});
  rg_ctx::GroupGraph* gg = nullptr;
  for (auto& g : L->g_graphs)
    if (g.exec && g.key == key) gg = &g;
  if (!gg) {
    gg = &L->g_graphs[L->g_graph_next];
    L->g_graph_next ^= 1;
    if (gg->exec) CK(cudaGraphExecDestroy(gg->exec));
    gg->exec = nullptr;
    gg->key.clear();
    CK(cudaStreamBeginCapture(L->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaMemcpyAsync(L->g_dstreams, L->g_hstreams, sizeof(StreamDev) * n_desc, cudaMemcpyHostToDevice,
                                    L->stream);
    // an external event node: the event is recorded each time the graph runs (a plain record in a
    // capture only orders the capture's own streams)
    if (e == cudaSuccess) e = cudaEventRecordWithFlags(L->g_done, L->stream, cudaEventRecordExternal);
    if (e == cudaSuccess) e = cudaMemsetAsync(L->g_counters, 0, sizeof(int) * n_counters, L->stream);
    if (e == cudaSuccess) {
      launch_pipeline(fg, L->g_dstreams, n_desc, total_rows, L->g_counters, L->g_dtasks, L->g_ntasks, L->g_qbeg,
                      L->g_qend, T->deblock_sms, T->intra_sms, L->sms, seg, grid, T->timeout_ns, nullptr, seq, nullptr,
                      nullptr, L->stream, L->form != RG_FORM_PLAIN);
      for (int i = 0; i < n; i++)
        launch_error_to_host(L->g_counters, n_desc, total_rows, ctxs[i]->d_err + pslot[i],
                             ctxs[i]->d_err + 2 + 2 * pslot[i], L->stream);
      e = cudaGetLastError();
    }
    cudaGraph_t graph = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(L->stream, &graph);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&gg->exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      gg->exec = nullptr;
      cudaGetLastError();
      return fail(RG_ERR_CUDA, "%s: capturing the launch: %s", who, cudaGetErrorString(e));
    }
    gg->key = key;
    L->g_graph_captures++;
  }
  CK(cudaGraphLaunch(gg->exec, L->stream));
  L->g_graph_launches++;
  if (!L->g_order) CK(cudaEventCreateWithFlags(&L->g_order, cudaEventDisableTiming));
  CK(cudaEventRecord(L->g_order, L->stream));
  for (int i = 0; i < n; i++) {
    rg_ctx* c = ctxs[i];
    if (i) CK(cudaStreamWaitEvent(c->stream, L->g_order, 0));
    rg_ctx::Pending& p = c->pend[pslot[i]];
    CK(cudaEventRecord(p.done, c->stream));
    p.planes.assign(dev_planes[i], dev_planes[i] + (size_t)frames * c->S * 3);
    p.kinds.assign(kinds[i], kinds[i] + (size_t)frames * c->S);
    p.start = c->frames;
    p.frames = frames;
    p.sy = stride_y[i];
    p.suv = stride_uv[i];
    p.rec = rec_bases && rec_bases[i] ? rec_bases[i] : c->recs;
    p.out = nullptr;
    p.out_bytes = 0;
    p.hints.clear();
    c->pend_count++;
    for (int s = 0; s < c->S; s++) c->frames[s] += frames;
  }
  return RG_OK;
}

int rg_analyse_gops_group(rg_ctx* const* ctxs, int32_t n, const uint8_t* const* const* dev_planes,
                          const size_t* stride_y, const size_t* stride_uv, const int32_t* const* kinds,
                          int32_t frames) {
  return group_launch(ctxs, n, dev_planes, stride_y, stride_uv, kinds, frames, nullptr, false,
                      "rg_analyse_gops_group");
}

// rg_analyse_gops_group_async (bulk: each context's records copied out after the launch) and
// rg_analyse_gops_group_stream (each picture flagged as its records are final, fetched per picture).
static int group_async(rg_ctx* const* ctxs, int32_t n, const uint8_t* const* const* planes, const size_t* stride_y,
                       const size_t* stride_uv, const int32_t* const* kinds, int32_t frames, rg_mb_out* const* outs,
                       bool bulk, const char* who) {
  if (!ctxs || !planes || !stride_y || !stride_uv || !kinds || !outs || n < 1 || n > kMaxGroups)
    return fail(RG_ERR_INVALID, "%s: null argument or %d contexts (1..%d)", who, n, kMaxGroups);
  for (int i = 0; i < n; i++)
    if (!ctxs[i] || !planes[i] || !kinds[i] || !outs[i]) return fail(RG_ERR_INVALID, "%s: null argument %d", who, i);
  // each context's sources into its next staging slot (copy-in streams, overlapping the launches
  // still running)
  std::vector<std::vector<const uint8_t*>> dev(n);
  std::vector<const uint8_t* const*> devp(n);
  std::vector<int> slot(n);
  std::vector<rg_mb_out*> recs(n);
  std::vector<size_t> sy(n), suv(n);
  for (int i = 0; i < n; i++) {
    rg_ctx* c = ctxs[i];
    slot[i] = c->a_slot;
    int r = async_copy_in(c, slot[i], planes[i], stride_y[i], stride_uv[i], frames, dev[i], who);
    if (r) return r;
    devp[i] = dev[i].data();
    recs[i] = c->a_recs[slot[i]];
    sy[i] = c->cfg.width;
    suv[i] = (c->cfg.width + 1) / 2;
  }
  // at most one earlier call left in flight per context (the call two back, which last used this
  // staging slot, resolved -- re-run if a wait gave up -- and fetched): the launch is queued behind
  // the running one, whose pictures the caller fetches meanwhile. A wait that gives up in the
  // running launch re-runs both calls (resolve_oldest re-runs every pending call).
  for (int i = 0; i < n; i++)
    while (ctxs[i]->pend_count >= 2) {
      int r = resolve_oldest(ctxs[i]);
      if (r) return r;
    }
  // streamed: the slot's flags cleared (its last call was resolved and fetched), each picture's set
  // to 1 by the launch (a constant, so the launch's CUDA graph replays)
  std::vector<int*> readies(n);
  for (int i = 0; i < n; i++) {
    rg_ctx* c = ctxs[i];
    CK(cudaStreamWaitEvent(c->stream, c->a_in_done[slot[i]], 0));
    CK(cudaStreamWaitEvent(c->stream, c->a_out_done[slot[i]], 0));
    if (!bulk) memset((void*)c->h_ready[slot[i]], 0, sizeof(int) * (size_t)frames * c->S);
    readies[i] = c->d_ready[slot[i]];
  }
  int r = group_launch(ctxs, n, devp.data(), sy.data(), suv.data(), kinds, frames, recs.data(), true, who,
                       bulk ? nullptr : readies.data(), bulk ? 0 : 1);
  if (r) return r;
  // each context's records out on its copy-out stream once the launch is done (its stream waits
  // for the launch); its pending call copies them again if it has to be re-run
  for (int i = 0; i < n; i++) {
    rg_ctx* c = ctxs[i];
    const int sl = slot[i];
    c->a_slot = sl ^ 1;
    c->a_seq[sl] = bulk ? -1 : 1;  // bulk: no flag is ever set; a fetch waits for the launch's end
    c->a_frames[sl] = frames;
    c->a_compact[sl] = false;
    CK(cudaEventRecord(c->a_kern_done[sl], c->stream));
    const size_t bytes = sizeof(rg_mb_out) * c->n_mb * c->S * frames;
    CK(cudaStreamWaitEvent(c->a_out, c->a_kern_done[sl], 0));
    if (bulk) CK(cudaMemcpyAsync(outs[i], c->a_recs[sl], bytes, cudaMemcpyDeviceToHost, c->a_out));
    CK(cudaEventRecord(c->a_out_done[sl], c->a_out));
    c->a_out_ptr[sl] = outs[i];
    rg_ctx::Pending& p = c->pend[(c->pend_head + c->pend_count - 1) & 1];  // the call just queued
    p.out = outs[i];
    p.out_bytes = bytes;
  }
  return RG_OK;
}

int rg_analyse_gops_group_async(rg_ctx* const* ctxs, int32_t n, const uint8_t* const* const* planes,
                                const size_t* stride_y, const size_t* stride_uv, const int32_t* const* kinds,
                                int32_t frames, rg_mb_out* const* outs) {
  return group_async(ctxs, n, planes, stride_y, stride_uv, kinds, frames, outs, true, "rg_analyse_gops_group_async");
}

int rg_analyse_gops_group_stream(rg_ctx* const* ctxs, int32_t n, const uint8_t* const* const* planes,
                                 const size_t* stride_y, const size_t* stride_uv, const int32_t* const* kinds,
                                 int32_t frames, rg_mb_out* const* outs) {
  return group_async(ctxs, n, planes, stride_y, stride_uv, kinds, frames, outs, false, "rg_analyse_gops_group_stream");
}

int rg_group_graph_counts(const rg_ctx* c, int64_t* captures, int64_t* launches) {
  if (!c || !captures || !launches) return fail(RG_ERR_INVALID, "rg_group_graph_counts: null argument");
  *captures = c->g_graph_captures;
  *launches = c->g_graph_launches;
  return RG_OK;
}

int rg_copy_records_gops(rg_ctx* c, int32_t frames, rg_mb_out* out) {
  if (!c || !out) return fail(RG_ERR_INVALID, "rg_copy_records_gops: null argument");
  if (frames < 1 || frames > c->max_frames) return fail(RG_ERR_INVALID, "rg_copy_records_gops: frames %d", frames);
  int r = rg_sync(c);  // completes (or re-runs) the pending call first
  if (r) return r;
  CK(cudaMemcpyAsync(out, c->recs, sizeof(rg_mb_out) * c->n_mb * c->S * frames, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return RG_OK;
}

int rg_set_pipeline_tuning(rg_ctx* c, const rg_pipeline_tuning* t) {
  if (!c) return fail(RG_ERR_INVALID, "rg_set_pipeline_tuning: null context");
  rg_pipeline_tuning zero{};
  if (!t) t = &zero;
  int lag = t->lag, seg = t->seg, grid = t->grid, timeout_ms = t->timeout_ms, deblock_sms = t->deblock_sms,
      intra_sms = t->intra_sms;
  if (lag < 0 || lag > 4096) return fail(RG_ERR_INVALID, "rg_set_pipeline_tuning: lag %d outside 0..4096", lag);
  if (seg < 0 || seg > c->fp.mb_w) return fail(RG_ERR_INVALID, "rg_set_pipeline_tuning: seg %d outside 0..%d", seg, c->fp.mb_w);
  if (grid < 0 || timeout_ms < 0 || deblock_sms < -1 || intra_sms < -1)
    return fail(RG_ERR_INVALID, "rg_set_pipeline_tuning: negative argument");
  CK(cudaStreamSynchronize(c->stream));
  int new_seg = seg > 0 ? seg : kDefaultSeg;
  if (new_seg > c->fp.mb_w) new_seg = c->fp.mb_w;
  size_t need = pipeline_task_count(c->fp, c->max_frames, new_seg);
  if (need > c->tasks_cap) {
    int2* p = nullptr;
    if (cudaMalloc((void**)&p, sizeof(int2) * need) != cudaSuccess)
      return fail(RG_ERR_OOM, "rg_set_pipeline_tuning: work list of %zu segments", need);
    cudaFree(c->d_tasks);
    c->d_tasks = p;
    c->tasks_cap = need;
  }
  c->lag = lag > 0 ? lag : kDefaultLag;
  c->reach_y = c->reach_x = 4;
  c->reach_low = 0;
  c->seg = new_seg;
  c->deblock_sms = deblock_sms < 0 ? 0 : (deblock_sms > 0 ? deblock_sms : default_deblock_sms(c->sms));
  c->intra_sms = intra_sms < 0 ? 0 : (intra_sms > 0 ? intra_sms : default_intra_sms(c->sms));
  c->tasks_frames = -1;
  if (grid > 0) c->grid = grid;
  else c->grid = pipeline_grid(c->cfg.device, c->form != RG_FORM_PLAIN);
  c->timeout_ns = timeout_ms > 0 ? (unsigned long long)timeout_ms * 1000000ull : 2000000000ull;
  return RG_OK;
}

int32_t rg_pipeline_lag(const rg_ctx* c) {
  if (!c) return fail(RG_ERR_INVALID, "rg_pipeline_lag: null context");
  return c->lag > 0 ? c->lag : auto_lag(c);
}

// One source picture (host planes pl[3]) into device staging d (Y | U | V, unpadded rows): one copy
// when the planes lie back to back with unpadded rows, else one per plane; 2-D copies only for
// padded rows (they run at a fraction of the link's rate).
static cudaError_t copy_picture_in(uint8_t* d, const uint8_t* const* pl, int w, int h, size_t stride_y,
                                   size_t stride_uv, cudaStream_t st) {
  const int cw = (w + 1) / 2, ch = (h + 1) / 2;
  const size_t ny = (size_t)w * h, nc = (size_t)cw * ch;
  cudaError_t e = cudaSuccess;
  if (stride_y == (size_t)w && stride_uv == (size_t)cw) {
    if (pl[1] == pl[0] + ny && pl[2] == pl[1] + nc) return cudaMemcpyAsync(d, pl[0], ny + 2 * nc, cudaMemcpyHostToDevice, st);
    if ((e = cudaMemcpyAsync(d, pl[0], ny, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(d + ny, pl[1], nc, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    return cudaMemcpyAsync(d + ny + nc, pl[2], nc, cudaMemcpyHostToDevice, st);
  }
  if ((e = cudaMemcpy2DAsync(d, w, pl[0], stride_y, w, h, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
  if ((e = cudaMemcpy2DAsync(d + ny, cw, pl[1], stride_uv, cw, ch, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
  return cudaMemcpy2DAsync(d + ny + nc, cw, pl[2], stride_uv, cw, ch, cudaMemcpyHostToDevice, st);
}

int rg_analyse_gops(rg_ctx* c, const uint8_t* const* planes, size_t stride_y, size_t stride_uv, const int32_t* kinds,
                    int32_t frames, rg_mb_out* out) {
  if (!c || !planes || !kinds) return fail(RG_ERR_INVALID, "rg_analyse_gops: null argument");
  if (frames < 1 || frames > c->max_frames) return fail(RG_ERR_INVALID, "rg_analyse_gops: frames %d", frames);
  int w = c->cfg.width, h = c->cfg.height, cw = (w + 1) / 2, ch = (h + 1) / 2;
  if (stride_y < (size_t)w || stride_uv < (size_t)cw) return fail(RG_ERR_INVALID, "rg_analyse_gops: stride too small");
  int S = c->S;
  std::vector<const uint8_t*> dev(3 * (size_t)S * frames);
  for (int f = 0; f < frames; f++)
    for (int s = 0; s < S; s++) {
      const uint8_t* const* pl = planes + (f * S + s) * 3;
      if (!pl[0] || !pl[1] || !pl[2]) return fail(RG_ERR_INVALID, "rg_analyse_gops: picture %d stream %d null plane", f, s);
      uint8_t* d = c->srcs + c->src_bytes() * ((size_t)f * S + s);
      CK(copy_picture_in(d, pl, w, h, stride_y, stride_uv, c->stream));
      dev[(f * S + s) * 3] = d;
      dev[(f * S + s) * 3 + 1] = d + (size_t)w * h;
      dev[(f * S + s) * 3 + 2] = d + (size_t)w * h + (size_t)cw * ch;
    }
  int r = rg_analyse_gops_device(c, dev.data(), w, cw, kinds, frames);
  if (r) return r;
  if (out) return rg_copy_records_gops(c, frames, out);
  return rg_sync(c);
}

// Picture lag of the work order when none is set: the smallest under which no wait for the
// reference picture goes to a later segment of the work list, for the reach the context's searches
// have shown (the bound of pipeline_task_list: lag >= max(seg, 2) * (4 + rows) + seg + columns + 3).
// With reach 4 x 4 (about 64 samples) this is the work list's own default. A search reaching
// further only waits longer; if a wait gives up, the call is re-run exactly.
static int auto_lag(const rg_ctx* c) {
  const int a = c->seg > 2 ? c->seg : 2;
  return a * (4 + c->reach_y) + c->seg + c->reach_x + 3;
}

constexpr int kReachLowRuns = 2;
// The derived reach never goes below one macroblock row and column beyond zero motion: a diamond
// of at most 16 one-sample steps from still candidates reaches 16 samples further, so the first
// launch with motion after still pictures stays within the order's bound instead of waiting for
// segments no warp has taken (and re-running after the wait limit).
constexpr int kReachFloor = 1;

// The reach a completed launch's reference waits saw (1 + macroblocks, 0 = none): a larger one
// raises the derived lag at once; a smaller one lowers it after kReachLowRuns launches in a row,
// to the largest of them (not below kReachFloor).
static void observe_reach(rg_ctx* c, int oy, int ox) {
  if (oy <= 0) return;  // no P picture waited for a reference picture in that launch
  oy--;
  ox = ox > 0 ? ox - 1 : 0;
  if (oy > c->reach_y || ox > c->reach_x) {
    c->reach_y = std::max(c->reach_y, oy);
    c->reach_x = std::max(c->reach_x, ox);
    c->reach_low = 0;
  } else if (oy == c->reach_y && ox == c->reach_x) {
    c->reach_low = 0;
  } else {
    c->low_y = c->reach_low ? std::max(c->low_y, oy) : oy;
    c->low_x = c->reach_low ? std::max(c->low_x, ox) : ox;
    if (++c->reach_low >= kReachLowRuns) {
      c->reach_y = std::max(c->low_y, kReachFloor);
      c->reach_x = std::max(c->low_x, kReachFloor);
      c->reach_low = 0;
    }
  }
}

// Resolves the oldest pending pipelined call: waits for its launch and, if a wait of it gave up
// (a search reaching further than the picture lag allows, or another warp failing), re-runs it,
// picture by picture, on the per-diagonal path, which has no waits: each picture wrote its own
// ring slot and the reference it started from is untouched, so the results are identical. The
// host copy of an asynchronous call's records is made again.
static int resolve_oldest(rg_ctx* c) {
  if (!c->pend_count) return RG_OK;
  rg_ctx::Pending& p = c->pend[c->pend_head];
  CK(cudaEventSynchronize(p.done));
  const int oy = ((volatile int*)p.h_reach)[0], ox = ((volatile int*)p.h_reach)[1];
  if (*(volatile int*)p.h_err == 0) {
    observe_reach(c, oy, ox);
    c->pend_head ^= 1;
    c->pend_count--;
    return RG_OK;
  }
  // a wait gave up: order the next launches for at least the reach it saw, and no less than 4
  c->reach_y = std::max(std::max(c->reach_y, oy - 1), 4);
  c->reach_x = std::max(std::max(c->reach_x, ox - 1), 4);
  c->reach_low = 0;
  CK(cudaStreamSynchronize(c->stream));
  if (c->a_out) CK(cudaStreamSynchronize(c->a_out));  // its copy of the failed records may still run
  int S = c->S;
  c->frames = p.start;
  for (int k = 0; k < c->pend_count; k++) {
    rg_ctx::Pending& q = c->pend[(c->pend_head + k) & 1];
    for (int f = 0; f < q.frames; f++) {
      int r = enqueue_wavefront(c, q.planes.data() + (size_t)f * S * 3, q.sy, q.suv, q.kinds.data() + (size_t)f * S,
                                q.rec + (size_t)f * S * c->n_mb, -1,
                                q.hints.empty() ? nullptr : q.hints.data() + (size_t)f * S);
      if (r) return r;
    }
    CK(cudaStreamSynchronize(c->stream));
    if (q.out) CK(cudaMemcpy(q.out, q.rec, q.out_bytes, cudaMemcpyDeviceToHost));
    *(volatile int*)q.h_err = 0;
  }
  c->pend_head = 0;
  c->pend_count = 0;
  return RG_OK;
}

// Waits for the queued work of the context, resolving every pending pipelined call. wait_out: also
// wait for the copy-out stream of asynchronous calls.
static int resolve_pending(rg_ctx* c, bool wait_out) {
  while (c->pend_count) {
    int r = resolve_oldest(c);
    if (r) return r;
  }
  CK(cudaStreamSynchronize(c->stream));
  if (wait_out && c->a_out) CK(cudaStreamSynchronize(c->a_out));
  return RG_OK;
}

int rg_set_analysis_form(rg_ctx* c, int32_t form, int32_t search_range) {
  if (!c) return fail(RG_ERR_INVALID, "rg_set_analysis_form: null context");
  if (form != RG_FORM_PLAIN && form != RG_FORM_FULLSEARCH && form != RG_FORM_LEARNED)
    return fail(RG_ERR_INVALID, "rg_set_analysis_form: form %d", form);
  if (form != RG_FORM_PLAIN && c->cfg.profile == RG_PROFILE_BASELINE)
    return fail(RG_ERR_UNSUPPORTED, "rg_set_analysis_form: the search forms code partitions with CABAC (Main / High)");
  if (form != RG_FORM_PLAIN && (search_range < 1 || search_range > kMaxSearchRange))
    return fail(RG_ERR_INVALID, "rg_set_analysis_form: search range %d outside 1..%d", search_range, kMaxSearchRange);
  int r = resolve_pending(c, true);
  if (r) return r;
  if (form != RG_FORM_PLAIN && !c->mv4s) {
    size_t n = sizeof(MbMv4) * c->n_mb * c->nslots * c->S;
    if (cudaMalloc((void**)&c->mv4s, n) != cudaSuccess) return fail(RG_ERR_OOM, "rg_set_analysis_form: %zu bytes", n);
    CK(cudaMemset(c->mv4s, 0, n));
  }
  bool default_grid = c->grid == pipeline_grid(c->cfg.device, c->form != RG_FORM_PLAIN);
  c->form = form;
  if (form != RG_FORM_PLAIN) c->search_range = search_range;
  if (default_grid) c->grid = pipeline_grid(c->cfg.device, form != RG_FORM_PLAIN);
  c->hints.clear();
  return RG_OK;
}

int rg_set_hint_net(rg_ctx* c, rg_net* net) {
  if (!c) return fail(RG_ERR_INVALID, "rg_set_hint_net: null context");
  int r = resolve_pending(c, true);
  if (r) return r;
  if (net && !c->d_hints) {
    size_t n = sizeof(rg_mb_hint) * 2 * (size_t)c->max_frames * c->S * c->n_mb;
    if (cudaMalloc((void**)&c->d_hints, n) != cudaSuccess) return fail(RG_ERR_OOM, "rg_set_hint_net: %zu bytes", n);
  }
  c->net = net;
  return RG_OK;
}

int rg_set_search_tuning(rg_ctx* c, const int32_t* type_bits, int32_t walk) {
  if (!c) return fail(RG_ERR_INVALID, "rg_set_search_tuning: null context");
  if (walk < 0 || walk > 64) return fail(RG_ERR_INVALID, "rg_set_search_tuning: walk %d outside 0..64", walk);
  for (int k = 0; k < 4; k++) {
    int b = type_bits ? type_bits[k] : kDefaultTypeBits[k];
    if (b < 0 || b > 4096) return fail(RG_ERR_INVALID, "rg_set_search_tuning: type bits %d", b);
  }
  int r = resolve_pending(c, true);
  if (r) return r;
  for (int k = 0; k < 4; k++) c->type_bits[k] = (uint16_t)(type_bits ? type_bits[k] : kDefaultTypeBits[k]);
  c->walk = walk;
  return RG_OK;
}

int rg_set_hints(rg_ctx* c, const rg_mb_hint* const* dev_hints, int32_t count) {
  if (!c) return fail(RG_ERR_INVALID, "rg_set_hints: null context");
  if (count < 0 || (count > 0 && !dev_hints)) return fail(RG_ERR_INVALID, "rg_set_hints: %d hint arrays", count);
  if (c->form != RG_FORM_LEARNED) return fail(RG_ERR_STATE, "rg_set_hints: the context is not in the learned form");
  c->hints.assign(dev_hints, dev_hints + count);
  return RG_OK;
}

int rg_sync(rg_ctx* c) {
  if (!c) return fail(RG_ERR_INVALID, "rg_sync: null context");
  return resolve_pending(c, true);
}

// rg_analyse_gops_async (bulk: the records copied out after the launch) and rg_analyse_gops_stream
// (the host fetches each picture's records once the launch flags them final).
// The asynchronous calls' two slots of staging, records and events, allocated on first use.
static int async_setup(rg_ctx* c) {
  const int S = c->S;
  if (!c->a_in) {
    size_t nsrc = c->src_bytes() * S * c->max_frames, nrec = sizeof(rg_mb_out) * c->n_mb * S * c->max_frames;
    for (int i = 0; i < 2; i++) {
      if (cudaMalloc((void**)&c->a_srcs[i], nsrc) != cudaSuccess || cudaMalloc((void**)&c->a_recs[i], nrec) != cudaSuccess)
        return fail(RG_ERR_OOM, "rg_analyse_gops_async: staging of %zu + %zu bytes", nsrc, nrec);
      CK(cudaMemset(c->a_recs[i], 0, nrec));
      for (cudaEvent_t* e : {&c->a_in_done[i], &c->a_kern_done[i], &c->a_out_done[i]})
        CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
      size_t nflags = sizeof(int) * S * c->max_frames;
      if (cudaHostAlloc((void**)&c->h_ready[i], nflags, cudaHostAllocMapped) != cudaSuccess)
        return fail(RG_ERR_OOM, "rg_analyse_gops_async: %zu bytes of mapped host memory", nflags);
      memset(c->h_ready[i], 0, nflags);
      CK(cudaHostGetDevicePointer((void**)&c->d_ready[i], c->h_ready[i], 0));
    }
    CK(cudaStreamCreateWithFlags(&c->a_out, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->a_in, cudaStreamNonBlocking));
  }
  return RG_OK;
}

// Checks a call's host sources and copies them into slot `slot`'s staging on the copy-in stream, once
// the launch that last read that staging is done; dev receives the device planes.
static int async_copy_in(rg_ctx* c, int slot, const uint8_t* const* planes, size_t stride_y, size_t stride_uv,
                         int32_t frames, std::vector<const uint8_t*>& dev, const char* who) {
  if (frames < 1 || frames > c->max_frames) return fail(RG_ERR_INVALID, "%s: frames %d", who, frames);
  int w = c->cfg.width, h = c->cfg.height, cw = (w + 1) / 2, ch = (h + 1) / 2;
  if (stride_y < (size_t)w || stride_uv < (size_t)cw) return fail(RG_ERR_INVALID, "%s: stride too small", who);
  int S = c->S;
  for (int i = 0; i < 3 * S * frames; i++)
    if (!planes[i]) return fail(RG_ERR_INVALID, "%s: picture %d stream %d null plane", who, i / 3 / S, (i / 3) % S);
  int r = async_setup(c);
  if (r) return r;
  CK(cudaStreamWaitEvent(c->a_in, c->a_kern_done[slot], 0));
  dev.assign(3 * (size_t)S * frames, nullptr);
  const size_t ny = (size_t)w * h, nc = (size_t)cw * ch;
  for (int i = 0; i < S * frames; i++) {
    const uint8_t* const* pl = planes + 3 * i;
    uint8_t* d = c->a_srcs[slot] + c->src_bytes() * i;
    CK(copy_picture_in(d, pl, w, h, stride_y, stride_uv, c->a_in));
    dev[3 * i] = d;
    dev[3 * i + 1] = d + ny;
    dev[3 * i + 2] = d + ny + nc;
  }
  CK(cudaEventRecord(c->a_in_done[slot], c->a_in));
  return RG_OK;
}

static int async_gops(rg_ctx* c, const uint8_t* const* planes, size_t stride_y, size_t stride_uv, const int32_t* kinds,
                      int32_t frames, rg_mb_out* out, bool bulk) {
  if (!c || !planes || !kinds || !out) return fail(RG_ERR_INVALID, "rg_analyse_gops_async: null argument");
  int w = c->cfg.width, cw = (w + 1) / 2;
  int S = c->S;
  if (frames < 1 || frames > c->max_frames) return fail(RG_ERR_INVALID, "rg_analyse_gops_async: frames %d", frames);
  int slot = c->a_slot;
  std::vector<const uint8_t*> dev;
  {
    int r0 = async_copy_in(c, slot, planes, stride_y, stride_uv, frames, dev, "rg_analyse_gops_async");
    if (r0) return r0;
  }
  c->a_slot ^= 1;
  // The previous launch is resolved (waited for, re-run if it failed) before the launch stream is
  // told to wait for this copy: resolving ends with a synchronisation of that stream, which would
  // otherwise wait for the copy too and hold the caller for its whole duration.
  int r = resolve_pending(c, false);
  if (r) return r;
  // the launch waits for its sources and for the copy-out of this slot's previous records
  CK(cudaStreamWaitEvent(c->stream, c->a_in_done[slot], 0));
  CK(cudaStreamWaitEvent(c->stream, c->a_out_done[slot], 0));
  int seq = ++c->launch_seq;
  // compact records: this slot's mapped buffers (re)allocated to the current slot size; the slot's
  // previous call was resolved above, and its pictures were fetched before this call (the
  // two-calls rule), so nothing reads them any more
  CompactOut co{};
  c->a_compact[slot] = false;
  if (!bulk && c->compact_words > 0) {
    const int row = (c->fp.mb_w * c->compact_words + 3) & ~3;  // whole 16-byte stores
    const size_t rows = (size_t)S * c->max_frames * c->fp.mb_h;
    if (!c->h_cwords[slot] || c->c_row[slot] != row) {
      if (c->h_cwords[slot]) cudaFreeHost(c->h_cwords[slot]);
      if (c->h_cbytes[slot]) cudaFreeHost(c->h_cbytes[slot]);
      c->h_cwords[slot] = nullptr;
      c->h_cbytes[slot] = nullptr;
      if (cudaHostAlloc((void**)&c->h_cwords[slot], sizeof(uint32_t) * row * rows, cudaHostAllocMapped) != cudaSuccess ||
          cudaHostAlloc((void**)&c->h_cbytes[slot], sizeof(int) * rows, cudaHostAllocMapped) != cudaSuccess) {
        cudaGetLastError();
        return fail(RG_ERR_OOM, "rg_analyse_gops_stream: %zu bytes of mapped host memory for compact records",
                    sizeof(uint32_t) * row * rows);
      }
      CK(cudaHostGetDevicePointer((void**)&c->d_cwords[slot], c->h_cwords[slot], 0));
      CK(cudaHostGetDevicePointer((void**)&c->d_cbytes[slot], c->h_cbytes[slot], 0));
      c->c_row[slot] = row;
    }
    c->c_packed[slot].assign((size_t)S * frames, -1);
    co.words = c->d_cwords[slot];
    co.row_words = row;
    co.row_bytes = c->d_cbytes[slot];
    c->a_compact[slot] = true;
  }
  r = enqueue_gops(c, dev.data(), w, cw, kinds, frames, c->a_recs[slot], bulk ? nullptr : c->d_ready[slot], seq, true,
                   c->a_compact[slot] ? &co : nullptr);
  if (r) return r;
  c->a_seq[slot] = seq;
  c->a_frames[slot] = frames;
  CK(cudaEventRecord(c->a_kern_done[slot], c->stream));
  size_t bytes = sizeof(rg_mb_out) * c->n_mb * S * frames;
  CK(cudaStreamWaitEvent(c->a_out, c->a_kern_done[slot], 0));
  if (bulk) CK(cudaMemcpyAsync(out, c->a_recs[slot], bytes, cudaMemcpyDeviceToHost, c->a_out));
  CK(cudaEventRecord(c->a_out_done[slot], c->a_out));
  c->a_out_ptr[slot] = out;
  rg_ctx::Pending& p = c->pend[(c->pend_head + c->pend_count - 1) & 1];  // the call just queued
  p.out = out;
  p.out_bytes = bytes;
  return RG_OK;
}

int rg_analyse_gops_async(rg_ctx* c, const uint8_t* const* planes, size_t stride_y, size_t stride_uv,
                          const int32_t* kinds, int32_t frames, rg_mb_out* out) {
  return async_gops(c, planes, stride_y, stride_uv, kinds, frames, out, true);
}

int rg_analyse_gops_stream(rg_ctx* c, const uint8_t* const* planes, size_t stride_y, size_t stride_uv,
                           const int32_t* kinds, int32_t frames, rg_mb_out* out) {
  return async_gops(c, planes, stride_y, stride_uv, kinds, frames, out, false);
}

// Whether picture `picture` of the stream call writing into out is final: 1 yes (slot set), 0 not
// yet, 2 the launch ended without it, or a negative RG_ERR_*.
static int fetch_state(rg_ctx* c, const rg_mb_out* out, int32_t picture, const char* who, int& slot) {
  slot = c->a_out_ptr[0] == out ? 0 : (c->a_out_ptr[1] == out ? 1 : -1);
  if (slot < 0 || !c->h_ready[slot]) return fail(RG_ERR_STATE, "%s: no call in flight writes into out", who);
  if (picture < 0 || picture >= c->a_frames[slot] * c->S)
    return fail(RG_ERR_INVALID, "%s: picture %d of %d", who, picture, c->a_frames[slot] * c->S);
  volatile int* flag = c->h_ready[slot] + picture;
  if (*flag != c->a_seq[slot]) {
    // the launch flags a picture before it ends: after the end, an unflagged picture means a wait
    // gave up, and rg_analyse_gops_wait re-runs the call
    if (cudaEventQuery(c->a_kern_done[slot]) != cudaSuccess) return 0;
    if (*flag != c->a_seq[slot]) return 2;
  }
  std::atomic_thread_fence(std::memory_order_acquire);
  return 1;
}

// The picture's full records from the slot's device records into out.
static int fetch_dense(rg_ctx* c, rg_mb_out* out, int slot, int32_t picture) {
  CK(cudaSetDevice(c->cfg.device));
  thread_local cudaStream_t streams[16] = {};
  int dev = c->cfg.device & 15;
  if (!streams[dev]) CK(cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking));
  size_t n = (size_t)c->n_mb;
  CK(cudaMemcpyAsync(out + (size_t)picture * n, c->a_recs[slot] + (size_t)picture * n, sizeof(rg_mb_out) * n,
                     cudaMemcpyDeviceToHost, streams[dev]));
  CK(cudaStreamSynchronize(streams[dev]));
  return 1;
}

int rg_analyse_gops_fetch(rg_ctx* c, rg_mb_out* out, int32_t picture) {
  if (!c || !out) return fail(RG_ERR_INVALID, "rg_analyse_gops_fetch: null argument");
  int slot = -1;
  int st = fetch_state(c, out, picture, "rg_analyse_gops_fetch", slot);
  if (st != 1) return st;
  return fetch_dense(c, out, slot, picture);
}

int rg_analyse_gops_fetch_compact(rg_ctx* c, rg_mb_out* out, int32_t picture, const void** data, size_t* bytes) {
  if (!c || !out || !data || !bytes) return fail(RG_ERR_INVALID, "rg_analyse_gops_fetch_compact: null argument");
  *data = nullptr;
  *bytes = 0;
  int slot = -1;
  int st = fetch_state(c, out, picture, "rg_analyse_gops_fetch_compact", slot);
  if (st != 1) return st;
  if (c->a_compact[slot]) {
    // the picture's rows, each in its own slot, packed together in place on the first fetch
    int64_t& packed = c->c_packed[slot][picture];
    const int H = c->fp.mb_h, row = c->c_row[slot];
    uint32_t* base = c->h_cwords[slot] + (size_t)picture * H * row;
    if (packed == -1) {
      const volatile int* rb = c->h_cbytes[slot] + (size_t)picture * H;
      int64_t words = 0;
      for (int y = 0; y < H && packed == -1; y++)
        if (rb[y] < 0) packed = -2;  // a row did not fit its slot
      for (int y = 0; y < H && packed == -1; y++) {
        const int n = rb[y] / 4;
        if (y) memmove(base + words, base + (size_t)y * row, sizeof(uint32_t) * n);
        words += n;
      }
      if (packed == -1) packed = words * 4;
    }
    if (packed >= 0) {
      *data = base;
      *bytes = (size_t)packed;
      return 1;
    }
  }
  return fetch_dense(c, out, slot, picture);
}

int rg_set_record_compaction(rg_ctx* c, int32_t words_per_mb) {
  if (!c) return fail(RG_ERR_INVALID, "rg_set_record_compaction: null context");
  if (words_per_mb < 0 || (words_per_mb > 0 && words_per_mb < RG_COMPACT_MASK_WORDS) ||
      words_per_mb > RG_COMPACT_MASK_WORDS + (int)(sizeof(rg_mb_out) / 4))
    return fail(RG_ERR_INVALID, "rg_set_record_compaction: %d words per macroblock (0, or %d..%d)", words_per_mb,
                RG_COMPACT_MASK_WORDS, RG_COMPACT_MASK_WORDS + (int)(sizeof(rg_mb_out) / 4));
  if (c->pend_count) return fail(RG_ERR_STATE, "rg_set_record_compaction: calls in flight");
  c->compact_words = words_per_mb;
  return RG_OK;
}

int rg_analyse_gops_wait(rg_ctx* c, const rg_mb_out* out) {
  if (!c || !out) return fail(RG_ERR_INVALID, "rg_analyse_gops_wait: null argument");
  // resolve the pending calls up to the one copying into out
  int idx = -1;
  for (int k = 0; k < c->pend_count; k++)
    if (c->pend[(c->pend_head + k) & 1].out == out) idx = k;
  for (int k = 0; k <= idx && c->pend_count; k++) {
    int r = resolve_oldest(c);
    if (r) return r;
  }
  for (int i = 0; i < 2; i++)
    if (c->a_in && c->a_out_ptr[i] == out) CK(cudaEventSynchronize(c->a_out_done[i]));  // its copy out
  return RG_OK;
}

int rg_copy_records(rg_ctx* c, rg_mb_out* out) {
  if (!c || !out) return fail(RG_ERR_INVALID, "rg_copy_records: null argument");
  int r0 = rg_sync(c);
  if (r0) return r0;
  CK(cudaMemcpyAsync(out, c->recs, sizeof(rg_mb_out) * c->n_mb * c->S, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return RG_OK;
}

static int upload_planes(rg_ctx* c, int s, const uint8_t* y, const uint8_t* u, const uint8_t* v, size_t sy, size_t suv) {
  int w = c->cfg.width, h = c->cfg.height, cw = (w + 1) / 2, ch = (h + 1) / 2;
  uint8_t* d = c->srcs + c->src_bytes() * s;
  CK(cudaMemcpy2DAsync(d, w, y, sy, w, h, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpy2DAsync(d + (size_t)w * h, cw, u, suv, cw, ch, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpy2DAsync(d + (size_t)w * h + (size_t)cw * ch, cw, v, suv, cw, ch, cudaMemcpyHostToDevice, c->stream));
  return RG_OK;
}

int rg_analyse_batch(rg_ctx* c, const uint8_t* const* planes, size_t stride_y, size_t stride_uv, const int32_t* kinds,
                     rg_mb_out* out) {
  if (!c || !planes || !kinds) return fail(RG_ERR_INVALID, "rg_analyse_batch: null argument");
  {
    int r = resolve_pending(c, false);
    if (r) return r;
  }
  int w = c->cfg.width, cw = (w + 1) / 2;
  if (stride_y < (size_t)w || stride_uv < (size_t)cw) return fail(RG_ERR_INVALID, "rg_analyse_batch: stride too small");
  std::vector<const uint8_t*> dev(3 * c->S);
  for (int s = 0; s < c->S; s++) {
    if (!planes[3 * s] || !planes[3 * s + 1] || !planes[3 * s + 2])
      return fail(RG_ERR_INVALID, "rg_analyse_batch: stream %d null plane", s);
    int r = upload_planes(c, s, planes[3 * s], planes[3 * s + 1], planes[3 * s + 2], stride_y, stride_uv);
    if (r) return r;
    uint8_t* d = c->srcs + c->src_bytes() * s;
    dev[3 * s] = d;
    dev[3 * s + 1] = d + (size_t)w * c->cfg.height;
    dev[3 * s + 2] = d + (size_t)w * c->cfg.height + (size_t)cw * ((c->cfg.height + 1) / 2);
  }
  int r = rg_analyse_batch_device(c, dev.data(), w, cw, kinds);
  if (r) return r;
  if (out) return rg_copy_records(c, out);
  return rg_sync(c);
}

int rg_set_stream_qp(rg_ctx* c, int32_t stream, int32_t qp) {
  if (!c) return fail(RG_ERR_INVALID, "rg_set_stream_qp: null context");
  if (stream < 0 || stream >= c->S) return fail(RG_ERR_INVALID, "rg_set_stream_qp: stream %d of %d", stream, c->S);
  if (qp < 1 || qp > 51) return fail(RG_ERR_UNSUPPORTED, "rg_set_stream_qp: qp %d outside 1..51", qp);
  int r = resolve_pending(c, false);  // calls already queued keep the QP they were queued with
  if (r) return r;
  c->qps[stream] = stream_qp(qp);
  return RG_OK;
}

int rg_analyse_frame(rg_ctx* c, int32_t stream, const uint8_t* y, const uint8_t* u, const uint8_t* v, size_t stride_y,
                     size_t stride_uv, int32_t kind, rg_mb_out* out) {
  if (!c) return fail(RG_ERR_INVALID, "rg_analyse_frame: null context");
  if (stream < 0 || stream >= c->S) return fail(RG_ERR_INVALID, "rg_analyse_frame: stream %d of %d", stream, c->S);
  if (!y || !u || !v) return fail(RG_ERR_INVALID, "rg_analyse_frame: null plane");
  if (c->S == 1) {
    const uint8_t* planes[3] = {y, u, v};
    return rg_analyse_batch(c, planes, stride_y, stride_uv, &kind, out);
  }
  // one stream of a multi-stream context: its own wavefront launches
  int r = resolve_pending(c, false);
  if (r) return r;
  int w = c->cfg.width, cw = (w + 1) / 2;
  if (stride_y < (size_t)w || stride_uv < (size_t)cw) return fail(RG_ERR_INVALID, "rg_analyse_frame: stride too small");
  r = upload_planes(c, stream, y, u, v, stride_y, stride_uv);
  if (r) return r;
  uint8_t* d = c->srcs + c->src_bytes() * stream;
  const uint8_t* dev[3] = {d, d + (size_t)w * c->cfg.height, d + (size_t)w * c->cfg.height + (size_t)cw * ((c->cfg.height + 1) / 2)};
  std::vector<const rg_mb_hint*> hv;
  r = take_hints(c, 1, "rg_analyse_frame", hv);
  if (r) return r;
  r = enqueue_wavefront(c, dev, w, cw, &kind, nullptr, stream, hv.empty() ? nullptr : hv.data());
  if (r) return r;
  if (out) {
    CK(cudaMemcpyAsync(out, c->recs + (size_t)stream * c->n_mb, sizeof(rg_mb_out) * c->n_mb, cudaMemcpyDeviceToHost,
                       c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return RG_OK;
}

int rg_get_recon(rg_ctx* c, int32_t s, uint8_t* y, uint8_t* u, uint8_t* v, size_t sy, size_t suv) {
  if (!c || !y || !u || !v) return fail(RG_ERR_INVALID, "rg_get_recon: null argument");
  if (s < 0 || s >= c->S) return fail(RG_ERR_INVALID, "rg_get_recon: stream %d", s);
  if (c->frames[s] == 0) return fail(RG_ERR_STATE, "rg_get_recon: stream %d has no frame", s);
  int par = (c->frames[s] - 1) % c->nslots;
  int w = c->cfg.width, h = c->cfg.height, cw = (w + 1) / 2, ch = (h + 1) / 2;
  CK(cudaMemcpy2DAsync(y, sy, c->pic_plane(s, par, 0), c->fp.stride_y, w, h, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpy2DAsync(u, suv, c->pic_plane(s, par, 1), c->fp.stride_c, cw, ch, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpy2DAsync(v, suv, c->pic_plane(s, par, 2), c->fp.stride_c, cw, ch, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return RG_OK;
}

// Coded-size reconstruction after deblocking (for parity tests against the oracle).
int rg_get_recon_coded(rg_ctx* c, int32_t s, uint8_t* y, uint8_t* u, uint8_t* v) {
  if (!c || !y || !u || !v) return fail(RG_ERR_INVALID, "rg_get_recon_coded: null argument");
  if (s < 0 || s >= c->S || c->frames[s] == 0) return fail(RG_ERR_STATE, "rg_get_recon_coded: stream %d", s);
  int par = (c->frames[s] - 1) % c->nslots;
  int w = c->fp.mb_w * 16, h = c->fp.mb_h * 16;
  CK(cudaMemcpy2DAsync(y, w, c->pic_plane(s, par, 0), c->fp.stride_y, w, h, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpy2DAsync(u, w / 2, c->pic_plane(s, par, 1), c->fp.stride_c, w / 2, h / 2, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpy2DAsync(v, w / 2, c->pic_plane(s, par, 2), c->fp.stride_c, w / 2, h / 2, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return RG_OK;
}

int rg_get_recon_unfiltered(rg_ctx* c, int32_t s, uint8_t* y, uint8_t* u, uint8_t* v) {
  if (!c || !y || !u || !v) return fail(RG_ERR_INVALID, "rg_get_recon_unfiltered: null argument");
  if (!c->unf || !c->keep_unfiltered) return fail(RG_ERR_STATE, "rg_get_recon_unfiltered: enable rg_keep_unfiltered first");
  if (s < 0 || s >= c->S || c->frames[s] == 0) return fail(RG_ERR_STATE, "rg_get_recon_unfiltered: stream %d", s);
  size_t ny = (size_t)c->fp.mb_w * c->fp.mb_h * 256, nc = ny / 4;
  uint8_t* b = c->unf + c->unf_bytes() * s;
  CK(cudaMemcpyAsync(y, b, ny, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(u, b + ny, nc, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(v, b + ny + nc, nc, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return RG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Metrics: SSIM of Y/U/V, 5-scale MS-SSIM of Y and PSNR (evaluate_frame_quality,
// crates/ragdoll-pix/src/metrics.rs:328).
namespace {

const double kMsWeights[5] = {0.0448, 0.2856, 0.3001, 0.2363, 0.1333};

struct PlanePair {
  const uint8_t* a;
  long sa;
  const uint8_t* b;
  long sb;
  int w, h;
};

// Evaluates SSIM of each pair, MS-SSIM of pairs with want_ms, SSE of all, on stream st.
int device_metrics(const std::vector<PlanePair>& pairs, const std::vector<bool>& want_ms, cudaStream_t st,
                   std::vector<double>& ssim, std::vector<double>& ms, std::vector<unsigned long long>& sse) {
  int n = (int)pairs.size();
  // pyramid levels of the MS-SSIM pairs
  std::vector<SsimJob> jobs;
  std::vector<DecimateJob> djobs_per_level[4];
  std::vector<int> level_count(n, 1);
  size_t rows_total = 0, pyr_total = 0;
  for (int i = 0; i < n; i++) {
    rows_total += pairs[i].h / 4 + 1;
    if (want_ms[i]) {
      int w = pairs[i].w, h = pairs[i].h;
      for (int l = 1; l < 5; l++) {
        w >>= 1; h >>= 1;
        if (w < 8 || h < 8) break;
        pyr_total += 2 * (size_t)w * h;
        rows_total += h / 4 + 1;
        level_count[i]++;
      }
    }
  }
  float* rows = nullptr;
  double* outs = nullptr;
  unsigned long long* sses = nullptr;
  uint8_t* pyr = nullptr;
  SsimJob* d_jobs = nullptr;
  DecimateJob* d_djobs = nullptr;
  int total_jobs = 0;
  for (int i = 0; i < n; i++) total_jobs += want_ms[i] ? level_count[i] : 1;
  auto cleanup = [&]() {
    cudaFree(rows); cudaFree(outs); cudaFree(sses); cudaFree(pyr); cudaFree(d_jobs); cudaFree(d_djobs);
  };
  if (cudaMalloc(&rows, rows_total * sizeof(float) + 16) != cudaSuccess ||
      cudaMalloc(&outs, total_jobs * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&sses, n * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&pyr, pyr_total + 16) != cudaSuccess || cudaMalloc(&d_jobs, total_jobs * sizeof(SsimJob)) != cudaSuccess ||
      cudaMalloc(&d_djobs, (4 * n + 1) * sizeof(DecimateJob)) != cudaSuccess) {
    cleanup();
    return fail(RG_ERR_OOM, "metrics: device allocation failed");
  }
  cudaMemsetAsync(sses, 0, n * sizeof(unsigned long long), st);
  size_t rofs = 0, pofs = 0;
  int maxw = 0, maxh = 0;
  std::vector<int> job_of(n * 5, -1);
  // the n full-size planes first (jobs 0..n-1: the SSE launch reads those), pyramid levels after
  for (int i = 0; i < n; i++) {
    const PlanePair& p = pairs[i];
    SsimJob j{p.a, p.b, p.sa, p.sb, p.w, p.h, rows + rofs, outs + jobs.size(), sses + i};
    rofs += p.h / 4 + 1;
    job_of[i * 5] = (int)jobs.size();
    jobs.push_back(j);
    maxw = std::max(maxw, p.w);
    maxh = std::max(maxh, p.h);
  }
  for (int i = 0; i < n; i++) {
    const PlanePair& p = pairs[i];
    if (want_ms[i]) {
      const uint8_t* sa = p.a;
      const uint8_t* sb = p.b;
      long ssa = p.sa, ssb = p.sb;
      int w = p.w, h = p.h;
      for (int l = 1; l < level_count[i]; l++) {
        int nw = w >> 1, nh = h >> 1;
        uint8_t* da = pyr + pofs;
        uint8_t* db = da + (size_t)nw * nh;
        pofs += 2 * (size_t)nw * nh;
        djobs_per_level[l - 1].push_back(DecimateJob{sa, sb, ssa, ssb, w, h, da, db});
        SsimJob jl{da, db, nw, nw, nw, nh, rows + rofs, outs + jobs.size(), nullptr};
        rofs += nh / 4 + 1;
        job_of[i * 5 + l] = (int)jobs.size();
        jobs.push_back(jl);
        sa = da; sb = db; ssa = nw; ssb = nw; w = nw; h = nh;
      }
    }
  }
  // decimation levels in order, then every SSIM job in one launch
  std::vector<DecimateJob> all_d;
  std::vector<int> dofs;
  for (int l = 0; l < 4; l++) {
    dofs.push_back((int)all_d.size());
    all_d.insert(all_d.end(), djobs_per_level[l].begin(), djobs_per_level[l].end());
  }
  if (!all_d.empty()) CK(cudaMemcpyAsync(d_djobs, all_d.data(), all_d.size() * sizeof(DecimateJob), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_jobs, jobs.data(), jobs.size() * sizeof(SsimJob), cudaMemcpyHostToDevice, st));
  for (int l = 0; l < 4; l++) {
    int cnt = (int)djobs_per_level[l].size();
    if (!cnt) continue;
    int maxpix = 0;
    for (auto& d : djobs_per_level[l]) maxpix = std::max(maxpix, (d.src_w >> 1) * (d.src_h >> 1));
    launch_decimate(d_djobs + dofs[l], cnt, maxpix, st);
  }
  launch_ssim(d_jobs, (int)jobs.size(), maxw, maxh, st);
  launch_sse(d_jobs, n, st);
  std::vector<double> res(jobs.size());
  sse.assign(n, 0);
  CK(cudaMemcpyAsync(res.data(), outs, jobs.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(sse.data(), sses, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  cudaError_t e = cudaStreamSynchronize(st);
  cleanup();
  if (e != cudaSuccess) return fail(RG_ERR_CUDA, "metrics: %s", cudaGetErrorString(e));
  ssim.assign(n, 0.0);
  ms.assign(n, 0.0);
  for (int i = 0; i < n; i++) {
    ssim[i] = res[job_of[i * 5]];
    if (!want_ms[i]) continue;
    // ms_ssim_plane_u8 (crates/ragdoll-pix/src/metrics.rs:154)
    double s0 = std::min(1.0, std::max(0.0, ssim[i]));
    if (std::fabs(1.0 - s0) < 1e-12 || (pairs[i].w >> 1) < 8 || (pairs[i].h >> 1) < 8) { ms[i] = s0; continue; }
    double scores[5] = {s0, s0, s0, s0, s0};
    int active = level_count[i];
    for (int l = 1; l < active; l++) scores[l] = std::min(1.0, std::max(0.0, res[job_of[i * 5 + l]]));
    double wsum = 0.0;
    for (int l = 0; l < active; l++) wsum += kMsWeights[l];
    double prod = 1.0;
    for (int l = 0; l < active; l++) prod *= std::pow(std::max(scores[l], 1e-9), kMsWeights[l] / wsum);
    ms[i] = std::min(1.0, std::max(0.0, prod));
  }
  return RG_OK;
}

double psnr_of(unsigned long long sse, long n) {
  if (sse == 0) return INFINITY;
  double mse = (double)sse / (double)n;
  return 10.0 * std::log10((255.0 * 255.0) / mse);
}

// VMAF-Lite of one plane pair on the device (prev may be null); scores via vmaf_lite_score.
int device_vmaf(const uint8_t* a, long sa, const uint8_t* b, long sb, const uint8_t* prev, long sp, int w, int h,
                cudaStream_t st, double* score) {
  int bw = w >> 2, bh = h >> 2;
  if (bw == 0 || bh == 0) {
    *score = 100.0;
    return RG_OK;
  }
  double* buf = nullptr;
  VmafJob* d_job = nullptr;
  if (cudaMalloc(&buf, (3 * (size_t)bh + 3) * sizeof(double) + sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&d_job, sizeof(VmafJob)) != cudaSuccess) {
    cudaFree(buf);
    return fail(RG_ERR_OOM, "vmaf: device allocation failed");
  }
  unsigned long long* sad = (unsigned long long*)(buf + 3 * (size_t)bh + 3);
  VmafJob j{a, b, prev, sa, sb, sp, w, h, buf, buf + 3 * (size_t)bh, prev ? sad : nullptr};
  double res[3];
  unsigned long long sad_h = 0;
  cudaMemsetAsync(sad, 0, sizeof(unsigned long long), st);
  cudaMemcpyAsync(d_job, &j, sizeof j, cudaMemcpyHostToDevice, st);
  launch_vmaf(d_job, 1, h, st);
  cudaMemcpyAsync(res, buf + 3 * (size_t)bh, sizeof res, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&sad_h, sad, sizeof sad_h, cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  cudaFree(buf);
  cudaFree(d_job);
  if (e != cudaSuccess) return fail(RG_ERR_CUDA, "vmaf: %s", cudaGetErrorString(e));
  *score = vmaf_lite_score(res[0], res[1], res[2], (long)bw * bh, prev != nullptr, sad_h, (long)w * h);
  return RG_OK;
}

}  // namespace

extern "C" {

int rg_quality_frame(rg_ctx* c, int32_t s, const uint8_t* y, const uint8_t* u, const uint8_t* v, size_t sy, size_t suv,
                     rg_quality* q) {
  return rg_quality_frame_prev(c, s, y, u, v, sy, suv, nullptr, 0, q);
}

int rg_quality_frame_prev(rg_ctx* c, int32_t s, const uint8_t* y, const uint8_t* u, const uint8_t* v, size_t sy,
                          size_t suv, const uint8_t* prev_y, size_t stride_prev, rg_quality* q) {
  if (!c || !y || !u || !v || !q) return fail(RG_ERR_INVALID, "rg_quality_frame: null argument");
  if (s < 0 || s >= c->S || c->frames[s] == 0) return fail(RG_ERR_STATE, "rg_quality_frame: stream %d", s);
  int w = c->cfg.width, h = c->cfg.height, cw = (w + 1) / 2, ch = (h + 1) / 2;
  if (!c->m_src && cudaMalloc((void**)&c->m_src, c->src_bytes()) != cudaSuccess)
    return fail(RG_ERR_OOM, "rg_quality_frame: allocation failed");
  CK(cudaMemcpy2DAsync(c->m_src, w, y, sy, w, h, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpy2DAsync(c->m_src + (size_t)w * h, cw, u, suv, cw, ch, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpy2DAsync(c->m_src + (size_t)w * h + (size_t)cw * ch, cw, v, suv, cw, ch, cudaMemcpyHostToDevice, c->stream));
  int par = (c->frames[s] - 1) % c->nslots;
  std::vector<PlanePair> pairs = {
      {c->m_src, w, c->pic_plane(s, par, 0), c->fp.stride_y, w, h},
      {c->m_src + (size_t)w * h, cw, c->pic_plane(s, par, 1), c->fp.stride_c, cw, ch},
      {c->m_src + (size_t)w * h + (size_t)cw * ch, cw, c->pic_plane(s, par, 2), c->fp.stride_c, cw, ch}};
  std::vector<double> ss, ms;
  std::vector<unsigned long long> sse;
  int r = device_metrics(pairs, {true, false, false}, c->stream, ss, ms, sse);
  if (r) return r;
  q->ssim_y = ss[0];
  q->ssim_u = ss[1];
  q->ssim_v = ss[2];
  q->ssim_avg = (4.0 * ss[0] + ss[1] + ss[2]) / 6.0;
  q->ms_ssim = ms[0];
  q->psnr_y = psnr_of(sse[0], (long)w * h);
  q->psnr_u = psnr_of(sse[1], (long)cw * ch);
  q->psnr_v = psnr_of(sse[2], (long)cw * ch);
  // the rest of evaluate_frame_quality (crates/ragdoll-pix/src/metrics.rs:374-392)
  q->psnr_avg = psnr_of(sse[0] + sse[1] + sse[2], (long)w * h + 2L * cw * ch);
  if (std::isinf(q->psnr_y) && std::isinf(q->psnr_u) && std::isinf(q->psnr_v))
    q->psnr_yuv_611 = INFINITY;
  else
    q->psnr_yuv_611 = (6.0 * std::fmin(q->psnr_y, 100.0) + std::fmin(q->psnr_u, 100.0) + std::fmin(q->psnr_v, 100.0)) / 8.0;
  q->ssim_db = q->ssim_avg >= 1.0 ? INFINITY : -10.0 * std::log10(1.0 - q->ssim_avg);
  uint8_t* d_prev = nullptr;
  if (prev_y) {
    if (cudaMalloc(&d_prev, (size_t)w * h) != cudaSuccess) return fail(RG_ERR_OOM, "rg_quality_frame: allocation failed");
    CK(cudaMemcpy2DAsync(d_prev, w, prev_y, stride_prev, w, h, cudaMemcpyHostToDevice, c->stream));
  }
  r = device_vmaf(c->m_src, w, c->pic_plane(s, par, 0), c->fp.stride_y, d_prev, w, w, h, c->stream, &q->vmaf_lite);
  cudaFree(d_prev);
  return r;
}

int rg_vmaf_lite_plane(int32_t device, const uint8_t* ref, size_t stride_ref, const uint8_t* dist, size_t stride_dist,
                       int32_t width, int32_t height, const uint8_t* prev, size_t stride_prev, double* score) {
  if (!ref || !dist || !score || width < 1 || height < 1) return fail(RG_ERR_INVALID, "rg_vmaf_lite_plane: bad argument");
  CK(cudaSetDevice(device));
  size_t n = (size_t)width * height;
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, 3 * n) != cudaSuccess) return fail(RG_ERR_OOM, "rg_vmaf_lite_plane: allocation failed");
  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
    cudaFree(d);
    return fail(RG_ERR_CUDA, "rg_vmaf_lite_plane: stream creation failed");
  }
  int r = RG_OK;
  if (cudaMemcpy2DAsync(d, width, ref, stride_ref, width, height, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpy2DAsync(d + n, width, dist, stride_dist, width, height, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      (prev && cudaMemcpy2DAsync(d + 2 * n, width, prev, stride_prev, width, height, cudaMemcpyHostToDevice, st) != cudaSuccess)) {
    r = fail(RG_ERR_CUDA, "rg_vmaf_lite_plane: copy failed");
  } else {
    r = device_vmaf(d, width, d + n, width, prev ? d + 2 * n : nullptr, width, width, height, st, score);
  }
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  cudaFree(d);
  return r;
}

int rg_ssim_plane(int32_t device, const uint8_t* a, size_t stride_a, const uint8_t* b, size_t stride_b, int32_t width,
                  int32_t height, double* ssim, double* ms_ssim) {
  if (!a || !b || width < 1 || height < 1) return fail(RG_ERR_INVALID, "rg_ssim_plane: bad argument");
  if (width < 8 || height < 8) return fail(RG_ERR_INVALID, "rg_ssim_plane: plane smaller than one 8x8 window");
  CK(cudaSetDevice(device));
  size_t n = (size_t)width * height;
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, 2 * n) != cudaSuccess) return fail(RG_ERR_OOM, "rg_ssim_plane: allocation failed");
  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
    cudaFree(d);
    return fail(RG_ERR_CUDA, "rg_ssim_plane: stream creation failed");
  }
  int r = RG_OK;
  if (cudaMemcpy2DAsync(d, width, a, stride_a, width, height, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpy2DAsync(d + n, width, b, stride_b, width, height, cudaMemcpyHostToDevice, st) != cudaSuccess) {
    r = fail(RG_ERR_CUDA, "rg_ssim_plane: copy failed");
  } else {
    std::vector<double> ss, ms;
    std::vector<unsigned long long> sse;
    r = device_metrics({{d, width, d + n, width, width, height}}, {ms_ssim != nullptr}, st, ss, ms, sse);
    if (!r) {
      if (ssim) *ssim = ss[0];
      if (ms_ssim) *ms_ssim = ms[0];
    }
  }
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  cudaFree(d);
  return r;
}

int rg_ssim_batch_device(int32_t device, const uint8_t* const* dev_a, const uint8_t* const* dev_b, int32_t n,
                         int32_t width, int32_t height, size_t stride_a, size_t stride_b, double* ssim, double* ms_ssim,
                         void* cuda_stream) {
  if (!dev_a || !dev_b || n < 1 || (!ssim && !ms_ssim)) return fail(RG_ERR_INVALID, "rg_ssim_batch_device: bad argument");
  if (width < 8 || height < 8) return fail(RG_ERR_INVALID, "rg_ssim_batch_device: plane smaller than one 8x8 window");
  if (stride_a < (size_t)width || stride_b < (size_t)width) return fail(RG_ERR_INVALID, "rg_ssim_batch_device: stride");
  CK(cudaSetDevice(device));
  std::vector<PlanePair> pairs;
  for (int i = 0; i < n; i++) {
    if (!dev_a[i] || !dev_b[i]) return fail(RG_ERR_INVALID, "rg_ssim_batch_device: null plane %d", i);
    pairs.push_back({dev_a[i], (long)stride_a, dev_b[i], (long)stride_b, width, height});
  }
  std::vector<double> ss, ms;
  std::vector<unsigned long long> sse;
  int r = device_metrics(pairs, std::vector<bool>(n, ms_ssim != nullptr), (cudaStream_t)cuda_stream, ss, ms, sse);
  if (r) return r;
  for (int i = 0; i < n; i++) {
    if (ssim) ssim[i] = ss[i];
    if (ms_ssim) ms_ssim[i] = ms[i];
  }
  return RG_OK;
}

int64_t rg_pipeline_work_list(int32_t mb_w, int32_t mb_h, int32_t streams, int32_t frames, int32_t lag, int32_t seg,
                              int32_t split, const int32_t* kinds, int32_t* tasks, int64_t cap, int32_t* queues) {
  if (mb_w < 1 || mb_h < 1 || streams < 1 || frames < 1 || seg < 1 || lag < 0 || !tasks || !queues)
    return fail(RG_ERR_INVALID, "rg_pipeline_work_list: bad argument");
  FrameParams fp{};
  fp.mb_w = mb_w;
  fp.mb_h = mb_h;
  fp.n_streams = streams;
  size_t n = pipeline_task_count(fp, frames, seg);
  if ((int64_t)n > cap) return fail(RG_ERR_INVALID, "rg_pipeline_work_list: %zu segments exceed cap %lld", n, (long long)cap);
  std::vector<int2> list(n);
  int qb[kPipeQueues], qe[kPipeQueues];
  pipeline_task_list(fp, frames, lag, seg, split != 0, kinds, list.data(), qb, qe);
  for (size_t i = 0; i < n; i++) {
    tasks[2 * i] = list[i].x;
    tasks[2 * i + 1] = list[i].y;
  }
  for (int q = 0; q < kPipeQueues; q++) {
    queues[2 * q] = qb[q];
    queues[2 * q + 1] = qe[q];
  }
  return (int64_t)n;
}

}  // extern "C"
