// The encoder around the engine (host code): ragdoll's H264Encoder (crates/ragdoll-codec/src/h264.rs:2996,
// encode_frame :3153) and the wave loop of GopRingEncoder (crates/ragdoll-pipeline/src/lib.rs:543-597)
// with the macroblock loop on the GPU. A picture is analysed, reconstructed and deblocked by the
// engine, and its access unit is written on the host from the engine's records.
//
// Waves: rg_encoder_submit queues the copy in and the persistent launch of `frames` pictures of every
// stream behind the wave in flight, and returns; rg_encoder_collect writes the wave's pictures on a
// pool of threads, each as soon as the launch flags its records final (rg_analyse_gops_stream /
// _fetch), so the writing overlaps the launch. Every picture is one slice whose entropy coder
// starts afresh, and its frame_num / POC / idr_pic_id are known when it is submitted, so the
// pictures of one stream are written in parallel too. With two waves in flight the GPU goes from
// one launch to the next while the host writes.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "bitstream.h"

namespace {

int efail(int code, const char* fmt, ...) {
  char buf[256];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  rg::set_last_error(buf);
  return code;
}

// Fixed set of worker threads; run() hands out items 0..n-1 to them and to the calling thread.
class Pool {
 public:
  explicit Pool(int threads) {
    for (int i = 1; i < threads; i++) threads_.emplace_back([this, i] { loop(i); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> g(m_);
      stop_ = true;
    }
    go_.notify_all();
    for (auto& t : threads_) t.join();
  }
  int size() const { return (int)threads_.size() + 1; }
  void run(int items, const std::function<void(int item, int worker)>& fn) {
    {
      std::lock_guard<std::mutex> g(m_);
      fn_ = &fn;
      items_ = items;
      next_ = 0;
      busy_ = (int)threads_.size();
      gen_++;
    }
    go_.notify_all();
    work(0);
    std::unique_lock<std::mutex> g(m_);
    done_.wait(g, [this] { return busy_ == 0; });
    fn_ = nullptr;
  }

 private:
  void work(int worker) {
    for (int k; (k = next_.fetch_add(1)) < items_;) (*fn_)(k, worker);
  }
  void loop(int worker) {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> g(m_);
        go_.wait(g, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      work(worker);
      std::lock_guard<std::mutex> g(m_);
      if (--busy_ == 0) done_.notify_one();
    }
  }

  std::vector<std::thread> threads_;
  std::mutex m_;
  std::condition_variable go_, done_;
  const std::function<void(int, int)>* fn_ = nullptr;
  int items_ = 0, busy_ = 0;
  std::atomic<int> next_{0};
  uint64_t gen_ = 0;
  bool stop_ = false;
};

struct Wave {
  rg_mb_out* recs = nullptr;  // pinned, frames * streams * n_mb, picture-major
  int frames = 0;
  std::vector<int> qp;        // per stream
  bool written = false;       // its access units are in rg_encoder::aus, not yet handed out
  std::vector<uint8_t> idr;
  std::vector<uint32_t> since, idr_id;
  std::chrono::steady_clock::time_point submitted;
  std::vector<double> latency_ms;  // per picture: submit -> access unit written
  std::atomic<int64_t> record_bytes{0};  // records brought to the host (compact or full)
};


}  // namespace

struct rg_encoder {
  rg_config cfg{};
  int fps_num = 30, fps_den = 1, keyint = 30;
  rg_ctx* ctx = nullptr;
  int n_mb = 0;
  std::vector<int64_t> coded;    // per stream: pictures so far
  std::vector<uint32_t> idrs;    // per stream: IDR pictures so far
  std::vector<uint32_t> since;   // per stream: pictures since its last IDR
  std::vector<int> qp;           // per stream: fixed QP
  Wave waves[2];
  int head = 0, pending = 0;     // oldest wave in flight, waves in flight
  Pool* pool = nullptr;
  std::vector<rg_writer*> writers;               // one per pool thread
  std::vector<std::vector<uint8_t>> aus;         // access units of the wave being written
  std::vector<rg_mb_out> one;                    // records of rg_encode_frame
  std::vector<double> last_latency_ms;           // of the wave collected last
  int64_t last_record_bytes = 0;                 // of the wave collected last

  // Counters of the next picture of stream s, then advances them.
  void next_picture(int s, uint8_t& idr, uint32_t& since_idr, uint32_t& idr_id) {
    idr = coded[s] % keyint == 0;
    if (idr) since[s] = 0;
    since_idr = since[s];
    idr_id = idrs[s];
    if (idr) idrs[s]++;
    since[s]++;
    coded[s]++;
  }
};

extern "C" {

rg_encoder* rg_encoder_create(const rg_config* cfg, int32_t fps_num, int32_t fps_den, int32_t keyint, int32_t threads) {
  if (!cfg) {
    efail(RG_ERR_INVALID, "rg_encoder_create: null config");
    return nullptr;
  }
  if (keyint < 1 || fps_num < 1 || fps_den < 1) {
    efail(RG_ERR_INVALID, "rg_encoder_create: keyint %d, rate %d/%d", keyint, fps_num, fps_den);
    return nullptr;
  }
  rg_writer* probe = rg_writer_create(cfg, fps_num, fps_den);  // checks size, profile, QP, rate
  if (!probe) return nullptr;
  rg_writer_destroy(probe);
  rg_ctx* ctx = rg_create(cfg);
  if (!ctx) return nullptr;
  rg_encoder* e = new rg_encoder();
  e->cfg = *cfg;
  e->fps_num = fps_num;
  e->fps_den = fps_den;
  e->keyint = keyint;
  e->ctx = ctx;
  int mw = 0, mh = 0;
  rg_mb_dims(ctx, &mw, &mh);
  e->n_mb = mw * mh;
  int S = std::max(cfg->num_streams, 1);
  e->coded.assign(S, 0);
  e->idrs.assign(S, 0);
  e->since.assign(S, 0);
  e->qp.assign(S, cfg->qp);
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  e->pool = new Pool(threads);
  for (int i = 0; i < threads; i++) e->writers.push_back(rg_writer_create(cfg, fps_num, fps_den));
  return e;
}

void rg_encoder_destroy(rg_encoder* e) {
  if (!e) return;
  rg_sync(e->ctx);
  delete e->pool;
  for (rg_writer* w : e->writers) rg_writer_destroy(w);
  for (Wave& w : e->waves)
    if (w.recs) cudaFreeHost(w.recs);
  rg_destroy(e->ctx);
  delete e;
}

int32_t rg_encoder_threads(const rg_encoder* e) { return e ? e->pool->size() : 0; }

rg_ctx* rg_encoder_context(rg_encoder* e) { return e ? e->ctx : nullptr; }

int rg_encoder_set_stream_qp(rg_encoder* e, int32_t stream, int32_t qp) {
  if (!e) return efail(RG_ERR_INVALID, "rg_encoder_set_stream_qp: null encoder");
  if (stream < 0 || stream >= (int)e->coded.size()) return efail(RG_ERR_INVALID, "rg_encoder_set_stream_qp: stream %d", stream);
  if (e->coded[stream]) return efail(RG_ERR_STATE, "rg_encoder_set_stream_qp: stream %d has pictures already", stream);
  int r = rg_set_stream_qp(e->ctx, stream, qp);
  if (r) return r;
  e->qp[stream] = qp;
  return RG_OK;
}

int64_t rg_encode_frame(rg_encoder* e, int32_t stream, const uint8_t* y, const uint8_t* u, const uint8_t* v,
                        size_t stride_y, size_t stride_uv, uint8_t* out, size_t cap) {
  if (!e || !out) return efail(RG_ERR_INVALID, "rg_encode_frame: null argument");
  if (stream < 0 || stream >= (int)e->coded.size()) return efail(RG_ERR_INVALID, "rg_encode_frame: stream %d", stream);
  if (e->pending) return efail(RG_ERR_STATE, "rg_encode_frame: waves submitted and not collected");
  e->one.resize(e->n_mb);
  uint8_t idr;
  uint32_t since_idr, idr_id;
  const int64_t coded = e->coded[stream];
  const uint32_t idrs = e->idrs[stream], since = e->since[stream];
  e->next_picture(stream, idr, since_idr, idr_id);
  int r = rg_analyse_frame(e->ctx, stream, y, u, v, stride_y, stride_uv, idr ? RG_FRAME_IDR : RG_FRAME_P, e->one.data());
  std::vector<uint8_t> au;
  if (!r) r = rg::writer_access_unit(e->writers[0], e->one.data(), idr, since_idr, idr_id, e->qp[stream], au);
  if (r) {  // the picture was not coded: the stream's counters stay where they were
    e->coded[stream] = coded;
    e->idrs[stream] = idrs;
    e->since[stream] = since;
    return r;
  }
  if (au.size() > cap) return efail(RG_ERR_INVALID, "rg_encode_frame: %zu-byte access unit, %zu-byte buffer", au.size(), cap);
  memcpy(out, au.data(), au.size());
  return (int64_t)au.size();
}

}  // extern "C"

namespace {

// The next wave of encoder e (frames pictures of every stream): its pinned records, picture
// counters and kinds; the counters before it in `saved` (restored by rollback when the wave is
// not queued).
struct WaveStart {
  std::vector<int64_t> coded;
  std::vector<uint32_t> idrs, since;
  std::vector<int32_t> kinds;
};
int start_wave(rg_encoder* e, int32_t frames, const char* who, WaveStart& ws) {
  const int S = (int)e->coded.size();
  if (frames < 1 || frames > std::max(e->cfg.max_frames, 1))
    return efail(RG_ERR_INVALID, "%s: %d pictures per stream (max_frames %d)", who, frames, e->cfg.max_frames);
  if (e->pending == 2) return efail(RG_ERR_STATE, "%s: two waves in flight; collect one first", who);
  Wave& w = e->waves[(e->head + e->pending) & 1];
  if (!w.recs) {  // both waves' pinned records at once: pinning takes a while, and not mid-stream
    size_t bytes = sizeof(rg_mb_out) * e->n_mb * S * std::max(e->cfg.max_frames, 1);
    for (Wave& v : e->waves)
      if (!v.recs && cudaHostAlloc((void**)&v.recs, bytes, cudaHostAllocDefault) != cudaSuccess) {
        v.recs = nullptr;
        cudaGetLastError();
        return efail(RG_ERR_OOM, "%s: %zu bytes of pinned host memory", who, bytes);
      }
  }
  w.submitted = std::chrono::steady_clock::now();
  w.frames = frames;
  w.qp = e->qp;
  w.idr.resize((size_t)frames * S);
  w.since.resize((size_t)frames * S);
  w.idr_id.resize((size_t)frames * S);
  ws.kinds.assign((size_t)frames * S, 0);
  ws.coded = e->coded;
  ws.idrs = e->idrs;
  ws.since = e->since;
  for (int f = 0; f < frames; f++)
    for (int s = 0; s < S; s++) {
      const size_t i = (size_t)f * S + s;
      e->next_picture(s, w.idr[i], w.since[i], w.idr_id[i]);
      ws.kinds[i] = w.idr[i] ? RG_FRAME_IDR : RG_FRAME_P;
    }
  return RG_OK;
}
void rollback_wave(rg_encoder* e, const WaveStart& ws) {
  e->coded = ws.coded;
  e->idrs = ws.idrs;
  e->since = ws.since;
}

}  // namespace

extern "C" {

int rg_encoder_submit(rg_encoder* e, const uint8_t* const* planes, size_t stride_y, size_t stride_uv, int32_t frames) {
  if (!e || !planes) return efail(RG_ERR_INVALID, "rg_encoder_submit: null argument");
  WaveStart ws;
  int r = start_wave(e, frames, "rg_encoder_submit", ws);
  if (r) return r;
  Wave& w = e->waves[(e->head + e->pending) & 1];
  r = rg_analyse_gops_stream(e->ctx, planes, stride_y, stride_uv, ws.kinds.data(), frames, w.recs);
  if (r) {
    rollback_wave(e, ws);
    return r;
  }
  e->pending++;
  return RG_OK;
}

int rg_encoder_submit_group(rg_encoder* const* encs, int32_t n, const uint8_t* const* const* planes,
                            const size_t* stride_y, const size_t* stride_uv, int32_t frames) {
  if (!encs || !planes || !stride_y || !stride_uv || n < 1)
    return efail(RG_ERR_INVALID, "rg_encoder_submit_group: null argument or %d encoders", n);
  std::vector<WaveStart> ws(n);
  std::vector<rg_ctx*> ctxs(n);
  std::vector<const int32_t*> kinds(n);
  std::vector<rg_mb_out*> outs(n);
  for (int i = 0; i < n; i++) {
    rg_encoder* e = encs[i];
    int r = e ? start_wave(e, frames, "rg_encoder_submit_group", ws[i]) : efail(RG_ERR_INVALID, "rg_encoder_submit_group: null encoder %d", i);
    if (r) {
      for (int j = 0; j < i; j++) rollback_wave(encs[j], ws[j]);
      return r;
    }
    ctxs[i] = e->ctx;
    kinds[i] = ws[i].kinds.data();
    outs[i] = e->waves[(e->head + e->pending) & 1].recs;
  }
  int r = rg_analyse_gops_group_stream(ctxs.data(), n, planes, stride_y, stride_uv, kinds.data(), frames, outs.data());
  if (r) {
    for (int i = 0; i < n; i++) rollback_wave(encs[i], ws[i]);
    return r;
  }
  for (int i = 0; i < n; i++) encs[i]->pending++;
  return RG_OK;
}

int64_t rg_encoder_collect(rg_encoder* e, uint8_t* out, size_t cap, int64_t* sizes) {
  if (!e || !sizes) return efail(RG_ERR_INVALID, "rg_encoder_collect: null argument");
  if (!e->pending) return efail(RG_ERR_STATE, "rg_encoder_collect: no wave in flight");
  Wave& w = e->waves[e->head];
  const int S = (int)e->coded.size(), n = w.frames * S;
  if (!w.written) {
    // Pictures are written as the launch finishes them (picture-major order is roughly the order
    // they become final); one the launch could not finish is written after the call is re-run.
    if ((int)e->aus.size() < n) e->aus.resize(n);
    w.latency_ms.assign(n, 0.0);
    std::vector<uint8_t> later(n, 0);
    std::atomic<int> err{0};
    w.record_bytes = 0;
    // data null: the picture's full records in w.recs
    auto write = [&](int i, int worker, const void* data, size_t bytes) {
      int rc;
      if (data) {
        rg::RecordReader rd(data, bytes);
        rc = rg::writer_access_unit(e->writers[worker], rd, w.idr[i], w.since[i], w.idr_id[i], w.qp[i % S], e->aus[i]);
      } else {
        rc = rg::writer_access_unit(e->writers[worker], w.recs + (size_t)i * e->n_mb, w.idr[i], w.since[i],
                                    w.idr_id[i], w.qp[i % S], e->aus[i]);
        bytes = sizeof(rg_mb_out) * e->n_mb;
      }
      w.record_bytes += (int64_t)bytes;
      if (rc) err.store(rc);
      w.latency_ms[i] =
          std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w.submitted).count();
    };
    {  // a wave of rg_encoder_submit or of rg_encoder_submit_group alike
      e->pool->run(n, [&](int i, int worker) {
        const void* data = nullptr;
        size_t bytes = 0;
        for (int spins = 0;; spins++) {
          int st = rg_analyse_gops_fetch_compact(e->ctx, w.recs, i, &data, &bytes);
          if (st == 1) break;
          if (st != 0) {
            later[i] = 1;
            return;
          }
          std::this_thread::sleep_for(std::chrono::microseconds(spins < 64 ? 20 : 200));
        }
        write(i, worker, data, bytes);
      });
      int r = rg_analyse_gops_wait(e->ctx, w.recs);  // the launch's end; a re-run if a wait gave up
      if (r) return r;
      std::vector<int> rest;
      for (int i = 0; i < n; i++)
        if (later[i]) rest.push_back(i);
      if (!rest.empty()) e->pool->run((int)rest.size(), [&](int k, int worker) { write(rest[k], worker, nullptr, 0); });
    }
    if (err.load()) return err.load();
    w.written = true;
  }
  size_t total = 0;
  for (int i = 0; i < n; i++) {
    sizes[i] = (int64_t)e->aus[i].size();
    total += e->aus[i].size();
  }
  if (!out) return (int64_t)total;  // a size query: the wave stays to be collected
  if (cap < total) return efail(RG_ERR_INVALID, "rg_encoder_collect: %zu bytes of access units, %zu-byte buffer", total, cap);
  size_t at = 0;
  for (int i = 0; i < n; i++) {
    memcpy(out + at, e->aus[i].data(), e->aus[i].size());
    at += e->aus[i].size();
  }
  w.written = false;
  e->last_latency_ms = w.latency_ms;
  e->last_record_bytes = w.record_bytes.load();
  e->head ^= 1;
  e->pending--;
  return (int64_t)total;
}

int rg_encoder_set_form(rg_encoder* e, int32_t form, int32_t search_range, rg_net* net) {
  if (!e) return efail(RG_ERR_INVALID, "rg_encoder_set_form: null encoder");
  if (e->pending) return efail(RG_ERR_STATE, "rg_encoder_set_form: waves in flight");
  int r = rg_set_analysis_form(e->ctx, form, search_range);
  if (r) return r;
  return rg_set_hint_net(e->ctx, form == RG_FORM_LEARNED ? net : nullptr);
}

int rg_encoder_new_gops(rg_encoder* e) {
  if (!e) return efail(RG_ERR_INVALID, "rg_encoder_new_gops: null encoder");
  std::fill(e->coded.begin(), e->coded.end(), 0);
  std::fill(e->idrs.begin(), e->idrs.end(), 0u);
  std::fill(e->since.begin(), e->since.end(), 0u);
  return RG_OK;
}

int64_t rg_encoder_record_bytes(const rg_encoder* e) {
  if (!e) return efail(RG_ERR_INVALID, "rg_encoder_record_bytes: null encoder");
  return e->last_record_bytes;
}

int32_t rg_encoder_latencies(const rg_encoder* e, double* ms, int32_t n) {
  if (!e) return efail(RG_ERR_INVALID, "rg_encoder_latencies: null encoder");
  int32_t k = (int32_t)e->last_latency_ms.size();
  if (ms)
    for (int32_t i = 0; i < std::min(n, k); i++) ms[i] = e->last_latency_ms[i];
  return k;
}

}  // extern "C"
