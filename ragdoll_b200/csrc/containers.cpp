// Containers for the encoder's access units (host code, no GPU): fast-start MP4 and Matroska
// muxing of Annex-B access units, and demuxing of both back to Annex-B.
//
// MP4 (ISO/IEC 14496-12, AVC file format 14496-15) with the box set, order and field values of
// ragdoll's muxer (crates/ragdoll-format/src/mp4.rs:1746 Mp4Muxer::finish, :2138 ftyp, :2149
// moov, :2188 mvhd, :2206 trak, :2465 stsd): ftyp, moov (mvhd, trak (tkhd, mdia (mdhd, hdlr,
// minf (vmhd, dinf, stbl (stsd (avc1 (avcC, colr, pasp)), stts, stsc, stsz, stco | co64,
// stss))))), mdat; one sample per chunk; samples are 4-byte length-prefixed NAL units with the
// parameter sets and access unit delimiters moved out (crates/ragdoll-format/src/mpegts.rs:123)
// into the avcC record (mpegts.rs:273). The track timescale is 90 kHz and picture i starts at
// round(i * 90000 * fps_den / fps_num); the movie timescale is 1000.
//
// Matroska follows crates/ragdoll-format/src/mkv.rs:906 MkvMuxer::finish: EBML header, Segment
// (SeekHead with 8-byte positions, Info, Tracks, Clusters of SimpleBlocks started at every
// keyframe or 30 s, Cues for the clusters holding a keyframe), element sizes as minimal EBML
// variable-length integers (crates/ragdoll-core/src/bitstream.rs:996), timestamps in ms.
//
// Both muxers reproduce the reference's own files bit for bit given the same access units
// (qa/corpus/synth/clip_160x90_30fps.mp4, clip_320x180_25fps.mkv).
#include <algorithm>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/ragdoll_cuda.h"

namespace rg {
void set_last_error(const char* msg);
}

namespace {

int cfail(int code, const char* fmt, ...) {
  char buf[256];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  rg::set_last_error(buf);
  return code;
}

constexpr int64_t kTrackTimescale = 90000;

// Rounds a * b / c to the nearest integer, halves away from zero (a, b >= 0, c > 0).
int64_t rescale(int64_t a, int64_t b, int64_t c) {
  const __int128 n = (__int128)a * b;
  return (int64_t)((2 * n + c) / (2 * (__int128)c));
}

// --- Annex-B access units ----------------------------------------------------------------

struct Nal {
  const uint8_t* p;
  size_t n;
};

// NAL units of an Annex-B buffer (3- or 4-byte start codes; trailing zero bytes of a unit
// belong to the next start code).
std::vector<Nal> split_annex_b(const uint8_t* d, size_t n) {
  std::vector<Nal> out;
  size_t i = 0, start = SIZE_MAX;
  while (i + 2 < n) {
    if (d[i] == 0 && d[i + 1] == 0 && d[i + 2] == 1) {
      if (start != SIZE_MAX) {
        size_t e = i;
        while (e > start && d[e - 1] == 0) e--;
        out.push_back({d + start, e - start});
      }
      i += 3;
      start = i;
    } else {
      i++;
    }
  }
  if (start != SIZE_MAX && start < n) out.push_back({d + start, n - start});
  return out;
}

// Big-endian byte sink with box / element size patching.
struct Sink {
  std::vector<uint8_t> b;
  void u8(unsigned v) { b.push_back((uint8_t)v); }
  void u16(unsigned v) { u8(v >> 8); u8(v & 0xFF); }
  void u32(uint32_t v) { u16(v >> 16); u16(v & 0xFFFF); }
  void u64(uint64_t v) { u32((uint32_t)(v >> 32)); u32((uint32_t)v); }
  void raw(const void* p, size_t n) {
    const uint8_t* q = (const uint8_t*)p;
    b.insert(b.end(), q, q + n);
  }
  void str(const char* s) { raw(s, strlen(s)); }
  void zeros(size_t n) { b.insert(b.end(), n, 0); }
  void patch32(size_t at, uint32_t v) {
    for (int k = 0; k < 4; k++) b[at + k] = (uint8_t)(v >> (24 - 8 * k));
  }
  void patch64(size_t at, uint64_t v) {
    patch32(at, (uint32_t)(v >> 32));
    patch32(at + 4, (uint32_t)v);
  }
  // ISO boxes: a 32-bit size written when the box closes.
  size_t open(const char* type) {
    size_t at = b.size();
    u32(0);
    raw(type, 4);
    return at;
  }
  size_t open_full(const char* type, uint32_t version_flags) {
    size_t at = open(type);
    u32(version_flags);
    return at;
  }
  void close(size_t at) { patch32(at, (uint32_t)(b.size() - at)); }
};

// --- EBML --------------------------------------------------------------------------------

void ebml_id(Sink& s, uint32_t id) {
  int n = id > 0xFFFFFF ? 4 : id > 0xFFFF ? 3 : id > 0xFF ? 2 : 1;
  for (int k = n - 1; k >= 0; k--) s.u8((id >> (8 * k)) & 0xFF);
}

// Minimal-width size field; the all-ones value of each width is reserved ("unknown").
void ebml_size(Sink& s, uint64_t v) {
  int w = 1;
  while (w < 8 && v >= (1ull << (7 * w)) - 1) w++;
  const uint64_t coded = v | (1ull << (7 * w));
  for (int k = w - 1; k >= 0; k--) s.u8((coded >> (8 * k)) & 0xFF);
}

void ebml_bytes(Sink& s, uint32_t id, const void* p, size_t n) {
  ebml_id(s, id);
  ebml_size(s, n);
  s.raw(p, n);
}

void ebml_uint(Sink& s, uint32_t id, uint64_t v) {
  uint8_t be[8];
  for (int k = 0; k < 8; k++) be[k] = (uint8_t)(v >> (56 - 8 * k));
  int first = 0;
  while (first < 7 && be[first] == 0) first++;
  ebml_bytes(s, id, be + first, 8 - first);
}

void ebml_f64(Sink& s, uint32_t id, double v) {
  uint64_t bits;
  memcpy(&bits, &v, 8);
  uint8_t be[8];
  for (int k = 0; k < 8; k++) be[k] = (uint8_t)(bits >> (56 - 8 * k));
  ebml_bytes(s, id, be, 8);
}

void ebml_master(Sink& s, uint32_t id, const Sink& body) { ebml_bytes(s, id, body.b.data(), body.b.size()); }

enum : uint32_t {
  kEbml = 0x1A45DFA3, kDocType = 0x4282, kDocTypeVersion = 0x4287, kDocTypeReadVersion = 0x4285,
  kSegment = 0x18538067, kSeekHead = 0x114D9B74, kSeek = 0x4DBB, kSeekId = 0x53AB, kSeekPosition = 0x53AC,
  kInfo = 0x1549A966, kTimestampScale = 0x2AD7B1, kDuration = 0x4489, kMuxingApp = 0x4D80, kWritingApp = 0x5741,
  kTracks = 0x1654AE6B, kTrackEntry = 0xAE, kTrackNumber = 0xD7, kTrackUid = 0x73C5, kTrackType = 0x83,
  kDefaultDuration = 0x23E383, kCodecId = 0x86, kCodecPrivate = 0x63A2, kVideo = 0xE0, kPixelWidth = 0xB0,
  kPixelHeight = 0xBA, kColour = 0x55B0, kMatrixCoefficients = 0x55B1, kBitsPerChannel = 0x55B2, kRange = 0x55B9,
  kTransferCharacteristics = 0x55BA, kPrimaries = 0x55BB, kCluster = 0x1F43B675, kTimestamp = 0xE7,
  kSimpleBlock = 0xA3, kBlockGroup = 0xA0, kBlock = 0xA1, kCues = 0x1C53BB6B, kCuePoint = 0xBB, kCueTime = 0xB3,
  kCueTrackPositions = 0xB7, kCueTrack = 0xF7, kCueClusterPosition = 0xF1,
};

const char kAppName[] = "Ragdoll v0.1.0";  // Info MuxingApp / WritingApp (mkv.rs:937-938)

}  // namespace

struct rg_mux {
  int container, width, height, fps_num, fps_den;
  std::vector<uint8_t> sps, pps;
  std::vector<uint8_t> data;     // concatenated length-prefixed samples
  std::vector<size_t> offset;    // sample start in data
  std::vector<uint8_t> key;      // sample holds an IDR slice
};

namespace {

std::vector<uint8_t> avcc_record(const rg_mux* m) {
  std::vector<uint8_t> r;
  const auto& s = m->sps;
  r.push_back(1);                          // configurationVersion
  r.push_back(s[1]);                       // AVCProfileIndication
  r.push_back(s[2]);                       // profile_compatibility
  r.push_back(s[3]);                       // AVCLevelIndication
  r.push_back(0xFF);                       // lengthSizeMinusOne = 3
  r.push_back(0xE1);                       // one SPS
  r.push_back((uint8_t)(s.size() >> 8));
  r.push_back((uint8_t)s.size());
  r.insert(r.end(), s.begin(), s.end());
  r.push_back(1);                          // one PPS
  r.push_back((uint8_t)(m->pps.size() >> 8));
  r.push_back((uint8_t)m->pps.size());
  r.insert(r.end(), m->pps.begin(), m->pps.end());
  return r;
}

// Start of picture i and its duration, in 90 kHz ticks.
int64_t pic_ticks(const rg_mux* m, int64_t i) { return rescale(i, kTrackTimescale * m->fps_den, m->fps_num); }
int64_t pic_duration(const rg_mux* m, size_t i) {
  const size_t n = m->offset.size();
  if (i + 1 < n) return std::max<int64_t>(1, pic_ticks(m, i + 1) - pic_ticks(m, i));
  return std::max<int64_t>(1, rescale(1, kTrackTimescale * m->fps_den, m->fps_num));
}

size_t sample_size(const rg_mux* m, size_t i) {
  return (i + 1 < m->offset.size() ? m->offset[i + 1] : m->data.size()) - m->offset[i];
}

void matrix(Sink& s) {
  const uint32_t unity[9] = {0x00010000, 0, 0, 0, 0x00010000, 0, 0, 0, 0x40000000};
  for (uint32_t v : unity) s.u32(v);
}

std::vector<uint8_t> build_mp4(const rg_mux* m) {
  const size_t n = m->offset.size();
  const uint64_t payload = m->data.size();
  const bool co64 = payload > 0xFFFFFFFFull - 16ull * 1024 * 1024;
  const uint64_t mdat_header = payload + 8 > 0xFFFFFFFFull ? 16 : 8;

  int64_t total = 0;
  for (size_t i = 0; i < n; i++) total += pic_duration(m, i);
  const uint32_t movie_dur = (uint32_t)std::min<int64_t>(rescale(total, 1000, kTrackTimescale), 0xFFFFFFFF);

  Sink s;
  size_t ftyp = s.open("ftyp");
  s.str("isom");
  s.u32(512);
  s.str("isomiso2avc1mp41");
  s.close(ftyp);

  size_t moov = s.open("moov");
  size_t mvhd = s.open_full("mvhd", 0);
  s.u32(0); s.u32(0);                      // creation / modification time
  s.u32(1000);                             // movie timescale
  s.u32(movie_dur);
  s.u32(0x00010000); s.u16(0x0100);        // rate 1.0, volume 1.0
  s.zeros(10);
  matrix(s);
  s.zeros(24);
  s.u32(2);                                // next track id
  s.close(mvhd);

  size_t trak = s.open("trak");
  size_t tkhd = s.open_full("tkhd", 3);    // enabled, in movie
  s.u32(0); s.u32(0);
  s.u32(1);                                // track id
  s.u32(0);
  s.u32(movie_dur);
  s.zeros(8);
  s.u16(0); s.u16(0); s.u16(0); s.u16(0);  // layer, group, volume, reserved
  matrix(s);
  s.u32((uint32_t)m->width << 16);
  s.u32((uint32_t)m->height << 16);
  s.close(tkhd);

  size_t mdia = s.open("mdia");
  size_t mdhd = s.open_full("mdhd", 0);
  s.u32(0); s.u32(0);
  s.u32((uint32_t)kTrackTimescale);
  s.u32((uint32_t)std::min<int64_t>(total, 0xFFFFFFFF));
  s.u16(0x55C4);                           // language "und"
  s.u16(0);
  s.close(mdhd);
  size_t hdlr = s.open_full("hdlr", 0);
  s.u32(0);
  s.str("vide");
  s.zeros(12);
  s.raw("Ragdoll Video Handler", 22);      // handler name with its terminating NUL (mp4.rs:2316)
  s.close(hdlr);

  size_t minf = s.open("minf");
  size_t vmhd = s.open_full("vmhd", 1);
  s.zeros(8);
  s.close(vmhd);
  size_t dinf = s.open("dinf");
  size_t dref = s.open_full("dref", 0);
  s.u32(1);
  size_t url = s.open_full("url ", 1);     // media in this file
  s.close(url);
  s.close(dref);
  s.close(dinf);

  size_t stbl = s.open("stbl");
  size_t stsd = s.open_full("stsd", 0);
  s.u32(1);
  size_t avc1 = s.open("avc1");
  s.zeros(6);
  s.u16(1);                                // data reference index
  s.zeros(16);
  s.u16((unsigned)m->width);
  s.u16((unsigned)m->height);
  s.u32(0x00480000); s.u32(0x00480000);    // 72 dpi
  s.u32(0);
  s.u16(1);                                // frames per sample
  s.zeros(32);                             // compressor name
  s.u16(0x0018);                           // depth
  s.u16(0xFFFF);                           // pre_defined = -1
  size_t avcc = s.open("avcC");
  const std::vector<uint8_t> rec = avcc_record(m);
  s.raw(rec.data(), rec.size());
  s.close(avcc);
  size_t colr = s.open("colr");            // BT.709, limited range
  s.str("nclx");
  s.u16(1); s.u16(1); s.u16(1);
  s.u8(0);
  s.close(colr);
  size_t pasp = s.open("pasp");
  s.u32(1); s.u32(1);
  s.close(pasp);
  s.close(avc1);
  s.close(stsd);

  std::vector<std::pair<uint32_t, uint32_t>> runs;
  for (size_t i = 0; i < n; i++) {
    const uint32_t d = (uint32_t)pic_duration(m, i);
    if (!runs.empty() && runs.back().second == d) runs.back().first++;
    else runs.push_back({1, d});
  }
  size_t stts = s.open_full("stts", 0);
  s.u32((uint32_t)runs.size());
  for (auto& r : runs) { s.u32(r.first); s.u32(r.second); }
  s.close(stts);
  size_t stsc = s.open_full("stsc", 0);    // every chunk holds one sample
  s.u32(1); s.u32(1); s.u32(1); s.u32(1);
  s.close(stsc);
  size_t stsz = s.open_full("stsz", 0);
  s.u32(0);
  s.u32((uint32_t)n);
  for (size_t i = 0; i < n; i++) s.u32((uint32_t)sample_size(m, i));
  s.close(stsz);
  size_t stco = s.open_full(co64 ? "co64" : "stco", 0);
  s.u32((uint32_t)n);
  const size_t first_entry = s.b.size();
  for (size_t i = 0; i < n; i++) {
    if (co64) s.u64(0); else s.u32(0);
  }
  s.close(stco);
  size_t keys = 0;
  for (size_t i = 0; i < n; i++) keys += m->key[i];
  if (keys != n) {
    size_t stss = s.open_full("stss", 0);
    s.u32((uint32_t)keys);
    for (size_t i = 0; i < n; i++)
      if (m->key[i]) s.u32((uint32_t)(i + 1));
    s.close(stss);
  }
  s.close(stbl);
  s.close(minf);
  s.close(mdia);
  s.close(trak);
  s.close(moov);

  const uint64_t data_start = s.b.size() + mdat_header;
  for (size_t i = 0; i < n; i++) {
    const uint64_t at = data_start + m->offset[i];
    if (co64) s.patch64(first_entry + 8 * i, at);
    else s.patch32(first_entry + 4 * i, (uint32_t)at);
  }
  if (mdat_header == 16) {
    s.u32(1);
    s.str("mdat");
    s.u64(payload + 16);
  } else {
    s.u32((uint32_t)(payload + 8));
    s.str("mdat");
  }
  s.raw(m->data.data(), m->data.size());
  return std::move(s.b);
}

std::vector<uint8_t> build_mkv(const rg_mux* m) {
  const size_t n = m->offset.size();
  // Picture timing in ms, through the 90 kHz track clock.
  std::vector<int64_t> pts_ms(n), dur_ms(n);
  int64_t end_ms = 0;
  for (size_t i = 0; i < n; i++) {
    pts_ms[i] = rescale(pic_ticks(m, (int64_t)i), 1000, kTrackTimescale);
    dur_ms[i] = std::max<int64_t>(1, rescale(pic_duration(m, i), 1000, kTrackTimescale));
    end_ms = std::max(end_ms, pts_ms[i] + dur_ms[i]);
  }

  Sink ebml_body;
  ebml_bytes(ebml_body, kDocType, "matroska", 8);
  ebml_uint(ebml_body, kDocTypeVersion, 4);
  ebml_uint(ebml_body, kDocTypeReadVersion, 2);

  Sink info;
  ebml_uint(info, kTimestampScale, 1000000);
  if (end_ms > 0) ebml_f64(info, kDuration, (double)end_ms);
  ebml_bytes(info, kMuxingApp, kAppName, sizeof kAppName - 1);
  ebml_bytes(info, kWritingApp, kAppName, sizeof kAppName - 1);

  Sink entry;
  ebml_uint(entry, kTrackNumber, 1);
  ebml_uint(entry, kTrackUid, 1001);
  ebml_uint(entry, kTrackType, 1);
  ebml_bytes(entry, kCodecId, "V_MPEG4/ISO/AVC", 15);
  const std::vector<uint8_t> rec = avcc_record(m);
  ebml_bytes(entry, kCodecPrivate, rec.data(), rec.size());
  ebml_uint(entry, kDefaultDuration,
            (uint64_t)std::max<int64_t>(1, (int64_t)((__int128)1000000000 * m->fps_den / m->fps_num)));
  Sink colour;
  ebml_uint(colour, kMatrixCoefficients, 1);
  ebml_uint(colour, kTransferCharacteristics, 1);
  ebml_uint(colour, kPrimaries, 1);
  ebml_uint(colour, kRange, 1);  // limited
  ebml_uint(colour, kBitsPerChannel, 8);
  Sink video;
  ebml_uint(video, kPixelWidth, (uint64_t)m->width);
  ebml_uint(video, kPixelHeight, (uint64_t)m->height);
  ebml_master(video, kColour, colour);
  ebml_master(entry, kVideo, video);
  Sink tracks_body;
  ebml_master(tracks_body, kTrackEntry, entry);
  Sink tracks;
  ebml_master(tracks, kTracks, tracks_body);
  Sink info_el;
  ebml_master(info_el, kInfo, info);

  // Clusters: a new one at every keyframe, or when a block would sit more than 30 s away.
  struct Cluster {
    int64_t ts;
    size_t first, count;
    bool key;
  };
  std::vector<Cluster> clusters;
  for (size_t i = 0; i < n; i++) {
    const int64_t t = std::max<int64_t>(0, pts_ms[i]);
    bool fresh = clusters.empty();
    if (!fresh) {
      const int64_t rel = t - clusters.back().ts;
      fresh = rel < -30000 || rel > 30000 || (m->key[i] && clusters.back().count > 0);
    }
    if (fresh) clusters.push_back({t, i, 0, false});
    clusters.back().count++;
    clusters.back().key |= m->key[i] != 0;
  }
  std::vector<Sink> cl(clusters.size());
  for (size_t c = 0; c < clusters.size(); c++) {
    Sink body;
    ebml_uint(body, kTimestamp, (uint64_t)clusters[c].ts);
    for (size_t i = clusters[c].first; i < clusters[c].first + clusters[c].count; i++) {
      const size_t sz = sample_size(m, i);
      const int64_t rel = std::min<int64_t>(32767, std::max<int64_t>(-32768, std::max<int64_t>(0, pts_ms[i]) - clusters[c].ts));
      ebml_id(body, kSimpleBlock);
      ebml_size(body, 1 + 3 + sz);
      body.u8(0x81);                           // track 1
      body.u16((uint16_t)(int16_t)rel);
      body.u8(m->key[i] ? 0x80 : 0x00);
      body.raw(m->data.data() + m->offset[i], sz);
    }
    ebml_master(cl[c], kCluster, body);
  }

  auto seek_head = [&](uint64_t info_pos, uint64_t tracks_pos, bool cues, uint64_t cues_pos) {
    Sink body;
    const uint32_t ids[3] = {kInfo, kTracks, kCues};
    const uint64_t pos[3] = {info_pos, tracks_pos, cues_pos};
    for (int k = 0; k < (cues ? 3 : 2); k++) {
      Sink seek;
      const uint8_t id_be[4] = {(uint8_t)(ids[k] >> 24), (uint8_t)(ids[k] >> 16), (uint8_t)(ids[k] >> 8), (uint8_t)ids[k]};
      ebml_bytes(seek, kSeekId, id_be, 4);
      uint8_t p_be[8];
      for (int j = 0; j < 8; j++) p_be[j] = (uint8_t)(pos[k] >> (56 - 8 * j));
      ebml_bytes(seek, kSeekPosition, p_be, 8);
      ebml_master(body, kSeek, seek);
    }
    Sink el;
    ebml_master(el, kSeekHead, body);
    return el;
  };
  bool any_key = false;
  for (auto& c : clusters) any_key |= c.key;
  const uint64_t head_len = seek_head(0, 0, any_key, 0).b.size();
  const uint64_t info_pos = head_len;
  const uint64_t tracks_pos = info_pos + info_el.b.size();
  uint64_t pos = tracks_pos + tracks.b.size();
  Sink cues_body;
  for (size_t c = 0; c < clusters.size(); c++) {
    if (clusters[c].key) {
      Sink tp;
      ebml_uint(tp, kCueTrack, 1);
      ebml_uint(tp, kCueClusterPosition, pos);
      Sink pt;
      ebml_uint(pt, kCueTime, (uint64_t)clusters[c].ts);
      ebml_master(pt, kCueTrackPositions, tp);
      ebml_master(cues_body, kCuePoint, pt);
    }
    pos += cl[c].b.size();
  }
  Sink cues;
  if (!cues_body.b.empty()) ebml_master(cues, kCues, cues_body);
  const Sink head = seek_head(info_pos, tracks_pos, !cues.b.empty(), pos);

  Sink out;
  ebml_master(out, kEbml, ebml_body);
  ebml_id(out, kSegment);
  ebml_size(out, pos + cues.b.size());
  out.raw(head.b.data(), head.b.size());
  out.raw(info_el.b.data(), info_el.b.size());
  out.raw(tracks.b.data(), tracks.b.size());
  for (auto& c : cl) out.raw(c.b.data(), c.b.size());
  out.raw(cues.b.data(), cues.b.size());
  return std::move(out.b);
}

// --- demuxing ----------------------------------------------------------------------------

uint32_t be32(const uint8_t* p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }
uint64_t be64(const uint8_t* p) { return (uint64_t)be32(p) << 32 | be32(p + 4); }
uint16_t be16(const uint8_t* p) { return (uint16_t)(p[0] << 8 | p[1]); }

uint64_t gcd64(uint64_t a, uint64_t b) {
  while (b) { uint64_t t = a % b; a = b; b = t; }
  return a;
}

}  // namespace

struct rg_demux {
  rg_stream_info info{};
  std::vector<uint8_t> sps, pps;
  int len_size = 4;
  std::vector<uint8_t> data;             // the container, copied at open
  std::vector<uint64_t> at, size;        // sample ranges in data
};

namespace {

struct Box {
  const uint8_t* p;   // payload
  uint64_t n;         // payload bytes
  char type[5];
};

// Child boxes of [p, p + n); false on a malformed size.
bool boxes(const uint8_t* p, uint64_t n, std::vector<Box>& out) {
  uint64_t i = 0;
  while (i + 8 <= n) {
    uint64_t sz = be32(p + i), hdr = 8;
    if (sz == 1) {
      if (i + 16 > n) return false;
      sz = be64(p + i + 8);
      hdr = 16;
    } else if (sz == 0) {
      sz = n - i;
    }
    if (sz < hdr || sz > n - i) return false;
    Box b{p + i + hdr, sz - hdr, {}};
    memcpy(b.type, p + i + 4, 4);
    out.push_back(b);
    i += sz;
  }
  return true;
}

const Box* child(const std::vector<Box>& v, const char* t) {
  for (auto& b : v)
    if (!memcmp(b.type, t, 4)) return &b;
  return nullptr;
}

int parse_avcc(rg_demux* d, const uint8_t* p, uint64_t n) {
  if (n < 7 || p[0] != 1) return cfail(RG_ERR_INVALID, "demux: malformed avcC record");
  d->len_size = (p[4] & 3) + 1;
  uint64_t i = 6;
  const int nsps = p[5] & 0x1F;
  for (int k = 0; k < nsps; k++) {
    if (i + 2 > n || i + 2 + be16(p + i) > n) return cfail(RG_ERR_INVALID, "demux: truncated SPS in avcC");
    if (k == 0) d->sps.assign(p + i + 2, p + i + 2 + be16(p + i));
    i += 2 + be16(p + i);
  }
  if (i >= n) return cfail(RG_ERR_INVALID, "demux: avcC without PPS");
  const int npps = p[i++];
  for (int k = 0; k < npps; k++) {
    if (i + 2 > n || i + 2 + be16(p + i) > n) return cfail(RG_ERR_INVALID, "demux: truncated PPS in avcC");
    if (k == 0) d->pps.assign(p + i + 2, p + i + 2 + be16(p + i));
    i += 2 + be16(p + i);
  }
  if (d->sps.size() < 4 || d->pps.empty()) return cfail(RG_ERR_INVALID, "demux: avcC without parameter sets");
  d->info.profile_idc = d->sps[1];
  return 0;
}

int open_mp4(rg_demux* d) {
  std::vector<Box> top;
  if (!boxes(d->data.data(), d->data.size(), top)) return cfail(RG_ERR_INVALID, "demux: malformed MP4 box");
  const Box* moov = child(top, "moov");
  if (!moov) return cfail(RG_ERR_INVALID, "demux: MP4 without moov");
  std::vector<Box> mv;
  if (!boxes(moov->p, moov->n, mv)) return cfail(RG_ERR_INVALID, "demux: malformed moov");
  for (auto& trak : mv) {
    if (memcmp(trak.type, "trak", 4)) continue;
    std::vector<Box> tk, md, mi, st, sd;
    if (!boxes(trak.p, trak.n, tk)) continue;
    const Box* mdia = child(tk, "mdia");
    if (!mdia || !boxes(mdia->p, mdia->n, md)) continue;
    const Box* mdhd = child(md, "mdhd");
    const Box* minf = child(md, "minf");
    if (!mdhd || !minf || !boxes(minf->p, minf->n, mi)) continue;
    const Box* stbl = child(mi, "stbl");
    if (!stbl || !boxes(stbl->p, stbl->n, st)) continue;
    const Box* stsd = child(st, "stsd");
    if (!stsd || stsd->n < 8 + 8 + 78) continue;
    // First sample entry: 8-byte header, then 78 bytes of VisualSampleEntry before its boxes.
    const uint8_t* e = stsd->p + 8;
    const uint64_t esz = be32(e);
    if (memcmp(e + 4, "avc1", 4) && memcmp(e + 4, "avc3", 4)) continue;
    if (esz < 8 + 78 || esz > stsd->n - 8) return cfail(RG_ERR_INVALID, "demux: malformed avc1 entry");
    d->info.width = be16(e + 8 + 24);
    d->info.height = be16(e + 8 + 26);
    if (!boxes(e + 8 + 78, esz - 8 - 78, sd)) return cfail(RG_ERR_INVALID, "demux: malformed avc1 boxes");
    const Box* avcc = child(sd, "avcC");
    if (!avcc) return cfail(RG_ERR_INVALID, "demux: avc1 without avcC");
    int rc = parse_avcc(d, avcc->p, avcc->n);
    if (rc) return rc;
    const uint8_t* h = mdhd->p;
    const uint32_t timescale = h[0] == 1 ? be32(h + 20) : be32(h + 12);
    const Box* stts = child(st, "stts");
    const Box* stsc = child(st, "stsc");
    const Box* stsz = child(st, "stsz");
    const Box* stco = child(st, "stco");
    const Box* co64 = child(st, "co64");
    if (!stts || !stsc || !stsz || (!stco && !co64)) return cfail(RG_ERR_INVALID, "demux: incomplete sample table");
    if (stsz->n < 12) return cfail(RG_ERR_INVALID, "demux: malformed stsz");
    const uint32_t fixed = be32(stsz->p + 4), count = be32(stsz->p + 8);
    if (!fixed && stsz->n < 12 + 4ull * count) return cfail(RG_ERR_INVALID, "demux: truncated stsz");
    const Box* co = co64 ? co64 : stco;
    const int ow = co64 ? 8 : 4;
    if (co->n < 8) return cfail(RG_ERR_INVALID, "demux: malformed chunk offsets");
    const uint32_t chunks = be32(co->p + 4);
    if (co->n < 8 + (uint64_t)ow * chunks) return cfail(RG_ERR_INVALID, "demux: truncated chunk offsets");
    const uint32_t runs = stsc->n >= 8 ? be32(stsc->p + 4) : 0;
    if (!runs || stsc->n < 8 + 12ull * runs) return cfail(RG_ERR_INVALID, "demux: malformed stsc");
    uint32_t sample = 0;
    for (uint32_t r = 0; r < runs && sample < count; r++) {
      const uint32_t first = be32(stsc->p + 8 + 12 * r), per = be32(stsc->p + 12 + 12 * r);
      const uint32_t last = r + 1 < runs ? be32(stsc->p + 8 + 12 * (r + 1)) : chunks + 1;
      for (uint32_t c = first; c < last && c <= chunks && sample < count; c++) {
        uint64_t off = co64 ? be64(co->p + 8 + 8ull * (c - 1)) : be32(co->p + 8 + 4ull * (c - 1));
        for (uint32_t k = 0; k < per && sample < count; k++, sample++) {
          const uint64_t sz = fixed ? fixed : be32(stsz->p + 12 + 4ull * sample);
          if (off + sz > d->data.size()) return cfail(RG_ERR_INVALID, "demux: sample beyond the file");
          d->at.push_back(off);
          d->size.push_back(sz);
          off += sz;
        }
      }
    }
    if (sample != count) return cfail(RG_ERR_INVALID, "demux: sample table covers %u of %u samples", sample, count);
    if (stts->n >= 16 && be32(stts->p + 4) > 0 && timescale) {
      const uint64_t delta = be32(stts->p + 12), g = gcd64(timescale, delta ? delta : 1);
      d->info.fps_num = (int32_t)(timescale / g);
      d->info.fps_den = (int32_t)((delta ? delta : 1) / g);
    }
    d->info.container = RG_CONTAINER_MP4;
    return 0;
  }
  return cfail(RG_ERR_UNSUPPORTED, "demux: no H.264 video track in the MP4");
}

// EBML element at p (within end): id, payload range; false when malformed.
bool ebml_next(const uint8_t* p, const uint8_t* end, uint32_t& id, const uint8_t*& body, uint64_t& n) {
  if (p >= end) return false;
  int w = 1;
  while (w <= 4 && !(p[0] & (0x80 >> (w - 1)))) w++;
  if (w > 4 || p + w > end) return false;
  id = 0;
  for (int k = 0; k < w; k++) id = id << 8 | p[k];
  p += w;
  if (p >= end) return false;
  int s = 1;
  while (s <= 8 && !(p[0] & (0x80 >> (s - 1)))) s++;
  if (s > 8 || p + s > end) return false;
  uint64_t v = p[0] & (0xFF >> s);
  bool ones = v == (uint64_t)(0xFF >> s);
  for (int k = 1; k < s; k++) {
    v = v << 8 | p[k];
    ones &= p[k] == 0xFF;
  }
  p += s;
  body = p;
  n = ones ? (uint64_t)(end - p) : v;   // unknown size: up to the parent's end
  return n <= (uint64_t)(end - p);
}

uint64_t ebml_read_uint(const uint8_t* p, uint64_t n) {
  uint64_t v = 0;
  for (uint64_t k = 0; k < n && k < 8; k++) v = v << 8 | p[k];
  return v;
}

int open_mkv(rg_demux* d) {
  const uint8_t* p = d->data.data();
  const uint8_t* end = p + d->data.size();
  uint32_t id;
  const uint8_t* body;
  uint64_t n;
  if (!ebml_next(p, end, id, body, n) || id != kEbml) return cfail(RG_ERR_INVALID, "demux: not an EBML file");
  p = body + n;
  if (!ebml_next(p, end, id, body, n) || id != kSegment) return cfail(RG_ERR_INVALID, "demux: Matroska without Segment");
  const uint8_t* seg = body;
  const uint8_t* seg_end = body + n;
  uint64_t track = 0, default_ns = 0;
  for (const uint8_t* q = seg; q < seg_end;) {
    if (!ebml_next(q, seg_end, id, body, n)) return cfail(RG_ERR_INVALID, "demux: malformed Segment child");
    const uint8_t* next = body + n;
    if (id == kTracks) {
      for (const uint8_t* t = body; t < next;) {
        uint32_t tid;
        const uint8_t* tb;
        uint64_t tn;
        if (!ebml_next(t, next, tid, tb, tn)) return cfail(RG_ERR_INVALID, "demux: malformed Tracks");
        if (tid == kTrackEntry && !track) {
          uint64_t number = 0, type = 0;
          bool avc = false;
          const uint8_t* priv = nullptr;
          uint64_t priv_n = 0;
          int w = 0, h = 0;
          uint64_t dd = 0;
          for (const uint8_t* e = tb; e < tb + tn;) {
            uint32_t eid;
            const uint8_t* eb;
            uint64_t en;
            if (!ebml_next(e, tb + tn, eid, eb, en)) return cfail(RG_ERR_INVALID, "demux: malformed TrackEntry");
            if (eid == kTrackNumber) number = ebml_read_uint(eb, en);
            else if (eid == kTrackType) type = ebml_read_uint(eb, en);
            else if (eid == kCodecId) avc = en == 15 && !memcmp(eb, "V_MPEG4/ISO/AVC", 15);
            else if (eid == kCodecPrivate) { priv = eb; priv_n = en; }
            else if (eid == kDefaultDuration) dd = ebml_read_uint(eb, en);
            else if (eid == kVideo) {
              for (const uint8_t* v = eb; v < eb + en;) {
                uint32_t vid;
                const uint8_t* vb;
                uint64_t vn;
                if (!ebml_next(v, eb + en, vid, vb, vn)) return cfail(RG_ERR_INVALID, "demux: malformed Video");
                if (vid == kPixelWidth) w = (int)ebml_read_uint(vb, vn);
                if (vid == kPixelHeight) h = (int)ebml_read_uint(vb, vn);
                v = vb + vn;
              }
            }
            e = eb + en;
          }
          if (type == 1 && avc && priv) {
            int rc = parse_avcc(d, priv, priv_n);
            if (rc) return rc;
            track = number;
            d->info.width = w;
            d->info.height = h;
            default_ns = dd;
          }
        }
        t = tb + tn;
      }
    } else if (id == kCluster) {
      if (!track) return cfail(RG_ERR_UNSUPPORTED, "demux: cluster before an H.264 track entry");
      for (const uint8_t* c = body; c < next;) {
        uint32_t cid;
        const uint8_t* cb;
        uint64_t cn;
        if (!ebml_next(c, next, cid, cb, cn)) return cfail(RG_ERR_INVALID, "demux: malformed Cluster");
        const uint8_t* blk = nullptr;
        uint64_t bn = 0;
        if (cid == kSimpleBlock) { blk = cb; bn = cn; }
        if (cid == kBlockGroup) {
          for (const uint8_t* g = cb; g < cb + cn;) {
            uint32_t gid;
            const uint8_t* gb;
            uint64_t gn;
            if (!ebml_next(g, cb + cn, gid, gb, gn)) return cfail(RG_ERR_INVALID, "demux: malformed BlockGroup");
            if (gid == kBlock) { blk = gb; bn = gn; }
            g = gb + gn;
          }
        }
        if (blk) {
          int w = 1;
          while (w <= 8 && !(blk[0] & (0x80 >> (w - 1)))) w++;
          if (w > 8 || bn < (uint64_t)w + 3) return cfail(RG_ERR_INVALID, "demux: malformed block header");
          uint64_t num = blk[0] & (0xFF >> w);
          for (int k = 1; k < w; k++) num = num << 8 | blk[k];
          const uint8_t flags = blk[w + 2];
          if (num == track) {
            if (flags & 0x06) return cfail(RG_ERR_UNSUPPORTED, "demux: laced Matroska blocks");
            d->at.push_back((uint64_t)(blk + w + 3 - d->data.data()));
            d->size.push_back(bn - w - 3);
          }
        }
        c = cb + cn;
      }
    }
    q = next;
  }
  if (!track) return cfail(RG_ERR_UNSUPPORTED, "demux: no H.264 video track in the Matroska file");
  if (default_ns) {
    const uint64_t g = gcd64(1000000000ull, default_ns);
    d->info.fps_num = (int32_t)(1000000000ull / g);
    d->info.fps_den = (int32_t)(default_ns / g);
  }
  d->info.container = RG_CONTAINER_MKV;
  return 0;
}

bool sample_is_idr(const rg_demux* d, uint64_t at, uint64_t n) {
  const uint8_t* p = d->data.data() + at;
  uint64_t i = 0;
  while (i + d->len_size <= n) {
    uint64_t len = 0;
    for (int k = 0; k < d->len_size; k++) len = len << 8 | p[i + k];
    i += d->len_size;
    if (len == 0 || i + len > n) return false;
    if ((p[i] & 0x1F) == 5) return true;
    i += len;
  }
  return false;
}

}  // namespace

extern "C" {

rg_mux* rg_mux_create(int32_t container, int32_t width, int32_t height, int32_t fps_num, int32_t fps_den) {
  if (container != RG_CONTAINER_MP4 && container != RG_CONTAINER_MKV) {
    cfail(RG_ERR_INVALID, "rg_mux_create: unknown container %d", container);
    return nullptr;
  }
  if (width < 1 || height < 1 || width > 65535 || height > 65535) {
    cfail(RG_ERR_INVALID, "rg_mux_create: size %dx%d outside 1..65535", width, height);
    return nullptr;
  }
  if (fps_num < 1 || fps_den < 1) {
    cfail(RG_ERR_INVALID, "rg_mux_create: frame rate %d/%d", fps_num, fps_den);
    return nullptr;
  }
  rg_mux* m = new rg_mux();
  m->container = container;
  m->width = width;
  m->height = height;
  m->fps_num = fps_num;
  m->fps_den = fps_den;
  return m;
}

void rg_mux_destroy(rg_mux* m) { delete m; }

int rg_mux_write(rg_mux* m, const uint8_t* au, size_t size) {
  if (!m || (!au && size)) return cfail(RG_ERR_INVALID, "rg_mux_write: null argument");
  const std::vector<Nal> nals = split_annex_b(au, size);
  const size_t mark = m->data.size();
  bool key = false, slice = false;
  for (const Nal& u : nals) {
    if (!u.n) continue;
    const int type = u.p[0] & 0x1F;
    if (type == 7 || type == 8) {
      std::vector<uint8_t>& ps = type == 7 ? m->sps : m->pps;
      if (type == 7 && u.n < 4) {
        m->data.resize(mark);
        return cfail(RG_ERR_INVALID, "rg_mux_write: SPS of %zu bytes", u.n);
      }
      if (ps.empty()) {
        ps.assign(u.p, u.p + u.n);
      } else if (ps.size() != u.n || memcmp(ps.data(), u.p, u.n)) {
        m->data.resize(mark);
        return cfail(RG_ERR_UNSUPPORTED, "rg_mux_write: parameter sets change within the stream");
      }
      continue;
    }
    if (type == 9) continue;  // access unit delimiter
    key |= type == 5;
    slice |= type == 1 || type == 5;
    const uint32_t n = (uint32_t)u.n;
    const uint8_t len[4] = {(uint8_t)(n >> 24), (uint8_t)(n >> 16), (uint8_t)(n >> 8), (uint8_t)n};
    m->data.insert(m->data.end(), len, len + 4);
    m->data.insert(m->data.end(), u.p, u.p + u.n);
  }
  if (!slice) {
    m->data.resize(mark);
    return cfail(RG_ERR_INVALID, "rg_mux_write: access unit without a slice");
  }
  if (m->offset.empty() && (!key || m->sps.empty() || m->pps.empty())) {
    m->data.resize(mark);
    return cfail(RG_ERR_STATE, "rg_mux_write: the first access unit must be an IDR picture with SPS and PPS");
  }
  m->offset.push_back(mark);
  m->key.push_back(key);
  return 0;
}

int64_t rg_mux_finish(rg_mux* m, uint8_t* out, size_t cap) {
  if (!m) return cfail(RG_ERR_INVALID, "rg_mux_finish: null muxer");
  if (m->offset.empty()) return cfail(RG_ERR_STATE, "rg_mux_finish: no access units");
  const std::vector<uint8_t> file = m->container == RG_CONTAINER_MP4 ? build_mp4(m) : build_mkv(m);
  if (out) {
    if (cap < file.size()) return cfail(RG_ERR_INVALID, "rg_mux_finish: %zu-byte buffer for a %zu-byte file", cap, file.size());
    memcpy(out, file.data(), file.size());
  }
  return (int64_t)file.size();
}

rg_demux* rg_demux_open(const uint8_t* data, size_t size) {
  if (!data || size < 8) {
    cfail(RG_ERR_INVALID, "rg_demux_open: %zu bytes", data ? size : 0);
    return nullptr;
  }
  rg_demux* d = new rg_demux();
  d->data.assign(data, data + size);
  const bool ebml = be32(data) == kEbml;
  const int rc = ebml ? open_mkv(d) : open_mp4(d);
  if (rc) {
    delete d;
    return nullptr;
  }
  d->info.access_units = (int64_t)d->at.size();
  for (size_t i = 0; i < d->at.size(); i++) d->info.keyframes += sample_is_idr(d, d->at[i], d->size[i]);
  return d;
}

void rg_demux_destroy(rg_demux* d) { delete d; }

int rg_demux_info(const rg_demux* d, rg_stream_info* info) {
  if (!d || !info) return cfail(RG_ERR_INVALID, "rg_demux_info: null argument");
  *info = d->info;
  return 0;
}

int64_t rg_demux_access_unit(const rg_demux* d, int64_t index, uint8_t* out, size_t cap) {
  if (!d) return cfail(RG_ERR_INVALID, "rg_demux_access_unit: null demuxer");
  if (index < 0 || index >= (int64_t)d->at.size())
    return cfail(RG_ERR_INVALID, "rg_demux_access_unit: index %lld of %zu", (long long)index, d->at.size());
  const uint8_t* p = d->data.data() + d->at[index];
  const uint64_t n = d->size[index];
  std::vector<uint8_t> au;
  auto start = [&](const uint8_t* q, uint64_t len) {
    const uint8_t sc[4] = {0, 0, 0, 1};
    au.insert(au.end(), sc, sc + 4);
    au.insert(au.end(), q, q + len);
  };
  if (sample_is_idr(d, d->at[index], n)) {
    start(d->sps.data(), d->sps.size());
    start(d->pps.data(), d->pps.size());
  }
  uint64_t i = 0;
  while (i + d->len_size <= n) {
    uint64_t len = 0;
    for (int k = 0; k < d->len_size; k++) len = len << 8 | p[i + k];
    i += d->len_size;
    if (len == 0 || i + len > n) return cfail(RG_ERR_INVALID, "rg_demux_access_unit: malformed sample %lld", (long long)index);
    start(p + i, len);
    i += len;
  }
  if (out) {
    if (cap < au.size()) return cfail(RG_ERR_INVALID, "rg_demux_access_unit: %zu-byte buffer for %zu bytes", cap, au.size());
    memcpy(out, au.data(), au.size());
  }
  return (int64_t)au.size();
}

}  // extern "C"
