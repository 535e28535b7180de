"""H264Encoder with the macroblock loop on the GPU (rg_encoder_*, C++ host code around the engine).

``H264Encoder`` mirrors ragdoll's encoder (crates/ragdoll-codec/src/h264.rs:2996): ``encode_frame``
returns the Annex-B access unit of the next picture of a stream (an IDR picture every ``keyint``
pictures, SPS and PPS in front of it). ``submit`` / ``collect`` are the batched form, one wave of
GopRingEncoder::encode_wave (crates/ragdoll-pipeline/src/lib.rs:543): the next ``frames`` pictures
of every stream go to the GPU in one persistent launch, and their access units are written on the
host cores; with two waves in flight the GPU analyses one while the host writes the other.
"""
from __future__ import annotations

import ctypes
from typing import List, Sequence, Tuple

import numpy as np

from .engine import RG_PROFILE_HIGH, RgConfig, RgError, _u8, lib

Frame = Tuple[np.ndarray, np.ndarray, np.ndarray]


class H264Encoder:
    def __init__(self, width: int, height: int, qp: int, profile: int = RG_PROFILE_HIGH, fps=(30, 1),
                 keyint: int = 30, streams: int = 1, max_frames: int = 1, device: int = 0, threads: int = 0):
        cfg = RgConfig(width, height, profile, qp, streams, device, max_frames)
        self._destroy = lib().rg_encoder_destroy  # kept: the module's globals may go first at exit
        self.h = lib().rg_encoder_create(ctypes.byref(cfg), fps[0], fps[1], keyint, threads)
        if not self.h:
            raise RgError(-1, lib().rg_last_error().decode())
        self.width, self.height, self.streams, self.max_frames = width, height, streams, max_frames
        cw, ch = (width + 15) // 16 * 16, (height + 15) // 16 * 16
        self.bound = (cw * ch * 3 // 2) * 4 + (1 << 16)   # one access unit, generously
        self.buf = np.zeros(self.bound, np.uint8)
        self._inflight: List[list] = []                     # sources of waves not yet collected
        self._out = np.zeros(0, np.uint8)

    def set_stream_qp(self, stream: int, qp: int) -> None:
        """Fixed QP of one stream, before its first picture (rg_encoder_set_stream_qp)."""
        rc = lib().rg_encoder_set_stream_qp(self.h, stream, qp)
        if rc:
            raise RgError(rc, lib().rg_last_error().decode())

    @property
    def threads(self) -> int:
        return lib().rg_encoder_threads(self.h)

    def set_pipeline_tuning(self, **tuning) -> None:
        """Work order of the encoder's persistent launches (rg_set_pipeline_tuning on its context;
        keywords as Engine.set_pipeline_tuning), e.g. what ragdoll_b200.autotune picked; not while
        waves are in flight."""
        from .engine import RgPipelineTuning
        if self._inflight:
            raise RgError(-6, "set_pipeline_tuning: waves in flight")
        t = RgPipelineTuning(*(int(tuning.get(k, 0)) for k, _ in RgPipelineTuning._fields_))
        rc = lib().rg_set_pipeline_tuning(lib().rg_encoder_context(self.h), ctypes.byref(t))
        if rc:
            raise RgError(rc, lib().rg_last_error().decode())

    def set_record_compaction(self, words_per_mb: int) -> None:
        """Compact records of the encoder's waves (rg_set_record_compaction on its context, e.g.
        96 words per macroblock; 0, the default, turns them off); not while waves are in flight."""
        if self._inflight:
            raise RgError(-6, "set_record_compaction: waves in flight")
        rc = lib().rg_set_record_compaction(lib().rg_encoder_context(self.h), int(words_per_mb))
        if rc:
            raise RgError(rc, lib().rg_last_error().decode())

    def encode_frame(self, frame: Frame, stream: int = 0) -> bytes:
        y, u, v = (np.ascontiguousarray(p, np.uint8) for p in frame)
        n = lib().rg_encode_frame(self.h, stream, _u8(y), _u8(u), _u8(v), y.strides[0], u.strides[0],
                                  self.buf.ctypes.data, self.buf.size)
        if n < 0:
            raise RgError(n, lib().rg_last_error().decode())
        return self.buf[:n].tobytes()

    def submit(self, frames: Sequence[Sequence[Frame]]) -> None:
        """frames[f][s]: the next len(frames) pictures of every stream."""
        keep, ptrs = [], []
        for pics in frames:
            if len(pics) != self.streams:
                raise RgError(-1, f"submit: {len(pics)} pictures for {self.streams} streams")
            for y, u, v in pics:
                planes = [np.ascontiguousarray(p, np.uint8) for p in (y, u, v)]
                keep.append(planes)
                ptrs += [p.ctypes.data for p in planes]
        sy, suv = keep[0][0].strides[0], keep[0][1].strides[0]
        arr = (ctypes.c_void_p * len(ptrs))(*ptrs)
        rc = lib().rg_encoder_submit(self.h, arr, sy, suv, len(frames))
        if rc:
            raise RgError(rc, lib().rg_last_error().decode())
        self._inflight.append((keep, len(frames)))

    def _planes(self, frames):
        keep, ptrs = [], []
        for pics in frames:
            if len(pics) != self.streams:
                raise RgError(-1, f"submit: {len(pics)} pictures for {self.streams} streams")
            for y, u, v in pics:
                planes = [np.ascontiguousarray(p, np.uint8) for p in (y, u, v)]
                keep.append(planes)
                ptrs += [p.ctypes.data for p in planes]
        return keep, ptrs

    @staticmethod
    def submit_group(encoders: Sequence["H264Encoder"], frames: Sequence[Sequence[Sequence[Frame]]]) -> None:
        """frames[i][f][s]: the next len(frames[i]) pictures of every stream of encoders[i], all of
        them analysed by one persistent launch (rg_encoder_submit_group); collect each encoder's
        wave with its own collect()."""
        n = len(encoders)
        keeps, arrs, sy, suv = [], [], [], []
        for e, fr in zip(encoders, frames):
            keep, ptrs = e._planes(fr)
            keeps.append(keep)
            arrs.append((ctypes.c_void_p * len(ptrs))(*ptrs))
            sy.append(keep[0][0].strides[0])
            suv.append(keep[0][1].strides[0])
        planes = (ctypes.c_void_p * n)(*[ctypes.cast(a, ctypes.c_void_p) for a in arrs])
        hs = (ctypes.c_void_p * n)(*[e.h for e in encoders])
        rc = lib().rg_encoder_submit_group(hs, n, planes, (ctypes.c_size_t * n)(*sy), (ctypes.c_size_t * n)(*suv),
                                           len(frames[0]))
        if rc:
            raise RgError(rc, lib().rg_last_error().decode())
        for e, keep, fr in zip(encoders, keeps, frames):
            e._inflight.append((keep, len(fr)))

    def collect(self) -> List[List[bytes]]:
        """Access units of the oldest submitted wave, [f][s]."""
        if not self._inflight:
            raise RgError(-6, "collect: no wave in flight")
        frames = self._inflight[0][1]
        sizes = np.zeros(frames * self.streams, np.int64)
        total = lib().rg_encoder_collect(self.h, None, 0, sizes.ctypes.data)
        if total < 0:
            raise RgError(total, lib().rg_last_error().decode())
        if self._out.size < total:
            self._out = np.zeros(int(total * 1.25) + 1024, np.uint8)
        got = lib().rg_encoder_collect(self.h, self._out.ctypes.data, self._out.size, sizes.ctypes.data)
        if got != total:
            raise RgError(got if got < 0 else -1, lib().rg_last_error().decode())
        self._inflight.pop(0)
        data, at, out = self._out[:total].tobytes(), 0, []
        for f in range(frames):
            row = []
            for s in range(self.streams):
                n = int(sizes[f * self.streams + s])
                row.append(data[at:at + n])
                at += n
            out.append(row)
        return out

    def set_form(self, form: int, search_range: int = 32, net=None) -> None:
        """Analysis form of the next waves (rg_encoder_set_form): plain, full search, or learned with
        its candidate network (ragdoll_b200.learned.CandidateNet)."""
        rc = lib().rg_encoder_set_form(self.h, form, search_range, net.h if net is not None else None)
        if rc:
            raise RgError(rc, lib().rg_last_error().decode())
        self._net = net

    def new_gops(self) -> None:
        """The next submitted picture of every stream starts a new GOP (an IDR picture with
        idr_pic_id 0), as a fresh encoder per GOP chunk of the pipeline (rg_encoder_new_gops)."""
        rc = lib().rg_encoder_new_gops(self.h)
        if rc:
            raise RgError(rc, lib().rg_last_error().decode())

    def latencies(self) -> np.ndarray:
        """Milliseconds from submit to access unit written, per picture ([f][s]) of the wave
        collected last (rg_encoder_latencies)."""
        n = lib().rg_encoder_latencies(self.h, None, 0)
        if n < 0:
            raise RgError(n, lib().rg_last_error().decode())
        out = np.zeros(n, np.float64)
        lib().rg_encoder_latencies(self.h, out.ctypes.data, n)
        return out.reshape(-1, self.streams) if n else out

    def record_bytes(self) -> int:
        """Bytes of records the wave collected last brought to the host (rg_encoder_record_bytes):
        compact records, plus the full records of pictures handed out without them."""
        n = lib().rg_encoder_record_bytes(self.h)
        if n < 0:
            raise RgError(n, lib().rg_last_error().decode())
        return n

    def close(self) -> None:
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
