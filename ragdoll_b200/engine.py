"""ctypes binding of the sm_100a engine library (include/ragdoll_cuda.h).

:class:`Engine` wraps one ``rg_ctx``: a fixed picture size, profile and QP, and ``num_streams``
independent streams (GOPs) analysed side by side in one macroblock wavefront. Every call goes
through the C ABI; there is no CPU fallback -- loading fails loudly when the library or a CUDA
device is missing.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libragdoll_cuda.so"

RG_PROFILE_BASELINE, RG_PROFILE_MAIN, RG_PROFILE_HIGH = 0, 1, 2
RG_FRAME_IDR, RG_FRAME_P = 0, 1
PROFILES = {"baseline": RG_PROFILE_BASELINE, "main": RG_PROFILE_MAIN, "high": RG_PROFILE_HIGH}

ERRORS = {-1: "RG_ERR_INVALID", -2: "RG_ERR_OOM", -3: "RG_ERR_CUDA", -4: "RG_ERR_TIMEOUT",
          -5: "RG_ERR_UNSUPPORTED", -6: "RG_ERR_STATE"}

# rg_mb_out (include/ragdoll_cuda.h)
RECORD_DTYPE = np.dtype([
    ("mb_type", "u1"), ("i16_mode", "u1"), ("chroma_mode", "u1"), ("cbp", "u1"),
    ("transform_8x8", "u1"), ("qp", "u1"), ("qp_delta", "i1"), ("reserved0", "u1"),
    ("mv", "<i2", (2,)), ("mvd", "<i2", (2,)), ("i4_modes", "u1", (16,)),
    ("nz_mask", "<u2"), ("reserved1", "<u2"), ("luma", "<i2", (256,)), ("luma_dc", "<i2", (16,)),
    ("chroma_dc", "<i2", (2, 4)), ("chroma_ac", "<i2", (2, 4, 16)),
    ("part_mv", "<i2", (4, 2)), ("part_mvd", "<i2", (4, 2)), ("part_type", "u1"), ("reserved2", "u1", (3,)),
])
assert RECORD_DTYPE.itemsize == 888

# Analysis forms (rg_set_analysis_form) and the learned form's per-macroblock hint (rg_mb_hint).
RG_FORM_PLAIN, RG_FORM_FULLSEARCH, RG_FORM_LEARNED = 0, 1, 2
RG_MB_P_L0_16X8, RG_MB_P_L0_8X16, RG_MB_P_8X8 = 4, 5, 6
HINT_DTYPE = np.dtype([("part_mask", "u1"), ("flags", "u1"), ("mv_off", "i1", (2,)), ("i4_mask", "<u2", (16,)),
                       ("mv_coarse", "<i2", (2,))])
assert HINT_DTYPE.itemsize == 40

# Every symbol include/ragdoll_cuda.h declares.
EXPORTS = [
    "rg_last_error", "rg_version", "rg_create", "rg_destroy", "rg_mb_dims", "rg_analyse_frame",
    "rg_analyse_batch", "rg_analyse_batch_device", "rg_sync", "rg_copy_records", "rg_get_recon",
    "rg_get_recon_unfiltered", "rg_get_recon_coded", "rg_keep_unfiltered", "rg_cuda_stream",
    "rg_quality_frame", "rg_ssim_plane", "rg_ssim_plane_device_noalloc", "rg_analyse_gops",
    "rg_analyse_gops_device", "rg_copy_records_gops", "rg_set_pipeline_tuning", "rg_pipeline_lag", "rg_analyse_gops_async",
    "rg_writer_create", "rg_writer_destroy", "rg_writer_bound", "rg_writer_picture", "rg_pipeline_work_list",
    "rg_mux_create", "rg_mux_destroy", "rg_mux_write", "rg_mux_finish", "rg_demux_open", "rg_demux_destroy",
    "rg_demux_info", "rg_demux_access_unit", "rg_analyse_gops_wait", "rg_encoder_create", "rg_encoder_destroy",
    "rg_encoder_threads", "rg_encoder_context", "rg_encode_frame", "rg_encoder_submit", "rg_encoder_collect", "rg_encoder_latencies",
    "rg_quality_frame_prev",
    "rg_vmaf_lite_plane", "rg_set_stream_qp", "rg_encoder_set_stream_qp", "rg_analyse_gops_stream",
    "rg_analyse_gops_fetch", "rg_set_analysis_form", "rg_set_hints", "rg_encoder_new_gops",
    "rg_net_param_count", "rg_net_create", "rg_net_destroy", "rg_net_set_params", "rg_net_get_params",
    "rg_net_predict_hints", "rg_net_check", "rg_net_crops", "rg_net_forward_backward", "rg_net_adam_step",
    "rg_set_hint_net", "rg_encoder_set_form", "rg_ssim_batch_device", "rg_set_search_tuning",
    "rg_net_set_hint_policy", "rg_net_set_coarse_range", "rg_analyse_gops_group",
    "rg_set_record_compaction", "rg_analyse_gops_fetch_compact", "rg_records_compact", "rg_records_expand",
    "rg_writer_picture_compact", "rg_encoder_record_bytes", "rg_group_graph_counts",
    "rg_analyse_gops_group_async", "rg_analyse_gops_group_stream", "rg_encoder_submit_group",
]


class RgError(RuntimeError):
    """A negative RG_ERR_* return (RagdollError on the reference side)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class RgConfig(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("profile", ctypes.c_int32),
                ("qp", ctypes.c_int32), ("num_streams", ctypes.c_int32), ("device", ctypes.c_int32),
                ("max_frames", ctypes.c_int32)]


class RgPipelineTuning(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ("lag", "seg", "grid", "timeout_ms", "deblock_sms", "intra_sms")]


class RgStreamInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in
                ("container", "width", "height", "fps_num", "fps_den", "profile_idc")] + \
               [("access_units", ctypes.c_int64), ("keyframes", ctypes.c_int64)]


class RgQuality(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("ssim_y", "ssim_u", "ssim_v", "ssim_avg", "ms_ssim", "psnr_y", "psnr_u", "psnr_v",
                 "psnr_avg", "psnr_yuv_611", "ssim_db", "vmaf_lite")]


_lib = None


def lib() -> ctypes.CDLL:
    """Loads libragdoll_cuda.so (built in-tree by ragdoll_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        from . import build as _b
        _b.build()
    L = ctypes.CDLL(str(LIB_PATH))
    P = ctypes.c_void_p
    u8p = ctypes.POINTER(ctypes.c_uint8)
    L.rg_last_error.restype = ctypes.c_char_p
    L.rg_version.restype = ctypes.c_char_p
    L.rg_create.restype = P
    L.rg_create.argtypes = [ctypes.POINTER(RgConfig)]
    L.rg_destroy.argtypes = [P]
    L.rg_mb_dims.argtypes = [P, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
    L.rg_analyse_frame.argtypes = [P, ctypes.c_int32, u8p, u8p, u8p, ctypes.c_size_t, ctypes.c_size_t,
                                   ctypes.c_int32, P]
    L.rg_analyse_batch.argtypes = [P, P, ctypes.c_size_t, ctypes.c_size_t, P, P]
    L.rg_analyse_batch_device.argtypes = [P, P, ctypes.c_size_t, ctypes.c_size_t, P]
    L.rg_sync.argtypes = [P]
    L.rg_copy_records.argtypes = [P, P]
    L.rg_get_recon.argtypes = [P, ctypes.c_int32, u8p, u8p, u8p, ctypes.c_size_t, ctypes.c_size_t]
    L.rg_get_recon_coded.argtypes = [P, ctypes.c_int32, u8p, u8p, u8p]
    L.rg_get_recon_unfiltered.argtypes = [P, ctypes.c_int32, u8p, u8p, u8p]
    L.rg_keep_unfiltered.argtypes = [P, ctypes.c_int32]
    L.rg_cuda_stream.restype = P
    L.rg_cuda_stream.argtypes = [P]
    L.rg_quality_frame.argtypes = [P, ctypes.c_int32, u8p, u8p, u8p, ctypes.c_size_t, ctypes.c_size_t,
                                   ctypes.POINTER(RgQuality)]
    L.rg_ssim_plane.argtypes = [ctypes.c_int32, u8p, ctypes.c_size_t, u8p, ctypes.c_size_t,
                                ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_double),
                                ctypes.POINTER(ctypes.c_double)]
    L.rg_analyse_gops.argtypes = [P, P, ctypes.c_size_t, ctypes.c_size_t, P, ctypes.c_int32, P]
    L.rg_analyse_gops_device.argtypes = [P, P, ctypes.c_size_t, ctypes.c_size_t, P, ctypes.c_int32]
    L.rg_analyse_gops_group.argtypes = [P, ctypes.c_int32, P, P, P, P, ctypes.c_int32]
    L.rg_copy_records_gops.argtypes = [P, ctypes.c_int32, P]
    L.rg_analyse_gops_async.argtypes = [P, P, ctypes.c_size_t, ctypes.c_size_t, P, ctypes.c_int32, P]
    L.rg_pipeline_work_list.restype = ctypes.c_int64
    L.rg_pipeline_work_list.argtypes = [ctypes.c_int32] * 7 + [P, P, ctypes.c_int64, P]
    L.rg_writer_create.restype = P
    L.rg_writer_create.argtypes = [ctypes.POINTER(RgConfig), ctypes.c_int32, ctypes.c_int32]
    L.rg_writer_destroy.argtypes = [P]
    L.rg_writer_bound.restype = ctypes.c_size_t
    L.rg_writer_bound.argtypes = [P]
    L.rg_writer_picture.restype = ctypes.c_int64
    L.rg_writer_picture.argtypes = [P, P, ctypes.c_int32, P, ctypes.c_size_t]
    L.rg_set_pipeline_tuning.argtypes = [P, ctypes.POINTER(RgPipelineTuning)]
    L.rg_pipeline_lag.restype = ctypes.c_int32
    L.rg_pipeline_lag.argtypes = [P]
    L.rg_ssim_plane_device_noalloc.argtypes = [P, ctypes.c_size_t, P, ctypes.c_size_t, ctypes.c_int32,
                                               ctypes.c_int32, P, P]
    L.rg_analyse_gops_wait.argtypes = [P, P]
    L.rg_set_stream_qp.argtypes = [P, ctypes.c_int32, ctypes.c_int32]
    L.rg_analyse_gops_stream.argtypes = [P, P, ctypes.c_size_t, ctypes.c_size_t, P, ctypes.c_int32, P]
    L.rg_analyse_gops_fetch.argtypes = [P, P, ctypes.c_int32]
    L.rg_set_record_compaction.argtypes = [P, ctypes.c_int32]
    L.rg_analyse_gops_fetch_compact.argtypes = [P, P, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p),
                                                ctypes.POINTER(ctypes.c_size_t)]
    L.rg_records_compact.restype = ctypes.c_int64
    L.rg_records_compact.argtypes = [P, ctypes.c_int32, P, ctypes.c_size_t]
    L.rg_records_expand.argtypes = [P, ctypes.c_size_t, ctypes.c_int32, P]
    L.rg_writer_picture_compact.restype = ctypes.c_int64
    L.rg_writer_picture_compact.argtypes = [P, P, ctypes.c_size_t, ctypes.c_int32, P, ctypes.c_size_t]
    L.rg_encoder_record_bytes.restype = ctypes.c_int64
    L.rg_encoder_record_bytes.argtypes = [P]
    L.rg_group_graph_counts.argtypes = [P, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
    L.rg_analyse_gops_group_async.argtypes = [P, ctypes.c_int32, P, P, P, P, ctypes.c_int32, P]
    L.rg_encoder_submit_group.argtypes = [P, ctypes.c_int32, P, P, P, ctypes.c_int32]
    L.rg_analyse_gops_group_stream.argtypes = [P, ctypes.c_int32, P, P, P, P, ctypes.c_int32, P]
    L.rg_set_analysis_form.argtypes = [P, ctypes.c_int32, ctypes.c_int32]
    L.rg_set_hints.argtypes = [P, P, ctypes.c_int32]
    L.rg_encoder_new_gops.argtypes = [P]
    L.rg_set_hint_net.argtypes = [P, P]
    L.rg_set_search_tuning.argtypes = [P, P, ctypes.c_int32]
    L.rg_ssim_batch_device.argtypes = [ctypes.c_int32, P, P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                       ctypes.c_size_t, ctypes.c_size_t, P, P, P]
    L.rg_encoder_set_form.argtypes = [P, ctypes.c_int32, ctypes.c_int32, P]
    L.rg_net_param_count.restype = ctypes.c_int32
    L.rg_net_create.restype = P
    L.rg_net_create.argtypes = [ctypes.c_int32, ctypes.c_uint64]
    L.rg_net_destroy.argtypes = [P]
    L.rg_net_set_params.argtypes = [P, P, ctypes.c_int32]
    L.rg_net_get_params.argtypes = [P, P, ctypes.c_int32]
    L.rg_net_predict_hints.argtypes = [P, P, P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_size_t,
                                       P, P, P]
    L.rg_net_check.argtypes = [P, P]
    L.rg_net_set_hint_policy.argtypes = [P, ctypes.c_int32, ctypes.c_float, ctypes.c_int32, ctypes.c_float]
    L.rg_net_set_coarse_range.argtypes = [P, ctypes.c_int32]
    L.rg_net_crops.argtypes = [P, P, P, P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_size_t, P, P]
    L.rg_net_forward_backward.argtypes = [P, P, ctypes.c_int32, P, P, P, P, ctypes.c_float, P, P, P]
    L.rg_net_adam_step.argtypes = [P, ctypes.c_float]
    L.rg_encoder_set_stream_qp.argtypes = [P, ctypes.c_int32, ctypes.c_int32]
    L.rg_quality_frame_prev.argtypes = [P, ctypes.c_int32, u8p, u8p, u8p, ctypes.c_size_t, ctypes.c_size_t, u8p,
                                        ctypes.c_size_t, ctypes.POINTER(RgQuality)]
    L.rg_vmaf_lite_plane.argtypes = [ctypes.c_int32, u8p, ctypes.c_size_t, u8p, ctypes.c_size_t, ctypes.c_int32,
                                     ctypes.c_int32, u8p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_double)]
    L.rg_encoder_create.restype = P
    L.rg_encoder_create.argtypes = [ctypes.POINTER(RgConfig)] + [ctypes.c_int32] * 4
    L.rg_encoder_destroy.argtypes = [P]
    L.rg_encoder_threads.restype = ctypes.c_int32
    L.rg_encoder_threads.argtypes = [P]
    L.rg_encoder_context.restype = P
    L.rg_encoder_context.argtypes = [P]
    L.rg_encode_frame.restype = ctypes.c_int64
    L.rg_encode_frame.argtypes = [P, ctypes.c_int32, u8p, u8p, u8p, ctypes.c_size_t, ctypes.c_size_t, P,
                                  ctypes.c_size_t]
    L.rg_encoder_submit.argtypes = [P, P, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_int32]
    L.rg_encoder_collect.restype = ctypes.c_int64
    L.rg_encoder_collect.argtypes = [P, P, ctypes.c_size_t, P]
    L.rg_encoder_latencies.restype = ctypes.c_int32
    L.rg_encoder_latencies.argtypes = [P, P, ctypes.c_int32]
    L.rg_mux_create.restype = P
    L.rg_mux_create.argtypes = [ctypes.c_int32] * 5
    L.rg_mux_destroy.argtypes = [P]
    L.rg_mux_write.argtypes = [P, P, ctypes.c_size_t]
    L.rg_mux_finish.restype = ctypes.c_int64
    L.rg_mux_finish.argtypes = [P, P, ctypes.c_size_t]
    L.rg_demux_open.restype = P
    L.rg_demux_open.argtypes = [P, ctypes.c_size_t]
    L.rg_demux_destroy.argtypes = [P]
    L.rg_demux_info.argtypes = [P, ctypes.POINTER(RgStreamInfo)]
    L.rg_demux_access_unit.restype = ctypes.c_int64
    L.rg_demux_access_unit.argtypes = [P, ctypes.c_int64, P, ctypes.c_size_t]
    _lib = L
    return L


def _check(rc: int) -> None:
    if rc != 0:
        raise RgError(rc, lib().rg_last_error().decode())


COMPACT_MASK_WORDS = 7  # RG_COMPACT_MASK_WORDS


def compact_records(records: np.ndarray) -> bytes:
    """The compact form of records (rg_records_compact): per record, COMPACT_MASK_WORDS mask words
    of its nonzero 32-bit words, then those words in order."""
    recs = np.ascontiguousarray(records)
    cap = recs.size * (RECORD_DTYPE.itemsize + 4 * COMPACT_MASK_WORDS)
    out = np.zeros(max(cap, 4), np.uint8)
    n = lib().rg_records_compact(recs.ctypes.data, recs.size, out.ctypes.data, out.size)
    if n < 0:
        raise RgError(n, lib().rg_last_error().decode())
    return out[:n].tobytes()


def expand_records(data: bytes, n: int) -> np.ndarray:
    """Records back from their compact form (rg_records_expand)."""
    buf = np.frombuffer(data, np.uint8) if len(data) else np.zeros(4, np.uint8)
    out = np.zeros(n, RECORD_DTYPE)
    _check(lib().rg_records_expand(buf.ctypes.data, len(data), n, out.ctypes.data))
    return out


def _u8(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))


class Engine:
    """One ``rg_ctx``: ``num_streams`` streams of one size, profile and fixed QP."""

    def __init__(self, width: int, height: int, qp: int, profile: int = RG_PROFILE_BASELINE,
                 num_streams: int = 1, device: int = 0, max_frames: int = 1):
        self.width, self.height, self.qp, self.profile = width, height, qp, profile
        self.num_streams = num_streams
        self.max_frames = max(1, max_frames)
        cfg = RgConfig(width, height, profile, qp, num_streams, device, max_frames)
        h = lib().rg_create(ctypes.byref(cfg))
        if not h:
            raise RgError(-1, lib().rg_last_error().decode())
        self.h = h
        # kept on the instance: a context closed as the interpreter exits may outlive the module's globals
        self._destroy = lib().rg_destroy
        mw, mh = ctypes.c_int32(), ctypes.c_int32()
        _check(lib().rg_mb_dims(h, ctypes.byref(mw), ctypes.byref(mh)))
        self.mb_w, self.mb_h = mw.value, mh.value
        self.n_mb = self.mb_w * self.mb_h

    def close(self) -> None:
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def keep_unfiltered(self, enable: bool = True) -> None:
        _check(lib().rg_keep_unfiltered(self.h, 1 if enable else 0))

    @property
    def cuda_stream(self) -> int:
        return lib().rg_cuda_stream(self.h) or 0

    def analyse(self, frames, kinds) -> np.ndarray:
        """Analyses the next frame of every stream from host planes; returns the records
        ``[num_streams, mb_h * mb_w]``."""
        assert len(frames) == self.num_streams and len(kinds) == self.num_streams
        planes = (ctypes.c_void_p * (3 * self.num_streams))()
        keep = []
        sy = suv = None
        for s, (y, u, v) in enumerate(frames):
            y, u, v = (np.ascontiguousarray(p, dtype=np.uint8) for p in (y, u, v))
            keep += [y, u, v]
            if sy is None:
                sy, suv = y.strides[0], u.strides[0]
            assert y.strides[0] == sy and u.strides[0] == suv == v.strides[0]
            planes[3 * s], planes[3 * s + 1], planes[3 * s + 2] = y.ctypes.data, u.ctypes.data, v.ctypes.data
        k = (ctypes.c_int32 * self.num_streams)(*kinds)
        out = np.zeros((self.num_streams, self.n_mb), RECORD_DTYPE)
        _check(lib().rg_analyse_batch(self.h, planes, sy, suv, k, out.ctypes.data))
        return out

    def analyse_device(self, dev_planes, stride_y: int, stride_uv: int, kinds) -> None:
        """Queues the next frame of every stream from device planes (3 pointers per stream)."""
        planes = (ctypes.c_void_p * (3 * self.num_streams))(*dev_planes)
        k = (ctypes.c_int32 * self.num_streams)(*kinds)
        _check(lib().rg_analyse_batch_device(self.h, planes, stride_y, stride_uv, k))

    def analyse_gops(self, frames, kinds, out: np.ndarray | None = None) -> np.ndarray:
        """Pipelined form: ``frames[f][s]`` is picture f of stream s (host planes), ``kinds[f][s]``
        its kind; all pictures in one persistent launch. Returns records ``[F, S, n_mb]``, written
        into ``out`` when given (e.g. a view of pinned memory reused across calls)."""
        F, S = len(frames), self.num_streams
        planes = (ctypes.c_void_p * (3 * S * F))()
        keep = []
        sy = suv = None
        for f in range(F):
            assert len(frames[f]) == S
            for s, (y, u, v) in enumerate(frames[f]):
                y, u, v = (p if p.dtype == np.uint8 and p.strides[-1] == 1 else np.ascontiguousarray(p, dtype=np.uint8)
                           for p in (y, u, v))
                keep += [y, u, v]
                if sy is None:
                    sy, suv = y.strides[0], u.strides[0]
                i = (f * S + s) * 3
                planes[i], planes[i + 1], planes[i + 2] = y.ctypes.data, u.ctypes.data, v.ctypes.data
        k = (ctypes.c_int32 * (S * F))(*[kinds[f][s] for f in range(F) for s in range(S)])
        if out is None:
            out = np.zeros((F, S, self.n_mb), RECORD_DTYPE)
        assert out.shape == (F, S, self.n_mb) and out.dtype == RECORD_DTYPE and out.flags.c_contiguous
        _check(lib().rg_analyse_gops(self.h, planes, sy, suv, k, F, out.ctypes.data))
        return out

    def analyse_gops_async(self, frames, kinds, out: np.ndarray) -> None:
        """Queues ``analyse_gops`` and returns: the records land in ``out`` ([F, S, n_mb]) and the
        sources may be reused after ``sync()``. Pinned ``frames``/``out`` let the copies overlap the
        launches of neighbouring calls."""
        F, S = len(frames), self.num_streams
        assert out.shape == (F, S, self.n_mb) and out.dtype == RECORD_DTYPE and out.flags.c_contiguous
        planes = (ctypes.c_void_p * (3 * S * F))()
        sy = suv = None
        for f in range(F):
            assert len(frames[f]) == S
            for s, (y, u, v) in enumerate(frames[f]):
                for p in (y, u, v):
                    assert p.dtype == np.uint8 and p.strides[-1] == 1
                if sy is None:
                    sy, suv = y.strides[0], u.strides[0]
                i = (f * S + s) * 3
                planes[i], planes[i + 1], planes[i + 2] = y.ctypes.data, u.ctypes.data, v.ctypes.data
        k = (ctypes.c_int32 * (S * F))(*[kinds[f][s] for f in range(F) for s in range(S)])
        _check(lib().rg_analyse_gops_async(self.h, planes, sy, suv, k, F, out.ctypes.data))

    def analyse_gops_device(self, dev_planes, stride_y: int, stride_uv: int, kinds, frames: int) -> None:
        """Queues ``frames`` pictures of every stream from device planes ([f][s][y,u,v])."""
        planes = (ctypes.c_void_p * len(dev_planes))(*dev_planes)
        k = (ctypes.c_int32 * len(kinds))(*kinds)
        _check(lib().rg_analyse_gops_device(self.h, planes, stride_y, stride_uv, k, frames))

    @staticmethod
    def analyse_gops_group(engines, dev_planes, stride_y, stride_uv, kinds, frames: int) -> None:
        """rg_analyse_gops_group: ``frames`` pictures of every stream of every engine (each its own
        picture size) in one persistent launch on the first engine's stream. dev_planes[i] /
        kinds[i]: engine i's arguments as analyse_gops_device takes them; stride_y / stride_uv: one
        per engine."""
        n = len(engines)
        P = ctypes.c_void_p
        ctxs = (P * n)(*[e.h for e in engines])
        plane_arrays = [(P * len(p))(*p) for p in dev_planes]
        kind_arrays = [(ctypes.c_int32 * len(k))(*k) for k in kinds]
        planes = (P * n)(*[ctypes.cast(a, P) for a in plane_arrays])
        ks = (P * n)(*[ctypes.cast(a, P) for a in kind_arrays])
        sy = (ctypes.c_size_t * n)(*stride_y)
        suv = (ctypes.c_size_t * n)(*stride_uv)
        _check(lib().rg_analyse_gops_group(ctxs, n, planes, sy, suv, ks, frames))

    def set_analysis_form(self, form: int, search_range: int = 32) -> None:
        """Plain (byte-identical Balanced), full-search or learned analysis of the next calls
        (rg_set_analysis_form); the search forms need a Main or High profile context."""
        _check(lib().rg_set_analysis_form(self.h, form, search_range))

    def set_search_tuning(self, type_bits=None, walk: int = 4) -> None:
        """Search forms' partition type bits (16x16, 16x8, 8x16, 8x8; None: defaults) and the learned
        form's window re-centrings (rg_set_search_tuning)."""
        tb = (ctypes.c_int32 * 4)(*type_bits) if type_bits is not None else None
        _check(lib().rg_set_search_tuning(self.h, tb, walk))

    def set_hint_net(self, net) -> None:
        """The candidate network (ragdoll_b200.learned.CandidateNet or None) the learned form runs
        on each pipelined call's own sources when no hints were set (rg_set_hint_net)."""
        _check(lib().rg_set_hint_net(self.h, net.h if net is not None else None))
        self._hint_net = net

    def set_hints_device(self, dev_hints) -> None:
        """The learned form's hints of the next call: device addresses of one rg_mb_hint array
        (n_mb records, HINT_DTYPE) per picture and stream, in the call's [f][s] order."""
        arr = (ctypes.c_void_p * len(dev_hints))(*dev_hints)
        _check(lib().rg_set_hints(self.h, arr, len(dev_hints)))

    def set_pipeline_tuning(self, lag: int = 0, seg: int = 0, grid: int = 0, timeout_ms: int = 0,
                            deblock_sms: int = 0, intra_sms: int = 0) -> None:
        """Pipelined-mode work order (0 = library defaults): lag macroblock-times between the
        pictures of a stream, seg macroblocks per work segment, grid resident warps, the limit
        of one device wait, the SMs that take deblocking segments first and the next SMs that
        take IDR-picture analysis first (-1 = no such queue)."""
        t = RgPipelineTuning(lag, seg, grid, timeout_ms, deblock_sms, intra_sms)
        _check(lib().rg_set_pipeline_tuning(self.h, ctypes.byref(t)))

    def pipeline_lag(self) -> int:
        """The picture lag the next pipelined launch uses: the set one, or with lag 0 the one
        derived from the reach of the searches of the launches so far."""
        r = lib().rg_pipeline_lag(self.h)
        _check(r if r < 0 else 0)
        return r

    def records_gops(self, frames: int) -> np.ndarray:
        out = np.zeros((frames, self.num_streams, self.n_mb), RECORD_DTYPE)
        _check(lib().rg_copy_records_gops(self.h, frames, out.ctypes.data))
        return out

    def sync(self) -> None:
        _check(lib().rg_sync(self.h))

    def records(self) -> np.ndarray:
        out = np.zeros((self.num_streams, self.n_mb), RECORD_DTYPE)
        _check(lib().rg_copy_records(self.h, out.ctypes.data))
        return out

    def recon(self, stream: int = 0):
        w, h = self.width, self.height
        cw, ch = (w + 1) // 2, (h + 1) // 2
        y = np.zeros((h, w), np.uint8)
        u = np.zeros((ch, cw), np.uint8)
        v = np.zeros((ch, cw), np.uint8)
        _check(lib().rg_get_recon(self.h, stream, _u8(y), _u8(u), _u8(v), w, cw))
        return y, u, v

    def recon_coded(self, stream: int = 0):
        cw, ch = self.mb_w * 16, self.mb_h * 16
        y = np.zeros((ch, cw), np.uint8)
        u = np.zeros((ch // 2, cw // 2), np.uint8)
        v = np.zeros((ch // 2, cw // 2), np.uint8)
        _check(lib().rg_get_recon_coded(self.h, stream, _u8(y), _u8(u), _u8(v)))
        return y, u, v

    def recon_unfiltered(self, stream: int = 0):
        cw, ch = self.mb_w * 16, self.mb_h * 16
        y = np.zeros((ch, cw), np.uint8)
        u = np.zeros((ch // 2, cw // 2), np.uint8)
        v = np.zeros((ch // 2, cw // 2), np.uint8)
        _check(lib().rg_get_recon_unfiltered(self.h, stream, _u8(y), _u8(u), _u8(v)))
        return y, u, v

    def set_stream_qp(self, stream: int, qp: int) -> None:
        """Fixed QP of one stream (rg_set_stream_qp); streams of different QPs share launches."""
        _check(lib().rg_set_stream_qp(self.h, stream, qp))

    def quality(self, frame, stream: int = 0, prev=None) -> dict:
        """evaluate_frame_quality of the stream's last reconstruction against its source ``frame``;
        ``prev`` (the previous source frame) adds VMAF-Lite's motion term."""
        y, u, v = (np.ascontiguousarray(p, dtype=np.uint8) for p in frame)
        q = RgQuality()
        if prev is None:
            _check(lib().rg_quality_frame(self.h, stream, _u8(y), _u8(u), _u8(v), y.strides[0], u.strides[0],
                                          ctypes.byref(q)))
        else:
            py = np.ascontiguousarray(prev[0], dtype=np.uint8)
            _check(lib().rg_quality_frame_prev(self.h, stream, _u8(y), _u8(u), _u8(v), y.strides[0], u.strides[0],
                                               _u8(py), py.strides[0], ctypes.byref(q)))
        return {n: getattr(q, n) for n, _ in RgQuality._fields_}


def ssim_plane(a: np.ndarray, b: np.ndarray, device: int = 0):
    """(SSIM, MS-SSIM) of two 8-bit planes on the GPU (ssim_plane_u8 / ms_ssim_plane_u8)."""
    a = np.ascontiguousarray(a, dtype=np.uint8)
    b = np.ascontiguousarray(b, dtype=np.uint8)
    s, m = ctypes.c_double(), ctypes.c_double()
    _check(lib().rg_ssim_plane(device, _u8(a), a.strides[0], _u8(b), b.strides[0], a.shape[1], a.shape[0],
                               ctypes.byref(s), ctypes.byref(m)))
    return s.value, m.value


def vmaf_lite_plane(ref: np.ndarray, dist: np.ndarray, prev: np.ndarray = None, device: int = 0) -> float:
    """VMAF-Lite of two 8-bit planes on the GPU (vmaf_lite_plane_u8); prev: previous reference plane."""
    r = np.ascontiguousarray(ref, dtype=np.uint8)
    d = np.ascontiguousarray(dist, dtype=np.uint8)
    out = ctypes.c_double()
    if prev is None:
        _check(lib().rg_vmaf_lite_plane(device, _u8(r), r.strides[0], _u8(d), d.strides[0], r.shape[1], r.shape[0],
                                        None, 0, ctypes.byref(out)))
    else:
        q = np.ascontiguousarray(prev, dtype=np.uint8)
        _check(lib().rg_vmaf_lite_plane(device, _u8(r), r.strides[0], _u8(d), d.strides[0], r.shape[1], r.shape[0],
                                        _u8(q), q.strides[0], ctypes.byref(out)))
    return out.value


def ssim_batch_device(dev_a, dev_b, width: int, height: int, stride_a: int, stride_b: int, device: int = 0,
                      stream: int = 0, ms: bool = True):
    """SSIM and MS-SSIM of len(dev_a) device plane pairs in shared launches (rg_ssim_batch_device);
    returns two numpy arrays (MS-SSIM None when ms is False)."""
    n = len(dev_a)
    A = ctypes.c_void_p * n
    s, m = np.zeros(n), (np.zeros(n) if ms else None)
    _check(lib().rg_ssim_batch_device(device, A(*dev_a), A(*dev_b), n, width, height, stride_a, stride_b,
                                      s.ctypes.data, m.ctypes.data if ms else None, stream or None))
    return s, m


def ssim_plane_device_noalloc(dev_a: int, stride_a: int, dev_b: int, stride_b: int, width: int, height: int,
                              dev_out: int, stream: int = 0) -> None:
    """Queues SSIM / MS-SSIM of two device planes into ``dev_out`` (two device doubles) on
    ``stream`` without any device allocation (rg_ssim_plane_device_noalloc)."""
    _check(lib().rg_ssim_plane_device_noalloc(dev_a, stride_a, dev_b, stride_b, width, height, dev_out,
                                               stream or None))


class BitstreamWriter:
    """Annex-B writer of one stream from engine records (rg_writer_*; host code): CAVLC slices
    for Baseline, CABAC slices for Main and High."""

    def __init__(self, width: int, height: int, qp: int, fps=(30, 1), profile: int = RG_PROFILE_BASELINE):
        cfg = RgConfig(width, height, profile, qp, 1, 0, 1)
        self._destroy = lib().rg_writer_destroy  # kept: the module's globals may go first at exit
        self.h = lib().rg_writer_create(ctypes.byref(cfg), fps[0], fps[1])
        if not self.h:
            raise RgError(-1, lib().rg_last_error().decode())
        self.buf = np.zeros(lib().rg_writer_bound(self.h), np.uint8)

    def picture(self, records: np.ndarray, kind: int) -> bytes:
        records = np.ascontiguousarray(records, dtype=RECORD_DTYPE)
        n = lib().rg_writer_picture(self.h, records.ctypes.data, kind, self.buf.ctypes.data, self.buf.size)
        if n < 0:
            raise RgError(n, lib().rg_last_error().decode())
        return self.buf[:n].tobytes()

    def picture_compact(self, data: bytes, kind: int) -> bytes:
        """The access unit from the picture's compact records (rg_writer_picture_compact)."""
        buf = np.frombuffer(data, np.uint8) if len(data) else np.zeros(4, np.uint8)
        n = lib().rg_writer_picture_compact(self.h, buf.ctypes.data, len(data), kind, self.buf.ctypes.data,
                                            self.buf.size)
        if n < 0:
            raise RgError(n, lib().rg_last_error().decode())
        return self.buf[:n].tobytes()

    def close(self) -> None:
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class CavlcWriter(BitstreamWriter):
    """The Baseline (CAVLC) writer."""

    def __init__(self, width: int, height: int, qp: int, fps=(30, 1)):
        super().__init__(width, height, qp, fps, RG_PROFILE_BASELINE)
