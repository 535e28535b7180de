"""ctypes bindings of the CPU oracle (oracle/liboracle.so) for the tests.

The oracle is test infrastructure: a scalar restatement of ragdoll's Balanced encoder and SSIM
path that the GPU engine is checked against. Nothing in the product imports this module.
"""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
LIB_PATH = ROOT / "oracle" / "liboracle.so"

MB_TYPES = {0: "P_Skip", 1: "P_L0_16x16", 2: "I16x16", 3: "I4x4", 4: "P_L0_16x8", 5: "P_L0_8x16", 6: "P_8x8"}


class MbOut(ctypes.Structure):
    """Mirror of rg_mb_out (include/ragdoll_cuda.h)."""
    _fields_ = [
        ("mb_type", ctypes.c_uint8), ("i16_mode", ctypes.c_uint8), ("chroma_mode", ctypes.c_uint8),
        ("cbp", ctypes.c_uint8), ("transform_8x8", ctypes.c_uint8), ("qp", ctypes.c_uint8),
        ("qp_delta", ctypes.c_int8), ("reserved0", ctypes.c_uint8),
        ("mv", ctypes.c_int16 * 2), ("mvd", ctypes.c_int16 * 2),
        ("i4_modes", ctypes.c_uint8 * 16), ("nz_mask", ctypes.c_uint16), ("reserved1", ctypes.c_uint16),
        ("luma", ctypes.c_int16 * 256), ("luma_dc", ctypes.c_int16 * 16),
        ("chroma_dc", ctypes.c_int16 * 8), ("chroma_ac", ctypes.c_int16 * 128),
        ("part_mv", ctypes.c_int16 * 8), ("part_mvd", ctypes.c_int16 * 8), ("part_type", ctypes.c_uint8),
        ("reserved2", ctypes.c_uint8 * 3),
    ]


RECORD_DTYPE = np.dtype([
    ("mb_type", "u1"), ("i16_mode", "u1"), ("chroma_mode", "u1"), ("cbp", "u1"),
    ("transform_8x8", "u1"), ("qp", "u1"), ("qp_delta", "i1"), ("reserved0", "u1"),
    ("mv", "<i2", (2,)), ("mvd", "<i2", (2,)), ("i4_modes", "u1", (16,)),
    ("nz_mask", "<u2"), ("reserved1", "<u2"), ("luma", "<i2", (256,)), ("luma_dc", "<i2", (16,)),
    ("chroma_dc", "<i2", (2, 4)), ("chroma_ac", "<i2", (2, 4, 16)),
    ("part_mv", "<i2", (4, 2)), ("part_mvd", "<i2", (4, 2)), ("part_type", "u1"), ("reserved2", "u1", (3,)),
])
assert RECORD_DTYPE.itemsize == ctypes.sizeof(MbOut)

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
        L = ctypes.CDLL(str(LIB_PATH))
        u8p = ctypes.POINTER(ctypes.c_uint8)
        L.oracle_enc_create.restype = ctypes.c_void_p
        L.oracle_enc_create.argtypes = [ctypes.c_int] * 7
        L.oracle_enc_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_enc_frame.restype = ctypes.c_long
        L.oracle_enc_frame.argtypes = [ctypes.c_void_p, u8p, u8p, u8p, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_void_p, u8p, ctypes.c_long, ctypes.POINTER(ctypes.c_int)]
        L.oracle_enc_recon.argtypes = [ctypes.c_void_p, u8p, u8p, u8p, ctypes.c_int]
        L.oracle_mb_dims.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.oracle_record_size.restype = ctypes.c_int
        L.oracle_enc_set_form.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.oracle_enc_set_hints.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_enc_set_search_tuning.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.oracle_pixel_ops.restype = ctypes.c_ulonglong
        L.oracle_pixel_ops.argtypes = [ctypes.c_int]
        for fn in ("oracle_ssim_plane", "oracle_ms_ssim_plane", "oracle_psnr_plane"):
            f = getattr(L, fn)
            f.restype = ctypes.c_double
            f.argtypes = [u8p, ctypes.c_long, u8p, ctypes.c_long, ctypes.c_int, ctypes.c_int]
        L.oracle_sse_plane.restype = ctypes.c_uint64
        L.oracle_sse_plane.argtypes = [u8p, ctypes.c_long, u8p, ctypes.c_long, ctypes.c_int, ctypes.c_int]
        L.oracle_vmaf_lite_plane.restype = ctypes.c_double
        L.oracle_vmaf_lite_plane.argtypes = [u8p, ctypes.c_long, u8p, ctypes.c_long, ctypes.c_int, ctypes.c_int,
                                             u8p, ctypes.c_long]
        assert L.oracle_record_size() == RECORD_DTYPE.itemsize
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))


class OracleEncoder:
    """CPU restatement of H264Encoder (Balanced, fixed QP)."""

    def __init__(self, width, height, qp, profile=0, keyint=30, fps=(30, 1)):
        self.width, self.height = width, height
        self.h = lib().oracle_enc_create(width, height, profile, qp, keyint, fps[0], fps[1])
        mw, mh = ctypes.c_int(), ctypes.c_int()
        lib().oracle_mb_dims(self.h, ctypes.byref(mw), ctypes.byref(mh))
        self.mb_w, self.mb_h = mw.value, mh.value
        self.last_idr = False

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_enc_destroy(self.h)
            self.h = None

    def set_form(self, form, search_range=32):
        """Search forms (1 full search, 2 learned): decisions and reconstruction only, no bitstream."""
        lib().oracle_enc_set_form(self.h, form, search_range)

    def set_search_tuning(self, type_bits=(1, 16, 16, 40), walk=4):
        tb = (ctypes.c_int * 4)(*type_bits)
        lib().oracle_enc_set_search_tuning(self.h, tb, walk)

    def set_hints(self, hints):
        """The learned form's hints of the next frame (a HINT_DTYPE array of mb_w * mb_h records)."""
        self._hints = np.ascontiguousarray(hints)
        lib().oracle_enc_set_hints(self.h, self._hints.ctypes.data)

    def encode(self, frame):
        """Returns (annex_b_bytes, records[mb_h*mb_w])."""
        y, u, v = (np.ascontiguousarray(p) for p in frame)
        recs = np.zeros(self.mb_w * self.mb_h, RECORD_DTYPE)
        cap = 8 * (y.size + 2 * u.size) + 4096
        bits = np.zeros(cap, np.uint8)
        idr = ctypes.c_int()
        n = lib().oracle_enc_frame(self.h, _p(y), _p(u), _p(v), y.strides[0], u.strides[0],
                                   recs.ctypes.data, _p(bits), cap, ctypes.byref(idr))
        assert n >= 0
        self.last_idr = bool(idr.value)
        return bits[:n].tobytes(), recs

    def recon(self, filtered=True):
        cw, ch = self.mb_w * 16, self.mb_h * 16
        y = np.zeros((ch, cw), np.uint8)
        u = np.zeros((ch // 2, cw // 2), np.uint8)
        v = np.zeros((ch // 2, cw // 2), np.uint8)
        lib().oracle_enc_recon(self.h, _p(y), _p(u), _p(v), 1 if filtered else 0)
        return y, u, v


def pixel_ops(reset=False) -> int:
    """Pixel differences evaluated by the oracle's SAD / SSD / SATD over the frames encoded so far
    (all threads of the process); reset=True also zeroes the count."""
    return int(lib().oracle_pixel_ops(1 if reset else 0))


def ssim_plane(a, b):
    a = np.ascontiguousarray(a); b = np.ascontiguousarray(b)
    return lib().oracle_ssim_plane(_p(a), a.strides[0], _p(b), b.strides[0], a.shape[1], a.shape[0])


def ms_ssim_plane(a, b):
    a = np.ascontiguousarray(a); b = np.ascontiguousarray(b)
    return lib().oracle_ms_ssim_plane(_p(a), a.strides[0], _p(b), b.strides[0], a.shape[1], a.shape[0])


def psnr_plane(a, b):
    a = np.ascontiguousarray(a); b = np.ascontiguousarray(b)
    return lib().oracle_psnr_plane(_p(a), a.strides[0], _p(b), b.strides[0], a.shape[1], a.shape[0])


def sse_plane(a, b):
    a = np.ascontiguousarray(a); b = np.ascontiguousarray(b)
    return lib().oracle_sse_plane(_p(a), a.strides[0], _p(b), b.strides[0], a.shape[1], a.shape[0])


def vmaf_lite_plane(ref, dist, prev=None):
    r = np.ascontiguousarray(ref); d = np.ascontiguousarray(dist)
    if prev is None:
        return lib().oracle_vmaf_lite_plane(_p(r), r.strides[0], _p(d), d.strides[0], r.shape[1], r.shape[0], None, 0)
    q = np.ascontiguousarray(prev)
    return lib().oracle_vmaf_lite_plane(_p(r), r.strides[0], _p(d), d.strides[0], r.shape[1], r.shape[0],
                                        _p(q), q.strides[0])


def quality_report(ref, dist, prev=None):
    """evaluate_frame_quality (crates/ragdoll-pix/src/metrics.rs:328) from the oracle's plane metrics."""
    import math
    psnr = [psnr_plane(ref[p], dist[p]) for p in range(3)]
    ssim = [ssim_plane(ref[p], dist[p]) for p in range(3)]
    sse = sum(sse_plane(ref[p], dist[p]) for p in range(3))
    n = sum(ref[p].size for p in range(3))
    psnr_avg = math.inf if sse == 0 else 10.0 * math.log10((255.0 * 255.0) / (sse / n))
    if all(math.isinf(v) for v in psnr):
        psnr_611 = math.inf
    else:
        psnr_611 = (6.0 * min(psnr[0], 100.0) + min(psnr[1], 100.0) + min(psnr[2], 100.0)) / 8.0
    ssim_avg = (4.0 * ssim[0] + ssim[1] + ssim[2]) / 6.0
    ssim_db = math.inf if ssim_avg >= 1.0 else -10.0 * math.log10(1.0 - ssim_avg)
    return {"psnr_y": psnr[0], "psnr_u": psnr[1], "psnr_v": psnr[2], "psnr_avg": psnr_avg,
            "psnr_yuv_611": psnr_611, "ssim_y": ssim[0], "ssim_u": ssim[1], "ssim_v": ssim[2],
            "ssim_avg": ssim_avg, "ssim_db": ssim_db, "ms_ssim": ms_ssim_plane(ref[0], dist[0]),
            "vmaf_lite": vmaf_lite_plane(ref[0], dist[0], None if prev is None else prev[0])}


def split_annex_b(data: bytes) -> list[bytes]:
    """NAL units of an Annex-B byte stream (4-byte start codes as the encoder writes them)."""
    out, i, n = [], 0, len(data)
    starts = []
    while i + 3 < n:
        if data[i] == 0 and data[i + 1] == 0 and data[i + 2] == 0 and data[i + 3] == 1:
            starts.append(i + 4)
            i += 4
        else:
            i += 1
    for k, s in enumerate(starts):
        e = starts[k + 1] - 4 if k + 1 < len(starts) else n
        out.append(data[s:e])
    return out


def read_nal_fixture(path) -> list[bytes]:
    data = Path(path).read_bytes()
    out, p = [], 0
    while p < len(data):
        ln = struct.unpack(">I", data[p:p + 4])[0]
        out.append(data[p + 4:p + 4 + ln])
        p += 4 + ln
    return out
