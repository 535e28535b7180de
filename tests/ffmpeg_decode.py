"""An independent H.264 decoder for the tests: FFmpeg's libavcodec, through its public C API.

The FFmpeg libraries come with the opencv-python wheel of this environment; they are loaded from
that wheel's library folder by absolute path (their own dependencies first). ``decode`` feeds
Annex-B access units to the h264 decoder and returns every output picture as 8-bit Y, U, V
planes exactly as decoded (no colour conversion), so a test can require the decoded pictures to
equal the encoder's reconstruction sample for sample. ``available()`` is False when the libraries
are missing; tests then skip.

Structure offsets used (libavutil / libavcodec public headers, stable across these major
versions): AVPacket.data at 24; AVFrame.data[] at 0, linesize[] at 64, width/height at 104/108,
format at 116 (AV_PIX_FMT_YUV420P = 0).
"""
from __future__ import annotations

import ctypes
import glob
import os
from typing import List, Sequence, Tuple

import numpy as np

AV_CODEC_ID_H264 = 27
AVERROR_EAGAIN = -11
AVERROR_EOF = -0x20464F45

_libs = None


def _load():
    global _libs
    if _libs is not None:
        return _libs
    _libs = {}
    try:
        import cv2  # noqa: F401  (locates the wheel)
        folder = os.path.join(os.path.dirname(os.path.dirname(cv2.__file__)), "opencv_python_headless.libs")
    except ImportError:
        return _libs
    pending = sorted(glob.glob(os.path.join(folder, "*.so*")))
    for _ in range(len(pending) + 1):
        rest = []
        for p in pending:
            try:
                _libs[os.path.basename(p).split("-")[0]] = ctypes.CDLL(p, mode=ctypes.RTLD_GLOBAL)
            except OSError:
                rest.append(p)
        if not rest or rest == pending:
            break
        pending = rest
    if "libavcodec" in _libs:
        L = _libs["libavcodec"]
        P = ctypes.c_void_p
        L.avcodec_find_decoder.restype = P
        L.avcodec_find_decoder.argtypes = [ctypes.c_int]
        L.avcodec_alloc_context3.restype = P
        L.avcodec_alloc_context3.argtypes = [P]
        L.avcodec_open2.argtypes = [P, P, P]
        L.avcodec_send_packet.argtypes = [P, P]
        L.avcodec_receive_frame.argtypes = [P, P]
        L.avcodec_free_context.argtypes = [ctypes.POINTER(P)]
        L.av_packet_alloc.restype = P
        L.av_packet_free.argtypes = [ctypes.POINTER(P)]
        L.av_packet_unref.argtypes = [P]
        L.av_new_packet.argtypes = [P, ctypes.c_int]
        U = _libs["libavutil"]
        U.av_frame_alloc.restype = P
        U.av_frame_free.argtypes = [ctypes.POINTER(P)]
        U.av_frame_unref.argtypes = [P]
    return _libs


def available() -> bool:
    libs = _load()
    return "libavcodec" in libs and bool(libs["libavcodec"].avcodec_find_decoder(AV_CODEC_ID_H264))


Frame = Tuple[np.ndarray, np.ndarray, np.ndarray]


def _take(frame: int) -> Frame:
    ptrs = (ctypes.c_void_p * 3).from_address(frame)
    lines = (ctypes.c_int * 3).from_address(frame + 64)
    w, h, fmt = (ctypes.c_int * 4).from_address(frame + 104)[0:1] + \
        (ctypes.c_int * 4).from_address(frame + 104)[1:2] + (ctypes.c_int * 4).from_address(frame + 104)[3:4]
    if fmt != 0:
        raise RuntimeError(f"decoder output format {fmt}, expected yuv420p")
    out = []
    for k, (pw, ph) in enumerate(((w, h), ((w + 1) // 2, (h + 1) // 2), ((w + 1) // 2, (h + 1) // 2))):
        buf = (ctypes.c_uint8 * (lines[k] * ph)).from_address(ptrs[k])
        out.append(np.frombuffer(buf, np.uint8).reshape(ph, lines[k])[:, :pw].copy())
    return tuple(out)


def decode(access_units: Sequence[bytes]) -> List[Frame]:
    """Decodes Annex-B access units in order; returns the output pictures (cropped planes)."""
    libs = _load()
    L, U = libs["libavcodec"], libs["libavutil"]
    codec = L.avcodec_find_decoder(AV_CODEC_ID_H264)
    ctx = ctypes.c_void_p(L.avcodec_alloc_context3(codec))
    if L.avcodec_open2(ctx, codec, None) < 0:
        raise RuntimeError("avcodec_open2 failed")
    pkt = ctypes.c_void_p(L.av_packet_alloc())
    frame = ctypes.c_void_p(U.av_frame_alloc())
    out: List[Frame] = []

    def drain():
        while True:
            rc = L.avcodec_receive_frame(ctx, frame)
            if rc in (AVERROR_EAGAIN, AVERROR_EOF):
                return
            if rc < 0:
                raise RuntimeError(f"avcodec_receive_frame: {rc}")
            out.append(_take(frame.value))
            U.av_frame_unref(frame)

    try:
        for au in access_units:
            if L.av_new_packet(pkt, len(au)) < 0:
                raise RuntimeError("av_new_packet failed")
            data = ctypes.c_void_p.from_address(pkt.value + 24).value
            ctypes.memmove(data, au, len(au))
            rc = L.avcodec_send_packet(ctx, pkt)
            L.av_packet_unref(pkt)
            if rc < 0:
                raise RuntimeError(f"avcodec_send_packet: {rc}")
            drain()
        L.avcodec_send_packet(ctx, None)
        drain()
    finally:
        U.av_frame_free(ctypes.byref(frame))
        L.av_packet_free(ctypes.byref(pkt))
        L.avcodec_free_context(ctypes.byref(ctx))
    return out
