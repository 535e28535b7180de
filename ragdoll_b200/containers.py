"""Containers for the encoder's output and input (host code, no GPU).

* ``mux`` / ``Muxer``: fast-start MP4 or Matroska from Annex-B access units (rg_mux_*, C++),
  byte-identical to ragdoll's muxers (crates/ragdoll-format/src/mp4.rs:1746,
  crates/ragdoll-format/src/mkv.rs:906).
* ``Demuxer``: the same two containers back to Annex-B access units (rg_demux_*).
* ``write_y4m`` / ``read_y4m``: YUV4MPEG2 with the header ragdoll writes
  (crates/ragdoll-format/src/y4m.rs:334: ``W H F Ip A1:1 C420mpeg2 XCOLORRANGE=LIMITED``) and the
  tokens its demuxer reads (y4m.rs:19-110), 8-bit 4:2:0 only.
"""
from __future__ import annotations

import ctypes
from typing import Iterable, List, Sequence, Tuple

import numpy as np

from .engine import RgError, RgStreamInfo, lib

RG_CONTAINER_MP4, RG_CONTAINER_MKV = 0, 1
CONTAINERS = {"mp4": RG_CONTAINER_MP4, "mkv": RG_CONTAINER_MKV}


def _err(code: int) -> RgError:
    return RgError(code, lib().rg_last_error().decode())


class Muxer:
    """One H.264 track: ``write(access_unit)`` per picture in decoding order, then ``finish()``."""

    def __init__(self, container: str, width: int, height: int, fps: Tuple[int, int] = (30, 1)):
        self._destroy = lib().rg_mux_destroy  # kept: the module's globals may go first at exit
        self.h = lib().rg_mux_create(CONTAINERS[container], width, height, fps[0], fps[1])
        if not self.h:
            raise _err(-1)

    def write(self, access_unit: bytes) -> None:
        buf = (ctypes.c_uint8 * len(access_unit)).from_buffer_copy(access_unit)
        rc = lib().rg_mux_write(self.h, buf, len(access_unit))
        if rc:
            raise _err(rc)

    def finish(self) -> bytes:
        n = lib().rg_mux_finish(self.h, None, 0)
        if n < 0:
            raise _err(n)
        out = (ctypes.c_uint8 * n)()
        m = lib().rg_mux_finish(self.h, out, n)
        if m != n:
            raise _err(m if m < 0 else -1)
        return bytes(out)

    def close(self) -> None:
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def mux(container: str, width: int, height: int, access_units: Iterable[bytes],
        fps: Tuple[int, int] = (30, 1)) -> bytes:
    m = Muxer(container, width, height, fps)
    try:
        for au in access_units:
            m.write(au)
        return m.finish()
    finally:
        m.close()


class Demuxer:
    """The first H.264 track of an MP4 or Matroska file as Annex-B access units."""

    def __init__(self, data: bytes):
        buf = (ctypes.c_uint8 * len(data)).from_buffer_copy(data)
        self._destroy = lib().rg_demux_destroy  # kept: the module's globals may go first at exit
        self.h = lib().rg_demux_open(buf, len(data))
        if not self.h:
            raise _err(-1)
        info = RgStreamInfo()
        rc = lib().rg_demux_info(self.h, ctypes.byref(info))
        if rc:
            raise _err(rc)
        self.container = "mp4" if info.container == RG_CONTAINER_MP4 else "mkv"
        self.width, self.height = info.width, info.height
        self.fps = (info.fps_num, info.fps_den)
        self.profile_idc = info.profile_idc
        self.keyframes = info.keyframes
        self.count = info.access_units

    def __len__(self) -> int:
        return self.count

    def access_unit(self, i: int) -> bytes:
        n = lib().rg_demux_access_unit(self.h, i, None, 0)
        if n < 0:
            raise _err(n)
        out = (ctypes.c_uint8 * n)()
        m = lib().rg_demux_access_unit(self.h, i, out, n)
        if m != n:
            raise _err(m if m < 0 else -1)
        return bytes(out)

    def access_units(self) -> List[bytes]:
        return [self.access_unit(i) for i in range(self.count)]

    def close(self) -> None:
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


Frame = Tuple[np.ndarray, np.ndarray, np.ndarray]


def write_y4m(width: int, height: int, frames: Sequence[Frame], fps: Tuple[int, int] = (30, 1)) -> bytes:
    """8-bit 4:2:0 YUV4MPEG2 with ragdoll's header line (y4m.rs:334) and ``FRAME`` markers."""
    head = f"YUV4MPEG2 W{width} H{height} F{max(fps[0], 1)}:{max(fps[1], 1)} Ip A1:1 C420mpeg2 XCOLORRANGE=LIMITED\n"
    cw, ch = (width + 1) // 2, (height + 1) // 2
    parts = [head.encode()]
    for y, u, v in frames:
        if y.shape != (height, width) or u.shape != (ch, cw) or v.shape != (ch, cw):
            raise RgError(-1, f"write_y4m: planes {y.shape} {u.shape} {v.shape} for {width}x{height}")
        parts += [b"FRAME\n", np.ascontiguousarray(y, np.uint8).tobytes(),
                  np.ascontiguousarray(u, np.uint8).tobytes(), np.ascontiguousarray(v, np.uint8).tobytes()]
    return b"".join(parts)


def read_y4m(data: bytes):
    """Returns (width, height, (fps_num, fps_den), frames) of an 8-bit 4:2:0 YUV4MPEG2 stream."""
    if not data.startswith(b"YUV4MPEG2 "):
        raise RgError(-1, "read_y4m: missing 'YUV4MPEG2 ' stream header")
    end = data.find(b"\n")
    if end < 0:
        raise RgError(-1, "read_y4m: unterminated stream header")
    width = height = 0
    fps = (25, 1)
    for tok in data[10:end].decode().split():
        if tok[0] == "W":
            width = int(tok[1:])
        elif tok[0] == "H":
            height = int(tok[1:])
        elif tok[0] == "F":
            a, b = tok[1:].split(":")
            fps = (int(a), int(b))
        elif tok[0] == "C" and not tok[1:].startswith("420"):
            raise RgError(-5, f"read_y4m: chroma format {tok[1:]} (only 4:2:0)")
    if width < 1 or height < 1:
        raise RgError(-1, "read_y4m: missing width or height")
    cw, ch = (width + 1) // 2, (height + 1) // 2
    size = width * height + 2 * cw * ch
    frames, p = [], end + 1
    while p < len(data):
        q = data.find(b"\n", p)
        if q < 0 or not data[p:q].startswith(b"FRAME"):
            raise RgError(-1, "read_y4m: expected a FRAME marker")
        p = q + 1
        if p + size > len(data):
            raise RgError(-1, "read_y4m: truncated frame payload")
        buf = np.frombuffer(data, np.uint8, size, p)
        frames.append((buf[:width * height].reshape(height, width).copy(),
                       buf[width * height:width * height + cw * ch].reshape(ch, cw).copy(),
                       buf[width * height + cw * ch:].reshape(ch, cw).copy()))
        p += size
    return width, height, fps, frames
