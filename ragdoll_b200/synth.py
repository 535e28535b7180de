"""Seeded synthetic video sources.

Two generators:

* :func:`synth_video_frame` restates ragdoll's procedural test picture (SMPTE-style luma step
  bars over a moving diagonal gradient, blocky moving chroma), the source of the reference's
  pinned corpus clips (crates/ragdoll-pipeline/src/lib.rs:2919-2952).
* :func:`grating_clip` produces the seeded benchmark clips: a sum of four sinusoidal gratings
  plus blurred uniform noise, shifted per frame by a quarter-sample global motion, with
  independently moving textured rectangles; chroma is the field decimated 2x plus 128.

Frames are ``(y, u, v)`` tuples of C-contiguous ``uint8`` numpy arrays (``VideoFrame``
Yuv420p layout: chroma planes ``ceil(w/2) x ceil(h/2)``).
"""
from __future__ import annotations

import numpy as np


def synth_video_frame(width: int, height: int, frame_idx: int):
    """Procedural frame ``frame_idx`` (crates/ragdoll-pipeline/src/lib.rs:2919)."""
    shift = frame_idx * 4
    y = np.empty((height, width), np.uint8)
    xs = np.arange(width)
    bars = (16 + ((xs * 8) // max(width, 1)) * 28).astype(np.uint8)
    top = height // 3
    y[:top, :] = bars[None, :]
    yy = np.arange(top, height)[:, None]
    g = ((xs[None, :] + yy + shift) >> 2) & 0xFF
    y[top:, :] = (16 + (g * 219) // 255).astype(np.uint8)
    cw, ch = (width + 1) // 2, (height + 1) // 2
    cx = np.arange(cw)
    cy = np.arange(ch)
    u_row = (96 + (((cx + shift // 2) // 16) & 0x3F)).astype(np.uint8)
    v_col = (160 - (((cy + shift // 2) // 16) & 0x3F)).astype(np.uint8)
    u = np.ascontiguousarray(np.broadcast_to(u_row[None, :], (ch, cw)))
    v = np.ascontiguousarray(np.broadcast_to(v_col[:, None], (ch, cw)))
    return y, u, v


def _blur_1d(a: np.ndarray, sigma: float, axis: int) -> np.ndarray:
    r = int(np.ceil(3 * sigma))
    k = np.exp(-0.5 * (np.arange(-r, r + 1) / sigma) ** 2)
    k /= k.sum()
    pad = [(0, 0)] * a.ndim
    pad[axis] = (r, r)
    ap = np.pad(a, pad, mode="reflect")
    out = np.zeros_like(a)
    for i, w in enumerate(k):
        sl = [slice(None)] * a.ndim
        sl[axis] = slice(i, i + a.shape[axis])
        out += w * ap[tuple(sl)]
    return out


def grating_clip(width: int, height: int, frames: int, seed: int, motion: float = 8.0,
                 rects: int = 6):
    """Seeded grating clip: a list of ``frames`` Yuv420p frames.

    Luma is the sum of 4 sinusoidal gratings (periods 8-64 px, random orientation and phase)
    plus Gaussian-blurred (sigma 1.5) uniform noise of amplitude +-20, clamped to [16, 235].
    Each frame moves the whole field by a global shift drawn uniformly in +-``motion`` px at
    quarter-sample precision (the gratings are evaluated at the shifted coordinates and the
    noise field is resampled bilinearly), and ``rects`` textured rectangles of 64-256 px move
    independently. Chroma is the field decimated 2x (2x2 mean) around an offset of 128.
    """
    rng = np.random.default_rng(seed)
    periods = rng.uniform(8, 64, 4)
    angles = rng.uniform(0, np.pi, 4)
    phases = rng.uniform(0, 2 * np.pi, 4)
    amps = rng.uniform(12, 28, 4)
    steps = np.round(rng.uniform(-motion, motion, (frames, 2)) * 4) / 4
    steps[0] = 0
    pos = np.cumsum(steps, axis=0)
    ox = int(np.ceil(max(0.0, -pos[:, 0].min()))) + 2
    oy = int(np.ceil(max(0.0, -pos[:, 1].min()))) + 2
    nw = width + ox + int(np.ceil(max(0.0, pos[:, 0].max()))) + 3
    nh = height + oy + int(np.ceil(max(0.0, pos[:, 1].max()))) + 3
    noise = rng.uniform(-20, 20, (nh, nw)).astype(np.float32)
    noise = _blur_1d(_blur_1d(noise, 1.5, 0), 1.5, 1)
    rect_state = []
    for _ in range(rects):
        rw, rh = (int(v) for v in rng.integers(64, 257, 2))
        rx, ry = rng.uniform(0, max(1, width - rw)), rng.uniform(0, max(1, height - rh))
        vx, vy = rng.uniform(-motion, motion, 2)
        rect_state.append((rw, rh, rx, ry, vx, vy, rng.uniform(6, 24), rng.uniform(0, np.pi),
                           rng.uniform(40, 215)))
    ys, xs = np.mgrid[0:height, 0:width].astype(np.float32)
    base = []
    for p, a, ph in zip(periods, angles, phases):
        b = (2 * np.pi * (xs * np.cos(a) + ys * np.sin(a)) / p + ph).astype(np.float32)
        base.append((np.sin(b), np.cos(b)))
    cw, ch = (width + 1) // 2, (height + 1) // 2
    out = []
    for f in range(frames):
        gx, gy = pos[f]
        field = np.full((height, width), 126.0, np.float32)
        for (sb, cb), p, a, am in zip(base, periods, angles, amps):
            s = 2 * np.pi * (gx * np.cos(a) + gy * np.sin(a)) / p
            field += np.float32(am * np.cos(s)) * sb + np.float32(am * np.sin(s)) * cb
        # the static noise field sampled at the shifted grid: one global bilinear offset
        x0, y0 = int(np.floor(gx)) + ox, int(np.floor(gy)) + oy
        fx, fy = np.float32(gx - np.floor(gx)), np.float32(gy - np.floor(gy))
        n00 = noise[y0:y0 + height, x0:x0 + width]
        n01 = noise[y0:y0 + height, x0 + 1:x0 + 1 + width]
        n10 = noise[y0 + 1:y0 + 1 + height, x0:x0 + width]
        n11 = noise[y0 + 1:y0 + 1 + height, x0 + 1:x0 + 1 + width]
        field += (1 - fx) * (1 - fy) * n00 + fx * (1 - fy) * n01 + (1 - fx) * fy * n10 + fx * fy * n11
        for rw, rh, rx, ry, vx, vy, tp, ta, bse in rect_state:
            x0r, y0r = int(round(rx + vx * f)), int(round(ry + vy * f))
            xa, xb = max(0, x0r), min(width, x0r + rw)
            ya, yb = max(0, y0r), min(height, y0r + rh)
            if xa < xb and ya < yb:
                lx, ly = xs[ya:yb, xa:xb] - x0r, ys[ya:yb, xa:xb] - y0r
                field[ya:yb, xa:xb] = bse + 30 * np.sin(
                    2 * np.pi * (lx * np.cos(ta) + ly * np.sin(ta)) / tp)
        y = np.clip(np.rint(field), 16, 235).astype(np.uint8)
        fp = np.pad(field, ((0, 2 * ch - height), (0, 2 * cw - width)), mode="edge")
        c = fp.reshape(ch, 2, cw, 2).mean(axis=(1, 3)) - 126.0
        u = np.clip(np.rint(c * 0.5 + 128), 16, 240).astype(np.uint8)
        v = np.clip(np.rint(-c * 0.4 + 128), 16, 240).astype(np.uint8)
        out.append((np.ascontiguousarray(y), np.ascontiguousarray(u), np.ascontiguousarray(v)))
    return out
