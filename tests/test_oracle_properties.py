"""The reference encoder's own property tests, restated against the CPU oracle (no GPU).

* decimation_scores_follow_x264 (crates/ragdoll-codec/src/h264/enc.rs:4189): the x264 decimation
  score of five level patterns, known answers 0 / 3 / 0 / 9 / 6.
* transform_8x8_paths_match_the_reference (enc.rs:4119): at every QP, with noise residuals, the
  oracle's High-profile 8x8 path (quant_luma_8x8_inter, enc.rs:2041, and recon_8x8, enc.rs:2020)
  gives the levels of sub8x8_dct_u8 + quantize_block8x8 (crates/ragdoll-codec/src/h264.rs:1374,
  :1387) for every coded block, and reconstructs as add8x8_idct_u8 of dequantize_block8x8
  (h264.rs:1634, :1403). The second path is restated here in numpy from those functions and
  crates/ragdoll-simd/src/fixed.rs:392 forward_dct8x8 / :457 inverse_idct8x8, independently of the
  oracle's C++.
"""
import ctypes

import numpy as np

from oracle_lib import lib

QUANT8_MF = [[13107, 11428, 20972, 12222, 16777, 15481], [11916, 10826, 19174, 11058, 14980, 14290],
             [10082, 8943, 15978, 9675, 12710, 11985], [9362, 8228, 14913, 8931, 11984, 11259],
             [8192, 7346, 13159, 7740, 10486, 9777], [7282, 6428, 11570, 6830, 9118, 8640]]
DEQUANT8 = [[20, 18, 32, 19, 25, 24], [22, 19, 35, 21, 28, 26], [26, 23, 42, 24, 33, 31],
            [28, 25, 45, 26, 35, 33], [32, 28, 51, 30, 40, 38], [36, 32, 58, 34, 46, 43]]


def _pos8(i):
    r, c = (i >> 3) & 3, i & 3
    if r == 0 and c == 0:
        return 0
    if r in (1, 3) and c in (1, 3):
        return 1
    if r == 2 and c == 2:
        return 2
    if (r == 0 and c in (1, 3)) or (r in (1, 3) and c == 0):
        return 3
    if (r, c) in ((0, 2), (2, 0)):
        return 4
    return 5


def _fdct8_pass(a):
    a0, a1, a2, a3 = a[0] + a[7], a[1] + a[6], a[2] + a[5], a[3] + a[4]
    a4, a5, a6, a7 = a[0] - a[7], a[1] - a[6], a[2] - a[5], a[3] - a[4]
    b0, b1, b2, b3 = a0 + a3, a1 + a2, a0 - a3, a1 - a2
    b4 = a5 + a6 + ((a4 >> 1) + a4)
    b5 = a4 - a7 - ((a6 >> 1) + a6)
    b6 = a4 + a7 - ((a5 >> 1) + a5)
    b7 = a5 - a6 + ((a7 >> 1) + a7)
    return [b0 + b1, b4 + (b7 >> 2), b2 + (b3 >> 1), b5 + (b6 >> 2), b0 - b1, b6 - (b5 >> 2),
            (b2 >> 1) - b3, (b4 >> 2) - b7]


def forward_dct8x8(block):
    """fixed.rs:392 (rows, then columns; i32 intermediates, i16 result)."""
    t = [0] * 64
    for r in range(8):
        t[r * 8:r * 8 + 8] = _fdct8_pass([int(v) for v in block[r * 8:r * 8 + 8]])
    out = [0] * 64
    for c in range(8):
        col = _fdct8_pass([t[k * 8 + c] for k in range(8)])
        for k in range(8):
            out[k * 8 + c] = ((col[k] + 32768) & 0xFFFF) - 32768
    return out


def _idct8_pass(c):
    a0, a2 = c[0] + c[4], c[0] - c[4]
    a4, a6 = (c[2] >> 1) - c[6], c[2] + (c[6] >> 1)
    b0, b2, b4, b6 = a0 + a6, a2 + a4, a2 - a4, a0 - a6
    a1 = -c[3] + c[5] - c[7] - (c[7] >> 1)
    a3 = c[1] + c[7] - c[3] - (c[3] >> 1)
    a5 = -c[1] + c[7] + c[5] + (c[5] >> 1)
    a7 = c[3] + c[5] + c[1] + (c[1] >> 1)
    b1, b3, b5, b7 = a1 + (a7 >> 2), a3 + (a5 >> 2), (a3 >> 2) - a5, a7 - (a1 >> 2)
    return [b0 + b7, b2 + b5, b4 + b3, b6 + b1, b6 - b1, b4 - b3, b2 - b5, b0 - b7]


def inverse_idct8x8(coeff):
    """fixed.rs:457 with the (x + 32) >> 6 normalisation."""
    t = [0] * 64
    for r in range(8):
        t[r * 8:r * 8 + 8] = _idct8_pass([int(v) for v in coeff[r * 8:r * 8 + 8]])
    out = [0] * 64
    for c in range(8):
        col = _idct8_pass([t[k * 8 + c] for k in range(8)])
        for k in range(8):
            out[k * 8 + c] = (col[k] + 32) >> 6
    return out


def quantize_block8x8(coeffs, qp, intra):
    """h264.rs:1387."""
    qp = min(qp, 51)
    qbits = 16 + qp // 6
    f = (1 << qbits) // (3 if intra else 6)
    out = []
    for i, c in enumerate(coeffs):
        level = min((abs(c) * QUANT8_MF[qp % 6][_pos8(i)] + f) >> qbits, 32767)
        out.append(-level if c < 0 else level)
    return out


def dequantize_block8x8(levels, qp):
    """h264.rs:1403."""
    qp = min(qp, 51)
    qd, rem = qp // 6, qp % 6
    out = []
    for i, lv in enumerate(levels):
        v = DEQUANT8[rem][_pos8(i)]
        d = int(lv) * (v << (qd - 2)) if qd >= 2 else (int(lv) * v + (1 << (1 - qd))) >> (2 - qd)
        out.append(max(-32768, min(32767, d)))
    return out


def _xorshift(seed):
    x = seed

    def nxt():
        nonlocal x
        x ^= (x << 13) & 0xFFFFFFFF
        x ^= x >> 17
        x ^= (x << 5) & 0xFFFFFFFF
        return x
    return nxt


def test_decimation_scores_follow_x264():
    L = lib()
    L.oracle_decimate_score.restype = ctypes.c_uint
    L.oracle_decimate_score.argtypes = [ctypes.c_void_p, ctypes.c_int]

    def score(c):
        a = np.array(c, np.int16)
        return L.oracle_decimate_score(a.ctypes.data, 16)

    def one_at(i, v):
        c = [0] * 16
        c[i] = v
        return c
    two = one_at(0, 1)
    two[1] = -1
    assert [score([0] * 16), score(one_at(0, 1)), score(one_at(15, -1)), score(one_at(1, 2)), score(two)] == \
        [0, 3, 0, 9, 6]


def test_transform_8x8_paths_match_the_reference():
    L = lib()
    L.oracle_quant_luma_8x8.restype = ctypes.c_int
    L.oracle_quant_luma_8x8.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    L.oracle_recon_8x8.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    nxt = _xorshift(0x2468ACE1)
    coded_blocks = 0
    for qp in range(52):
        src = np.zeros(256, np.uint8)
        for i in range(256):
            r = nxt() % 7
            src[i] = 0 if r == 0 else (255 if r == 1 else nxt() & 255)
        pred = np.array([nxt() % 256 for _ in range(256)], np.uint8)
        for fine in (False, True):
            q8 = np.zeros((4, 64), np.int16)
            cbp = L.oracle_quant_luma_8x8(src.ctypes.data, pred.ctypes.data, qp, int(fine), q8.ctypes.data)
            for b in range(4):
                o = (b >> 1) * 128 + (b & 1) * 8
                diff = [int(src[o + y * 16 + x]) - int(pred[o + y * 16 + x]) for y in range(8) for x in range(8)]
                want = quantize_block8x8(forward_dct8x8(diff), qp, fine)
                if cbp & (1 << b):
                    coded_blocks += 1
                    assert q8[b].tolist() == want, f"qp {qp} fine {fine} block {b}"
                a = pred.copy()
                wl = np.array(want, np.int16)
                L.oracle_recon_8x8(a[o:].ctypes.data, 16, wl.ctypes.data, qp)
                res = inverse_idct8x8(dequantize_block8x8(want, qp))
                bb = pred.copy()
                for y in range(8):
                    for x in range(8):
                        bb[o + y * 16 + x] = max(0, min(255, int(bb[o + y * 16 + x]) + res[y * 8 + x]))
                assert np.array_equal(a, bb), f"qp {qp} fine {fine} block {b} reconstruction"
    assert coded_blocks > 100
