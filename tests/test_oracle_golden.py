"""Pins the CPU oracle to the reference's own encoder output.

The reference cannot be built here (Rust, no toolchain), so the oracle -- a C++ restatement of
ragdoll's Balanced encoder -- is checked against the byte-pinned clips of the reference's corpus
(qa/corpus/manifest.toml): ragdoll's Balanced / Constrained Baseline / QP 20 encodings of
synth_video_frame, in 15-frame GOPs as `ragdoll transcode` cuts them
(crates/ragdoll-pipeline/src/lib.rs:210, :580-585). Every slice NAL, the SPS and the PPS must be
byte-identical.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle_lib import MB_TYPES, OracleEncoder, read_nal_fixture, split_annex_b
from ragdoll_b200.synth import synth_video_frame

GOLDEN = Path(__file__).resolve().parent / "golden"


def encode_gops(width, height, frames, qp, fps, gop=15):
    nals, types = [], {}
    for g0 in range(0, frames, gop):
        n = min(gop, frames - g0)
        enc = OracleEncoder(width, height, qp, profile=0, keyint=n + 1, fps=fps)
        for i in range(n):
            data, recs = enc.encode(synth_video_frame(width, height, g0 + i))
            nals += split_annex_b(data)
            for t in recs["mb_type"]:
                types[MB_TYPES[int(t)]] = types.get(MB_TYPES[int(t)], 0) + 1
    return nals, types


@pytest.mark.parametrize("fixture,w,h,frames,fps", [
    ("clip_160x90_qp20.nal", 160, 90, 30, (30, 1)),
    ("clip_320x180_qp20.nal", 320, 180, 15, (25, 1)),
])
def test_oracle_matches_pinned_corpus(fixture, w, h, frames, fps):
    gold = read_nal_fixture(GOLDEN / fixture)
    nals, types = encode_gops(w, h, frames, 20, fps)
    params = [n for n in nals if n[0] & 0x1F in (7, 8)]
    slices = [n for n in nals if n[0] & 0x1F in (1, 5)]
    assert params[0] == gold[0], "SPS differs"
    assert params[1] == gold[1], "PPS differs"
    assert len(slices) == len(gold) - 2
    for i, (a, b) in enumerate(zip(slices, gold[2:])):
        assert a == b, f"slice {i} differs ({len(a)} vs {len(b)} bytes)"
    # the pinned clips exercise every macroblock kind of the Balanced P and I paths
    assert set(types) == {"I4x4", "I16x16", "P_Skip", "P_L0_16x16"}


def test_golden_provenance():
    meta = json.loads((GOLDEN / "golden.json").read_text())
    assert meta["clip_160x90_qp20.nal"]["source_sha256"].startswith("a14d81e8")
    assert meta["clip_160x90_qp20.nal"]["source_size"] == 3779
    assert meta["clip_320x180_qp20.nal"]["source_size"] == 4050


def test_synth_generator_deterministic():
    a = synth_video_frame(64, 36, 3)
    b = synth_video_frame(64, 36, 3)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert a[1].shape == (18, 32)


def _crop(frame, w, h):
    y, u, v = frame
    cw, ch = (w + 1) // 2, (h + 1) // 2
    return (np.ascontiguousarray(y[:h, :w]), np.ascontiguousarray(u[:ch, :cw]),
            np.ascontiguousarray(v[:ch, :cw]))


def test_oracle_matches_cli_transcode_and_metrics_snapshots():
    """`ragdoll transcode v.mp4 text_t.mp4 --qp 30` then `ragdoll metrics v.mp4 text_t.mp4`
    (crates/ragdoll-cli/tests/cli.rs:125-160, golden/transcode.txt, golden/metrics.txt).

    The decode of v.mp4 is the QP 20 encoder's reconstruction (the reference's recon == decode
    contract, crates/ragdoll-codec/src/h264.rs:4326); re-encoding it at QP 30 must give the pinned
    2382-byte MP4 (ftyp 32 + moov 919 + mdat 8 + length-prefixed slices: the avcC and tables
    have equal sizes at both QPs) and the pinned PSNR / SSIM / MS-SSIM averages.
    """
    from oracle_lib import ms_ssim_plane, psnr_plane, quality_report, ssim_plane

    meta = json.loads((GOLDEN / "golden.json").read_text())["cli_snapshots"]
    w, h = 160, 90
    r1 = []
    for g in range(2):
        enc = OracleEncoder(w, h, 20, keyint=16)
        for i in range(15):
            enc.encode(synth_video_frame(w, h, g * 15 + i))
            r1.append(_crop(enc.recon(), w, h))
    r2, payload = [], 0
    for g in range(2):
        enc = OracleEncoder(w, h, 30, keyint=16)
        for i in range(15):
            data, _ = enc.encode(r1[g * 15 + i])
            payload += sum(4 + len(n) for n in split_annex_b(data) if n[0] & 0x1F in (1, 5))
            r2.append(_crop(enc.recon(), w, h))
    assert 32 + 919 + 8 + payload == meta["transcode_qp30_mp4_bytes"]
    n = len(r1)
    psnr = [sum(psnr_plane(a[p], b[p]) for a, b in zip(r1, r2)) / n for p in range(3)]
    ssim = [sum(ssim_plane(a[p], b[p]) for a, b in zip(r1, r2)) / n for p in range(3)]
    ms = sum(ms_ssim_plane(a[0], b[0]) for a, b in zip(r1, r2)) / n
    m = meta["metrics"]
    assert round(psnr[0], 2) == m["psnr_y"]
    assert round(psnr[1], 2) == m["psnr_u"]
    assert round(psnr[2], 2) == m["psnr_v"]
    assert round(ssim[0], 5) == m["ssim_y"]
    assert round((4 * ssim[0] + ssim[1] + ssim[2]) / 6, 5) == m["ssim_avg"]
    assert round(ms, 5) == m["ms_ssim"]
    # the rest of the report (evaluate_media_metrics, crates/ragdoll-pipeline/src/lib.rs:2879: each
    # frame against the previous reference frame for VMAF-Lite's motion term, then the mean)
    reps = [quality_report(a, b, r1[i - 1] if i else None) for i, (a, b) in enumerate(zip(r1, r2))]
    for key, digits in (("psnr_avg", 2), ("psnr_yuv_611", 2), ("ssim_db", 2), ("vmaf_lite", 2)):
        assert round(sum(r[key] for r in reps) / n, digits) == m[key], key


def test_pixel_op_counter():
    """The oracle's count of integer work (pixel differences of every SAD / SSD / SATD its
    decisions evaluate -- the denominator of the kernel's integer-pipe figures) is deterministic
    and covers at least the three-way 16x16 SATD of every intra macroblock."""
    from oracle_lib import pixel_ops
    w, h = 96, 64
    frames = [synth_video_frame(w, h, i) for i in range(3)]
    counts = []
    for _ in range(2):
        enc = OracleEncoder(w, h, 26, profile=2, keyint=30)
        pixel_ops(reset=True)
        per = []
        for f in frames:
            enc.encode(f)
            per.append(pixel_ops(reset=True))
        counts.append(per)
    assert counts[0] == counts[1]
    assert counts[0][0] >= (w // 16) * (h // 16) * 3 * 256
    assert all(c > 0 for c in counts[0])
