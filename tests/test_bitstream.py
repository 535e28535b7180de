"""The library's bitstream writer (host code, no GPU) against the reference corpus and the oracle.

* CAVLC (Baseline): fed the macroblock records the oracle chose for the reference corpus clips,
  the product writer must emit exactly the pinned SPS, PPS and slice NAL units of
  qa/corpus/synth/clip_160x90_30fps.mp4 and clip_320x180_25fps.mkv (two / one 15-picture GOPs,
  QP 20), and exactly the oracle's bytes on grating clips at several QPs and sizes.
* CABAC (Main, High with 8x8 transforms): the product writer (the arithmetic coder of the
  standard, per-macroblock context summaries) and the oracle (a restatement of the reference's
  cabac.rs engine and h264.rs / enc.rs glue) must give the same bytes; the reference holds no
  CABAC output of its own encoder, so both are further pinned by decoding: FFmpeg's H.264 decoder
  must turn the stream into exactly the oracle's reconstruction, every plane of every picture.
GPU records go through the same writer in test_gpu_bitstream.py.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle_lib import OracleEncoder, read_nal_fixture, split_annex_b
from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, BitstreamWriter, CavlcWriter, RgError
from ragdoll_b200.synth import grating_clip, synth_video_frame

GOLDEN = Path(__file__).resolve().parent / "golden"


def writer_gops(width, height, frames, qp, fps, gop=15):
    """Oracle decisions, product bitstream: one oracle and one writer per GOP."""
    nals = []
    for g0 in range(0, len(frames), gop):
        n = min(gop, len(frames) - g0)
        orc = OracleEncoder(width, height, qp, profile=0, keyint=n + 1, fps=fps)
        wr = CavlcWriter(width, height, qp, fps=fps)
        for i in range(n):
            ref_bytes, recs = orc.encode(frames[g0 + i])
            au = wr.picture(recs, RG_FRAME_IDR if orc.last_idr else RG_FRAME_P)
            assert au == ref_bytes, f"picture {g0 + i}: writer {len(au)} B, oracle {len(ref_bytes)} B"
            nals += split_annex_b(au)
    return nals


@pytest.mark.parametrize("fixture,w,h,frames,fps", [
    ("clip_160x90_qp20.nal", 160, 90, 30, (30, 1)),
    ("clip_320x180_qp20.nal", 320, 180, 15, (25, 1)),
])
def test_writer_reproduces_pinned_corpus(fixture, w, h, frames, fps):
    gold = read_nal_fixture(GOLDEN / fixture)
    nals = writer_gops(w, h, [synth_video_frame(w, h, i) for i in range(frames)], 20, fps)
    params = [n for n in nals if n[0] & 0x1F in (7, 8)]
    slices = [n for n in nals if n[0] & 0x1F in (1, 5)]
    assert params[0] == gold[0] and params[1] == gold[1]
    assert len(slices) == len(gold) - 2
    for i, (a, b) in enumerate(zip(slices, gold[2:])):
        assert a == b, f"slice {i} differs"


@pytest.mark.parametrize("w,h,qp", [(176, 144, 12), (208, 120, 26), (250, 138, 40), (96, 64, 51)])
def test_writer_matches_oracle_bytes(w, h, qp):
    frames = grating_clip(w, h, 6, seed=w + qp, motion=6.0, rects=3)
    writer_gops(w, h, frames, qp, (30, 1), gop=4)


def test_writer_rejects_bad_calls():
    from ragdoll_b200.engine import RECORD_DTYPE, RgConfig, lib
    import ctypes
    cfg = RgConfig(64, 64, 7, 26, 1, 0, 1)
    assert not lib().rg_writer_create(ctypes.byref(cfg), 30, 1)
    assert b"profile" in lib().rg_last_error()
    for profile in (0, 2):
        wr = BitstreamWriter(64, 64, 26, profile=profile)
        with pytest.raises(RgError):
            wr.picture(np.zeros(16, RECORD_DTYPE), RG_FRAME_P)  # P before any IDR
        recs = np.zeros(16, RECORD_DTYPE)
        recs["mb_type"] = 0  # P_Skip
        with pytest.raises(RgError):
            wr.picture(recs, RG_FRAME_IDR)                    # P_Skip in an IDR picture


def cabac_gop(w, h, qp, profile, frames, keyint):
    """Oracle decisions and bytes, product bytes, oracle reconstructions."""
    orc = OracleEncoder(w, h, qp, profile=profile, keyint=keyint)
    wr = BitstreamWriter(w, h, qp, profile=profile)
    aus, recons = [], []
    for i, fr in enumerate(frames):
        want, recs = orc.encode(fr)
        got = wr.picture(recs, RG_FRAME_IDR if orc.last_idr else RG_FRAME_P)
        assert got == want, f"picture {i}: writer {len(got)} B, oracle {len(want)} B"
        aus.append(got)
        recons.append([p.copy() for p in orc.recon()])
    return aus, recons


@pytest.mark.parametrize("w,h,qp,profile", [
    (176, 144, 26, 1), (176, 144, 26, 2), (208, 120, 12, 2), (250, 138, 30, 2),
    (96, 64, 40, 1), (64, 48, 51, 2), (48, 32, 1, 2), (16, 16, 22, 2),
])
def test_cabac_writer_matches_oracle_and_decodes(w, h, qp, profile):
    import ffmpeg_decode
    frames = grating_clip(w, h, 7, seed=5 + w + qp, motion=6.0, rects=2)
    aus, recons = cabac_gop(w, h, qp, profile, frames, keyint=4)
    for n in split_annex_b(aus[0])[:1]:
        assert n[1] == (77 if profile == 1 else 100)          # profile_idc
    if not ffmpeg_decode.available():
        pytest.skip("FFmpeg libraries not found")
    pics = ffmpeg_decode.decode(aus)
    assert len(pics) == len(recons)
    for i, (p, r) in enumerate(zip(pics, recons)):
        for k in range(3):
            assert np.array_equal(p[k], r[k][:p[k].shape[0], :p[k].shape[1]]), f"picture {i} plane {k}"


def test_cabac_streams_use_every_syntax_path():
    """The clips above reach 8x8 transforms, I_4x4 / I_16x16 / P_Skip / P_L0_16x16 macroblocks,
    levels beyond the unary prefix (>= 15) and vectors beyond the mvd prefix (|mvd| >= 9)."""
    seen = {"t8": 0, "big_level": 0, "big_mvd": 0, "types": set()}
    for w, h, qp in ((208, 120, 12), (176, 144, 26), (48, 32, 1)):
        orc = OracleEncoder(w, h, qp, profile=2, keyint=4)
        for fr in grating_clip(w, h, 7, seed=5 + w + qp, motion=6.0, rects=2):
            _, recs = orc.encode(fr)
            seen["t8"] += int((recs["transform_8x8"] != 0).sum())
            seen["big_level"] += int((np.abs(recs["luma"]) >= 15).sum())
            seen["big_mvd"] += int((np.abs(recs["mvd"]) >= 9).sum())
            seen["types"] |= set(int(t) for t in recs["mb_type"])
    assert seen["t8"] and seen["big_level"] and seen["big_mvd"]
    assert len(seen["types"]) == 4
