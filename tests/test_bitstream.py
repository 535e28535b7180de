"""The library's CAVLC writer (host code, no GPU) against the reference corpus.

Fed the macroblock records the oracle chose for the reference corpus clips, the product writer
must emit exactly the pinned SPS, PPS and slice NAL units of qa/corpus/synth/clip_160x90_30fps.mp4
and clip_320x180_25fps.mkv (two / one 15-picture GOPs, QP 20, Baseline), and exactly the oracle's
bytes on grating clips with every macroblock kind at several QPs and sizes. GPU records go through
the same writer in test_gpu_bitstream.py.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle_lib import OracleEncoder, read_nal_fixture, split_annex_b
from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, CavlcWriter, RgError
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


def test_writer_rejects_cabac_profiles_and_bad_calls():
    from ragdoll_b200.engine import RECORD_DTYPE, RgConfig, lib
    import ctypes
    cfg = RgConfig(64, 64, 2, 26, 1, 0, 1)
    assert not lib().rg_writer_create(ctypes.byref(cfg), 30, 1)
    assert b"CABAC" in lib().rg_last_error()
    wr = CavlcWriter(64, 64, 26)
    with pytest.raises(RgError):
        wr.picture(np.zeros(16, RECORD_DTYPE), RG_FRAME_P)  # P before any IDR
