"""Bitstreams from GPU decisions (GPU tests): the engine's records, written by the library's
writer, must give the reference corpus's NAL units byte for byte (CAVLC), and the oracle's access
units on the 1280x720 Baseline QP 30 configuration, on the 1920x1080 High QP 26 configuration
(CABAC, 8x8 transforms) and on batched Main-profile streams of the pipelined launch. The High
stream must also decode, through FFmpeg's H.264 decoder, to exactly the engine's reconstruction.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle_lib import OracleEncoder, read_nal_fixture, split_annex_b
from ragdoll_b200.synth import grating_clip, synth_video_frame

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("fixture,w,h,frames,fps", [
    ("clip_160x90_qp20.nal", 160, 90, 30, (30, 1)),
    ("clip_320x180_qp20.nal", 320, 180, 15, (25, 1)),
])
def test_gpu_records_reproduce_pinned_corpus(fixture, w, h, frames, fps):
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, CavlcWriter, Engine
    gold = read_nal_fixture(GOLDEN / fixture)
    eng = Engine(w, h, 20, profile=0)
    nals = []
    for g0 in range(0, frames, 15):
        wr = CavlcWriter(w, h, 20, fps=fps)
        for i in range(min(15, frames - g0)):
            kind = RG_FRAME_IDR if i == 0 else RG_FRAME_P
            recs = eng.analyse([synth_video_frame(w, h, g0 + i)], [kind])[0]
            nals += split_annex_b(wr.picture(recs, kind))
    params = [n for n in nals if n[0] & 0x1F in (7, 8)]
    slices = [n for n in nals if n[0] & 0x1F in (1, 5)]
    assert params[0] == gold[0] and params[1] == gold[1]
    assert len(slices) == len(gold) - 2
    for i, (a, b) in enumerate(zip(slices, gold[2:])):
        assert a == b, f"slice {i} differs"


def test_gpu_720p_baseline_bitstream_matches_oracle():
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, CavlcWriter, Engine
    w, h, qp = 1280, 720, 30
    frames = grating_clip(w, h, 5, seed=1001, motion=8.0, rects=6)
    eng = Engine(w, h, qp, profile=0)
    orc = OracleEncoder(w, h, qp, profile=0, keyint=30)
    wr = CavlcWriter(w, h, qp)
    for i, fr in enumerate(frames):
        want, _ = orc.encode(fr)
        kind = RG_FRAME_IDR if orc.last_idr else RG_FRAME_P
        got = wr.picture(eng.analyse([fr], [kind])[0], kind)
        assert got == want, f"picture {i}: {len(got)} vs {len(want)} bytes"


def test_gpu_pipelined_streams_bitstreams_match_oracle():
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, CavlcWriter, Engine
    w, h, qp, S, F = 320, 180, 28, 4, 6
    clips = [grating_clip(w, h, F, seed=40 + s, motion=8.0, rects=3) for s in range(S)]
    eng = Engine(w, h, qp, profile=0, num_streams=S, max_frames=F)
    kinds = [[RG_FRAME_IDR if f == 0 else RG_FRAME_P] * S for f in range(F)]
    recs = eng.analyse_gops([[clips[s][f] for s in range(S)] for f in range(F)], kinds)
    for s in range(S):
        orc = OracleEncoder(w, h, qp, profile=0, keyint=F + 1)
        wr = CavlcWriter(w, h, qp)
        for f in range(F):
            want, _ = orc.encode(clips[s][f])
            assert wr.picture(recs[f, s], kinds[f][s]) == want, f"stream {s} picture {f}"


def test_gpu_1080p_high_cabac_bitstream_matches_oracle_and_decodes():
    import ffmpeg_decode
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, BitstreamWriter, Engine
    w, h, qp = 1920, 1080, 26
    frames = grating_clip(w, h, 3, seed=2001, motion=24.0, rects=12)
    eng = Engine(w, h, qp, profile=2)
    orc = OracleEncoder(w, h, qp, profile=2, keyint=15)
    wr = BitstreamWriter(w, h, qp, profile=2)
    aus, recons = [], []
    for i, fr in enumerate(frames):
        want, _ = orc.encode(fr)
        kind = RG_FRAME_IDR if orc.last_idr else RG_FRAME_P
        got = wr.picture(eng.analyse([fr], [kind])[0], kind)
        assert got == want, f"picture {i}: {len(got)} vs {len(want)} bytes"
        aus.append(got)
        recons.append([p.copy() for p in eng.recon_coded(0)])
    if not ffmpeg_decode.available():
        pytest.skip("FFmpeg libraries not found")
    for i, (p, r) in enumerate(zip(ffmpeg_decode.decode(aus), recons)):
        for k in range(3):
            assert np.array_equal(p[k], r[k][:p[k].shape[0], :p[k].shape[1]]), f"picture {i} plane {k}"


def test_gpu_pipelined_main_streams_bitstreams_match_oracle():
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, BitstreamWriter, Engine
    w, h, qp, S, F = 320, 180, 28, 4, 6
    clips = [grating_clip(w, h, F, seed=50 + s, motion=8.0, rects=3) for s in range(S)]
    eng = Engine(w, h, qp, profile=1, num_streams=S, max_frames=F)
    kinds = [[RG_FRAME_IDR if f == 0 else RG_FRAME_P] * S for f in range(F)]
    recs = eng.analyse_gops([[clips[s][f] for s in range(S)] for f in range(F)], kinds)
    for s in range(S):
        orc = OracleEncoder(w, h, qp, profile=1, keyint=F + 1)
        wr = BitstreamWriter(w, h, qp, profile=1)
        for f in range(F):
            want, _ = orc.encode(clips[s][f])
            assert wr.picture(recs[f, s], kinds[f][s]) == want, f"stream {s} picture {f}"
