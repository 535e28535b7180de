"""Bit-exact parity of the sm_100a engine with the CPU oracle (GPU tests).

Every record field (macroblock type, modes, vectors, coded block pattern, every level), the
reconstruction before deblocking and the deblocked reference picture must be identical after
every frame, for I and P frames, Baseline / Main / High (8x8 transform decision), at several
QPs and at picture sizes that are not macroblock multiples (edge replication of the source,
picture-edge availability, MvBounds at the borders).
"""
import numpy as np
import pytest

from gpu_parity_util import run_parity
from ragdoll_b200.synth import grating_clip, synth_video_frame

pytestmark = pytest.mark.gpu


def _engine(w, h, qp, profile, streams=1):
    from ragdoll_b200.engine import Engine
    e = Engine(w, h, qp, profile=profile, num_streams=streams)
    e.keep_unfiltered(True)
    return e


@pytest.mark.parametrize("qp", [20, 30])
def test_corpus_clip_parity(qp):
    w, h = 160, 90
    frames = [synth_video_frame(w, h, i) for i in range(8)]
    eng = _engine(w, h, qp, 0)
    fails = run_parity(frames, w, h, qp, 0, keyint=16, engine=eng)
    assert not fails, "\n".join(fails)


@pytest.mark.parametrize("w,h,qp,profile", [
    (176, 144, 26, 2),
    (208, 120, 22, 0),
    (250, 138, 34, 2),
    (96, 64, 40, 1),
    (320, 176, 12, 2),
])
def test_grating_parity(w, h, qp, profile):
    frames = grating_clip(w, h, 6, seed=7 + w + qp, motion=6.0, rects=3)
    eng = _engine(w, h, qp, profile)
    fails = run_parity(frames, w, h, qp, profile, keyint=4, engine=eng)
    assert not fails, "\n".join(fails)


def test_batched_streams_match_single():
    """Streams analysed side by side in one wavefront give the same records as alone."""
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, Engine
    w, h, qp = 128, 80, 28
    clips = [grating_clip(w, h, 3, seed=s, motion=4.0, rects=2) for s in range(3)]
    batch = Engine(w, h, qp, profile=2, num_streams=3)
    solo = [Engine(w, h, qp, profile=2) for _ in range(3)]
    for f in range(3):
        kind = RG_FRAME_IDR if f == 0 else RG_FRAME_P
        rb = batch.analyse([c[f] for c in clips], [kind] * 3)
        for s in range(3):
            rs = solo[s].analyse([clips[s][f]], [kind])[0]
            assert rb[s].tobytes() == rs.tobytes()
            assert all(np.array_equal(a, b) for a, b in zip(batch.recon(s), solo[s].recon()))
