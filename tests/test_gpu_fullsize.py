"""Parity at the full sizes of the benchmark configurations (GPU tests).

* 1280x720 Constrained Baseline QP 30 (global motion +-8 px, 6 rectangles): every record field
  and both reconstructions identical to the oracle, picture by picture.
* 1920x1080 High QP 26 (global motion +-24 px, 12 rectangles): the same on the first pictures
  of a GOP (IDR + P).
* 1920x1080, 8 GOPs x 5 pictures: the persistent pipelined launch and the per-diagonal launches
  give identical records and deblocked references (two independent schedules of the same
  wavefront), and a second pipelined run repeats the first bit for bit.
"""
import numpy as np
import pytest

from gpu_parity_util import run_parity
from ragdoll_b200.synth import grating_clip

pytestmark = pytest.mark.gpu


def test_720p_baseline_qp30_matches_oracle():
    from ragdoll_b200.engine import Engine
    w, h, qp = 1280, 720, 30
    frames = grating_clip(w, h, 5, seed=1001, motion=8.0, rects=6)
    eng = Engine(w, h, qp, profile=0)
    eng.keep_unfiltered(True)
    fails = run_parity(frames, w, h, qp, 0, keyint=30, engine=eng)
    assert not fails, "\n".join(fails)


def test_1080p_high_qp26_matches_oracle():
    from ragdoll_b200.engine import Engine
    w, h, qp = 1920, 1080, 26
    frames = grating_clip(w, h, 3, seed=2001, motion=24.0, rects=12)
    eng = Engine(w, h, qp, profile=2)
    eng.keep_unfiltered(True)
    fails = run_parity(frames, w, h, qp, 2, keyint=15, engine=eng)
    assert not fails, "\n".join(fails)


def test_1080p_pipelined_equals_per_diagonal_and_repeats():
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, Engine
    w, h, qp, gops, nf = 1920, 1080, 26, 8, 5
    clips = [grating_clip(w, h, nf, seed=3000 + g, motion=24.0, rects=12) for g in range(gops)]
    kinds = [[RG_FRAME_IDR if f == 0 else RG_FRAME_P] * gops for f in range(nf)]
    pics = [[clips[g][f] for g in range(gops)] for f in range(nf)]

    diag = Engine(w, h, qp, profile=2, num_streams=gops)
    want = np.stack([diag.analyse(pics[f], kinds[f]) for f in range(nf)])
    want_ref = [diag.recon_coded(g) for g in range(gops)]

    pipe = Engine(w, h, qp, profile=2, num_streams=gops, max_frames=nf)
    for run in range(2):
        got = pipe.analyse_gops(pics, kinds)
        assert got.tobytes() == want.tobytes(), f"run {run}: records differ"
        for g in range(gops):
            for a, b in zip(want_ref[g], pipe.recon_coded(g)):
                assert np.array_equal(a, b), f"run {run}: stream {g} reference picture differs"
        # the next run starts a new GOP on every stream (IDR first), from the same input
