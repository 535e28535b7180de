"""The launch-shape autotuner (GPU tests).

* It times every candidate shape on a sample wave and returns the fastest, as tuning keywords.
* The shape changes the time only: an encoder running the tuned shape writes the oracle's access
  units, and an engine gives the same records under every candidate.
"""
import numpy as np
import pytest

from oracle_lib import OracleEncoder
from ragdoll_b200.synth import grating_clip

pytestmark = pytest.mark.gpu


def test_autotune_picks_a_candidate_and_keeps_the_results():
    from ragdoll_b200.autotune import autotune_pipeline
    from ragdoll_b200.encoder import H264Encoder
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, Engine
    w, h, qp, S, F = 128, 80, 28, 3, 4
    clips = [grating_clip(w, h, 2 * F, seed=600 + s, motion=5.0, rects=2) for s in range(S)]
    wave = [[clips[s][f] for s in range(S)] for f in range(F)]
    kinds = [[RG_FRAME_IDR if f == 0 else RG_FRAME_P] * S for f in range(F)]
    cands = [{"per_sm": 2, "seg": 1}, {"per_sm": 8, "seg": 2}, {"per_sm": 16, "seg": 1}]
    tuning, table = autotune_pipeline(w, h, qp, 2, wave, kinds, candidates=cands, repeats=2)
    assert [c for c, _ in table] == cands and all(ms > 0 for _, ms in table)
    best = min(table, key=lambda t: t[1])[0]
    assert tuning["seg"] == best["seg"] and tuning["grid"] % best["per_sm"] == 0
    # same records under every candidate
    ref = None
    for c in cands:
        eng = Engine(w, h, qp, profile=2, num_streams=S, max_frames=F)
        eng.set_pipeline_tuning(seg=c["seg"], grid=c["per_sm"] * 4)
        recs = eng.analyse_gops(wave, kinds)
        ref = recs if ref is None else ref
        assert recs.tobytes() == ref.tobytes(), c
    # an encoder on the tuned shape writes the oracle's access units
    enc = H264Encoder(w, h, qp, profile=2, keyint=30, streams=S, max_frames=F, threads=2)
    enc.set_pipeline_tuning(**tuning)
    enc.submit(wave)
    got = enc.collect()
    for s in range(S):
        orc = OracleEncoder(w, h, qp, profile=2, keyint=30)
        for f in range(F):
            assert got[f][s] == orc.encode(clips[s][f])[0], f"stream {s} picture {f}"
