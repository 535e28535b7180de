"""The encoder (GPU engine + host writer) against the oracle (GPU tests).

* encode_frame, stream by stream across an IDR boundary: every access unit equals the oracle's
  (CAVLC Baseline and CABAC High).
* submit / collect with two waves in flight (the GPU analyses one wave while the host writes the
  other): every access unit of every stream equals the oracle's, and one stream, muxed to MP4 and
  demuxed, decodes through FFmpeg to exactly the oracle's reconstruction; every picture's
  submit-to-written latency is reported and bounded by the wall time since its submit.
* Calls out of order are refused without disturbing the streams.
"""
import numpy as np
import pytest

from oracle_lib import OracleEncoder
from ragdoll_b200.synth import grating_clip

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("profile,qp", [(0, 30), (2, 26), (1, 34)])
def test_encode_frame_matches_oracle(profile, qp):
    from ragdoll_b200.encoder import H264Encoder
    w, h, S, N, keyint = 176, 144, 2, 7, 4
    clips = [grating_clip(w, h, N, seed=70 + s + qp, motion=6.0, rects=2) for s in range(S)]
    enc = H264Encoder(w, h, qp, profile=profile, keyint=keyint, streams=S)
    orcs = [OracleEncoder(w, h, qp, profile=profile, keyint=keyint) for _ in range(S)]
    for i in range(N):
        for s in range(S):
            want, _ = orcs[s].encode(clips[s][i])
            assert enc.encode_frame(clips[s][i], stream=s) == want, f"stream {s} picture {i}"


def test_waves_in_flight_match_oracle_and_decode():
    import ffmpeg_decode
    from ragdoll_b200.containers import Demuxer, mux
    from ragdoll_b200.encoder import H264Encoder
    w, h, qp, S, F, waves, keyint = 320, 180, 26, 3, 5, 3, 8
    clips = [grating_clip(w, h, F * waves, seed=90 + s, motion=8.0, rects=3) for s in range(S)]
    enc = H264Encoder(w, h, qp, profile=2, keyint=keyint, streams=S, max_frames=F, threads=4)
    got, t_sub = [], []
    import time
    for k in range(waves):
        t_sub.append(time.perf_counter())
        enc.submit([[clips[s][k * F + f] for s in range(S)] for f in range(F)])
        if k >= 1:
            got += enc.collect()
            lat = enc.latencies()   # of wave k - 1: submit -> access unit written, per picture
            assert lat.shape == (F, S) and (lat > 0).all()
            assert lat.max() <= 1000 * (time.perf_counter() - t_sub[k - 1]) + 1
    got += enc.collect()
    assert len(got) == F * waves
    for s in range(S):
        orc = OracleEncoder(w, h, qp, profile=2, keyint=keyint)
        recons = []
        for i in range(F * waves):
            want, _ = orc.encode(clips[s][i])
            assert got[i][s] == want, f"stream {s} picture {i}"
            recons.append([p.copy() for p in orc.recon()])
        if s == 0 and ffmpeg_decode.available():
            aus = Demuxer(mux("mp4", w, h, [got[i][0] for i in range(F * waves)])).access_units()
            for i, (p, r) in enumerate(zip(ffmpeg_decode.decode(aus), recons)):
                for c in range(3):
                    assert np.array_equal(p[c], r[c][:p[c].shape[0], :p[c].shape[1]]), f"picture {i} plane {c}"


def test_out_of_order_calls_are_refused():
    from ragdoll_b200.encoder import H264Encoder
    from ragdoll_b200.engine import RgError
    w, h = 64, 48
    clip = grating_clip(w, h, 8, seed=3, motion=2.0, rects=1)
    enc = H264Encoder(w, h, 28, profile=1, keyint=30, streams=1, max_frames=2, threads=2)
    with pytest.raises(RgError):
        enc.collect()
    enc.submit([[clip[0]], [clip[1]]])
    enc.submit([[clip[2]], [clip[3]]])
    with pytest.raises(RgError):
        enc.submit([[clip[4]]])                 # a third wave
    with pytest.raises(RgError):
        enc.encode_frame(clip[4])               # waves in flight
    with pytest.raises(RgError):
        enc.submit([[clip[4]]] * 3)             # more pictures than max_frames
    a = enc.collect() + enc.collect()
    b = [[enc.encode_frame(clip[i])] for i in range(4, 8)]
    orc = OracleEncoder(w, h, 28, profile=1, keyint=30)
    for i, row in enumerate(a + b):
        assert row[0] == orc.encode(clip[i])[0], f"picture {i}"


def test_mixed_sizes_and_qps_like_the_batched_configuration():
    """The batched-streams configuration scaled down: four picture sizes, four streams each,
    Main profile (CABAC), a QP drawn from 20..36 per stream -- one encoder per size, each stream at
    its own QP in the same launches; every access unit equals the oracle's."""
    from ragdoll_b200.encoder import H264Encoder
    rng = np.random.default_rng(64)
    sizes, per_size, F = [(64, 48), (160, 96), (320, 180), (352, 288)], 4, 3
    for (w, h) in sizes:
        qps = [int(q) for q in rng.integers(20, 37, per_size)]
        clips = [grating_clip(w, h, F, seed=w + h + s, motion=4.0, rects=2) for s in range(per_size)]
        enc = H264Encoder(w, h, 28, profile=1, keyint=30, streams=per_size, max_frames=F, threads=4)
        for s, q in enumerate(qps):
            enc.set_stream_qp(s, q)
        enc.submit([[clips[s][f] for s in range(per_size)] for f in range(F)])
        got = enc.collect()
        for s, q in enumerate(qps):
            orc = OracleEncoder(w, h, q, profile=1, keyint=30)
            for f in range(F):
                assert got[f][s] == orc.encode(clips[s][f])[0], f"{w}x{h} stream {s} (QP {q}) picture {f}"
        with pytest.raises(Exception):
            enc.set_stream_qp(0, 30)              # the stream has pictures already
