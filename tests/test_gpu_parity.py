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


@pytest.mark.parametrize("w,h,qp,profile,streams,frames,tuning", [
    (176, 144, 26, 2, 3, 5, {}),
    (250, 138, 30, 0, 2, 4, {}),
    (64, 32, 22, 1, 4, 6, {}),
    (176, 144, 26, 2, 3, 5, {"deblock_sms": -1, "seg": 8}),
    (208, 120, 24, 2, 2, 5, {"deblock_sms": 16, "grid": 64, "lag": 40}),
    (176, 144, 26, 2, 3, 5, {"deblock_sms": 20, "intra_sms": 40}),
    (176, 144, 26, 2, 3, 5, {"deblock_sms": 3, "intra_sms": 2, "grid": 100}),
    (16, 16, 26, 2, 2, 3, {}),                  # one macroblock
    (48, 16, 28, 1, 2, 3, {}),                  # one row
    (16, 64, 30, 0, 2, 3, {"grid": 8}),         # one column
])
def test_pipelined_gops_match_oracle(w, h, qp, profile, streams, frames, tuning):
    """One persistent launch for all pictures of several GOPs (pictures of a GOP overlapping)
    gives the oracle's records and deblocked reconstruction for every picture -- with separate
    analysis / deblocking queues (default) or one mixed queue, at several segment lengths, lags
    and grid sizes."""
    from oracle_lib import OracleEncoder
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, Engine
    from gpu_parity_util import first_record_mismatch, first_pixel_mismatch

    clips = [grating_clip(w, h, frames, seed=100 + 7 * s + w, motion=6.0, rects=2) for s in range(streams)]
    eng = Engine(w, h, qp, profile=profile, num_streams=streams, max_frames=frames)
    if tuning:
        eng.set_pipeline_tuning(**tuning)
    kinds = [[RG_FRAME_IDR if f == 0 else RG_FRAME_P] * streams for f in range(frames)]
    recs = eng.analyse_gops([[clips[s][f] for s in range(streams)] for f in range(frames)], kinds)
    for s in range(streams):
        orc = OracleEncoder(w, h, qp, profile=profile, keyint=frames + 1)
        for f in range(frames):
            _, ref = orc.encode(clips[s][f])
            m = first_record_mismatch(ref, recs[f, s], orc.mb_w)
            assert m is None, f"stream {s} picture {f}: {m}"
        # the last picture's reference (deblocked, coded size) stays on the device
        for p, (a, b) in enumerate(zip(orc.recon(True), eng.recon_coded(s))):
            assert first_pixel_mismatch(a, b) is None, f"stream {s} plane {p}"
    # a second call continues the streams with P pictures from the kept references
    more = [grating_clip(w, h, 2, seed=900 + s, motion=3.0, rects=1) for s in range(streams)]
    eng.analyse_gops([[more[s][f] for s in range(streams)] for f in range(2)], [[RG_FRAME_P] * streams] * 2)


def test_pipelined_wait_timeout_falls_back_to_exact_path():
    """Failure detection without a GPU fault: one resident warp and a lag of one macroblock-time
    make a picture's first segment wait for deblocking of the previous picture that no warp will
    ever take (a flag nothing sets). The wait gives up after 300 ms, the launch stops with an
    error status the host reads, and the call is re-run on the per-diagonal path: results stay
    exact, the context usable."""
    from oracle_lib import OracleEncoder
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, Engine
    from gpu_parity_util import first_record_mismatch

    w, h, qp, frames = 96, 96, 28, 3
    clip = grating_clip(w, h, frames, seed=77, motion=4.0, rects=1)
    eng = Engine(w, h, qp, profile=2, num_streams=1, max_frames=frames)
    eng.set_pipeline_tuning(lag=1, grid=1, timeout_ms=300)
    recs = eng.analyse_gops([[clip[f]] for f in range(frames)], [[RG_FRAME_IDR]] + [[RG_FRAME_P]] * (frames - 1))
    orc = OracleEncoder(w, h, qp, profile=2, keyint=frames + 1)
    for f in range(frames):
        _, ref = orc.encode(clip[f])
        assert first_record_mismatch(ref, recs[f, 0], orc.mb_w) is None
    eng.set_pipeline_tuning()
    more = grating_clip(w, h, 2, seed=78, motion=4.0, rects=1)
    eng.analyse_gops([[more[0]], [more[1]]], [[RG_FRAME_P], [RG_FRAME_P]])


def test_async_gops_match_sync_and_recover_from_timeout():
    """Asynchronous host-buffer calls, queued back to back into alternating output buffers, give
    the records of the synchronous call; a call whose wait is made to run out (one warp, lag 1)
    is re-run before the next call starts, and its records in the caller's buffer are exact."""
    from ragdoll_b200.engine import RECORD_DTYPE, RG_FRAME_IDR, RG_FRAME_P, Engine
    w, h, qp, S, F = 176, 144, 26, 3, 4
    clips = [grating_clip(w, h, 2 * F, seed=500 + s, motion=5.0, rects=2) for s in range(S)]
    batches = [[[clips[s][b * F + f] for s in range(S)] for f in range(F)] for b in range(2)]
    kinds = [[[RG_FRAME_IDR if (b == 0 and f == 0) else RG_FRAME_P] * S for f in range(F)] for b in range(2)]

    sync = Engine(w, h, qp, profile=2, num_streams=S, max_frames=F)
    want = [sync.analyse_gops(batches[b], kinds[b]) for b in range(2)]

    for tuning in ({}, {"lag": 1, "grid": 1, "timeout_ms": 300}):
        eng = Engine(w, h, qp, profile=2, num_streams=S, max_frames=F)
        if tuning:
            eng.set_pipeline_tuning(**tuning)
        outs = [np.zeros((F, S, eng.n_mb), RECORD_DTYPE) for _ in range(2)]
        for b in range(2):
            eng.analyse_gops_async(batches[b], kinds[b], outs[b])
        eng.sync()
        for b in range(2):
            assert outs[b].tobytes() == want[b].tobytes(), f"{tuning} batch {b}"
        for s in range(S):
            for a, c in zip(sync.recon_coded(s), eng.recon_coded(s)):
                assert np.array_equal(a, c)


@pytest.mark.parametrize("w,h,qp,profile", [
    (16, 16, 26, 2),     # one macroblock
    (48, 16, 30, 0),     # one row of three
    (16, 64, 22, 1),     # one column of four
    (33, 17, 1, 2),      # ragged in both directions, lowest QP
    (72, 40, 51, 2),     # highest QP
    (80, 48, 1, 0),      # lowest QP, Baseline
])
def test_edge_shapes_and_qps(w, h, qp, profile):
    frames = grating_clip(w, h, 4, seed=w * 7 + h + qp, motion=5.0, rects=1)
    eng = _engine(w, h, qp, profile)
    fails = run_parity(frames, w, h, qp, profile, keyint=3, engine=eng)
    assert not fails, "\n".join(fails)


def test_pipelined_many_small_streams():
    """32 streams of 48x32 pictures in one persistent launch: every picture equals the oracle."""
    from oracle_lib import OracleEncoder
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, Engine
    from gpu_parity_util import first_record_mismatch
    w, h, qp, S, F = 48, 32, 28, 32, 4
    clips = [grating_clip(w, h, F, seed=3000 + s, motion=3.0, rects=1) for s in range(S)]
    eng = Engine(w, h, qp, profile=2, num_streams=S, max_frames=F)
    kinds = [[RG_FRAME_IDR if f == 0 else RG_FRAME_P] * S for f in range(F)]
    recs = eng.analyse_gops([[clips[s][f] for s in range(S)] for f in range(F)], kinds)
    for s in range(S):
        orc = OracleEncoder(w, h, qp, profile=2, keyint=F + 1)
        for f in range(F):
            _, ref = orc.encode(clips[s][f])
            assert first_record_mismatch(ref, recs[f, s], orc.mb_w) is None, f"stream {s} picture {f}"


@pytest.mark.parametrize("pipelined", [False, True])
def test_streams_of_different_qps_in_one_launch(pipelined):
    """Four streams at QP 20 / 26 / 31 / 36 (rg_set_stream_qp) analysed together, per-diagonal
    and in one persistent launch: each equals the oracle at its own QP."""
    from oracle_lib import OracleEncoder
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, Engine
    from gpu_parity_util import first_record_mismatch
    w, h, F, qps = 160, 96, 4, [20, 26, 31, 36]
    S = len(qps)
    clips = [grating_clip(w, h, F, seed=600 + s, motion=5.0, rects=2) for s in range(S)]
    eng = Engine(w, h, 28, profile=2, num_streams=S, max_frames=F if pipelined else 1)
    for s, q in enumerate(qps):
        eng.set_stream_qp(s, q)
    kinds = [[RG_FRAME_IDR if f == 0 else RG_FRAME_P] * S for f in range(F)]
    if pipelined:
        recs = eng.analyse_gops([[clips[s][f] for s in range(S)] for f in range(F)], kinds)
    else:
        recs = np.stack([eng.analyse([clips[s][f] for s in range(S)], kinds[f]) for f in range(F)])
    for s, q in enumerate(qps):
        orc = OracleEncoder(w, h, q, profile=2, keyint=F + 1)
        for f in range(F):
            _, ref = orc.encode(clips[s][f])
            assert first_record_mismatch(ref, recs[f, s], orc.mb_w) is None, f"stream {s} (QP {q}) picture {f}"
        assert np.array_equal(orc.recon()[0], eng.recon_coded(s)[0]), f"stream {s} reference picture"


@pytest.mark.parametrize("give_up", [False, True])
def test_streamed_records_arrive_per_picture_and_match(give_up):
    """rg_analyse_gops_stream / _fetch: every picture's records, fetched as soon as the launch flags
    them final (while it still runs), equal those of the bulk call; fetching out of range or
    without a call is refused. give_up: one warp and a lag of one macroblock-time make a wait run
    out (no fault); fetch then reports the unfinished pictures (2) and rg_analyse_gops_wait re-runs
    the call, after which every record is exact."""
    import ctypes
    from ragdoll_b200.engine import RECORD_DTYPE, RG_FRAME_IDR, RG_FRAME_P, Engine, lib
    w, h, qp, S, F = 320, 180, 26, 4, 6
    clips = [grating_clip(w, h, F, seed=700 + s, motion=6.0, rects=2) for s in range(S)]
    pics = [[clips[s][f] for s in range(S)] for f in range(F)]
    kinds = [[RG_FRAME_IDR if f == 0 else RG_FRAME_P] * S for f in range(F)]
    bulk = Engine(w, h, qp, profile=2, num_streams=S, max_frames=F).analyse_gops(pics, kinds)
    eng = Engine(w, h, qp, profile=2, num_streams=S, max_frames=F)
    if give_up:
        eng.set_pipeline_tuning(lag=1, grid=1, timeout_ms=300)
    out = np.zeros((F, S, eng.n_mb), RECORD_DTYPE)
    planes = [np.ascontiguousarray(p) for f in range(F) for s in range(S) for p in pics[f][s]]
    ptrs = (ctypes.c_void_p * len(planes))(*[p.ctypes.data for p in planes])
    k = (ctypes.c_int32 * (F * S))(*[kinds[f][s] for f in range(F) for s in range(S)])
    L = lib()
    assert L.rg_analyse_gops_fetch(eng.h, out.ctypes.data, 0) < 0          # no call yet
    assert L.rg_analyse_gops_stream(eng.h, ptrs, w, (w + 1) // 2, k, F, out.ctypes.data) == 0
    assert L.rg_analyse_gops_fetch(eng.h, out.ctypes.data, F * S) < 0      # out of range
    done, unfinished = set(), set()
    while len(done) + len(unfinished) < F * S:
        for i in range(F * S):
            if i not in done and i not in unfinished:
                st = L.rg_analyse_gops_fetch(eng.h, out.ctypes.data, i)
                assert st in (0, 1, 2), st
                if st == 1:
                    done.add(i)
                elif st == 2:
                    unfinished.add(i)
    assert bool(unfinished) == give_up
    assert L.rg_analyse_gops_wait(eng.h, out.ctypes.data) == 0
    assert out.tobytes() == bulk.tobytes()


def test_source_layouts_give_the_same_records():
    """Host sources as separate planes, as one Y|U|V buffer per picture (copied in one piece) and
    with padded rows (2-D copies), through the synchronous and the asynchronous host-buffer calls:
    the same records every time."""
    from ragdoll_b200.engine import RECORD_DTYPE, RG_FRAME_IDR, RG_FRAME_P, Engine
    w, h, qp, S, F = 96, 64, 27, 2, 3
    cw, ch = w // 2, h // 2
    clips = [grating_clip(w, h, F, seed=321 + s, motion=5.0, rects=1) for s in range(S)]
    kinds = [[RG_FRAME_IDR if f == 0 else RG_FRAME_P] * S for f in range(F)]

    def packed(y, u, v):
        buf = np.concatenate([y.reshape(-1), u.reshape(-1), v.reshape(-1)])
        return buf[:w * h].reshape(h, w), buf[w * h:w * h + cw * ch].reshape(ch, cw), buf[w * h + cw * ch:].reshape(ch, cw)

    def padded(y, u, v):
        out = []
        for p in (y, u, v):
            wide = np.zeros((p.shape[0], p.shape[1] + 32), np.uint8)
            wide[:, :p.shape[1]] = p
            out.append(wide[:, :p.shape[1]])
        return tuple(out)

    layouts = {"planes": lambda y, u, v: (y, u, v), "packed": packed, "padded": padded}
    got = {}
    for name, lay in layouts.items():
        frames = [[lay(*clips[s][f]) for s in range(S)] for f in range(F)]
        got[name + "/sync"] = Engine(w, h, qp, profile=2, num_streams=S, max_frames=F).analyse_gops(frames, kinds)
        eng = Engine(w, h, qp, profile=2, num_streams=S, max_frames=F)
        out = np.zeros((F, S, eng.n_mb), RECORD_DTYPE)
        eng.analyse_gops_async(frames, kinds, out)
        eng.sync()
        got[name + "/async"] = out
    ref = got["planes/sync"]
    for k, v in got.items():
        assert v.tobytes() == ref.tobytes(), k


def test_derived_lag_follows_the_reach_of_the_searches():
    """With lag 0 the work order's picture lag follows the reach of the searches: 24 (reach 4 x 4,
    one-macroblock segments) for the first launch, 15 after two launches of still pictures (no reach
    beyond zero motion, held at the floor of one macroblock row and column a diamond can walk from
    still candidates), and not below that for a launch with motion. The records and the
    deblocked references equal those of a context with the lag fixed at 24."""
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, Engine

    w, h, qp, S, F = 176, 144, 26, 2, 4
    still = [grating_clip(w, h, 1, seed=300 + s, motion=0.0, rects=0)[0] for s in range(S)]
    moving = [grating_clip(w, h, F, seed=310 + s, motion=24.0, rects=2) for s in range(S)]
    auto = Engine(w, h, qp, profile=2, num_streams=S, max_frames=F)
    fixed = Engine(w, h, qp, profile=2, num_streams=S, max_frames=F)
    fixed.set_pipeline_tuning(lag=24)
    assert auto.pipeline_lag() == 24 and fixed.pipeline_lag() == 24
    calls = [([[still[s] for s in range(S)]] * F, [[RG_FRAME_IDR] * S] + [[RG_FRAME_P] * S] * (F - 1))]
    calls += [([[still[s] for s in range(S)]] * F, [[RG_FRAME_P] * S] * F)] * 3
    calls += [([[moving[s][f] for s in range(S)] for f in range(F)], [[RG_FRAME_P] * S] * F)]
    lags = []
    for pics, kinds in calls:
        a = auto.analyse_gops(pics, kinds)
        b = fixed.analyse_gops(pics, kinds)
        assert a.tobytes() == b.tobytes()
        lags.append(auto.pipeline_lag())
    assert lags[0] == 24 and lags[1:4] == [15, 15, 15], lags
    assert lags[4] >= 15, lags
    assert fixed.pipeline_lag() == 24
    for s in range(S):
        assert all(np.array_equal(x, y) for x, y in zip(auto.recon_coded(s), fixed.recon_coded(s)))


@pytest.mark.gpu
@pytest.mark.parametrize("form,words,give_up", [("plain", 48, False), ("plain", 7, False), ("plain", 48, True),
                                                ("fullsearch", 96, False)])
def test_compact_records_written_by_the_launch(form, words, give_up):
    """rg_set_record_compaction: the launch writes each picture's compact records into mapped host
    memory as its rows complete; rg_analyse_gops_fetch_compact hands them out, and they are exactly
    rg_records_compact of the bulk call's records. A picture with a macroblock row whose compact
    records exceed the row's slot (words per macroblock x its macroblocks; here rows of the IDR
    pictures at 48, every row at 7, the mask words alone) comes as full records instead. give_up: a wait runs out (one warp, lag one
    macroblock-time); the unfinished pictures come from the re-run as full records."""
    import ctypes
    from ragdoll_b200.engine import (RECORD_DTYPE, RG_FORM_FULLSEARCH, RG_FRAME_IDR, RG_FRAME_P, Engine,
                                     compact_records, lib)
    w, h, qp, S, F = 320, 180, 24, 3, 5
    clips = [grating_clip(w, h, F, seed=900 + s, motion=6.0, rects=2) for s in range(S)]
    pics = [[clips[s][f] for s in range(S)] for f in range(F)]
    kinds = [[RG_FRAME_IDR if f == 0 else RG_FRAME_P] * S for f in range(F)]

    def engine():
        e = Engine(w, h, qp, profile=2, num_streams=S, max_frames=F)
        if form == "fullsearch":
            e.set_analysis_form(RG_FORM_FULLSEARCH, 16)
        return e
    bulk = engine().analyse_gops(pics, kinds)
    eng = engine()
    L = lib()
    assert L.rg_set_record_compaction(eng.h, 3) < 0                       # fewer than the mask words
    assert L.rg_set_record_compaction(eng.h, words) == 0
    if give_up:
        eng.set_pipeline_tuning(lag=1, grid=1, timeout_ms=300)
    out = np.zeros((F, S, eng.n_mb), RECORD_DTYPE)
    planes = [np.ascontiguousarray(p) for f in range(F) for s in range(S) for p in pics[f][s]]
    ptrs = (ctypes.c_void_p * len(planes))(*[p.ctypes.data for p in planes])
    k = (ctypes.c_int32 * (F * S))(*[kinds[f][s] for f in range(F) for s in range(S)])
    assert L.rg_analyse_gops_stream(eng.h, ptrs, w, (w + 1) // 2, k, F, out.ctypes.data) == 0
    assert L.rg_set_record_compaction(eng.h, 0) < 0                       # a call in flight
    data, nbytes = ctypes.c_void_p(), ctypes.c_size_t()
    compact, dense, unfinished = {}, set(), set()
    while len(compact) + len(dense) + len(unfinished) < F * S:
        for i in range(F * S):
            if i in compact or i in dense or i in unfinished:
                continue
            st = L.rg_analyse_gops_fetch_compact(eng.h, out.ctypes.data, i, ctypes.byref(data), ctypes.byref(nbytes))
            assert st in (0, 1, 2), st
            if st == 1 and data.value:
                compact[i] = ctypes.string_at(data.value, nbytes.value)
            elif st == 1:
                dense.add(i)
            elif st == 2:
                unfinished.add(i)
    assert L.rg_analyse_gops_wait(eng.h, out.ctypes.data) == 0
    flat = bulk.reshape(F * S, -1)
    for i, c in compact.items():
        assert c == compact_records(flat[i]), f"picture {i}"
    got = out.reshape(F * S, -1)
    for i in dense | unfinished:
        assert got[i].tobytes() == flat[i].tobytes(), f"picture {i}"
    mb_w = (w + 15) // 16
    fits = {i for i in range(F * S)
            if all(len(compact_records(row)) <= 4 * words * mb_w for row in flat[i].reshape(-1, mb_w))}
    assert set(compact) == fits - unfinished
    assert dense == set(range(F * S)) - fits - unfinished
    assert bool(unfinished) == give_up
    if words == 7:
        assert not compact
    elif not give_up:   # (a wait that gives up early may leave no picture finished)
        assert compact and (words == 96 or dense)
    assert L.rg_set_record_compaction(eng.h, 0) == 0
