"""One persistent launch over several contexts of different picture sizes (rg_analyse_gops_group)
against each context analysed alone (rg_analyse_gops_device), GPU tests.

The batched configuration transcodes many independent streams of several sizes; the group call
analyses all of them in one launch whose work list interleaves the sizes' segments by key. It must
not change a single decision: every record and every reconstruction of every context equals the one
the same context gives alone, over three calls in a row (the second continuing each GOP from the
reference the first left, the third starting new GOPs), in the plain form (with a QP per stream)
and in the full-search form. The launch is a CUDA graph captured per launch shape: the third call,
of the first one's shape, replays the first one's graph.
"""
import numpy as np
import pytest

from ragdoll_b200.synth import grating_clip

pytestmark = pytest.mark.gpu

SIZES = [(160, 96, 3), (96, 64, 2), (208, 80, 1)]   # width, height, streams
F = 3                                               # pictures per call


def _clips():
    return [[grating_clip(w, h, 2 * F, seed=700 + 10 * i + s, motion=6.0, rects=2) for s in range(S)]
            for i, (w, h, S) in enumerate(SIZES)]


def _engines(form, qps):
    from ragdoll_b200.engine import RG_PROFILE_MAIN, Engine
    engs = []
    for i, (w, h, S) in enumerate(SIZES):
        e = Engine(w, h, 28, profile=RG_PROFILE_MAIN, num_streams=S, max_frames=F)
        if form:
            e.set_analysis_form(form, 16)
        for s in range(S):
            e.set_stream_qp(s, qps[i][s])
        engs.append(e)
    return engs


def _call_args(clips, call):
    """Device planes ([f][s][y,u,v]) and kinds of every context for call `call` (0: IDR + P, 1: P)."""
    import torch
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P
    keep, planes, kinds, sy, suv = [], [], [], [], []
    for i, (w, h, S) in enumerate(SIZES):
        cw = (w + 1) // 2
        p, k = [], []
        for f in range(F):
            for s in range(S):
                for plane in clips[i][s][call * F + f]:
                    t = torch.from_numpy(np.ascontiguousarray(plane)).cuda()
                    keep.append(t)
                    p.append(t.data_ptr())
                k.append(RG_FRAME_IDR if call == 0 and f == 0 else RG_FRAME_P)
        planes.append(p)
        kinds.append(k)
        sy.append(w)
        suv.append(cw)
    return keep, planes, kinds, sy, suv


@pytest.mark.parametrize("form", [0, 1])
def test_group_launch_equals_each_context_alone(form):
    import torch

    from ragdoll_b200.engine import Engine
    rng = np.random.default_rng(form)
    qps = [rng.integers(20, 37, S).tolist() for _, _, S in SIZES]
    clips = _clips()
    group = _engines(form, qps)
    alone = _engines(form, qps)
    for e in group:   # a fixed lag: the launch shape does not follow the reach the calls observe
        e.set_pipeline_tuning(lag=64)
    for call in range(3):
        # call 2 repeats call 0's pictures and kinds (an IDR picture starts each stream's next GOP):
        # the same launch shape, so its graph is replayed
        keep, planes, kinds, sy, suv = _call_args(clips, call % 2)
        Engine.analyse_gops_group(group, planes, sy, suv, kinds, F)
        for i, e in enumerate(alone):
            e.analyse_gops_device(planes[i], sy[i], suv[i], kinds[i], F)
        torch.cuda.synchronize()
        for i, (w, h, S) in enumerate(SIZES):
            got = group[i].records_gops(F)
            want = alone[i].records_gops(F)
            assert got.tobytes() == want.tobytes(), f"call {call}, size {w}x{h}: records differ"
            for s in range(S):
                for a, b in zip(group[i].recon(s), alone[i].recon(s)):
                    assert np.array_equal(a, b), f"call {call}, size {w}x{h}, stream {s}: reconstruction differs"
        del keep
    import ctypes
    from ragdoll_b200.engine import lib
    captures, launches = ctypes.c_int64(), ctypes.c_int64()
    assert lib().rg_group_graph_counts(group[0].h, ctypes.byref(captures), ctypes.byref(launches)) == 0
    assert (captures.value, launches.value) == (2, 3)
    for e in group + alone:
        e.close()


def test_group_launch_rejects_mixed_forms_and_duplicates():
    from ragdoll_b200.engine import RG_FORM_FULLSEARCH, RG_PROFILE_MAIN, Engine, RgError
    a = Engine(96, 64, 28, profile=RG_PROFILE_MAIN, max_frames=1)
    b = Engine(64, 48, 28, profile=RG_PROFILE_MAIN, max_frames=1)
    b.set_analysis_form(RG_FORM_FULLSEARCH, 8)
    with pytest.raises(RgError):
        Engine.analyse_gops_group([a, b], [[0] * 3, [0] * 3], [96, 64], [48, 32], [[0], [0]], 1)
    with pytest.raises(RgError):
        Engine.analyse_gops_group([a, a], [[0] * 3, [0] * 3], [96, 96], [48, 48], [[0], [0]], 1)
    a.close()
    b.close()


@pytest.mark.parametrize("give_up", [False, True])
def test_group_encoder_waves_equal_each_encoder_alone(give_up):
    """rg_encoder_submit_group: the waves of encoders of three sizes (a QP per stream), analysed by
    one launch per wave and collected per encoder, give exactly the access units of the same
    encoders submitting alone, over two waves. give_up: one warp and a lag of one macroblock-time
    make a wait run out; each context re-runs its pictures and the access units are still exact."""
    from ragdoll_b200.encoder import H264Encoder
    from ragdoll_b200.engine import RG_PROFILE_MAIN
    rng = np.random.default_rng(11)
    qps = [rng.integers(20, 37, S).tolist() for _, _, S in SIZES]
    clips = _clips()

    def encoders():
        out = []
        for i, (w, h, S) in enumerate(SIZES):
            e = H264Encoder(w, h, 28, profile=RG_PROFILE_MAIN, keyint=2 * F, streams=S, max_frames=F, threads=2)
            for s in range(S):
                e.set_stream_qp(s, qps[i][s])
            out.append(e)
        return out
    group, alone = encoders(), encoders()
    if give_up:   # the launch takes the largest grid of any context: one warp everywhere
        for e in group:
            e.set_pipeline_tuning(lag=1, grid=1, timeout_ms=300)
    waves = [[[[clips[i][s][wv * F + f] for s in range(S)] for f in range(F)] for i, (_, _, S) in enumerate(SIZES)]
             for wv in range(2)]
    got, want = [], []
    for wv in range(2):
        H264Encoder.submit_group(group, waves[wv])
        got.append([e.collect() for e in group])
        for e, fr in zip(alone, waves[wv]):
            e.submit(fr)
        want.append([e.collect() for e in alone])
    for wv in range(2):
        for i, (w, h, S) in enumerate(SIZES):
            assert got[wv][i] == want[wv][i], f"wave {wv}, size {w}x{h}: access units differ"
    for e in group + alone:
        e.close()


def test_group_async_records_equal_each_context_alone():
    """rg_analyse_gops_group_async: host sources of three sizes in, one launch, each context's
    records copied into its own host buffer -- the records of each context analysed alone."""
    import ctypes

    from ragdoll_b200.engine import RECORD_DTYPE, RG_FRAME_IDR, RG_FRAME_P, lib
    rng = np.random.default_rng(3)
    qps = [rng.integers(20, 37, S).tolist() for _, _, S in SIZES]
    clips = _clips()
    group, alone = _engines(0, qps), _engines(0, qps)
    L = lib()
    n = len(SIZES)
    keep, arrs, outs, kinds = [], [], [], []
    for i, (w, h, S) in enumerate(SIZES):
        ptrs, k = [], []
        for f in range(F):
            for s in range(S):
                for p in clips[i][s][f]:
                    a = np.ascontiguousarray(p)
                    keep.append(a)
                    ptrs.append(a.ctypes.data)
                k.append(RG_FRAME_IDR if f == 0 else RG_FRAME_P)
        arrs.append((ctypes.c_void_p * len(ptrs))(*ptrs))
        kinds.append((ctypes.c_int32 * len(k))(*k))
        outs.append(np.zeros((F, S, group[i].n_mb), RECORD_DTYPE))
    P = ctypes.c_void_p
    rc = L.rg_analyse_gops_group_async((P * n)(*[e.h for e in group]), n,
                                       (P * n)(*[ctypes.cast(a, P) for a in arrs]),
                                       (ctypes.c_size_t * n)(*[w for w, _, _ in SIZES]),
                                       (ctypes.c_size_t * n)(*[(w + 1) // 2 for w, _, _ in SIZES]),
                                       (P * n)(*[ctypes.cast(k, P) for k in kinds]), F,
                                       (P * n)(*[o.ctypes.data for o in outs]))
    assert rc == 0
    for i, (w, h, S) in enumerate(SIZES):
        assert L.rg_analyse_gops_wait(group[i].h, outs[i].ctypes.data) == 0
        want = alone[i].analyse_gops([[clips[i][s][f] for s in range(S)] for f in range(F)],
                                     [[RG_FRAME_IDR if f == 0 else RG_FRAME_P] * S for f in range(F)])
        assert outs[i].tobytes() == want.tobytes(), f"size {w}x{h}: records differ"
    for e in group + alone:
        e.close()
