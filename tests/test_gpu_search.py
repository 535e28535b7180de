"""The full-search and learned forms against the oracle (GPU tests).

Neither form exists in the reference; the oracle restates the same decisions (oracle/h264_oracle.cpp
code_p_mb_search) and the GPU must equal it field by field -- partition type, every partition's
vector and vector difference, levels -- and pixel by pixel (reconstruction before and after
deblocking), picture by picture:

* full search on the per-diagonal path and in the pipelined persistent launch (several streams);
* the learned form with seeded hints (partition subsets, vector offsets, intra 4x4 mode subsets)
  uploaded to the device, as the candidate network's kernel writes them;
* the CABAC stream the library's writer makes from the full search's records (partitioned
  macroblocks included) decodes, through FFmpeg's H.264 decoder, to exactly the engine's
  reconstruction.
"""
import numpy as np
import pytest

from gpu_parity_util import SEARCH_FIELDS, first_pixel_mismatch, first_record_mismatch
from oracle_lib import OracleEncoder
from ragdoll_b200.synth import grating_clip

pytestmark = pytest.mark.gpu


def random_hints(n_mb, seed):
    from ragdoll_b200.engine import HINT_DTYPE
    rng = np.random.default_rng(seed)
    h = np.zeros(n_mb, HINT_DTYPE)
    for i in range(n_mb):
        parts = rng.choice(4, size=3, replace=False)
        h["part_mask"][i] = sum(1 << int(p) for p in parts)
        h["mv_off"][i] = rng.integers(-12, 13, 2)
        if rng.random() < 0.7:  # a coarse vector (even integer samples) on most macroblocks
            h["flags"][i] = 1
            h["mv_coarse"][i] = 8 * rng.integers(-6, 7, 2)
        for b in range(16):
            modes = rng.choice(9, size=3, replace=False)
            h["i4_mask"][i, b] = sum(1 << int(m) for m in modes)
    return h


def _oracle(w, h, qp, profile, keyint, form, rng_):
    o = OracleEncoder(w, h, qp, profile=profile, keyint=keyint)
    o.set_form(form, rng_)
    return o


@pytest.mark.parametrize("profile,qp,rng_", [(2, 26, 16), (1, 30, 8), (2, 22, 32)])
def test_fullsearch_per_diagonal_matches_oracle(profile, qp, rng_):
    from ragdoll_b200.engine import RG_FORM_FULLSEARCH, RG_FRAME_IDR, RG_FRAME_P, Engine
    w, h, N = 176, 144, 4
    frames = grating_clip(w, h, N, seed=500 + qp, motion=6.0, rects=3)
    eng = Engine(w, h, qp, profile=profile)
    eng.keep_unfiltered(True)
    eng.set_analysis_form(RG_FORM_FULLSEARCH, rng_)
    orc = _oracle(w, h, qp, profile, 30, 1, rng_)
    types = set()
    for f, fr in enumerate(frames):
        _, want = orc.encode(fr)
        got = eng.analyse([fr], [RG_FRAME_IDR if f == 0 else RG_FRAME_P])[0]
        m = first_record_mismatch(want, got, orc.mb_w, SEARCH_FIELDS)
        assert m is None, f"picture {f}: {m}"
        types |= set(got["mb_type"].tolist())
        for p, (a, b) in enumerate(zip(orc.recon(filtered=False), eng.recon_unfiltered(0))):
            assert first_pixel_mismatch(a, b) is None, f"picture {f} unfiltered plane {p}: {first_pixel_mismatch(a, b)}"
        for p, (a, b) in enumerate(zip(orc.recon(filtered=True), eng.recon_coded(0))):
            assert first_pixel_mismatch(a, b) is None, f"picture {f} deblocked plane {p}: {first_pixel_mismatch(a, b)}"
    assert types & {4, 5, 6}, f"no partitioned macroblock coded: {sorted(types)}"


def test_fullsearch_pipelined_streams_match_oracle():
    from ragdoll_b200.engine import RG_FORM_FULLSEARCH, RG_FRAME_IDR, RG_FRAME_P, Engine
    w, h, qp, S, F, R = 320, 192, 26, 3, 5, 24
    clips = [grating_clip(w, h, F, seed=600 + s, motion=10.0, rects=3) for s in range(S)]
    eng = Engine(w, h, qp, profile=2, num_streams=S, max_frames=F)
    eng.set_analysis_form(RG_FORM_FULLSEARCH, R)
    kinds = [[RG_FRAME_IDR if f == 0 else RG_FRAME_P] * S for f in range(F)]
    got = eng.analyse_gops([[clips[s][f] for s in range(S)] for f in range(F)], kinds)
    for s in range(S):
        orc = _oracle(w, h, qp, 2, F + 1, 1, R)
        for f in range(F):
            _, want = orc.encode(clips[s][f])
            m = first_record_mismatch(want, got[f, s], orc.mb_w, SEARCH_FIELDS)
            assert m is None, f"stream {s} picture {f}: {m}"
        for p, (a, b) in enumerate(zip(orc.recon(filtered=True), eng.recon_coded(s))):
            assert first_pixel_mismatch(a, b) is None, f"stream {s} final reference plane {p}"


def test_learned_with_given_hints_matches_oracle():
    import torch

    from ragdoll_b200.engine import RG_FORM_LEARNED, RG_FRAME_IDR, RG_FRAME_P, Engine
    w, h, qp, S, F, R = 240, 160, 26, 2, 4, 16
    clips = [grating_clip(w, h, F, seed=700 + s, motion=8.0, rects=3) for s in range(S)]
    eng = Engine(w, h, qp, profile=2, num_streams=S, max_frames=F)
    eng.set_analysis_form(RG_FORM_LEARNED, R)
    hints = [[random_hints(eng.n_mb, 10 * f + s) for s in range(S)] for f in range(F)]
    dev = [[torch.from_numpy(hints[f][s].view(np.uint8)).cuda() for s in range(S)] for f in range(F)]
    eng.set_hints_device([dev[f][s].data_ptr() for f in range(F) for s in range(S)])
    kinds = [[RG_FRAME_IDR if f == 0 else RG_FRAME_P] * S for f in range(F)]
    got = eng.analyse_gops([[clips[s][f] for s in range(S)] for f in range(F)], kinds)
    for s in range(S):
        orc = _oracle(w, h, qp, 2, F + 1, 2, R)
        for f in range(F):
            orc.set_hints(hints[f][s])
            _, want = orc.encode(clips[s][f])
            m = first_record_mismatch(want, got[f, s], orc.mb_w, SEARCH_FIELDS)
            assert m is None, f"stream {s} picture {f}: {m}"
        for p, (a, b) in enumerate(zip(orc.recon(filtered=True), eng.recon_coded(s))):
            assert first_pixel_mismatch(a, b) is None, f"stream {s} final reference plane {p}"


def test_learned_form_needs_hints():
    from ragdoll_b200.engine import RG_FORM_LEARNED, RG_FRAME_IDR, Engine, RgError
    fr = grating_clip(64, 48, 1, seed=1, motion=0.0, rects=0)[0]
    eng = Engine(64, 48, 26, profile=2)
    eng.set_analysis_form(RG_FORM_LEARNED, 16)
    with pytest.raises(RgError) as e:
        eng.analyse([fr], [RG_FRAME_IDR])
    assert e.value.code == -6
    base = Engine(64, 48, 26, profile=0)
    with pytest.raises(RgError) as e:
        base.set_analysis_form(RG_FORM_LEARNED, 16)
    assert e.value.code == -5


def test_fullsearch_stream_decodes_to_the_reconstruction():
    import ffmpeg_decode
    from ragdoll_b200.engine import RG_FORM_FULLSEARCH, RG_FRAME_IDR, RG_FRAME_P, BitstreamWriter, Engine
    w, h, qp, N = 320, 180, 26, 6
    frames = grating_clip(w, h, N, seed=800, motion=9.0, rects=4)
    eng = Engine(w, h, qp, profile=2)
    eng.set_analysis_form(RG_FORM_FULLSEARCH, 24)
    wr = BitstreamWriter(w, h, qp, profile=2)
    aus, recons, types = [], [], set()
    for f, fr in enumerate(frames):
        kind = RG_FRAME_IDR if f == 0 else RG_FRAME_P
        recs = eng.analyse([fr], [kind])[0]
        types |= set(recs["mb_type"].tolist())
        aus.append(wr.picture(recs, kind))
        recons.append([p.copy() for p in eng.recon_coded(0)])
    assert types & {4, 5, 6}
    if not ffmpeg_decode.available():
        pytest.skip("FFmpeg libraries not found")
    dec = ffmpeg_decode.decode(aus)
    assert len(dec) == N
    for f, (p, r) in enumerate(zip(dec, recons)):
        for k in range(3):
            assert np.array_equal(p[k], r[k][:p[k].shape[0], :p[k].shape[1]]), f"picture {f} plane {k}"
