"""The search forms' CPU oracle and the CABAC writer's partition syntax (no GPU).

The oracle's full-search and learned decisions (partitioned macroblocks included), written by the
library's host CABAC writer, must decode through an independent H.264 decoder (FFmpeg) to exactly
the oracle's reconstruction, picture by picture; the learned form with every candidate allowed
must decide as the full search does within the hint's window.
"""
import numpy as np
import pytest

from oracle_lib import OracleEncoder
from ragdoll_b200.synth import grating_clip


def _encode(w, h, qp, profile, form, rng_, frames, hints=None):
    orc = OracleEncoder(w, h, qp, profile=profile, keyint=len(frames) + 1)
    orc.set_form(form, rng_)
    recs, recons = [], []
    for f, fr in enumerate(frames):
        if hints is not None:
            orc.set_hints(hints[f])
        _, r = orc.encode(fr)
        recs.append(r)
        recons.append([p.copy() for p in orc.recon()])
    return recs, recons


@pytest.mark.parametrize("profile,qp,form", [(2, 26, 1), (1, 32, 1), (2, 22, 2)])
def test_search_form_streams_decode_to_the_oracle_reconstruction(profile, qp, form):
    import ffmpeg_decode
    from ragdoll_b200.engine import HINT_DTYPE, RG_FRAME_IDR, RG_FRAME_P, BitstreamWriter
    w, h, N = 160, 96, 5
    frames = grating_clip(w, h, N, seed=900 + qp, motion=7.0, rects=3)
    hints = None
    if form == 2:
        rng = np.random.default_rng(qp)
        n = ((w + 15) // 16) * ((h + 15) // 16)
        hints = []
        for _ in range(N):
            hh = np.zeros(n, HINT_DTYPE)
            hh["part_mask"] = rng.integers(1, 16, n)
            hh["mv_off"] = rng.integers(-8, 9, (n, 2))
            hh["flags"] = rng.integers(0, 2, n)
            hh["mv_coarse"] = 8 * rng.integers(-5, 6, (n, 2))
            hh["i4_mask"] = rng.integers(1, 512, (n, 16))
            hints.append(hh)
    recs, recons = _encode(w, h, qp, profile, form, 16, frames, hints)
    types = set(np.concatenate([r["mb_type"] for r in recs]).tolist())
    assert types & {4, 5, 6}, sorted(types)
    wr = BitstreamWriter(w, h, qp, profile=profile)
    aus = [wr.picture(recs[f], RG_FRAME_IDR if f == 0 else RG_FRAME_P) for f in range(N)]
    if not ffmpeg_decode.available():
        pytest.skip("FFmpeg libraries not found")
    dec = ffmpeg_decode.decode(aus)
    assert len(dec) == N
    for f, (p, r) in enumerate(zip(dec, recons)):
        for k in range(3):
            assert np.array_equal(p[k], r[k][:p[k].shape[0], :p[k].shape[1]]), f"picture {f} plane {k}"
