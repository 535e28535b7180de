"""Containers (host code, no GPU): MP4 / Matroska muxing and demuxing, YUV4MPEG2.

* The muxers, fed the access units of the pinned corpus clips, reproduce the reference's files
  bit for bit (SHA-256 and size from qa/corpus/manifest.toml, kept in tests/golden/golden.json):
  clip_160x90_30fps.mp4 (two 15-picture GOPs, 30 fps) and clip_320x180_25fps.mkv (25 fps).
* Demuxing gives back the access units, the size, the frame rate and the keyframes.
* write_y4m of synth_video_frame reproduces qa/corpus/synth/clip_64x36_30fps.y4m.
* The streams decode, through FFmpeg's H.264 decoder, to exactly the oracle's reconstruction.
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from oracle_lib import OracleEncoder, read_nal_fixture, split_annex_b
from ragdoll_b200.containers import Demuxer, Muxer, mux, read_y4m, write_y4m
from ragdoll_b200.engine import RgError
from ragdoll_b200.synth import grating_clip, synth_video_frame

GOLDEN = Path(__file__).resolve().parent / "golden"
SC = b"\x00\x00\x00\x01"

# qa/corpus/manifest.toml: clip_64x36_30fps.y4m
Y4M_SIZE, Y4M_SHA256 = 20834, "f3725781f178a93dc53fcc3f0780a271efbcb67347bbb7b43bd4eab50ee9a433"


def fixture_access_units(name):
    nals = read_nal_fixture(GOLDEN / name)
    return [SC + nals[0] + SC + nals[1] + SC + nals[2]] + [SC + n for n in nals[3:]]


CASES = [("clip_160x90_qp20.nal", "mp4", 160, 90, (30, 1)), ("clip_320x180_qp20.nal", "mkv", 320, 180, (25, 1))]


@pytest.mark.parametrize("fixture,container,w,h,fps", CASES)
def test_muxer_reproduces_corpus_file(fixture, container, w, h, fps):
    gold = json.loads((GOLDEN / "golden.json").read_text())[fixture]
    data = mux(container, w, h, fixture_access_units(fixture), fps)
    assert len(data) == gold["source_size"]
    assert hashlib.sha256(data).hexdigest() == gold["source_sha256"]


@pytest.mark.parametrize("fixture,container,w,h,fps", CASES)
def test_demuxer_round_trip(fixture, container, w, h, fps):
    aus = fixture_access_units(fixture)
    d = Demuxer(mux(container, w, h, aus, fps))
    assert (d.container, d.width, d.height, d.fps, len(d)) == (container, w, h, fps, len(aus))
    assert d.profile_idc == 66
    back = d.access_units()
    keys = [i for i, au in enumerate(back) if any(n[0] & 0x1F == 5 for n in split_annex_b(au))]
    assert d.keyframes == len(keys) == len(aus) // 15 + (len(aus) % 15 > 0)
    params = split_annex_b(aus[0])[:2]
    for i, (a, b) in enumerate(zip(aus, back)):
        want = [n for n in split_annex_b(a) if n[0] & 0x1F not in (7, 8)]
        if i in keys:
            want = params + want   # the demuxer puts the parameter sets before every IDR picture
        assert split_annex_b(b) == want, f"access unit {i}"


@pytest.mark.parametrize("container", ["mp4", "mkv"])
def test_fractional_rates_and_many_gops(container):
    w, h = 64, 48
    orc, aus = None, []
    for i in range(40):
        if i % 7 == 0:
            orc = OracleEncoder(w, h, 30, profile=0, keyint=8, fps=(30000, 1001))
        aus.append(orc.encode(grating_clip(w, h, 1, seed=i, motion=0.0, rects=1)[0])[0])
    d = Demuxer(mux(container, w, h, aus, (30000, 1001)))
    assert len(d) == 40 and d.keyframes == 6
    if container == "mp4":
        assert d.fps == (30000, 1001)
    else:
        assert abs(d.fps[0] / d.fps[1] - 30000 / 1001) < 1e-6   # DefaultDuration: whole nanoseconds
    assert [split_annex_b(a)[-1] for a in aus] == [split_annex_b(b)[-1] for b in d.access_units()]


def test_mux_errors():
    aus = fixture_access_units("clip_160x90_qp20.nal")
    m = Muxer("mp4", 160, 90)
    with pytest.raises(RgError):
        m.write(aus[1])                       # a P picture first
    with pytest.raises(RgError):
        m.write(b"\x00\x00\x01\x09\xf0")        # no slice
    with pytest.raises(RgError):
        m.finish()                            # nothing written
    m.write(aus[0])
    other = read_nal_fixture(GOLDEN / "clip_320x180_qp20.nal")
    with pytest.raises(RgError):
        m.write(SC + other[0] + SC + other[1] + SC + other[2])   # parameter sets change
    assert len(m.finish()) > 0
    with pytest.raises(KeyError):
        Muxer("avi", 16, 16)
    with pytest.raises(RgError):
        Muxer("mp4", 0, 16)
    with pytest.raises(RgError):
        Demuxer(b"\x00" * 64)
    with pytest.raises(RgError):
        Demuxer(mux("mp4", 160, 90, aus)[:600])   # moov cut short


def test_y4m_reproduces_corpus_file():
    frames = [synth_video_frame(64, 36, i) for i in range(6)]
    data = write_y4m(64, 36, frames, (30, 1))
    assert len(data) == Y4M_SIZE
    assert hashlib.sha256(data).hexdigest() == Y4M_SHA256
    w, h, fps, back = read_y4m(data)
    assert (w, h, fps, len(back)) == (64, 36, (30, 1), 6)
    for a, b in zip(frames, back):
        for p, q in zip(a, b):
            assert np.array_equal(p, q)


def test_oracle_stream_decodes_to_its_reconstruction():
    """Independent decoder: FFmpeg's h264 decoder turns the stream (muxed, demuxed) into
    exactly the oracle's reconstruction, every plane of every picture."""
    import ffmpeg_decode
    if not ffmpeg_decode.available():
        pytest.skip("FFmpeg libraries not found")
    w, h = 160, 90
    aus, recons = [], []
    for g0 in (0, 15):
        orc = OracleEncoder(w, h, 20, profile=0, keyint=16)
        for i in range(15):
            aus.append(orc.encode(synth_video_frame(w, h, g0 + i))[0])
            recons.append([p.copy() for p in orc.recon()])
    back = Demuxer(mux("mp4", w, h, aus)).access_units()
    pics = ffmpeg_decode.decode(back)
    assert len(pics) == len(recons)
    for i, (p, r) in enumerate(zip(pics, recons)):
        for k in range(3):
            assert np.array_equal(p[k], r[k][:p[k].shape[0], :p[k].shape[1]]), f"picture {i} plane {k}"
