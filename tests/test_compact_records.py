"""The compact record form (host code, no GPU): per macroblock, 7 mask words of the record's
nonzero 32-bit words, then those words in order.

* rg_records_compact / rg_records_expand round-trip the oracle's records of grating clips and
  random records bit for bit, and the size is 28 bytes + 4 per nonzero word;
* a hand-made record gives the exact words;
* the writers give the same access unit from the compact form as from the records (CAVLC and
  CABAC, the oracle's bytes), and reject truncated, overlong and malformed streams.
The device side (the launch writing the form into mapped host memory) is compared with these
host functions in test_gpu_parity.py.
"""
import numpy as np
import pytest

from oracle_lib import OracleEncoder
from ragdoll_b200.engine import (COMPACT_MASK_WORDS, RECORD_DTYPE, RG_FRAME_IDR, RG_FRAME_P, BitstreamWriter,
                                 RgError, compact_records, expand_records)
from ragdoll_b200.synth import grating_clip

WORDS = RECORD_DTYPE.itemsize // 4


def nonzero_words(recs):
    return int((np.ascontiguousarray(recs).view(np.uint32) != 0).sum())


def oracle_records(w, h, qp, profile, n=5):
    orc = OracleEncoder(w, h, qp, profile=profile, keyint=4)
    out = []
    for fr in grating_clip(w, h, n, seed=w + qp, motion=6.0, rects=2):
        want, recs = orc.encode(fr)
        out.append((want, recs.copy(), RG_FRAME_IDR if orc.last_idr else RG_FRAME_P))
    return out


def test_round_trip_and_size_on_oracle_records():
    for _, recs, _ in oracle_records(208, 120, 22, 2):
        data = compact_records(recs)
        assert len(data) == 4 * (COMPACT_MASK_WORDS * recs.size + nonzero_words(recs))
        back = expand_records(data, recs.size)
        assert back.tobytes() == recs.tobytes()
        assert len(data) < recs.nbytes / 2   # mostly zero levels, even in intra pictures at QP 22


def test_round_trip_random_and_extreme_records():
    rng = np.random.default_rng(7)
    words = rng.integers(0, 2**32, size=(9, WORDS), dtype=np.uint64).astype(np.uint32)
    words[1] = 0                                  # an all-zero record: mask words only
    words[2] = 0xFFFFFFFF                         # every word nonzero: 7 + 222 words
    words[3, ::3] = 0
    words[4, :] = 0
    words[4, WORDS - 1] = 1                       # the last word only (bit 29 of mask word 6)
    recs = words.view(RECORD_DTYPE).reshape(-1)
    data = compact_records(recs)
    assert len(data) == 4 * (COMPACT_MASK_WORDS * 9 + int((words != 0).sum()))
    assert expand_records(data, 9).tobytes() == recs.tobytes()
    # the last record's words: mask words 0..5 zero, mask word 6 = 1 << 29, then the word
    tail = np.frombuffer(data, np.uint32)[-COMPACT_MASK_WORDS - 1 - 8 * 0:]
    w4 = np.frombuffer(compact_records(recs[4:5]), np.uint32)
    assert w4.tolist() == [0, 0, 0, 0, 0, 0, 1 << 29, 1]
    assert len(tail) == COMPACT_MASK_WORDS + 1


def test_known_words_of_a_hand_made_record():
    r = np.zeros(1, RECORD_DTYPE)
    r["mb_type"] = 2
    r["qp"] = 26
    r["mv"] = (-3, 5)
    r["luma"][0, 17] = 4                          # word 9 + 8 = 17 (low half)
    r["part_type"] = 255
    got = np.frombuffer(compact_records(r), np.uint32).tolist()
    w = r.view(np.uint32)
    mask = [0] * COMPACT_MASK_WORDS
    for k in np.flatnonzero(w):
        mask[k // 32] |= 1 << (k % 32)
    assert got == mask + [int(x) for x in w[w != 0]]
    assert mask[0] == (1 << 0) | (1 << 1) | (1 << 2) | (1 << 17)   # mb_type, qp, mv, the level
    assert mask[6] == 1 << (221 - 192)                                # part_type


@pytest.mark.parametrize("w,h,qp,profile", [(176, 144, 26, 0), (208, 120, 12, 2), (96, 64, 30, 1)])
def test_writer_from_compact_records_equals_oracle(w, h, qp, profile):
    dense = BitstreamWriter(w, h, qp, profile=profile)
    compact = BitstreamWriter(w, h, qp, profile=profile)
    for want, recs, kind in oracle_records(w, h, qp, profile):
        assert compact.picture_compact(compact_records(recs), kind) == want
        assert dense.picture(recs, kind) == want


def test_compact_streams_that_are_not_a_picture_are_rejected():
    (_, recs, kind), = oracle_records(64, 48, 26, 2, n=1)
    data = compact_records(recs)
    wr = BitstreamWriter(64, 48, 26, profile=2)
    for bad in (data[:-4], data + b"\0\0\0\0", data[:4 * COMPACT_MASK_WORDS - 4], b""):
        with pytest.raises(RgError):
            wr.picture_compact(bad, kind)
        with pytest.raises(RgError):
            expand_records(bad, recs.size)
    bad = bytearray(data)
    bad[4 * (COMPACT_MASK_WORDS - 1) + 3] |= 0x80   # a mask bit past the record's 222 words
    with pytest.raises(RgError):
        expand_records(bytes(bad), recs.size)
    with pytest.raises(RgError):
        compact_records(recs[:0]) or expand_records(data, recs.size + 1)
    assert wr.picture_compact(data, kind)        # the writer is still usable
