"""Shared helpers of the GPU parity tests: run the oracle and the engine on the same frames and
report the first differing macroblock field."""
from __future__ import annotations

import numpy as np

from oracle_lib import OracleEncoder

FIELDS = ["mb_type", "i16_mode", "chroma_mode", "cbp", "transform_8x8", "qp", "mv", "mvd",
          "i4_modes", "luma", "luma_dc", "chroma_dc", "chroma_ac"]
# the search forms' partition fields
SEARCH_FIELDS = FIELDS + ["part_mv", "part_mvd", "part_type"]


def first_record_mismatch(a: np.ndarray, b: np.ndarray, mb_w: int, fields=FIELDS):
    """(mb_x, mb_y, field, oracle value, engine value) of the first difference, else None."""
    for i in range(len(a)):
        for f in fields:
            if f == "i4_modes" and a[i]["mb_type"] != 3:
                continue
            if not np.array_equal(a[i][f], b[i][f]):
                return (i % mb_w, i // mb_w, f, a[i][f].tolist(), b[i][f].tolist(),
                        int(a[i]["mb_type"]), int(b[i]["mb_type"]))
    return None


def first_pixel_mismatch(a: np.ndarray, b: np.ndarray):
    d = np.argwhere(a != b)
    if len(d) == 0:
        return None
    y, x = d[0]
    return int(x), int(y), int(a[y, x]), int(b[y, x]), int(len(d))


def run_parity(frames, width, height, qp, profile, keyint, engine, stream=0, check_unfiltered=True):
    """Encodes `frames` with the oracle and the engine stream, comparing records, unfiltered and
    deblocked reconstructions after every frame. Returns a list of failure strings."""
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P

    orc = OracleEncoder(width, height, qp, profile=profile, keyint=keyint)
    fails = []
    for fi, fr in enumerate(frames):
        _, ref_recs = orc.encode(fr)
        kind = RG_FRAME_IDR if orc.last_idr else RG_FRAME_P
        recs = engine.analyse([fr], [kind])[0]
        m = first_record_mismatch(ref_recs, recs, orc.mb_w)
        if m:
            fails.append(f"frame {fi} ({'I' if orc.last_idr else 'P'}) records: mb ({m[0]},{m[1]}) field {m[2]} "
                         f"oracle={m[3]} engine={m[4]} types {m[5]}/{m[6]}")
        if check_unfiltered:
            ou = orc.recon(filtered=False)
            gu = engine.recon_unfiltered(stream)
            for p, (x, y) in enumerate(zip(ou, gu)):
                pm = first_pixel_mismatch(x, y)
                if pm:
                    fails.append(f"frame {fi} unfiltered plane {p}: first diff at {pm[:2]} {pm[2]} vs {pm[3]} ({pm[4]} px)")
        of = orc.recon(filtered=True)
        gf = engine.recon_coded(stream)
        for p, (x, y) in enumerate(zip(of, gf)):
            pm = first_pixel_mismatch(x, y)
            if pm:
                fails.append(f"frame {fi} deblocked plane {p}: first diff at {pm[:2]} {pm[2]} vs {pm[3]} ({pm[4]} px)")
        if fails:
            break
    return fails
