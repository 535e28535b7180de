"""Regenerates the golden fixtures of tests/golden from the reference's pinned corpus.

Run from the repository root where the reference tree is mounted (it is not needed afterwards):

    python tests/golden/make_golden.py /path/to/ragdoll

Fixtures written:

* ``clip_160x90_qp20.nal``: the NAL units of qa/corpus/synth/clip_160x90_30fps.mp4 (SHA-256
  pinned in qa/corpus/manifest.toml), in decoding order, each prefixed by a 4-byte big-endian
  length: first the SPS and PPS of the avcC box, then every NAL of every sample. The clip is
  ragdoll's Balanced / Constrained Baseline / QP 20 encoding of synth_video_frame(160, 90, i),
  i = 0..29, in two independent 15-frame GOPs (crates/ragdoll-pipeline/src/lib.rs:2919-3078).
* ``clip_320x180_qp20.nal``: the same for qa/corpus/synth/clip_320x180_25fps.mkv (15 frames).
* ``golden.json``: provenance (source sizes and SHA-256) and the CLI snapshot numbers of
  crates/ragdoll-cli/tests/golden/{transcode,metrics}.txt.
"""
from __future__ import annotations

import hashlib
import json
import re
import struct
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def mp4_nals(data: bytes) -> list[bytes]:
    """SPS/PPS of avcC, then the length-prefixed NALs of each sample (stsz/stco/stsc)."""
    boxes = {}

    def walk(off, end, path):
        while off < end:
            size, typ = struct.unpack(">I4s", data[off:off + 8])
            t = typ.decode()
            p = path + "/" + t
            boxes.setdefault(p, []).append((off, size))
            if t in ("moov", "trak", "mdia", "minf", "stbl", "dinf"):
                walk(off + 8, off + size, p)
            elif t == "stsd":
                walk(off + 16, off + size, p)
            elif t == "avc1":
                walk(off + 8 + 78, off + size, p)
            off += size

    walk(0, len(data), "")
    stbl = "/moov/trak/mdia/minf/stbl"
    off, size = boxes[stbl + "/stsd/avc1/avcC"][0]
    c = data[off + 8:off + size]
    nals = []
    n_sps = c[5] & 0x1F
    pos = 6
    for _ in range(n_sps):
        ln = struct.unpack(">H", c[pos:pos + 2])[0]
        nals.append(c[pos + 2:pos + 2 + ln])
        pos += 2 + ln
    n_pps = c[pos]
    pos += 1
    for _ in range(n_pps):
        ln = struct.unpack(">H", c[pos:pos + 2])[0]
        nals.append(c[pos + 2:pos + 2 + ln])
        pos += 2 + ln
    nal_len = (c[4] & 3) + 1

    off, size = boxes[stbl + "/stsz"][0]
    b = data[off + 8:off + size]
    sample_size, count = struct.unpack(">II", b[4:12])
    sizes = [sample_size] * count if sample_size else list(struct.unpack(f">{count}I", b[12:12 + 4 * count]))
    off, size = boxes[stbl + "/stco"][0]
    b = data[off + 8:off + size]
    n = struct.unpack(">I", b[4:8])[0]
    chunk_offs = struct.unpack(f">{n}I", b[8:8 + 4 * n])
    off, size = boxes[stbl + "/stsc"][0]
    b = data[off + 8:off + size]
    n = struct.unpack(">I", b[4:8])[0]
    stsc = [struct.unpack(">III", b[8 + 12 * i:20 + 12 * i]) for i in range(n)]
    si = 0
    for ci, coff in enumerate(chunk_offs):
        per = [e[1] for e in stsc if e[0] - 1 <= ci][-1]
        pos = coff
        for _ in range(per):
            end = pos + sizes[si]
            p = pos
            while p < end:
                ln = int.from_bytes(data[p:p + nal_len], "big")
                nals.append(data[p + nal_len:p + nal_len + ln])
                p += nal_len + ln
            pos = end
            si += 1
    assert si == len(sizes)
    return nals


def mkv_nals(data: bytes) -> list[bytes]:
    """CodecPrivate (avcC) SPS/PPS, then the NALs of every SimpleBlock/Block, in file order."""
    def vint(p, keep_marker):
        b0 = data[p]
        ln = 1
        mask = 0x80
        while not (b0 & mask):
            mask >>= 1
            ln += 1
        v = b0 if keep_marker else b0 & (mask - 1)
        for i in range(1, ln):
            v = (v << 8) | data[p + i]
        return v, ln

    masters = {0x18538067, 0x1F43B675, 0x1654AE6B, 0xAE, 0xA0}
    out = []
    priv = None

    def walk(p, end):
        nonlocal priv
        while p < end:
            eid, l1 = vint(p, True)
            size, l2 = vint(p + l1, False)
            body = p + l1 + l2
            if size == (1 << (7 * l2)) - 1:  # unknown size
                size = end - body
            if eid in masters:
                walk(body, body + size)
            elif eid == 0x63A2:
                priv = data[body:body + size]
            elif eid in (0xA3, 0xA1):
                _, tl = vint(body, False)
                q = body + tl + 3
                while q < body + size:
                    ln = int.from_bytes(data[q:q + 4], "big")
                    out.append(data[q + 4:q + 4 + ln])
                    q += 4 + ln
            p = body + size

    walk(0, len(data))
    c = priv
    hdr = []
    n_sps = c[5] & 0x1F
    pos = 6
    for _ in range(n_sps):
        ln = struct.unpack(">H", c[pos:pos + 2])[0]
        hdr.append(c[pos + 2:pos + 2 + ln])
        pos += 2 + ln
    n_pps = c[pos]
    pos += 1
    for _ in range(n_pps):
        ln = struct.unpack(">H", c[pos:pos + 2])[0]
        hdr.append(c[pos + 2:pos + 2 + ln])
        pos += 2 + ln
    return hdr + out


def pack(nals: list[bytes]) -> bytes:
    return b"".join(struct.pack(">I", len(n)) + n for n in nals)


def main(ref_root: str) -> None:
    ref = Path(ref_root)
    meta = {}
    for name, fn, out in [("clip_160x90_30fps.mp4", mp4_nals, "clip_160x90_qp20.nal"),
                          ("clip_320x180_25fps.mkv", mkv_nals, "clip_320x180_qp20.nal")]:
        data = (ref / "qa/corpus/synth" / name).read_bytes()
        nals = fn(data)
        (HERE / out).write_bytes(pack(nals))
        meta[out] = {"source": "qa/corpus/synth/" + name, "source_size": len(data),
                     "source_sha256": hashlib.sha256(data).hexdigest(), "nal_units": len(nals)}
    golden = ref / "crates/ragdoll-cli/tests/golden"
    text = (golden / "metrics.txt").read_text()
    num = r"([0-9]+\.[0-9]+)"
    pm = re.search(r"Y=" + num + r" dB \| U=" + num + r" dB \| V=" + num + r" dB \| Avg=" + num +
                   r" dB \(6:1:1=" + num + r" dB\)", text)
    sm = re.search(r"Y=" + num + r" \(" + num + r" dB\) \| Avg=" + num + r" \| 5-Scale MS-SSIM=" + num, text)
    vm = re.search(r"VMAF-Lite\s*: " + num, text)
    tm = re.search(r"out=([0-9]+) B", (golden / "transcode.txt").read_text())
    meta["cli_snapshots"] = {
        "transcode_qp30_mp4_bytes": int(tm.group(1)),
        "metrics": {"psnr_y": float(pm.group(1)), "psnr_u": float(pm.group(2)), "psnr_v": float(pm.group(3)),
                    "psnr_avg": float(pm.group(4)), "psnr_yuv_611": float(pm.group(5)),
                    "ssim_y": float(sm.group(1)), "ssim_db": float(sm.group(2)), "ssim_avg": float(sm.group(3)),
                    "ms_ssim": float(sm.group(4)), "vmaf_lite": float(vm.group(1))},
        "source": "crates/ragdoll-cli/tests/golden/transcode.txt, metrics.txt",
    }
    (HERE / "golden.json").write_text(json.dumps(meta, indent=2) + "\n")
    print(json.dumps(meta, indent=2))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <checkout of oddurs/ragdoll>")
    main(sys.argv[1])
