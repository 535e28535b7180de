"""GOP-parallel encoding over ranks (ragdoll_b200.multi_gpu) on CPU: two gloo ranks, as one
process per GPU would run, with the oracle as each rank's chunk encoder (the GPU encoder's access
units equal the oracle's, tests/test_gpu_encoder.py). The gathered stream must be byte for byte the
one rank's stream -- the reference's determinism contract (crates/ragdoll-pipeline/tests/
determinism.rs: transcode bytes do not depend on the thread count) -- with chunks assigned round robin.
"""
import datetime
import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent
W, H, QP, GOP, N = 96, 64, 28, 4, 14   # 4 chunks, the last one shorter


def _clip():
    sys.path.insert(0, str(ROOT))
    from ragdoll_b200.synth import grating_clip
    return grating_clip(W, H, N, seed=77, motion=5.0, rects=2)


def _oracle_chunks(chunks):
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_lib import OracleEncoder
    out = []
    for frames in chunks:
        enc = OracleEncoder(W, H, QP, profile=1, keyint=len(frames))   # a fresh encoder per chunk
        out.append([enc.encode(f)[0] for f in frames])
    return out


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    from ragdoll_b200.multi_gpu import chunks_of, encode_gop_parallel, my_chunks
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    seen = []

    def encode(chunks):
        seen.append(len(chunks))
        return _oracle_chunks(chunks)
    aus = encode_gop_parallel(_clip(), GOP, encode, dist)
    mine = my_chunks(len(chunks_of(N, GOP)), rank, world)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, mine, seen, None if aus is None else b"".join(aus), None if aus is None else len(aus)))


def test_two_ranks_give_the_one_rank_bytes():
    from ragdoll_b200.multi_gpu import encode_gop_parallel
    want = encode_gop_parallel(_clip(), GOP, _oracle_chunks, None)
    assert len(want) == N
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results[0][1] == [0, 2] and results[1][1] == [1, 3]
    assert results[1][3] is None, "only rank 0 gathers"
    assert results[0][4] == N and results[0][3] == b"".join(want)


import pytest  # noqa: E402


@pytest.mark.gpu
def test_gpu_chunk_encoder_gives_the_oracle_bytes():
    """One rank on the GPU: its chunks side by side in the encoder's waves (chunks of one length per
    wave, each a fresh GOP), gathered in chunk order -- the oracle's bytes."""
    from ragdoll_b200.multi_gpu import encode_gop_parallel, gpu_chunk_encoder
    frames = _clip()
    want = encode_gop_parallel(frames, GOP, _oracle_chunks, None)
    got = encode_gop_parallel(frames, GOP, gpu_chunk_encoder(W, H, QP, 1, device=0, threads=2), None)
    assert got == want
