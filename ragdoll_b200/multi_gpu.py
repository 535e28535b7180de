"""GOP-parallel encoding over several GPUs (one process per GPU), ragdoll's parallel_gop_map
(crates/ragdoll-pipeline/src/lib.rs:110-157) spread over ranks instead of host threads.

A clip is cut into GOP chunks of `gop` pictures (GOP_FRAMES = 15, lib.rs:210); chunk k goes to rank
k % world. Each rank encodes its chunks with its own encoder, one fresh GOP per chunk (as the
pipeline's fresh H264Encoder per chunk, lib.rs:580-585), all of them side by side in its GPU's
persistent launches. There is no collective on the data path: the ranks' access units are gathered
to rank 0 once, after encoding, and concatenated in chunk order -- the same bytes whatever the
number of ranks (the reference's determinism contract, crates/ragdoll-pipeline/tests/determinism.rs).
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

Frame = Tuple["np.ndarray", "np.ndarray", "np.ndarray"]  # noqa: F821


def chunks_of(n_frames: int, gop: int) -> List[range]:
    """The GOP chunks of a clip of n_frames pictures (the last one may be shorter)."""
    return [range(s, min(s + gop, n_frames)) for s in range(0, n_frames, gop)]


def my_chunks(n_chunks: int, rank: int, world: int) -> List[int]:
    """Chunks of `rank`: round robin."""
    return list(range(rank, n_chunks, world))


def gpu_chunk_encoder(width: int, height: int, qp: int, profile: int, device: int, threads: int = 0):
    """Encoder of equally long chunks on `device`: all of a rank's chunks as the streams of one
    H264Encoder wave (ragdoll_b200.encoder), each a fresh GOP. Returns fn(chunks) -> [[au, ...] per chunk]."""
    def encode(chunk_frames: Sequence[Sequence[Frame]]):
        from .encoder import H264Encoder
        if not chunk_frames:
            return []
        lens = {len(c) for c in chunk_frames}
        out = []
        for L in sorted(lens):  # chunks of one length share a wave
            group = [i for i, c in enumerate(chunk_frames) if len(c) == L]
            enc = H264Encoder(width, height, qp, profile=profile, keyint=L, streams=len(group), max_frames=L,
                              device=device, threads=threads)
            enc.new_gops()
            enc.submit([[chunk_frames[i][f] for i in group] for f in range(L)])
            aus = enc.collect()
            enc.close()
            for k, i in enumerate(group):
                out.append((i, [aus[f][k] for f in range(L)]))
        return [a for _, a in sorted(out, key=lambda t: t[0])]
    return encode


def encode_gop_parallel(frames: Sequence[Frame], gop: int, encode_chunks: Callable, dist=None) -> Optional[List[bytes]]:
    """Encodes `frames` GOP-parallel over the ranks of the process group `dist` (torch.distributed,
    or None for one rank). encode_chunks(list of chunks' frames) -> list of each chunk's access
    units. Returns every access unit in display order on rank 0, None on the others."""
    rank = dist.get_rank() if dist is not None else 0
    world = dist.get_world_size() if dist is not None else 1
    chunks = chunks_of(len(frames), gop)
    mine = my_chunks(len(chunks), rank, world)
    coded = encode_chunks([[frames[i] for i in chunks[k]] for k in mine])
    local = list(zip(mine, coded))
    if dist is None:
        gathered = [local]
    else:
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(local, gathered, dst=0)
    if rank != 0:
        return None
    by_chunk = dict(kv for part in gathered for kv in part)
    return [au for k in range(len(chunks)) for au in by_chunk[k]]
