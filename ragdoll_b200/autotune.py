"""Autotuner of the pipelined launch shape.

The persistent launch's best shape depends on the workload: how many warps per SM it keeps
resident (more warps overlap more waits, until they slow every macroblock on the critical path or
sit polling for work a small picture cannot offer) and how many macroblocks a work segment spans.
``autotune_pipeline`` times candidate shapes on a sample wave of the workload -- one persistent
launch per try, sources already on the device, CUDA events on the engine's stream -- and returns
the fastest, for ``Engine.set_pipeline_tuning`` / ``H264Encoder.set_pipeline_tuning``. Every shape
gives the same records (the tests check it); only the time differs. No counterpart in the
reference (its GOP threads have no device schedule).
"""
from __future__ import annotations

import statistics
from typing import Dict, List, Sequence, Tuple

import numpy as np

from .engine import Engine

# warps per SM x macroblocks per segment (lag, queues: library defaults)
DEFAULT_CANDIDATES = [{"per_sm": p, "seg": s} for p in (4, 8, 12, 16) for s in (1, 2)]


def autotune_pipeline(width: int, height: int, qp: int, profile: int, frames: Sequence[Sequence[Tuple]],
                      kinds: Sequence[Sequence[int]], candidates: List[Dict] | None = None, repeats: int = 3,
                      device: int = 0) -> Tuple[Dict, List[Tuple[Dict, float]]]:
    """frames[f][s] = (y, u, v) host planes and kinds[f][s] of a sample wave. Returns
    (tuning keywords of the fastest candidate, [(candidate, median launch ms)])."""
    import torch

    cands = candidates or DEFAULT_CANDIDATES
    F, S = len(frames), len(frames[0])
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    cw, ch = (width + 1) // 2, (height + 1) // 2
    fb = width * height + 2 * cw * ch
    host = np.empty((F * S, fb), np.uint8)
    for f in range(F):
        for s in range(S):
            y, u, v = frames[f][s]
            host[f * S + s] = np.concatenate([np.ascontiguousarray(p).reshape(-1)[:n] for p, n in
                                              ((y, width * height), (u, cw * ch), (v, cw * ch))])
    dev = torch.from_numpy(host).to(f"cuda:{device}")
    base = dev.data_ptr()
    ptrs = []
    for i in range(F * S):
        p = base + i * fb
        ptrs += [p, p + width * height, p + width * height + cw * ch]
    flat_kinds = [int(kinds[f][s]) for f in range(F) for s in range(S)]
    eng = Engine(width, height, qp, profile=profile, num_streams=S, device=device, max_frames=F)
    stream = torch.cuda.ExternalStream(eng.cuda_stream, device=f"cuda:{device}")
    table = []
    try:
        for c in cands:
            tuning = {k: v for k, v in c.items() if k != "per_sm"}
            tuning["grid"] = int(c.get("per_sm", 0)) * sms
            eng.set_pipeline_tuning(**tuning)
            eng.analyse_gops_device(ptrs, width, cw, flat_kinds, F)   # warm (task list, caches)
            times = []
            for _ in range(repeats):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                eng.analyse_gops_device(ptrs, width, cw, flat_kinds, F)
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
            eng.sync()
            table.append((dict(c), statistics.median(times)))
    finally:
        eng.close()
    best = min(table, key=lambda t: t[1])[0]
    tuning = {k: v for k, v in best.items() if k != "per_sm"}
    tuning["grid"] = int(best.get("per_sm", 0)) * sms
    return tuning, table
