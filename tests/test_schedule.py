"""The pipelined kernel's work order never waits for work that no warp can take (CPU test).

rg_pipeline_work_list returns the library's own work list for a shape. A discrete-event simulation
then runs warps over it the way pipeline_kernel does: each warp holds one segment, takes tickets
from its role's queue in order and falls back to the other queues when its own is empty, and
advances a macroblock per step only when the kernel's waits are met:

* analysis of (x, y): (x - 1, y) analysed, (x + 1, y - 1) analysed (two ahead of the row above);
  in a P picture the co-located macroblock of the previous picture analysed and the previous
  picture deblocked over the search region, taken here as `reach` macroblocks beyond zero motion;
* deblocking of (x, y): (x - 1, y) deblocked, (x + 1, y) and (x, y + 1) analysed,
  (x + 1, y - 1) deblocked.

With the default lag (searches up to four macroblock rows beyond zero motion) every shape and warp
mix must finish; a lag far below the reach must be able to stall (which the kernel turns into a
timeout and an exact re-run on the per-diagonal path).
"""
import ctypes

import numpy as np
import pytest

from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, lib


def work_list(mb_w, mb_h, streams, frames, lag, seg, split, kinds):
    cap = 2 * frames * streams * mb_h * ((mb_w + seg - 1) // seg)
    tasks = np.zeros(2 * cap, np.int32)
    queues = np.zeros(6, np.int32)
    k = None
    if kinds is not None:
        k = np.ascontiguousarray(kinds, np.int32)
    n = lib().rg_pipeline_work_list(mb_w, mb_h, streams, frames, lag, seg, split,
                                    k.ctypes.data if k is not None else None,
                                    tasks.ctypes.data, cap, queues.ctypes.data)
    assert n == cap
    return tasks[:2 * n].reshape(n, 2), [(int(queues[2 * q]), int(queues[2 * q + 1])) for q in range(3)]


ORDER = {0: (0, 1, 2), 1: (1, 2, 0), 2: (2, 0, 1)}  # queue order per warp role, as in the kernel


def simulate(mb_w, mb_h, streams, frames, lag, seg, reach, warps, idr_every=None):
    """warps = (analysis, deblocking, IDR-analysis) warp counts. Returns steps, or None on a stall."""
    W, H, S, F = mb_w, mb_h, streams, frames
    kinds = np.full(F * S, RG_FRAME_P, np.int32)
    for f in range(F):
        if f == 0 or (idr_every and f % idr_every == 0):
            kinds[f * S:(f + 1) * S] = RG_FRAME_IDR
    split = 1 if warps[1] else 0
    tasks, queues = work_list(W, H, S, F, lag, seg, split, kinds if warps[2] else None)
    ana = np.zeros(F * S * H, np.int64)
    db = np.zeros(F * S * H, np.int64)
    ticket = [q[0] for q in queues]
    held = []  # [role, task, x]

    def take(role):
        for q in ORDER[role]:
            if ticket[q] < queues[q][1]:
                t = ticket[q]
                ticket[q] += 1
                return t
        return None

    for role, n in enumerate(warps):
        for _ in range(n):
            t = take(role)
            if t is not None:
                held.append([role, t, (int(tasks[t, 1]) >> 1) & 0x7FFF])
    total, done, steps = 2 * F * S * H * W, 0, 0
    while done < total:
        steps += 1
        moved, pub = 0, []
        for w in held:
            if w[1] is None:
                continue
            ps, packed = int(tasks[w[1], 0]), int(tasks[w[1], 1])
            f, y, x0, deblock = ps // S, packed >> 16, (packed >> 1) & 0x7FFF, packed & 1
            x = w[2]
            A, D = ps * H, ps * H
            if not deblock:
                ok = ana[A + y] >= x and (y == 0 or ana[A + y - 1] >= min(x + 2, W))
                if ok and f > 0 and kinds[ps] == RG_FRAME_P:
                    pa, pd = (ps - S) * H, (ps - S) * H
                    xx, rr = min(x + 2 + reach, W - 1), min(y + 2 + reach, H - 1)
                    ok = ana[pa + y] >= x + 1 and (db[pd + rr + 1] >= xx + 1 if rr < H - 1 else db[pd + rr] >= min(xx + 2, W))
                if ok:
                    pub.append((ana, A + y, x + 1))
            else:
                ok = (db[D + y] >= x and ana[A + y] >= min(x + 2, W)
                      and (y + 1 >= H or ana[A + y + 1] >= min(x + 1, W))
                      and (y == 0 or db[D + y - 1] >= min(x + 2, W)))
                if ok:
                    pub.append((db, D + y, x + 1))
            if ok:
                moved += 1
                done += 1
                w[2] += 1
                if w[2] >= min(x0 + seg, W):
                    t = take(w[0])
                    w[1] = t
                    if t is not None:
                        w[2] = (int(tasks[t, 1]) >> 1) & 0x7FFF
        for arr, i, v in pub:
            assert arr[i] == v - 1      # every macroblock once, in order along its row
            arr[i] = v
        if not moved:
            return None
    assert (ana == W).all() and (db == W).all()
    return steps


@pytest.mark.parametrize("shape", [
    (8, 5, 2, 4),      # tiny picture, two streams
    (20, 12, 3, 6),
    (40, 23, 2, 5),    # 640x360
])
@pytest.mark.parametrize("warps", [(1, 0, 0), (3, 1, 1), (12, 4, 6), (40, 10, 20), (2, 1, 0)])
@pytest.mark.parametrize("reach", [0, 2, 4])
@pytest.mark.parametrize("seg", [1, 2])
def test_default_order_never_stalls(shape, warps, reach, seg):
    W, H, S, F = shape
    assert simulate(W, H, S, F, 0, seg, reach, warps) is not None


def test_longer_segments_and_gops_in_one_call():
    assert simulate(24, 10, 2, 8, 0, 8, 2, (6, 2, 3), idr_every=4) is not None
    assert simulate(24, 10, 3, 6, 40, 4, 4, (9, 3, 0)) is not None


def test_lag_below_the_reach_can_stall():
    """One warp and lag 1: a P picture's first segment comes before the deblocking it waits
    for -- the situation the kernel's time limit and exact re-run exist for."""
    assert simulate(8, 6, 1, 3, 1, 2, 0, (1, 0, 0)) is None


def test_work_list_covers_every_segment_once():
    W, H, S, F, seg = 13, 7, 3, 4, 2
    kinds = np.full(F * S, RG_FRAME_P, np.int32)
    kinds[:S] = RG_FRAME_IDR
    tasks, queues = work_list(W, H, S, F, 0, seg, 1, kinds)
    seen = {(int(t[0]), int(t[1])) for t in tasks}
    segs = (W + seg - 1) // seg
    assert len(seen) == len(tasks) == 2 * F * S * H * segs
    assert queues[0][0] == 0 and queues[2][1] == len(tasks)
    for q in range(3):
        for t in tasks[queues[q][0]:queues[q][1]]:
            f, deblock = int(t[0]) // S, int(t[1]) & 1
            want = 1 if deblock else (2 if kinds[int(t[0])] == RG_FRAME_IDR else 0)
            assert want == q
