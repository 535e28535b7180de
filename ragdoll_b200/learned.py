"""The learned analysis form: its candidate network (rg_net_*), training on the full search's
decisions, and the hints the engine's learned form reads.

The network and the form have no counterpart in the reference. Training data is the full-search
form's own decisions on seeded synthetic clips (ragdoll_b200.synth): for every macroblock, its
24 x 24 luma window in the picture and in the previous picture (the crop), the partition type the
full search found cheapest (P pictures), the intra 4x4 mode of each block (intra 4x4 macroblocks of
IDR pictures) and the offset of the 16x16 vector from its predictor (P_L0_16x16 macroblocks). Every
kernel -- crops, forward, backward, Adam and the tensor-core inference -- is in the library; torch
only holds device memory.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from .engine import (HINT_DTYPE, RG_FORM_FULLSEARCH, RG_FRAME_IDR, RG_FRAME_P, RG_MB_P_L0_16X8, RgError, _check,
                     lib)

WEIGHTS = Path(__file__).resolve().parent / "weights" / "candidate_net.f32"
# the offset head's weights and biases in the parameter vector (rg_net_params order)
_C = 32
OFFSET_HEAD = slice(_C * 2 * 9 + _C + 2 * (_C * _C * 9 + _C) + 4 * _C + 4,
                    _C * 2 * 9 + _C + 2 * (_C * _C * 9 + _C) + 4 * _C + 4 + 2 * _C + 2)
N_LOGITS = 150
# decoding-order 4x4 block -> raster index
DEC_TO_RASTER = np.array([((b >> 1) & 1) * 4 + (b & 1) + ((b >> 3) & 1) * 8 + ((b >> 2) & 1) * 2 for b in range(16)])


class CandidateNet:
    """rg_net: parameters on `device`, f32 training state, BF16 tensor-core inference."""

    def __init__(self, device: int = 0, seed: int = 1, params: np.ndarray | None = None):
        self._destroy = lib().rg_net_destroy
        self.h = lib().rg_net_create(device, seed)
        if not self.h:
            raise RgError(-1, lib().rg_last_error().decode())
        self.device = device
        self.n_params = lib().rg_net_param_count()
        if params is not None:
            self.set_params(params)

    @classmethod
    def trained(cls, device: int = 0) -> "CandidateNet":
        """The network with the weights shipped in the package (ragdoll_b200/weights)."""
        return cls(device, params=np.fromfile(WEIGHTS, np.float32))

    def close(self) -> None:
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def params(self) -> np.ndarray:
        out = np.zeros(self.n_params, np.float32)
        _check(lib().rg_net_get_params(self.h, out.ctypes.data, self.n_params))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        _check(lib().rg_net_set_params(self.h, p.ctypes.data, p.size))

    def predict_hints(self, cur, prev, width: int, height: int, stride: int, hints, logits=None, stream: int = 0) -> None:
        """Queues the hints of len(cur) pictures: device addresses of each picture's luma, its previous
        picture's luma (itself for an IDR picture), its hint array and (optionally) its logits."""
        n = len(cur)
        A = ctypes.c_void_p * n
        lg = A(*logits) if logits is not None else None
        _check(lib().rg_net_predict_hints(self.h, A(*cur), A(*prev), n, width, height, stride, A(*hints), lg,
                                          stream or None))

    def set_hint_policy(self, part_k: int = 3, part_margin: float = float("inf"), i4_k: int = 3,
                        i4_margin: float = float("inf")) -> None:
        """Candidates the hints keep (rg_net_set_hint_policy): the best partition type, then the next
        ones up to part_k while within part_margin of the best logit; intra 4x4 modes alike."""
        _check(lib().rg_net_set_hint_policy(self.h, part_k, part_margin, i4_k, i4_margin))

    def set_coarse_range(self, search_range: int = 32) -> None:
        """Range (samples, even, 0: off) of the coarse motion pass that follows the network in
        predict_hints and fills the hints' mv_coarse (rg_net_set_coarse_range)."""
        _check(lib().rg_net_set_coarse_range(self.h, search_range))

    def check(self, stream: int = 0) -> None:
        _check(lib().rg_net_check(self.h, stream or None))

    def crops(self, cur, prev, mb_xy: np.ndarray, width: int, height: int, stride: int, out_ptr: int, stream: int = 0):
        n = len(cur)
        A = ctypes.c_void_p * n
        xy = np.ascontiguousarray(mb_xy, np.int32)
        _check(lib().rg_net_crops(self.h, A(*cur), A(*prev), xy.ctypes.data, n, width, height, stride, out_ptr,
                                  stream or None))

    def forward_backward(self, crops_ptr: int, n: int, part_ptr: int, i4_ptr: int, mv_ptr: int, mvv_ptr: int,
                         mv_weight: float = 0.25, logits_ptr: int = 0, want_grads: bool = False):
        """One forward and backward pass over n device crops; returns (loss, grads or None)."""
        loss = ctypes.c_float()
        grads = np.zeros(self.n_params, np.float32) if want_grads else None
        _check(lib().rg_net_forward_backward(self.h, crops_ptr, n, part_ptr, i4_ptr, mv_ptr, mvv_ptr, mv_weight,
                                             logits_ptr or None, ctypes.byref(loss),
                                             grads.ctypes.data if want_grads else None))
        return loss.value, grads

    def adam_step(self, lr: float) -> None:
        _check(lib().rg_net_adam_step(self.h, lr))


def labels_from_records(recs: np.ndarray, idr: bool):
    """Training labels of one picture's records (full-search form): partition type (-1 none), the
    intra 4x4 mode of each raster block (-1 none), the 16x16 offset target (vector difference / 16
    quarter samples) and its validity."""
    n = len(recs)
    part = np.full(n, -1, np.int32)
    i4 = np.full((n, 16), -1, np.int32)
    mv = np.zeros((n, 2), np.float32)
    mvv = np.zeros(n, np.int32)
    if idr:
        sel = recs["mb_type"] == 3
        i4[sel] = recs["i4_modes"][sel][:, np.argsort(DEC_TO_RASTER)]
    else:
        pt = recs["part_type"].astype(np.int32)
        part[pt != 255] = pt[pt != 255]
        sel = recs["mb_type"] == 1
        mv[sel] = recs["mvd"][sel].astype(np.float32) / 16.0
        mvv[sel] = 1
    return part, i4, mv, mvv


def generate_training_set(n_clips: int, width: int, height: int, frames: int, search_range: int = 32,
                          qps=(22, 26, 30, 34), device: int = 0, seed0: int = 50000, streams: int = 8,
                          labels: str = "fullsearch"):
    """Runs a labelling form on seeded clips (each a GOP: IDR + P pictures, `streams` clips per
    pipelined launch, QPs cycling through `qps`) and returns device tensors: crops [N][2][24][24] u8,
    part [N], i4 [N][16], mv [N][2], mvv [N]. labels "fullsearch": the full-search form's decisions;
    "learned": the learned form's own search with every candidate open (all four partition types,
    all nine intra 4x4 modes, the coarse motion vector, no network offset) -- the choices the
    restricted search is to reproduce."""
    import torch

    from .engine import RG_FORM_LEARNED, RG_PROFILE_HIGH, Engine
    from .synth import grating_clip

    if labels not in ("fullsearch", "learned"):
        raise ValueError(f"labels {labels!r}")
    dev = torch.device("cuda", device)
    net = CandidateNet(device)
    opener = None
    if labels == "learned":
        # a network whose hints keep every candidate and offer no offset: only its coarse pass matters
        opener = CandidateNet(device, seed=1)
        p = opener.params()
        p[OFFSET_HEAD] = 0.0
        opener.set_params(p)
        opener.set_hint_policy(4, float("inf"), 9, float("inf"))
    crops, parts, i4s, mvs, mvvs = [], [], [], [], []
    cw, ch = (width + 1) // 2, (height + 1) // 2
    for c0 in range(0, n_clips, streams):
        S = min(streams, n_clips - c0)
        qp = qps[(c0 // streams) % len(qps)]
        clips = [grating_clip(width, height, frames, seed=seed0 + c0 + s, motion=24.0, rects=12) for s in range(S)]
        eng = Engine(width, height, qp, profile=RG_PROFILE_HIGH, num_streams=S, max_frames=frames, device=device)
        if opener is None:
            eng.set_analysis_form(RG_FORM_FULLSEARCH, search_range)
        else:
            eng.set_analysis_form(RG_FORM_LEARNED, search_range)
            eng.set_hint_net(opener)
        kinds = [[RG_FRAME_IDR if f == 0 else RG_FRAME_P] * S for f in range(frames)]
        recs = eng.analyse_gops([[clips[s][f] for s in range(S)] for f in range(frames)], kinds)
        eng.close()
        luma = torch.from_numpy(np.stack([[clips[s][f][0] for f in range(frames)] for s in range(S)])).to(dev)
        mb_w, mb_h = (width + 15) // 16, (height + 15) // 16
        xy = np.stack(np.meshgrid(np.arange(mb_w), np.arange(mb_h)), -1).reshape(-1, 2).astype(np.int32)
        for s in range(S):
            for f in range(frames):
                cur = luma[s, f].data_ptr()
                prev = luma[s, f - 1].data_ptr() if f > 0 else cur
                out = torch.empty((len(xy), 2, 24, 24), dtype=torch.uint8, device=dev)
                net.crops([cur] * len(xy), [prev] * len(xy), xy, width, height, width, out.data_ptr())
                p, i, m, v = labels_from_records(recs[f, s], f == 0)
                crops.append(out)
                parts.append(p); i4s.append(i); mvs.append(m); mvvs.append(v)
        del luma
    net.close()
    if opener is not None:
        opener.close()
    t = lambda a: torch.from_numpy(np.concatenate(a)).to(dev)  # noqa: E731
    return torch.cat(crops), t(parts), t(i4s), t(mvs), t(mvvs)


def train(net: CandidateNet, data, epochs: int = 2, batch: int = 256, lr: float = 2e-3, lr_end: float = 1e-4,
          mv_weight: float = 0.25, seed: int = 0, log=None):
    """Adam over shuffled batches with a cosine learning rate from lr to lr_end; returns the mean
    loss of each epoch."""
    import math

    import torch

    crops, part, i4, mv, mvv = data
    n = crops.shape[0]
    steps = epochs * (n // batch)
    g = torch.Generator(device="cpu").manual_seed(seed)
    losses, k = [], 0
    for e in range(epochs):
        perm = torch.randperm(n, generator=g).to(crops.device)
        tot, cnt = 0.0, 0
        for b0 in range(0, n - batch + 1, batch):
            idx = perm[b0:b0 + batch]
            bc, bp, bi, bm, bv = (x[idx].contiguous() for x in (crops, part, i4, mv, mvv))
            loss, _ = net.forward_backward(bc.data_ptr(), batch, bp.data_ptr(), bi.data_ptr(), bm.data_ptr(),
                                           bv.data_ptr(), mv_weight)
            rate = lr_end + 0.5 * (lr - lr_end) * (1 + math.cos(math.pi * k / max(steps, 1)))
            net.adam_step(rate)
            tot += loss
            cnt += 1
            k += 1
            if log and k % 500 == 0:
                log(f"step {k}/{steps} loss {tot / cnt:.4f}")
        losses.append(tot / max(cnt, 1))
    return losses


def hints_for(net: CandidateNet, luma_ptrs, prev_ptrs, width: int, height: int, stride: int, device: int = 0,
              stream: int = 0, with_logits: bool = False):
    """Device hint arrays (one torch tensor per picture) predicted for the given luma planes."""
    import torch

    mb_w, mb_h = (width + 15) // 16, (height + 15) // 16
    dev = torch.device("cuda", device)
    hints = [torch.empty(mb_w * mb_h * HINT_DTYPE.itemsize, dtype=torch.uint8, device=dev) for _ in luma_ptrs]
    logits = [torch.empty(mb_w * mb_h * N_LOGITS, dtype=torch.float32, device=dev) for _ in luma_ptrs] if with_logits else None
    net.predict_hints(luma_ptrs, prev_ptrs, width, height, stride, [h.data_ptr() for h in hints],
                      [l.data_ptr() for l in logits] if logits else None, stream)
    return hints, logits


def prior_hints(n_mb: int, part_order=(0, 1, 2), i4_modes=(2, 0, 1), mv_off=(0, 0)) -> np.ndarray:
    """Hints without the network: the same fixed candidates for every macroblock (by default the
    three partition types and intra 4x4 modes the training labels hold most often)."""
    h = np.zeros(n_mb, HINT_DTYPE)
    h["part_mask"] = sum(1 << p for p in part_order)
    h["mv_off"] = mv_off
    h["i4_mask"] = sum(1 << m for m in i4_modes)
    return h


__all__ = ["CandidateNet", "WEIGHTS", "generate_training_set", "train", "hints_for", "prior_hints",
           "labels_from_records", "RG_MB_P_L0_16X8"]
