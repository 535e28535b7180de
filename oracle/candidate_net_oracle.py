"""TEST INFRASTRUCTURE ONLY: a float64 numpy restatement of the learned form's candidate network
(forward, losses and backward), the checker of the library's GPU training kernels and of its
tensor-core inference. The network has no counterpart in the reference; this file restates the
definition documented in include/ragdoll_cuda.h (rg_net_*):

  x = (crop - 128) / 64, crop 2 x 24 x 24 (the picture's and the previous picture's luma)
  a1 = relu(conv3x3(x; W1, b1))  32 x 22 x 22
  a2 = relu(conv3x3(a1; W2, b2)) 32 x 20 x 20
  a3 = relu(conv3x3(a2; W3, b3)) 32 x 18 x 18
  g = mean(a3) over 18 x 18;  f_b = mean of a3 over rows/cols 1 + 4 by .. 4 + 4 by (4x4 block b raster)
  partition logits Wp g + bp, offset Wm g + bm, intra 4x4 logits of block b Wi f_b + bi
  loss = CE(partition) averaged over labelled samples + CE(intra 4x4) averaged over labelled blocks
         + mv_weight * Huber(offset - target) averaged over labelled samples (both components summed)

Nothing in the product imports this module.
"""
from __future__ import annotations

import numpy as np

C = 32
SHAPES = [("W1", (C, 2, 3, 3)), ("b1", (C,)), ("W2", (C, C, 3, 3)), ("b2", (C,)), ("W3", (C, C, 3, 3)), ("b3", (C,)),
          ("Wp", (4, C)), ("bp", (4,)), ("Wm", (2, C)), ("bm", (2,)), ("Wi", (9, C)), ("bi", (9,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(flat):
    out, at = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(flat[at:at + n], np.float64).reshape(shape)
        at += n
    return out


def pack(d):
    return np.concatenate([d[name].reshape(-1) for name, _ in SHAPES])


def conv(x, W, b):
    """valid 3x3: x [N][cin][h][h] -> [N][32][h-2][h-2]"""
    n, cin, h, _ = x.shape
    ho = h - 2
    cols = np.empty((n, cin, 3, 3, ho, ho))
    for dy in range(3):
        for dx in range(3):
            cols[:, :, dy, dx] = x[:, :, dy:dy + ho, dx:dx + ho]
    return np.einsum("nikluv,oikl->nouv", cols, W) + b[None, :, None, None], cols


def conv_back(dz, cols, W, x_shape):
    """gradients of a valid 3x3 conv: dW, db and dx"""
    dW = np.einsum("nouv,nikluv->oikl", dz, cols)
    db = dz.sum(axis=(0, 2, 3))
    n, cin, h, _ = x_shape
    ho = h - 2
    dx = np.zeros(x_shape)
    dcols = np.einsum("nouv,oikl->nikluv", dz, W)
    for dy in range(3):
        for dx_ in range(3):
            dx[:, :, dy:dy + ho, dx_:dx_ + ho] += dcols[:, :, dy, dx_]
    return dW, db, dx


def block_means(a3):
    """[N][32][18][18] -> [N][16][32] (raster 4x4 blocks of the central 16 x 16)"""
    n = a3.shape[0]
    c = a3[:, :, 1:17, 1:17].reshape(n, C, 4, 4, 4, 4)  # n, c, by, y, bx, x
    return c.mean(axis=(3, 5)).transpose(0, 2, 3, 1).reshape(n, 16, C)


def forward_backward(flat, crops, part, i4, mv, mvv, mv_weight=1.0):
    """crops uint8 [N][2][24][24]; part [N] (-1 none); i4 [N][16] (-1 none); mv [N][2]; mvv [N].
    Returns (loss, grads flat, logits [N][150])."""
    p = unpack(flat)
    x = (np.asarray(crops, np.float64) - 128.0) / 64.0
    z1, c1 = conv(x, p["W1"], p["b1"]); a1 = np.maximum(z1, 0)
    z2, c2 = conv(a1, p["W2"], p["b2"]); a2 = np.maximum(z2, 0)
    z3, c3 = conv(a2, p["W3"], p["b3"]); a3 = np.maximum(z3, 0)
    n = x.shape[0]
    g = a3.mean(axis=(2, 3))
    f = block_means(a3)
    lp = g @ p["Wp"].T + p["bp"]
    lm = g @ p["Wm"].T + p["bm"]
    li = f @ p["Wi"].T + p["bi"]          # [N][16][9]
    logits = np.concatenate([lp, lm, li.reshape(n, 144)], axis=1)
    part = np.asarray(part); i4 = np.asarray(i4); mv = np.asarray(mv, np.float64); mvv = np.asarray(mvv)
    npart, ni, nm = int((part >= 0).sum()), int((i4 >= 0).sum()), int((mvv != 0).sum())
    sp, si, sm = (1.0 / npart if npart else 0.0), (1.0 / ni if ni else 0.0), (1.0 / nm if nm else 0.0)
    loss = 0.0
    dlp = np.zeros_like(lp); dlm = np.zeros_like(lm); dli = np.zeros_like(li)
    for k in range(n):
        if part[k] >= 0:
            e = np.exp(lp[k] - lp[k].max()); s = e.sum()
            loss += sp * (np.log(s) + lp[k].max() - lp[k, part[k]])
            dlp[k] = sp * (e / s - np.eye(4)[part[k]])
        if mvv[k]:
            d = lm[k] - mv[k]
            loss += sm * mv_weight * np.where(np.abs(d) <= 1, 0.5 * d * d, np.abs(d) - 0.5).sum()
            dlm[k] = sm * mv_weight * np.where(np.abs(d) <= 1, d, np.sign(d))
        for b in range(16):
            lab = i4[k, b]
            if lab >= 0:
                e = np.exp(li[k, b] - li[k, b].max()); s = e.sum()
                loss += si * (np.log(s) + li[k, b].max() - li[k, b, lab])
                dli[k, b] = si * (e / s - np.eye(9)[lab])
    grads = {"Wp": dlp.T @ g, "bp": dlp.sum(0), "Wm": dlm.T @ g, "bm": dlm.sum(0),
             "Wi": np.einsum("nbo,nbc->oc", dli, f), "bi": dli.sum(axis=(0, 1))}
    dg = dlp @ p["Wp"] + dlm @ p["Wm"]           # [N][32]
    df = dli @ p["Wi"]                            # [N][16][32]
    da3 = np.repeat(np.repeat(dg[:, :, None, None] / 324.0, 18, 2), 18, 3)
    dfb = (df / 16.0).reshape(n, 4, 4, C).transpose(0, 3, 1, 2)  # n, c, by, bx
    da3[:, :, 1:17, 1:17] += np.repeat(np.repeat(dfb, 4, 2), 4, 3)
    dz3 = da3 * (z3 > 0)
    grads["W3"], grads["b3"], da2 = conv_back(dz3, c3, p["W3"], a2.shape)
    dz2 = da2 * (z2 > 0)
    grads["W2"], grads["b2"], da1 = conv_back(dz2, c2, p["W2"], a1.shape)
    dz1 = da1 * (z1 > 0)
    grads["W1"], grads["b1"], _ = conv_back(dz1, c1, p["W1"], x.shape)
    return loss, pack(grads), logits


def forward_bf16(flat, crops):
    """The tensor-core inference's arithmetic: BF16 inputs, weights and activations (rounded after
    each layer's ReLU), products accumulated exactly (float64 here, f32 on the GPU); f32 heads.
    Returns logits [N][150]."""
    def bf16(a):
        a = np.asarray(a, np.float32)
        u = a.view(np.uint32).astype(np.uint64)
        r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
        return r.astype(np.uint32).view(np.float32).astype(np.float64)
    p = unpack(flat)
    x = bf16((np.asarray(crops, np.float64) - 128.0) / 64.0)
    a1 = bf16(np.maximum(conv(x, bf16(p["W1"]), p["b1"])[0], 0))
    a2 = bf16(np.maximum(conv(a1, bf16(p["W2"]), p["b2"])[0], 0))
    a3 = bf16(np.maximum(conv(a2, bf16(p["W3"]), p["b3"])[0], 0))
    n = a3.shape[0]
    g = a3.mean(axis=(2, 3))
    f = block_means(a3)
    lp = g @ p["Wp"].T + p["bp"]
    lm = g @ p["Wm"].T + p["bm"]
    li = f @ p["Wi"].T + p["bi"]
    return np.concatenate([lp, lm, li.reshape(n, 144)], axis=1)
