"""Float64 restatement of the learned proposal's network (test
infrastructure: the checker of the FP16 tensor-core training kernels in
gpuupbp_b200/csrc/upbp_guide.cuh; nothing in the product imports it).

Network: 96 inputs (12-band frequency encoding of the position normalised to
the scene box, the direction of travel, a one-hot medium slot, one pad) ->
3 hidden layers of 64 ReLU units -> 48 outputs, of which 41 are used: 8 lobe
logits, 8 mean vectors (normalised), 8 log-kappas (kappa clamped to
[1e-2, 2e3]) and the logit of the selection probability a = 0.9
sigmoid(o[40]).  Loss of a row: -w log P(target), P = (1 - a) h + a q the
blend the renderer samples, h the phase function's pdf of the target
direction (a target's fifth value), q the 8-lobe von Mises-Fisher
mixture's, w the row weight divided by the batch mean weight.

`fp16_like_gpu` rounds the operands where the GPU kernels hold FP16 (inputs,
weights, the hidden activations after ReLU, the output gradients and the
hidden gradients after the ReLU mask), so that the remaining difference is
FP32 accumulation order only.
"""
from __future__ import annotations

import math

import numpy as np

BANDS, MEDIA, IN, HID, LOBES, OUT = 12, 20, 96, 64, 8, 48
LAYERS = [(IN, HID), (HID, HID), (HID, HID), (HID, OUT)]
KAPPA_MIN, KAPPA_MAX = 1e-2, 2e3


def param_layout():
    """Offsets of the four weight matrices (row-major [in][out]) and their
    biases in the flat parameter vector."""
    w_off, b_off, o = [], [], 0
    for i, n in LAYERS:
        w_off.append(o)
        o += i * n
    for _, n in LAYERS:
        b_off.append(o)
        o += n
    return w_off, b_off, o


def unpack(params: np.ndarray):
    w_off, b_off, _ = param_layout()
    Ws = [params[w_off[l]:w_off[l] + i * n].reshape(i, n) for l, (i, n) in enumerate(LAYERS)]
    bs = [params[b_off[l]:b_off[l] + n] for l, (_, n) in enumerate(LAYERS)]
    return Ws, bs


def encode(xn: np.ndarray, d: np.ndarray, slot: int) -> np.ndarray:
    """Input row of a normalised position, a direction of travel and a
    medium slot (the encoding of guide_encode)."""
    out = []
    for a in range(3):
        f = math.pi
        for _ in range(BANDS):
            out += [math.sin(f * xn[a]), math.cos(f * xn[a])]
            f *= 2.0
    out += list(d)
    out += [1.0 if m == slot else 0.0 for m in range(MEDIA)]
    out += [0.0] * (IN - len(out))
    return np.array(out)


def _h(a, on):
    return a.astype(np.float16).astype(np.float64) if on else a


def vmf_norm(k):
    return k / (2 * math.pi * (-np.expm1(-2 * k)))


ALPHA_MAX = 0.9
ALPHA_COL = 5 * LOBES


def row_loss_grad(o: np.ndarray, t: np.ndarray, wscale: float):
    """Loss and d loss / d output of one row (float64): -w log P with P =
    (1 - a) h + a q, h = t[4] the phase function's pdf of the target
    direction t[0:3], q the vMF mixture's, a = ALPHA_MAX sigmoid(o[40])."""
    lg = o[:LOBES]
    pi = np.exp(lg - lg.max())
    pi /= pi.sum()
    m = o[LOBES:4 * LOBES].reshape(LOBES, 3)
    mlen = np.maximum(np.linalg.norm(m, axis=1), 1e-6)
    mu = m / mlen[:, None]
    raw = np.exp(o[4 * LOBES:5 * LOBES])
    kap = np.clip(raw, KAPPA_MIN, KAPPA_MAX)
    w = t[:3]
    cosv = mu @ w
    val = vmf_norm(kap) * np.exp(kap * (cosv - 1))
    q = max(float(pi @ val), 1e-30)
    sig = 1.0 / (1.0 + math.exp(-o[ALPHA_COL]))
    a = ALPHA_MAX * sig
    h = float(t[4])
    P = max((1 - a) * h + a * q, 1e-30)
    wt = t[3] * wscale
    loss = -wt * math.log(P)
    sq = wt * a * q / P
    g = np.zeros(OUT)
    r = pi * val / q
    g[:LOBES] = sq * (pi - r)
    for j in range(LOBES):
        gmu = w * (-r[j] * kap[j])
        gm = (gmu - mu[j] * (gmu @ mu[j])) / mlen[j]
        g[LOBES + 3 * j:LOBES + 3 * j + 3] = sq * gm
        k = kap[j]
        e2 = math.exp(-2 * k)
        dlog = 1 / k - 2 * e2 / max(1 - e2, 1e-30) + (cosv[j] - 1)
        inside = 1.0 if KAPPA_MIN < raw[j] < KAPPA_MAX else 0.0
        g[4 * LOBES + j] = sq * (-r[j] * dlog * k * inside)
    g[ALPHA_COL] = -wt * (q - h) / P * ALPHA_MAX * sig * (1 - sig)
    return loss, g


def forward_backward(params: np.ndarray, X: np.ndarray, T: np.ndarray, fp16_like_gpu: bool = True):
    """Outputs, summed loss and gradient sums (flat, parameter layout) of
    a batch."""
    Ws, bs = unpack(params.astype(np.float64))
    Ws = [_h(W, fp16_like_gpu) for W in Ws]
    a = _h(X.astype(np.float64), fp16_like_gpu)
    acts = [a]
    for l in range(3):
        a = _h(np.maximum(a @ Ws[l] + bs[l], 0.0), fp16_like_gpu)
        acts.append(a)
    O = a @ Ws[3] + bs[3]
    wscale = len(T) / T[:, 3].sum()
    loss, dO = 0.0, np.zeros_like(O)
    for i in range(len(O)):
        li, gi = row_loss_grad(O[i], T[i].astype(np.float64), wscale)
        loss += li
        dO[i] = gi
    dY = _h(dO, fp16_like_gpu)
    gW, gb = [None] * 4, [None] * 4
    for l in range(3, -1, -1):
        gW[l] = acts[l].T @ dY
        gb[l] = dY.sum(axis=0)
        if l == 0:
            break
        dH = dY @ Ws[l].T
        dH = np.where(acts[l] > 0, dH, 0.0)
        dY = _h(dH, fp16_like_gpu)
    grads = np.concatenate([g.ravel() for g in gW] + list(gb))
    return O, loss, grads
