"""CPU restatement (numpy, FP64) of the learned coarse-grid correction.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA network in
gpe_b200/csrc/cnn_kernels.cuh.  No product path imports this module.

The reference has no learned component, so this file restates the network
defined for this project (include/gpe_cnn.h):

  a0 = (Re psi, Im psi, 0, ..., 0)                       16 channels
  pre_l = conv3d(a_l, W_l) + b_l,  a_{l+1} = GELU(pre_l)  l = 0, 1, 2
  delta = out_scale * (conv3d(a_3, W_3) + b_3)[..., 0:2]

conv3d: 3x3x3, periodic, out(p)[co] = sum_tap sum_ci W[tap][co][ci] a(p + d_tap)[ci],
tap = (dz+1)*9 + (dy+1)*3 + (dx+1).  GELU in its tanh form (Hendrycks &
Gimpel, 2016): 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))).  Loss of a pair (u, target):
mean over sites of |u + delta(u) - target|^2.

emulate=True mirrors the CUDA path's rounding points: weights, the packed
input, every GELU output, every stored pre-activation and every stored
gradient are rounded to bfloat16 (round to nearest even), as the kernels
store them; accumulation stays FP64 here (FP32 on the GPU).
emulate=False is the exact FP64 function and its exact gradient, the one
checked against finite differences.
"""
from __future__ import annotations

import math

import numpy as np

NL, NT, C = 4, 27, 16

def taps():
    """(dz, dy, dx) of tap index t = (dz+1)*9 + (dy+1)*3 + (dx+1)."""
    return [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(NT)]


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


_C = math.sqrt(2.0 / math.pi)
_A = 0.044715


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(_C * (x + _A * x ** 3)))


def gelu_grad(x):
    t = np.tanh(_C * (x + _A * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * _C * (1.0 + 3.0 * _A * x * x)


def shift(a, d):
    """s(p) = a(p + d), periodic; a indexed [z][y][x][c]."""
    dz, dy, dx = d
    return np.roll(a, shift=(-dz, -dy, -dx), axis=(0, 1, 2))


def conv(a, w):
    out = np.zeros(a.shape[:3] + (C,))
    for t, d in enumerate(taps()):
        out += np.einsum("zyxi,oi->zyxo", shift(a, d), w[t], optimize=True)
    return out


def conv_t(g, w):
    """Adjoint of conv: dx(p)[ci] = sum_tap sum_co g(p - d)[co] w[tap][co][ci]."""
    out = np.zeros(g.shape[:3] + (C,))
    for t, (dz, dy, dx) in enumerate(taps()):
        out += np.einsum("zyxo,oi->zyxi", shift(g, (-dz, -dy, -dx)), w[t], optimize=True)
    return out


def forward(psi, w, b, out_scale, emulate=True):
    """psi (nz, ny, nx) complex; w (4, 27, 16, 16); b (4, 16).
    Returns (delta (nz, ny, nx, 2), cache for backward)."""
    rnd = bf16 if emulate else (lambda v: np.asarray(v, dtype=np.float64))
    wr = rnd(w)
    b = np.asarray(b, dtype=np.float64)
    a = np.zeros(psi.shape + (C,))
    if emulate:
        a[..., 0] = bf16(np.asarray(psi.real, dtype=np.float32))
        a[..., 1] = bf16(np.asarray(psi.imag, dtype=np.float32))
    else:
        a[..., 0] = psi.real
        a[..., 1] = psi.imag
    acts, pres = [a], []
    for l in range(3):
        pre = conv(a, wr[l]) + b[l]
        pres.append(rnd(pre))
        a = rnd(gelu(pre))
        acts.append(a)
    out = conv(a, wr[3]) + b[3]
    delta = out_scale * out[..., :2]
    return delta, {"acts": acts, "pres": pres, "wr": wr, "emulate": emulate}


def loss_and_grad(u, target, w, b, out_scale, emulate=True):
    """Loss of one pair and (dW (4,27,16,16), db (4,16))."""
    rnd = bf16 if emulate else (lambda v: v)
    delta, cache = forward(u, w, b, out_scale, emulate)
    n = u.size
    er = u.real + delta[..., 0] - target.real
    ei = u.imag + delta[..., 1] - target.imag
    loss = float(np.sum(er * er + ei * ei) / n)
    g = np.zeros(u.shape + (C,))
    g[..., 0] = rnd(2.0 * er / n * out_scale)
    g[..., 1] = rnd(2.0 * ei / n * out_scale)
    dw = np.zeros((NL, NT, C, C))
    db = np.zeros((NL, C))
    acts, pres, wr = cache["acts"], cache["pres"], cache["wr"]
    for l in range(NL - 1, -1, -1):
        for t, d in enumerate(taps()):
            dw[l, t] = np.einsum("zyxo,zyxi->oi", g, shift(acts[l], d), optimize=True)
        db[l] = g.sum(axis=(0, 1, 2))
        if l > 0:
            g = rnd(conv_t(g, wr[l]) * gelu_grad(pres[l - 1]))
    mask_w, mask_b = masks()
    return loss, dw * mask_w, db * mask_b


def masks():
    """1 for the real parameters: layer 0 reads 2 input channels, layer 3
    writes 2 output channels."""
    mw = np.ones((NL, NT, C, C))
    mw[0, :, :, 2:] = 0
    mw[3, :, 2:, :] = 0
    mb = np.ones((NL, C))
    mb[3, 2:] = 0
    return mw, mb
