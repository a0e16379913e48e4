"""The con2prim-guess network restated in numpy, FP64.

TEST INFRASTRUCTURE ONLY: the checker of the CUDA network's forward pass and
gradients (black-hole-simulator_b200/csrc/bh_mlp.cu); nothing in the product
imports it.  The network has no counterpart in the reference (its con2prim
starts Newton at the bracket midpoint, conserved.cpp:170): 6 features of a
cell's conserved state -> 64 tanh -> 64 tanh -> 2 linear outputs, parameters
in the flat order W1 [64][6], b1 [64], W2 [64][64], b2 [64], W3 [2][64],
b3 [2], then mean[6] and 1/std[6] of the features.  Weights are used with
their BF16 roundings, as the device uses them.
"""
from __future__ import annotations

import numpy as np

NI, NH, NO = 6, 64, 2
SIZES = [("W1", (NH, NI)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NO, NH)), ("b3", (NO,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)


def bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even), as float64."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(w):
    out, o = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = np.asarray(w[o:o + k], np.float64).reshape(shape)
        o += k
    out["mean"] = np.asarray(w[o:o + NI], np.float64)
    out["istd"] = np.asarray(w[o + NI:o + 2 * NI], np.float64)
    return out


def features(pre, r):
    """[n][6] features from the con2prim preamble pre [5][n] (D, tau, Ssq,
    Bsq, SB) and r, rounded to float32 as the device rounds them."""
    D, tau, Ssq, Bsq, SB = pre
    x = np.stack([np.log(D), np.arcsinh(tau / D), np.log1p(Ssq / (D * D)), np.log1p(Bsq / D),
                  np.arcsinh(SB / (D * np.sqrt(D))), np.log(r)], 1)
    return x.astype(np.float32).astype(np.float64)


def forward(w, x):
    p = unpack(w)
    xn = (x - p["mean"]) * p["istd"]
    a1 = xn @ bf16(p["W1"]).T + bf16(p["b1"])
    h1 = np.tanh(a1)
    a2 = h1 @ bf16(p["W2"]).T + bf16(p["b2"])
    h2 = np.tanh(a2)
    y = h2 @ bf16(p["W3"]).T + bf16(p["b3"])
    return xn, h1, h2, y


def loss_and_grad(w, x, target):
    """Mean over cells of sum_o (y_o - t_o)^2 and its gradient with respect to
    the (BF16-rounded) weights, flat in parameter order."""
    p = unpack(w)
    xn, h1, h2, y = forward(w, x)
    n = len(x)
    e = y - target
    dy = 2.0 * e / n
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    d2 = (dy @ bf16(p["W3"])) * (1 - h2 * h2)
    g["W2"], g["b2"] = d2.T @ h1, d2.sum(0)
    d1 = (d2 @ bf16(p["W2"])) * (1 - h1 * h1)
    g["W1"], g["b1"] = d1.T @ xn, d1.sum(0)
    flat = np.concatenate([g[name].reshape(-1) for name, _ in SIZES])
    return float((e * e).sum()), flat
