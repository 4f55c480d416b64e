"""CPU restatement (numpy, FP64) of the learned preconditioner correction of
crtomo_stable_b200/csrc/crt_gnn.cu -- TEST INFRASTRUCTURE ONLY.

The reference has no learned component (its CG is preconditioned by cgfac
alone, src/cg_mod.f90:426-518), so this file restates the network the
device implements, with the same parameter layout, and is used by the tests
to check the device's loss and weight gradients.  Its own backward pass is
checked against finite differences (tests/test_gnn.py).

Network (per model cell i, width W = 32, L = 3 layers, no biases):
    h0_i  = tanh(x_i Win)
    m_i   = sum_d a[i, d] h_{l-1}[nbr[i, d]]               (nbr = -1: none)
    h_l,i = tanh(h_{l-1},i Ws_l + m_i Wn_l)
    out_i = h3_i Wout
    loss  = sum_i |out_i - t_i|^2 / tnorm2
The device evaluates every forward pass with the weights rounded to bf16
(round to nearest even) and sums in FP32; `loss_grad(..., bf16=True)` takes
the same rounded weights and sums in FP64.
"""
from __future__ import annotations

import numpy as np

W, L, F, O, D = 32, 3, 4, 2, 4
OFF_IN = 0
OFF_L = F * W
LSTRIDE = 2 * W * W
OFF_OUT = OFF_L + L * LSTRIDE
NPARAM = OFF_OUT + W * O


def bf16_round(w):
    """FP32 values rounded to the nearest bfloat16 (ties to even), as FP64."""
    u = np.ascontiguousarray(w, np.float32).view(np.uint32).astype(np.uint64)
    lsb = (u >> np.uint64(16)) & np.uint64(1)
    u = (u + np.uint64(0x7FFF) + lsb) & np.uint64(0xFFFF0000)
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(w):
    w = np.asarray(w, np.float64)
    win = w[OFF_IN:OFF_IN + F * W].reshape(F, W)
    layers = []
    for l in range(L):
        o = OFF_L + l * LSTRIDE
        layers.append((w[o:o + W * W].reshape(W, W), w[o + W * W:o + 2 * W * W].reshape(W, W)))
    wout = w[OFF_OUT:OFF_OUT + W * O].reshape(W, O)
    return win, layers, wout


def _aggregate(h, nbr, a):
    m = np.zeros_like(h)
    for d in range(D):
        j = nbr[:, d]
        ok = j >= 0
        m[ok] += a[ok, d, None] * h[j[ok]]
    return m


def _aggregate_t(g, nbr, a):
    """Transpose of _aggregate: out[j] += a[i, d] g[i] for nbr[i, d] = j."""
    out = np.zeros_like(g)
    for d in range(D):
        j = nbr[:, d]
        ok = j >= 0
        np.add.at(out, j[ok], a[ok, d, None] * g[ok])
    return out


def forward(w, x, nbr, a):
    win, layers, wout = unpack(w)
    h = [np.tanh(x @ win)]
    aggs = []
    for ws, wn in layers:
        m = _aggregate(h[-1], nbr, a)
        aggs.append(m)
        h.append(np.tanh(h[-1] @ ws + m @ wn))
    return h[-1] @ wout, h, aggs


def loss_grad(w, x, t, nbr, a, tnorm2, bf16=True):
    """(loss, gradient [NPARAM]) of one record, in FP64."""
    x = np.asarray(x, np.float64)
    t = np.asarray(t, np.float64)
    a = np.asarray(a, np.float64)
    wf = bf16_round(w) if bf16 else np.asarray(w, np.float64)
    win, layers, wout = unpack(wf)
    out, h, aggs = forward(wf, x, nbr, a)
    tinv = 1.0 / tnorm2 if tnorm2 > 0 else 0.0
    e = out - t
    loss = float((e * e).sum() * tinv)
    dout = 2.0 * e * tinv
    g = np.zeros(NPARAM)
    g[OFF_OUT:OFF_OUT + W * O] = (h[-1].T @ dout).ravel()
    dh = dout @ wout.T
    for l in range(L - 1, -1, -1):
        ws, wn = layers[l]
        du = dh * (1.0 - h[l + 1] ** 2)
        o = OFF_L + l * LSTRIDE
        g[o:o + W * W] = (h[l].T @ du).ravel()
        g[o + W * W:o + 2 * W * W] = (aggs[l].T @ du).ravel()
        dh = du @ ws.T + _aggregate_t(du @ wn.T, nbr, a)
    du0 = dh * (1.0 - h[0] ** 2)
    g[OFF_IN:OFF_IN + F * W] = (x.T @ du0).ravel()
    return loss, g
