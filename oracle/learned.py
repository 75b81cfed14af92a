"""CPU restatement of the learned convolution function (test infrastructure).

The learned form replaces a tabulated CF cache by a sinusoidal MLP (SIREN):

    inputs  x = (u, v, w, f, b): the tap's continuous offset from the sample
            in cells, u = jx - S + fracu/os and v = jy - S + fracv/os, divided
            by (S + 1); the w term of the plane divided by wmax; frequency and
            beam index mapped to [-1, 1] (0 when the CF does not depend on them)
    z0 = omega0 * (W0 x + b0),  h0 = sin(z0)                      (5 -> 64)
    zk = Wk h(k-1) + bk,        hk = sin(zk),  k = 1, 2, 3        (64 -> 64)
    y  = Wo h3 + bo                                               (64 -> 2)

y is (real, imaginary) of the tap divided by the CF table's largest |tap|.
Weights are stored in FP16 and every product is accumulated in FP32: the
forward and backward passes here use the FP16-rounded weights, and gradients
are applied to FP32 master weights (Adam).  The activations h0, h1, h2 are
rounded to FP16 (the operands of the kernels' tensor-core layers); the
rounding passes gradients straight through.  Nothing of this exists in the
reference: the targets are the reference's tabulated CFs
(WProjectVisGridder::initConvolutionFunction, restated in cf.py), and the
parameter layout below is the one the CUDA kernels use.

Parameter vector layout (float32, contiguous):
    W0 [5][64] (input-major), b0 [64],
    W1, W2, W3 [64][68] (input-major, rows padded to 68), b1, b2, b3 [64],
    Wo [64][2], bo [2]
"""
from __future__ import annotations

import numpy as np

NIN = 5
H = 64
HP = 68            # padded row of a hidden weight matrix
NOUT = 2
NHID = 3           # 64 -> 64 layers after the first
OMEGA0 = 30.0


def layout():
    off = {}
    o = 0
    off["W0"] = o; o += NIN * H
    off["b0"] = o; o += H
    for k in range(1, NHID + 1):
        off["W%d" % k] = o; o += H * HP
        off["b%d" % k] = o; o += H
    off["Wo"] = o; o += H * NOUT
    off["bo"] = o; o += NOUT
    off["total"] = o
    return off


OFF = layout()
NPARAM = OFF["total"]


def unpack(p):
    """Views of the weight matrices (the padding columns dropped)."""
    p = np.asarray(p)
    d = {"W0": p[OFF["W0"]:OFF["W0"] + NIN * H].reshape(NIN, H), "b0": p[OFF["b0"]:OFF["b0"] + H]}
    for k in range(1, NHID + 1):
        d["W%d" % k] = p[OFF["W%d" % k]:OFF["W%d" % k] + H * HP].reshape(H, HP)[:, :H]
        d["b%d" % k] = p[OFF["b%d" % k]:OFF["b%d" % k] + H]
    d["Wo"] = p[OFF["Wo"]:OFF["Wo"] + H * NOUT].reshape(H, NOUT)
    d["bo"] = p[OFF["bo"]:OFF["bo"] + NOUT]
    return d


def init_params(seed=0):
    """SIREN initialisation: first layer U(-1/n, 1/n), later layers
    U(-sqrt(6/n), sqrt(6/n)), biases likewise; padding columns zero."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, dtype=np.float32)
    p[OFF["W0"]:OFF["W0"] + NIN * H] = rng.uniform(-1.0 / NIN, 1.0 / NIN, NIN * H)
    p[OFF["b0"]:OFF["b0"] + H] = rng.uniform(-1.0 / NIN, 1.0 / NIN, H)
    lim = np.sqrt(6.0 / H)
    for k in range(1, NHID + 1):
        w = np.zeros((H, HP), dtype=np.float32)
        w[:, :H] = rng.uniform(-lim, lim, (H, H))
        p[OFF["W%d" % k]:OFF["W%d" % k] + H * HP] = w.ravel()
        p[OFF["b%d" % k]:OFF["b%d" % k] + H] = rng.uniform(-1.0 / np.sqrt(H), 1.0 / np.sqrt(H), H)
    p[OFF["Wo"]:OFF["Wo"] + H * NOUT] = rng.uniform(-lim, lim, H * NOUT)
    return p


def round16(p):
    """The FP16 weights the kernels compute with."""
    return np.asarray(p, dtype=np.float32).astype(np.float16).astype(np.float32)


def activations(z, round_act=True):
    """h_k = sin(z_k); with round_act, h0, h1, h2 rounded to FP16, as they
    enter the tensor-core layers; h3 (input of the FP32 output layer) never."""
    hs = [np.sin(zk) for zk in z]
    if round_act:
        for k in range(NHID):
            hs[k] = hs[k].astype(np.float16).astype(hs[k].dtype)
    return hs


def forward(p, X, dtype=np.float64, round_act=True):
    """y (n, 2) and the pre-activations, with the FP16-rounded weights (and
    FP16-rounded activations h0..h2 unless round_act is false)."""
    d = unpack(round16(p))
    X = np.asarray(X, dtype=dtype)
    z = [OMEGA0 * (X @ d["W0"].astype(dtype) + d["b0"].astype(dtype))]
    h = np.sin(z[0])
    if round_act:
        h = h.astype(np.float16).astype(dtype)
    for k in range(1, NHID + 1):
        z.append(h @ d["W%d" % k].astype(dtype) + d["b%d" % k].astype(dtype))
        h = np.sin(z[-1])
        if round_act and k < NHID:
            h = h.astype(np.float16).astype(dtype)
    y = h @ d["Wo"].astype(dtype) + d["bo"].astype(dtype)
    return y, z


def loss_and_grad(p, X, T, scale=1.0, dtype=np.float64, round_act=True):
    """L = scale * sum over samples of |y - t|^2 and dL/dp (padding columns 0);
    the FP16 rounding of the activations passes gradients straight through."""
    d = unpack(round16(p))
    X = np.asarray(X, dtype=dtype)
    T = np.asarray(T, dtype=dtype)
    y, z = forward(p, X, dtype, round_act)
    r = y - T
    L = scale * float(np.sum(r * r))
    g = np.zeros(NPARAM, dtype=np.float64)
    dy = 2.0 * scale * r
    hs = activations(z, round_act)
    g[OFF["Wo"]:OFF["Wo"] + H * NOUT] = (hs[-1].T @ dy).ravel()
    g[OFF["bo"]:OFF["bo"] + NOUT] = dy.sum(0)
    dh = dy @ d["Wo"].astype(dtype).T
    for k in range(NHID, 0, -1):
        dz = dh * np.cos(z[k])
        gw = np.zeros((H, HP))
        gw[:, :H] = hs[k - 1].T @ dz
        g[OFF["W%d" % k]:OFF["W%d" % k] + H * HP] = gw.ravel()
        g[OFF["b%d" % k]:OFF["b%d" % k] + H] = dz.sum(0)
        dh = dz @ d["W%d" % k].astype(dtype).T
    dz0 = dh * np.cos(z[0]) * OMEGA0
    g[OFF["W0"]:OFF["W0"] + NIN * H] = (X.T @ dz0).ravel()
    g[OFF["b0"]:OFF["b0"] + H] = dz0.sum(0)
    return L, g


def adam(p, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step on the FP32 master weights (in place); t counts from 1."""
    m[:] = b1 * m + (1 - b1) * g
    v[:] = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    p[:] = (p - lr * mh / (np.sqrt(vh) + eps)).astype(np.float32)
    pad_mask(p)


def pad_mask(p):
    for k in range(1, NHID + 1):
        w = p[OFF["W%d" % k]:OFF["W%d" % k] + H * HP].reshape(H, HP)
        w[:, H:] = 0


def tap_inputs(jx, jy, fu, fv, os_, support, wterm, wmax, freq=0.0, beam=0.0):
    """Network inputs of tap (jx, jy) of the CF plane (fu, fv) at w term wterm."""
    s1 = float(support + 1)
    u = (np.asarray(jx, dtype=np.float64) - support + np.asarray(fu, dtype=np.float64) / os_) / s1
    v = (np.asarray(jy, dtype=np.float64) - support + np.asarray(fv, dtype=np.float64) / os_) / s1
    w = np.broadcast_to(np.asarray(wterm, dtype=np.float64) / wmax, np.shape(u))
    f = np.broadcast_to(np.float64(freq), np.shape(u))
    b = np.broadcast_to(np.float64(beam), np.shape(u))
    return np.stack([u, v, w, f, b], axis=-1).astype(np.float32)
