"""CPU oracle of the learned pressure warm start (test infrastructure only).

The warm start has no counterpart in the reference, so this numpy restatement is its
checker: the same network, written with plain array arithmetic in float64, with bf16
rounding applied at exactly the points where the GPU stores bf16 (weights, activations and
back-propagated gradients), so GPU results must agree to FP32 accumulation-order error.
Its own gradients are checked against central finite differences in the tests.

Layouts follow the GPU: activations (B, H, W, C), weights (Cout, 3, 3, Cin).
"""
from __future__ import annotations

import numpy as np


def bf16(x) -> np.ndarray:
    """Round to the nearest bf16 (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    nan = np.isnan(f)
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    out[nan] = np.nan
    return out


def bf16_bits(x) -> np.ndarray:
    """bf16 bit patterns (uint16) of x, rounded to nearest even."""
    f = np.asarray(bf16(x), dtype=np.float32)
    return (f.view(np.uint32) >> 16).astype(np.uint16)


def from_bf16_bits(b) -> np.ndarray:
    return (np.asarray(b, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def _shifted(x, ky, kx):
    """x[b, y+ky-1, x+kx-1, c] with zero padding."""
    B, H, W, C = x.shape
    p = np.zeros((B, H + 2, W + 2, C))
    p[:, 1:H + 1, 1:W + 1] = x
    return p[:, ky:ky + H, kx:kx + W]


def conv3x3(x, w, b=None, relu=False):
    """out[b,y,x,co] = act(bias + sum_{ky,kx,ci} x[b,y+ky-1,x+kx-1,ci] w[co,ky,kx,ci])."""
    B, H, W, _ = x.shape
    out = np.zeros((B, H, W, w.shape[0]))
    for ky in range(3):
        for kx in range(3):
            out += np.einsum("bhwc,oc->bhwo", _shifted(x, ky, kx), w[:, ky, kx, :])
    if b is not None:
        out += b
    return np.maximum(out, 0) if relu else out


def conv3x3_wgrad(x, dout):
    """dw[co,ky,kx,ci] = sum dout[b,y,x,co] x[b,y+ky-1,x+kx-1,ci]; db[co] = sum dout."""
    Cout, Cin = dout.shape[-1], x.shape[-1]
    dw = np.zeros((Cout, 3, 3, Cin))
    for ky in range(3):
        for kx in range(3):
            dw[:, ky, kx, :] = np.einsum("bhwo,bhwc->oc", dout, _shifted(x, ky, kx))
    return dw, dout.sum(axis=(0, 1, 2))


def flip(w):
    """Weights of the input gradient: wt[ci,ky,kx,co] = w[co,2-ky,2-kx,ci]."""
    return np.ascontiguousarray(w[:, ::-1, ::-1, :].transpose(3, 1, 2, 0))


def conv3x3_dgrad(dout, w):
    """Gradient with respect to the input of conv3x3(x, w)."""
    return conv3x3(dout, flip(w))


# ---------------------------------------------------------------- the warm-start network

LAYERS = [(16, 32, 0, True), (32, 32, 0, True), (32, 64, 1, True), (64, 64, 1, True), (64, 64, 2, True),
          (64, 64, 3, True), (64, 64, 2, True), (64, 32, 1, True), (32, 32, 0, True), (32, 16, 0, False)]


def param_count():
    return sum(co * 9 * ci + co for ci, co, _, _ in LAYERS)


def unflatten(p):
    """Flat parameters (per layer w[Cout][3][3][Cin] then b[Cout]) -> [(w, b), ...]."""
    out, o = [], 0
    p = np.asarray(p, dtype=np.float64)
    for ci, co, _, _ in LAYERS:
        w = p[o:o + co * 9 * ci].reshape(co, 3, 3, ci)
        o += co * 9 * ci
        out.append((w, p[o:o + co]))
        o += co
    return out


def flatten(pairs):
    return np.concatenate([np.concatenate([w.ravel(), b.ravel()]) for w, b in pairs])


def _pool(x):
    return 0.25 * (((x[:, 0::2, 0::2] + x[:, 0::2, 1::2]) + x[:, 1::2, 0::2]) + x[:, 1::2, 1::2])


def _up(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def _pool_sum(x):
    return ((x[:, 0::2, 0::2] + x[:, 0::2, 1::2]) + x[:, 1::2, 0::2]) + x[:, 1::2, 1::2]


def _f32(x):
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def net_forward(params, x, quant=True):
    """Forward pass of the warm-start network on x (B, H, W, 16). Returns (out0, cache).

    With quant the weights, every stored activation and the pooled/upsampled sums are
    rounded to bf16 and the output to FP32, as on the GPU."""
    q = bf16 if quant else (lambda a: np.asarray(a, dtype=np.float64))
    f = _f32 if quant else (lambda a: np.asarray(a, dtype=np.float64))
    ws = [(q(w), f(b)) for w, b in unflatten(params)]

    def conv(l, inp):
        w, b = ws[l]
        y = conv3x3(inp, w, b, relu=LAYERS[l][3])
        return q(y) if l < 9 else f(y)

    A = [None] * 10
    x = q(x)
    A[0] = conv(0, x)
    A[1] = conv(1, A[0])
    P1 = q(_pool(A[1]))
    A[2] = conv(2, P1)
    A[3] = conv(3, A[2])
    P2 = q(_pool(A[3]))
    A[4] = conv(4, P2)
    P3 = q(_pool(A[4]))
    A[5] = conv(5, P3)
    U3 = q(_up(A[5]) + A[4])
    A[6] = conv(6, U3)
    U2 = q(_up(A[6]) + A[3])
    A[7] = conv(7, U2)
    U1 = q(_up(A[7]) + A[1])
    A[8] = conv(8, U1)
    out = conv(9, A[8])
    ins = [x, A[0], P1, A[2], P2, P3, U3, U2, U1, A[8]]
    return out[..., 0], (ws, A, ins, out)


def net_loss_grad(params, x, target, quant=True):
    """Loss mean((out0 - target)^2) and the flat gradient of all parameters."""
    q = bf16 if quant else (lambda a: np.asarray(a, dtype=np.float64))
    f = _f32 if quant else (lambda a: np.asarray(a, dtype=np.float64))
    out0, (ws, A, ins, out) = net_forward(params, x, quant)
    n = out0.size
    d = f(f(out0) - f(target))
    loss = float(np.mean(d * d))
    dout = np.zeros_like(out)
    dout[..., 0] = q(f(2.0 * d / n))
    grads = [None] * 10
    G = [None] * 10

    def back(l, Gl):
        g = dout if l == 9 else q(np.where(A[l] > 0, Gl, 0.0))
        dw, db = conv3x3_wgrad(ins[l], g)
        grads[l] = (dw, db)
        return conv3x3(g, flip(ws[l][0]))

    G[8] = back(9, None)
    G[1] = back(8, G[8])
    G[7] = _pool_sum(G[1])
    G[3] = back(7, G[7])
    G[6] = _pool_sum(G[3])
    G[4] = back(6, G[6])
    G[5] = _pool_sum(G[4])
    G[4] = G[4] + 0.25 * _up(back(5, G[5]))
    G[3] = G[3] + 0.25 * _up(back(4, G[4]))
    G[2] = back(3, G[3])
    G[1] = G[1] + 0.25 * _up(back(2, G[2]))
    G[0] = back(1, G[1])
    back(0, G[0])
    return loss, flatten(grads)
