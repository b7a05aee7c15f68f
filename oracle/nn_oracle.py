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
