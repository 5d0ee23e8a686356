"""CPU oracle of the learned confidence network (float64 numpy).

ORACLE INFRASTRUCTURE ONLY.  Imported by tests/ (to check the GPU kernels'
forward and backward passes) and nothing under fastfusion_b200/.

The network has no counterpart in the reference (its fusion weight is the
fixed ramp of update_functions.cpp:1187-1444); this file restates the
network as the library defines it, in float64, with the BF16 rounding of the
stored tensors (features, activations, weights) reproduced:

  features  z, n_x, n_y, n_z, valid  (8 channels, 5 used)
  a1 = bf16(relu(conv5x5(features; W1, b1)))     5 -> 16
  a2 = bf16(relu(conv5x5(a1; W2, b2)))          16 -> 16
  pred = conv5x5(a2; W3, b3)                    16 -> 1   (cm)
  confidence = (1 - max(pred, 0) / tau)^2 on [0, tau], else 0

conv5x5 is a 'same' correlation with zero padding:
  y[y, x, o] = b[o] + sum_{i, ky, kx} W[o, i, ky*5+kx] x[y+ky-2, x+kx-2, i].
Parameters are one flat vector W1[16][5][25] b1[16] W2[16][16][25] b2[16]
W3[1][16][25] b3[1] (8833 values).
"""
from __future__ import annotations

import numpy as np

HID, CIN, TAPS = 16, 5, 25
SHAPES = [("W1", (HID, CIN, TAPS)), ("b1", (HID,)), ("W2", (HID, HID, TAPS)), ("b2", (HID,)),
          ("W3", (1, HID, TAPS)), ("b3", (1,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16(x) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    nan = np.isnan(f)
    if nan.any():
        out[nan] = np.nan
    return out.reshape(np.shape(x))


def unpack(params) -> dict:
    p = np.asarray(params, dtype=np.float64).reshape(-1)
    assert p.size == N_PARAMS
    out, o = {}, 0
    for name, shp in SHAPES:
        k = int(np.prod(shp))
        out[name] = p[o:o + k].reshape(shp)
        o += k
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], dtype=np.float64).reshape(-1) for name, _ in SHAPES])


def features(depth_u16: np.ndarray, scaling: float, K) -> np.ndarray:
    """[H, W, 8] network input of one depth image (float64, BF16-rounded)."""
    fx, fy, cx, cy = (float(v) for v in K)
    z = depth_u16.astype(np.float64) * float(np.float32(scaling))
    H, W = z.shape
    zp = np.pad(z, 1)
    zl, zr = zp[1:-1, :-2], zp[1:-1, 2:]
    zu, zd = zp[:-2, 1:-1], zp[2:, 1:-1]
    xs = np.arange(W, dtype=np.float64)[None, :]
    ys = np.arange(H, dtype=np.float64)[:, None]
    ax = (xs + 1 - cx) * zr / fx - (xs - 1 - cx) * zl / fx
    ay = (ys - cy) * (zr - zl) / fy
    az = zr - zl
    bx = (xs - cx) * (zd - zu) / fx
    by = (ys + 1 - cy) * zd / fy - (ys - 1 - cy) * zu / fy
    bz = zd - zu
    n = np.stack([by * az - bz * ay, bz * ax - bx * az, bx * ay - by * ax], -1)
    ok = (z > 0) & (zl > 0) & (zr > 0) & (zu > 0) & (zd > 0)
    ln = np.linalg.norm(n, axis=-1)
    ok &= ln > 0
    n = np.where(ok[..., None], n / np.where(ln > 0, ln, 1.0)[..., None], 0.0)
    f = np.zeros((H, W, 8))
    f[..., 0] = z
    f[..., 1:4] = n
    f[..., 4] = (z > 0).astype(np.float64)
    return bf16(f)


def conv(x: np.ndarray, Wt: np.ndarray, b) -> np.ndarray:
    """'same' 5x5 correlation of x [n, H, W, Cin] with Wt [Cout, Cin, 25]."""
    n, H, W, _ = x.shape
    xp = np.pad(x, ((0, 0), (2, 2), (2, 2), (0, 0)))
    out = np.zeros((n, H, W, Wt.shape[0]))
    for tap in range(TAPS):
        ky, kx = divmod(tap, 5)
        out += xp[:, ky:ky + H, kx:kx + W, :] @ Wt[:, :, tap].T
    if b is not None:
        out += b
    return out


def conv_input_grad(dy: np.ndarray, Wt: np.ndarray) -> np.ndarray:
    """Gradient of conv's input: dx[.., i] = sum W[o, i, tap] dy[p - tap offset, o]."""
    n, H, W, _ = dy.shape
    dxp = np.zeros((n, H + 4, W + 4, Wt.shape[1]))
    for tap in range(TAPS):
        ky, kx = divmod(tap, 5)
        dxp[:, ky:ky + H, kx:kx + W, :] += dy @ Wt[:, :, tap]
    return dxp[:, 2:H + 2, 2:W + 2, :]


def conv_weight_grad(x: np.ndarray, dy: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    n, H, W, cin = x.shape
    xp = np.pad(x, ((0, 0), (2, 2), (2, 2), (0, 0)))
    dW = np.zeros((dy.shape[-1], cin, TAPS))
    for tap in range(TAPS):
        ky, kx = divmod(tap, 5)
        dW[:, :, tap] = np.einsum("nhwo,nhwi->oi", dy, xp[:, ky:ky + H, kx:kx + W, :])
    return dW, dy.sum(axis=(0, 1, 2))


def _params(params, rounding: bool) -> dict:
    return {k: (bf16(v) if rounding else v) for k, v in unpack(params).items()}


def forward(params, feat: np.ndarray, rounding: bool = True):
    """(a1, a2, pred) for feat [n, H, W, 8].  rounding: weights and stored
    activations rounded to BF16 as the library stores them (off for the
    finite-difference check of the backward pass)."""
    P = _params(params, rounding)
    x = np.asarray(feat, dtype=np.float64)[..., :CIN]
    r = bf16 if rounding else (lambda v: v)
    a1 = r(np.maximum(conv(x, P["W1"], P["b1"]), 0.0))
    a2 = r(np.maximum(conv(a1, P["W2"], P["b2"]), 0.0))
    pred = conv(a2, P["W3"], P["b3"])[..., 0]
    return a1, a2, pred


def backward(params, feat: np.ndarray, a1: np.ndarray, a2: np.ndarray, dpred: np.ndarray,
             rounding: bool = True) -> np.ndarray:
    """Flat parameter gradient of a loss with d(loss)/d(pred) = dpred [n, H, W]
    (the BF16 weights' gradient, applied to the FP32 master weights)."""
    P = _params(params, rounding)
    x = np.asarray(feat, dtype=np.float64)[..., :CIN]
    a1 = np.asarray(a1, dtype=np.float64)
    a2 = np.asarray(a2, dtype=np.float64)
    d3 = np.asarray(dpred, dtype=np.float64)[..., None]
    g = {}
    g["W3"], g["b3"] = conv_weight_grad(a2, d3)
    g2 = conv_input_grad(d3, P["W3"]) * (a2 > 0)
    g["W2"], g["b2"] = conv_weight_grad(a1, g2)
    g1 = conv_input_grad(g2, P["W2"]) * (a1 > 0)
    g["W1"], g["b1"] = conv_weight_grad(x, g1)
    return pack(g)


def mse(pred: np.ndarray, target: np.ndarray, inv_count: float):
    """(loss, dpred): squared error over target >= 0, scaled by inv_count."""
    m = target >= 0
    e = np.where(m, pred - target, 0.0)
    return float((e * e).sum() * inv_count), 2.0 * e * inv_count


def confidence(pred: np.ndarray, tau_cm: float) -> np.ndarray:
    c = np.maximum(1.0 - np.maximum(pred, 0.0) / tau_cm, 0.0)
    return c * c
