"""TEST INFRASTRUCTURE ONLY: the CPU oracle of the learned warm-start network.

A numpy restatement of omega_b200.learned.UNet3D (forward pass, mean squared
error and every parameter gradient) in FP64, with the values the GPU stores
in BF16 rounded to BF16 at the same points (network input, every conv
output, pooling, concatenation, every stored gradient), so the GPU's
gradients can be checked to the accuracy of its FP32 accumulation.  Only
tests import this module.

Layouts as the kernels: activations [B][Z][Y][X][C], conv weights
[27][Cout][Cin] with tap = (dz+1)*9 + (dy+1)*3 + (dx+1).
"""
from __future__ import annotations

import numpy as np

LAYERS = [(16, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (96, 32), (32, 32), (48, 16), (16, 16)]


def bf16(a):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def _taps():
    for tap in range(27):
        yield tap, tap // 9 - 1, (tap // 3) % 3 - 1, tap % 3 - 1


def conv3d(x, w, b=None):
    """out[v][co] = b[co] + sum_tap sum_ci x[v + off(tap)][ci] w[tap][co][ci], zero padding."""
    B, Z, Y, X, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((B, Z, Y, X, w.shape[1]))
    for tap, dz, dy, dx in _taps():
        xs = xp[:, 1 + dz:1 + dz + Z, 1 + dy:1 + dy + Y, 1 + dx:1 + dx + X, :]
        out += xs @ w[tap].T
    if b is not None:
        out += b
    return out


def conv3d_dgrad(dz, w):
    """d x[u][ci] = sum_tap sum_co dz[u - off(tap)][co] w[tap][co][ci]."""
    B, Z, Y, X, _ = dz.shape
    dp = np.pad(dz, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((B, Z, Y, X, w.shape[2]))
    for tap, ddz, ddy, ddx in _taps():
        ds = dp[:, 1 - ddz:1 - ddz + Z, 1 - ddy:1 - ddy + Y, 1 - ddx:1 - ddx + X, :]
        out += ds @ w[tap]
    return out


def conv3d_wgrad(x, dz):
    """dW[tap][co][ci] = sum_v dz[v][co] x[v + off(tap)][ci]."""
    B, Z, Y, X, ci = x.shape
    co = dz.shape[-1]
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    dw = np.zeros((27, co, ci))
    d2 = dz.reshape(-1, co)
    for tap, ddz, ddy, ddx in _taps():
        xs = xp[:, 1 + ddz:1 + ddz + Z, 1 + ddy:1 + ddy + Y, 1 + ddx:1 + ddx + X, :].reshape(-1, ci)
        dw[tap] = d2.T @ xs
    return dw


def avgpool2(x):
    B, Z, Y, X, C = x.shape
    return x.reshape(B, Z // 2, 2, Y // 2, 2, X // 2, 2, C).mean(axis=(2, 4, 6))


def avgpool2_bwd(d):
    return np.repeat(np.repeat(np.repeat(d, 2, axis=1), 2, axis=2), 2, axis=3) / 8.0


def up2(x):
    return np.repeat(np.repeat(np.repeat(x, 2, axis=1), 2, axis=2), 2, axis=3)


def up2_bwd(d):
    B, Z, Y, X, C = d.shape
    return d.reshape(B, Z // 2, 2, Y // 2, 2, X // 2, 2, C).sum(axis=(2, 4, 6))


def _vol(v, X, Y, Zs, Z):
    """Fortran-order (X, Y, Zs) volume -> [Z][Y][X] padded with zero slices."""
    a = np.asarray(v, dtype=np.float64).reshape((X, Y, Zs), order="F").transpose(2, 1, 0)
    return np.concatenate([a, np.zeros((Z - Zs, Y, X))], axis=0)


def forward_backward(ws, bs, head_w, head_b, osem, sens, sens_scale, target, shape):
    """Full network step; shape = (X, Y, Zs).  Returns dict with loss, pred,
    gw (list), gb (list), ghw, ghb."""
    X, Y, Zs = shape
    Z = (Zs + 3) // 4 * 4
    B = osem.shape[0]
    scale = np.array([1.0 / max(float(np.float32(np.mean(np.float32(osem[b])))), 1e-12) for b in range(B)])
    scale = scale.astype(np.float32).astype(np.float64)
    x0 = np.zeros((B, Z, Y, X, 16))
    for b in range(B):
        x0[b, :, :, :, 0] = _vol(osem[b], X, Y, Zs, Z) * scale[b]
        x0[b, :, :, :, 1] = _vol(sens, X, Y, Zs, Z) * sens_scale
    x0 = bf16(x0)
    relu = lambda t: np.maximum(t, 0.0)  # noqa: E731
    a1 = bf16(relu(conv3d(x0, ws[0], bs[0])))
    a2 = bf16(relu(conv3d(a1, ws[1], bs[1])))
    p1 = bf16(avgpool2(a2))
    a3 = bf16(relu(conv3d(p1, ws[2], bs[2])))
    a4 = bf16(relu(conv3d(a3, ws[3], bs[3])))
    p2 = bf16(avgpool2(a4))
    a5 = bf16(relu(conv3d(p2, ws[4], bs[4])))
    a6 = bf16(relu(conv3d(a5, ws[5], bs[5])))
    c2 = np.concatenate([up2(a6), a4], axis=-1)
    a7 = bf16(relu(conv3d(c2, ws[6], bs[6])))
    a8 = bf16(relu(conv3d(a7, ws[7], bs[7])))
    c1 = np.concatenate([up2(a8), a2], axis=-1)
    a9 = bf16(relu(conv3d(c1, ws[8], bs[8])))
    a10 = bf16(relu(conv3d(a9, ws[9], bs[9])))
    pred = x0[..., 0] + head_b + a10 @ head_w
    tgt = np.zeros((B, Z, Y, X))
    for b in range(B):
        tgt[b] = _vol(target[b], X, Y, Zs, Z) * scale[b]
    valid = np.zeros((B, Z, Y, X), dtype=bool)
    valid[:, :Zs] = True
    count = B * X * Y * Zs
    r = np.where(valid, pred - tgt, 0.0)
    loss = float(np.sum(r * r) / count)
    gr = 2.0 * r / count
    ghw = np.einsum("bzyx,bzyxc->c", gr, a10)
    ghb = float(np.sum(gr))
    gw, gb = [None] * 10, [None] * 10
    mask = lambda d, a: np.where(a > 0, d, 0.0)  # noqa: E731
    dz10 = bf16(mask(gr[..., None] * head_w, a10))

    def grads(i, src, dz):
        gw[i] = conv3d_wgrad(src, dz)
        gb[i] = dz.reshape(-1, dz.shape[-1]).sum(axis=0)

    grads(9, a9, dz10)
    dz9 = bf16(mask(conv3d_dgrad(dz10, ws[9]), a9))
    grads(8, c1, dz9)
    dc1 = bf16(conv3d_dgrad(dz9, ws[8]))
    da8 = bf16(up2_bwd(dc1[..., :32]))
    da2 = bf16(dc1[..., 32:])
    dz8 = mask(da8, a8)
    grads(7, a7, dz8)
    dz7 = bf16(mask(conv3d_dgrad(dz8, ws[7]), a7))
    grads(6, c2, dz7)
    dc2 = bf16(conv3d_dgrad(dz7, ws[6]))
    da6 = bf16(up2_bwd(dc2[..., :64]))
    da4 = bf16(dc2[..., 64:])
    dz6 = mask(da6, a6)
    grads(5, a5, dz6)
    dz5 = bf16(mask(conv3d_dgrad(dz6, ws[5]), a5))
    grads(4, p2, dz5)
    dp2 = bf16(conv3d_dgrad(dz5, ws[4]))
    da4 = bf16(da4 + avgpool2_bwd(dp2))
    dz4 = mask(da4, a4)
    grads(3, a3, dz4)
    dz3 = bf16(mask(conv3d_dgrad(dz4, ws[3]), a3))
    grads(2, p1, dz3)
    dp1 = bf16(conv3d_dgrad(dz3, ws[2]))
    da2 = bf16(da2 + avgpool2_bwd(dp1))
    dz2 = mask(da2, a2)
    grads(1, a1, dz2)
    dz1 = bf16(mask(conv3d_dgrad(dz2, ws[1]), a1))
    grads(0, x0, dz1)
    return {"loss": loss, "pred": pred, "gw": gw, "gb": gb, "ghw": ghw, "ghb": ghb, "scale": scale}
