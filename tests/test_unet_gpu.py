"""The learned warm start's kernels against the CPU oracle
(oracle/unet_oracle.py): every built convolution shape forward and as the
data gradient, the weight gradient, and the whole network's loss and
parameter gradients; plus a short training run that lowers the loss."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (96, 32), (48, 16), (32, 16), (64, 32), (32, 96),
          (16, 48)]


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-30))


def _bf(a, dev):
    import torch
    return torch.tensor(np.ascontiguousarray(a, dtype=np.float32), dtype=torch.bfloat16, device=dev).reshape(-1)


def _np(t, shape):
    return t.float().cpu().numpy().reshape(shape).astype(np.float64)


def _st(dev):
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def P(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


@pytest.mark.parametrize("ci,co", SHAPES)
def test_conv_forward_and_dgrad_match_oracle(cuda, ci, co):
    import torch
    from oracle import unet_oracle as uo
    from omega_b200 import _native
    rng = np.random.default_rng(ci * 100 + co)
    B, Z, Y, X = 2, 4, 6, 72        # X > 64: two blocks per row, the second partly masked
    x = uo.bf16(rng.normal(0, 1, (B, Z, Y, X, ci)))
    w = uo.bf16(rng.normal(0, 0.1, (27, co, ci)))
    b = rng.normal(0, 0.1, co).astype(np.float32)
    xt, wt, bt = _bf(x, cuda), _bf(w, cuda), torch.tensor(b, device=cuda)
    out = torch.empty(B * Z * Y * X * co, dtype=torch.bfloat16, device=cuda)
    _native.call("omb_unet_conv", ci, co, P(xt), P(wt), P(bt), P(out), None, 1, X, Y, Z, B, _st(cuda))
    ref = uo.bf16(np.maximum(uo.conv3d(x, w, b.astype(np.float64)), 0.0))
    assert _rel(_np(out, ref.shape), ref) < 4e-3
    # data gradient: the same kernel on flipped weights, masked by a ReLU input
    dz = uo.bf16(rng.normal(0, 1, (B, Z, Y, X, co)))
    mask = uo.bf16(rng.normal(0, 1, (B, Z, Y, X, ci)))
    wf = torch.empty_like(wt)
    _native.call("omb_unet_flip_weights", P(wt), P(wf), ci, co, _st(cuda))
    dx = torch.empty(B * Z * Y * X * ci, dtype=torch.bfloat16, device=cuda)
    dzt, mt = _bf(dz, cuda), _bf(mask, cuda)   # kept alive until the kernels have run
    _native.call("omb_unet_conv", co, ci, P(dzt), P(wf), None, P(dx), P(mt), 0, X, Y, Z, B, _st(cuda))
    refd = uo.bf16(np.where(mask > 0, uo.conv3d_dgrad(dz, w), 0.0))
    assert _rel(_np(dx, refd.shape), refd) < 4e-3


@pytest.mark.parametrize("ci,co", [(16, 16), (16, 32), (32, 64), (96, 32), (48, 16), (64, 64)])
def test_conv_wgrad_matches_oracle(cuda, ci, co):
    import torch
    from oracle import unet_oracle as uo
    from omega_b200 import _native
    rng = np.random.default_rng(7 + ci + co)
    B, Z, Y, X = 2, 6, 10, 24        # 2880 voxels: a partial last tile
    x = uo.bf16(rng.normal(0, 1, (B, Z, Y, X, ci)))
    dz = uo.bf16(rng.normal(0, 1, (B, Z, Y, X, co)))
    dw = torch.zeros(27 * co * ci, device=cuda)
    xt, dzt = _bf(x, cuda), _bf(dz, cuda)   # kept alive until the kernels have run
    _native.call("omb_unet_conv_wgrad", ci, co, P(xt), P(dzt), P(dw), X, Y, Z, B, _st(cuda))
    ref = uo.conv3d_wgrad(x, dz)
    assert _rel(dw.cpu().numpy().reshape(ref.shape), ref) < 1e-5
    if co in (16, 32, 64):
        db = torch.zeros(co, device=cuda)
        _native.call("omb_unet_bias_grad", co, P(dzt), P(db), B * Z * Y * X, _st(cuda))
        assert _rel(db.cpu().numpy(), dz.reshape(-1, co).sum(axis=0)) < 1e-5


def _tiny_problem(seed, X=16, Y=16, Zs=7, B=2):
    rng = np.random.default_rng(seed)
    n = X * Y * Zs
    xs = np.linspace(-1, 1, X)
    XX, YY, ZZ = np.meshgrid(xs, np.linspace(-1, 1, Y), np.linspace(-1, 1, Zs), indexing="ij")
    base = ((XX ** 2 + YY ** 2) < 0.7).astype(np.float64).ravel(order="F")
    osem = np.stack([base * rng.uniform(0.5, 2) + 0.2 * rng.random(n) for _ in range(B)]).astype(np.float32)
    target = np.stack([osem[b] * (1 + 0.3 * base) for b in range(B)]).astype(np.float32)
    sens = (1.0 + base).astype(np.float32)
    return osem, target, sens


def test_network_gradients_match_oracle(cuda):
    import torch
    from oracle import unet_oracle as uo
    from omega_b200.learned import UNet3D
    X, Y, Zs, B = 16, 16, 7, 2
    osem, target, sens = _tiny_problem(3, X, Y, Zs, B)
    net = UNet3D(X, Y, Zs, B, cuda, seed=5)
    rng = np.random.default_rng(9)
    net.head_w.copy_(torch.tensor(rng.normal(0, 0.3, 16).astype(np.float32)))
    net.head_b.fill_(0.05)
    for p in net.params:   # nonzero biases so every ReLU path is exercised
        p["b"].copy_(torch.tensor(rng.normal(0, 0.05, p["b"].numel()).astype(np.float32)))
    net._sync_weights()
    o_t = torch.tensor(osem, device=cuda).reshape(-1)
    t_t = torch.tensor(target, device=cuda).reshape(-1)
    s_t = torch.tensor(sens, device=cuda)
    net.loss.zero_()
    net.forward(o_t, X * Y * Zs, s_t, 0.5)
    net.backward(t_t, X * Y * Zs)
    torch.cuda.synchronize()
    ws = [uo.bf16(p["w"].cpu().numpy().reshape(27, co, ci)) for (ci, co), p in zip(uo.LAYERS, net.params)]
    bs = [p["b"].cpu().numpy().astype(np.float64) for p in net.params]
    ref = uo.forward_backward(ws, bs, net.head_w.cpu().numpy().astype(np.float64), float(net.head_b.item()),
                              osem, sens, 0.5, target, (X, Y, Zs))
    assert abs(net.loss.item() - ref["loss"]) < 2e-3 * ref["loss"]
    for i, ((ci, co), p) in enumerate(zip(uo.LAYERS, net.params)):
        g = p["gw"].cpu().numpy().reshape(27, co, ci)
        assert _rel(g, ref["gw"][i]) < 3e-2, (i, _rel(g, ref["gw"][i]))
        assert _rel(p["gb"].cpu().numpy(), ref["gb"][i]) < 3e-2, i
    assert _rel(net.gw_head.cpu().numpy(), ref["ghw"]) < 1e-2
    assert abs(net.gb_head.item() - ref["ghb"]) < 1e-2 * abs(ref["ghb"]) + 1e-6


def test_training_lowers_the_loss(cuda):
    import torch
    from omega_b200.learned import UNet3D
    X, Y, Zs, B = 16, 16, 7, 2
    osem, target, sens = _tiny_problem(4, X, Y, Zs, B)
    net = UNet3D(X, Y, Zs, B, cuda, seed=1)
    o_t = torch.tensor(osem, device=cuda).reshape(-1)
    t_t = torch.tensor(target, device=cuda).reshape(-1)
    s_t = torch.tensor(sens, device=cuda)
    losses = []
    for _ in range(60):
        net.loss.zero_()
        net.forward(o_t, X * Y * Zs, s_t, 0.5)
        net.backward(t_t, X * Y * Zs)
        net.adam_step(3e-3)
        losses.append(net.loss.item())
    assert losses[-1] < 0.3 * losses[0], (losses[0], losses[-1])
