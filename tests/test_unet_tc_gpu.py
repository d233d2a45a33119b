"""The tcgen05 (tensor-memory accumulator) convolution of the learned warm
start against the CPU oracle, for every built shape, forward (bias + ReLU)
and as the masked data gradient on flipped weights; no wait may time out."""
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


def P(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


@pytest.mark.parametrize("ci,co", SHAPES)
def test_tc_conv_matches_oracle(cuda, ci, co):
    import torch
    from oracle import unet_oracle as uo
    from omega_b200 import _native
    st = ctypes.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    rng = np.random.default_rng(ci * 101 + co)
    B, Z, Y, X = 2, 3, 5, 70          # 2100 voxels: a partial last tile of 128
    x = uo.bf16(rng.normal(0, 1, (B, Z, Y, X, ci)))
    w = uo.bf16(rng.normal(0, 0.1, (27, co, ci)))
    b = rng.normal(0, 0.1, co).astype(np.float32)
    xt, wt, bt = _bf(x, cuda), _bf(w, cuda), torch.tensor(b, device=cuda)
    out = torch.empty(B * Z * Y * X * co, dtype=torch.bfloat16, device=cuda)
    _native.call("omb_unet_conv_tc", ci, co, P(xt), P(wt), P(bt), P(out), None, 1, X, Y, Z, B, st)
    ref = uo.bf16(np.maximum(uo.conv3d(x, w, b.astype(np.float64)), 0.0))
    assert _rel(out.float().cpu().numpy().reshape(ref.shape), ref) < 4e-3
    dz = uo.bf16(rng.normal(0, 1, (B, Z, Y, X, co)))
    mask = uo.bf16(rng.normal(0, 1, (B, Z, Y, X, ci)))
    wf = torch.empty_like(wt)
    _native.call("omb_unet_flip_weights", P(wt), P(wf), ci, co, st)
    dzt, mt = _bf(dz, cuda), _bf(mask, cuda)
    dx = torch.empty(B * Z * Y * X * ci, dtype=torch.bfloat16, device=cuda)
    _native.call("omb_unet_conv_tc", co, ci, P(dzt), P(wf), None, P(dx), P(mt), 0, X, Y, Z, B, st)
    refd = uo.bf16(np.where(mask > 0, uo.conv3d_dgrad(dz, w), 0.0))
    assert _rel(dx.float().cpu().numpy().reshape(refd.shape), refd) < 4e-3
    flag = ctypes.c_int32(-1)
    _native.call("omb_unet_take_error", ctypes.byref(flag))
    assert flag.value == 0


@pytest.mark.parametrize("ci,co", SHAPES)
def test_tc_wgrad_matches_oracle(cuda, ci, co):
    """omb_unet_conv_wgrad_tc (tcgen05, the voxels as the reduction
    dimension) against the FP64 weight gradient and the mma.sync kernel, on
    a volume whose voxel count leaves partial stages and CTAs."""
    import torch
    from oracle import unet_oracle as uo
    from omega_b200 import _native
    st = ctypes.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    rng = np.random.default_rng(ci * 7 + co)
    B, Z, Y, X = 2, 7, 9, 70          # 8820 voxels: 2 CTAs of 8192, a partial last stage
    x = uo.bf16(rng.normal(0, 1, (B, Z, Y, X, ci)))
    dz = uo.bf16(rng.normal(0, 1, (B, Z, Y, X, co)))
    xt, dzt = _bf(x, cuda), _bf(dz, cuda)
    dw = torch.zeros(27 * co * ci, device=cuda)
    _native.call("omb_unet_conv_wgrad_tc", ci, co, P(xt), P(dzt), P(dw), X, Y, Z, B, st)
    ref = uo.conv3d_wgrad(x, dz)
    got = dw.cpu().numpy().reshape(ref.shape)
    assert _rel(got, ref) < 1e-5, _rel(got, ref)
    dw2 = torch.zeros_like(dw)
    _native.call("omb_unet_conv_wgrad", ci, co, P(xt), P(dzt), P(dw2), X, Y, Z, B, st)
    assert _rel(got, dw2.cpu().numpy().reshape(ref.shape)) < 1e-5
    flag = ctypes.c_int32(-1)
    _native.call("omb_unet_take_error", ctypes.byref(flag))
    assert flag.value == 0
