"""Learned OSEM warm start: a 3-D U-Net that maps the 2-iteration OSEM image
(plus the sensitivity image) to a 20-iteration-quality image, after which
plain OSEM continues.  The network is trained and run on the GPU by the
library's own kernels (include/omega_b200_unet.h): BF16 3x3x3 convolutions
on the tcgen05 tensor cores (FP32 accumulator in tensor memory) for the
forward pass and the data gradients, warp-level MMA for the weight
gradients, pooling,
upsampling, the loss and Adam.  torch only allocates device memory.

Architecture (3 levels, 16/32/64 channels, 3x3x3 convolutions + ReLU):
    enc1: 2(16 padded) -> 16 -> 16        (X x Y x Z)        skip1
    enc2: avgpool2, 16 -> 32 -> 32        (X/2 x Y/2 x Z/2)  skip2
    bott: avgpool2, 32 -> 64 -> 64        (X/4 x Y/4 x Z/4)
    dec2: up2 (+) skip2 = 96 -> 32 -> 32
    dec1: up2 (+) skip1 = 48 -> 16 -> 16
    head: prediction = input image + bias + w . features (1x1x1, 16 -> 1)
Inputs are normalised per study by the mean of its 2-iteration image; the
prediction is scaled back and clamped to a small positive floor, since the
multiplicative OSEM update cannot leave zero.  The reference has no learned
component; this is the warm start of the north star's "learned vs plain"
measurement.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native

# (cin, cout) of the ten 3x3x3 convolutions, in forward order
LAYERS = [(16, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (96, 32), (32, 32), (48, 16), (16, 16)]
FAN_IN = [2, 16, 16, 32, 32, 64, 96, 32, 48, 16]   # real input channels (layer 1 has 2 of its 16 padded)


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class UNet3D:
    """The network and its training state on one device.

    Volumes are (X, Y, Zs) Fortran-order images; the network works on Z =
    Zs rounded up to a multiple of 4 (extra slices are zero padding and are
    excluded from the loss).  `batch` studies go through one call."""

    # convolution engine of the forward pass and the data gradients:
    # "omb_unet_conv_tc" (tcgen05, accumulator in tensor memory) or
    # "omb_unet_conv" (warp-level mma.sync)
    conv_entry = "omb_unet_conv_tc"
    # weight gradients: "omb_unet_conv_wgrad" (mma.sync, the faster of the two on
    # every built shape) or "omb_unet_conv_wgrad_tc" (tcgen05)
    wgrad_entry = "omb_unet_conv_wgrad"

    def __init__(self, X, Y, Zs, batch, device, seed=0):
        import torch
        if X % 4 or Y % 4:
            raise ValueError("X and Y must be multiples of 4")
        self.X, self.Y, self.Zs = X, Y, Zs
        self.Z = (Zs + 3) // 4 * 4
        self.B = batch
        self.dev = torch.device(device)
        self.step_count = 0
        rng = np.random.default_rng(seed)
        self.params = []   # dicts: w (fp32 master), wb (bf16), wf (bf16 flipped), b, and Adam state
        for (ci, co), fan in zip(LAYERS, FAN_IN):
            std = np.sqrt(2.0 / (27 * fan))
            w = rng.normal(0.0, std, (27, co, ci)).astype(np.float32)
            if ci == 16 and fan == 2:
                w[:, :, 2:] = 0.0
            self.params.append(self._param(w, np.zeros(co, dtype=np.float32)))
        self.head_w = torch.zeros(16, device=self.dev)
        self.head_b = torch.zeros(1, device=self.dev)
        self.head_state = [torch.zeros(16, device=self.dev), torch.zeros(16, device=self.dev),
                           torch.zeros(1, device=self.dev), torch.zeros(1, device=self.dev)]
        self._alloc()

    # -- parameters -------------------------------------------------------
    def _param(self, w, b):
        import torch
        d = {"w": torch.from_numpy(w).to(self.dev).reshape(-1), "b": torch.from_numpy(b).to(self.dev)}
        d["wb"] = torch.empty(d["w"].numel(), dtype=torch.bfloat16, device=self.dev)
        d["wf"] = torch.empty_like(d["wb"])
        d["gw"] = torch.zeros_like(d["w"])
        d["gb"] = torch.zeros_like(d["b"])
        d["mw"], d["vw"] = torch.zeros_like(d["w"]), torch.zeros_like(d["w"])
        d["mb"], d["vb"] = torch.zeros_like(d["b"]), torch.zeros_like(d["b"])
        return d

    def _sync_weights(self):
        st = self._stream()
        for (ci, co), p in zip(LAYERS, self.params):
            _native.call("omb_unet_to_bf16", _p(p["w"]), _p(p["wb"]), p["w"].numel(), st)
            _native.call("omb_unet_flip_weights", _p(p["wb"]), _p(p["wf"]), ci, co, st)

    def state_dict(self):
        out = {"head_w": self.head_w.cpu().numpy(), "head_b": self.head_b.cpu().numpy(),
               "shape": np.array([self.X, self.Y, self.Zs])}
        for i, p in enumerate(self.params):
            out[f"w{i}"] = p["w"].cpu().numpy()
            out[f"b{i}"] = p["b"].cpu().numpy()
        return out

    def load_state_dict(self, sd):
        import torch
        for i, p in enumerate(self.params):
            p["w"].copy_(torch.from_numpy(np.asarray(sd[f"w{i}"], dtype=np.float32).reshape(-1)))
            p["b"].copy_(torch.from_numpy(np.asarray(sd[f"b{i}"], dtype=np.float32)))
        self.head_w.copy_(torch.from_numpy(np.asarray(sd["head_w"], dtype=np.float32)))
        self.head_b.copy_(torch.from_numpy(np.asarray(sd["head_b"], dtype=np.float32)))
        self._sync_weights()

    # -- buffers ------------------------------------------------------------
    def _alloc(self):
        import torch
        X, Y, Z, B = self.X, self.Y, self.Z, self.B
        n1, n2, n3 = B * X * Y * Z, B * X * Y * Z // 8, B * X * Y * Z // 64
        self.n = (n1, n2, n3)
        e = lambda n, c: torch.empty(n * c, dtype=torch.bfloat16, device=self.dev)  # noqa: E731
        self.a = {"x0": e(n1, 16), "a1": e(n1, 16), "a2": e(n1, 16), "p1": e(n2, 16), "a3": e(n2, 32),
                  "a4": e(n2, 32), "p2": e(n3, 32), "a5": e(n3, 64), "a6": e(n3, 64), "c2": e(n2, 96),
                  "a7": e(n2, 32), "a8": e(n2, 32), "c1": e(n1, 48), "a9": e(n1, 16), "a10": e(n1, 16)}
        self.d = {"z10": e(n1, 16), "z9": e(n1, 16), "c1": e(n1, 48), "a8": e(n2, 32), "a2": e(n1, 16),
                  "z7": e(n2, 32), "c2": e(n2, 96), "a6": e(n3, 64), "a4": e(n2, 32), "z5": e(n3, 64),
                  "p2": e(n3, 32), "z3": e(n2, 32), "p1": e(n2, 16), "z1": e(n1, 16)}
        self.pred = torch.empty(n1, dtype=torch.float32, device=self.dev)
        self.scale = torch.empty(B, dtype=torch.float32, device=self.dev)
        self.loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        self.gw_head = torch.zeros(16, device=self.dev)
        self.gb_head = torch.zeros(1, device=self.dev)
        self._sync_weights()

    def _stream(self):
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)

    # -- forward ------------------------------------------------------------
    def _conv(self, i, src, dst, level, relu=True):
        ci, co = LAYERS[i]
        X, Y, Z = self._dims(level)
        _native.call(self.conv_entry, ci, co, _p(src), _p(self.params[i]["wb"]), _p(self.params[i]["b"]), _p(dst),
                     None, 1 if relu else 0, X, Y, Z, self.B, self._stream())

    def _dims(self, level):
        f = 2 ** level
        return self.X // f, self.Y // f, self.Z // f

    def forward(self, osem, osem_stride, sens, sens_scale):
        """osem: device pointer-holder (tensor) of B FP32 volumes osem_stride
        apart; sens: FP32 volume.  Returns the FP32 prediction (normalised)."""
        import torch
        st = self._stream()
        a, B = self.a, self.B
        X, Y, Z = self.X, self.Y, self.Z
        nv = X * Y * self.Zs
        means = osem.reshape(B, -1)[:, :nv].mean(dim=1)
        torch.reciprocal(means.clamp_min(1e-12), out=self.scale)
        _native.call("omb_unet_make_input", _p(osem), osem_stride, _p(sens), _p(self.scale), float(sens_scale),
                     _p(a["x0"]), X, Y, Z, self.Zs, B, st)
        self._conv(0, a["x0"], a["a1"], 0)
        self._conv(1, a["a1"], a["a2"], 0)
        _native.call("omb_unet_avgpool", _p(a["a2"]), _p(a["p1"]), X, Y, Z, B, 16, 0, st)
        self._conv(2, a["p1"], a["a3"], 1)
        self._conv(3, a["a3"], a["a4"], 1)
        X2, Y2, Z2 = self._dims(1)
        _native.call("omb_unet_avgpool", _p(a["a4"]), _p(a["p2"]), X2, Y2, Z2, B, 32, 0, st)
        self._conv(4, a["p2"], a["a5"], 2)
        self._conv(5, a["a5"], a["a6"], 2)
        _native.call("omb_unet_up_concat", _p(a["a6"]), _p(a["a4"]), _p(a["c2"]), X2, Y2, Z2, B, 64, 32, st)
        self._conv(6, a["c2"], a["a7"], 1)
        self._conv(7, a["a7"], a["a8"], 1)
        _native.call("omb_unet_up_concat", _p(a["a8"]), _p(a["a2"]), _p(a["c1"]), X, Y, Z, B, 32, 16, st)
        self._conv(8, a["c1"], a["a9"], 0)
        self._conv(9, a["a9"], a["a10"], 0)
        _native.call("omb_unet_head_fwd", _p(a["a10"]), _p(a["x0"]), _p(self.head_w), _p(self.head_b),
                     _p(self.pred), self.n[0], st)
        return self.pred

    def predict_into(self, out, out_stride, floor_v):
        """Writes the de-normalised prediction of the last forward() into B
        Fortran-order FP32 volumes (out_stride apart)."""
        _native.call("omb_unet_head_out", _p(self.pred), _p(self.scale), _p(out), out_stride, float(floor_v),
                     self.X, self.Y, self.Z, self.Zs, self.B, self._stream())

    # -- backward -----------------------------------------------------------
    def _grads(self, i, src, dz, level):
        ci, co = LAYERS[i]
        X, Y, Z = self._dims(level)
        st = self._stream()
        p = self.params[i]
        _native.call(self.wgrad_entry, ci, co, _p(src), _p(dz), _p(p["gw"]), X, Y, Z, self.B, st)
        _native.call("omb_unet_bias_grad", co, _p(dz), _p(p["gb"]), X * Y * Z * self.B, st)

    def _dgrad(self, i, dz, dst, level, mask):
        ci, co = LAYERS[i]
        X, Y, Z = self._dims(level)
        _native.call(self.conv_entry, co, ci, _p(dz), _p(self.params[i]["wf"]), None, _p(dst), _p(mask), 0,
                     X, Y, Z, self.B, self._stream())

    def backward(self, target, target_stride):
        """Gradients of the mean squared error between the prediction and the
        target volumes (normalised by the same per-study scale)."""
        st = self._stream()
        a, d, B = self.a, self.d, self.B
        X, Y, Z = self.X, self.Y, self.Z
        X2, Y2, Z2 = self._dims(1)
        for p in self.params:
            p["gw"].zero_()
            p["gb"].zero_()
        self.gw_head.zero_()
        self.gb_head.zero_()
        d["a2"].zero_()
        d["a4"].zero_()
        _native.call("omb_unet_head_bwd", _p(a["a10"]), _p(self.pred), _p(target), target_stride, _p(self.scale),
                     _p(self.head_w), _p(d["z10"]), _p(self.gw_head), _p(self.gb_head), _p(self.loss),
                     X, Y, Z, self.Zs, B, st)
        self._grads(9, a["a9"], d["z10"], 0)
        self._dgrad(9, d["z10"], d["z9"], 0, a["a9"])
        self._grads(8, a["c1"], d["z9"], 0)
        self._dgrad(8, d["z9"], d["c1"], 0, None)
        _native.call("omb_unet_up_concat_bwd", _p(d["c1"]), _p(d["a8"]), _p(d["a2"]), X, Y, Z, B, 32, 16, st)
        _native.call("omb_unet_relu_mask", _p(d["a8"]), _p(a["a8"]), d["a8"].numel(), st)
        self._grads(7, a["a7"], d["a8"], 1)
        self._dgrad(7, d["a8"], d["z7"], 1, a["a7"])
        self._grads(6, a["c2"], d["z7"], 1)
        self._dgrad(6, d["z7"], d["c2"], 1, None)
        _native.call("omb_unet_up_concat_bwd", _p(d["c2"]), _p(d["a6"]), _p(d["a4"]), X2, Y2, Z2, B, 64, 32, st)
        _native.call("omb_unet_relu_mask", _p(d["a6"]), _p(a["a6"]), d["a6"].numel(), st)
        self._grads(5, a["a5"], d["a6"], 2)
        self._dgrad(5, d["a6"], d["z5"], 2, a["a5"])
        self._grads(4, a["p2"], d["z5"], 2)
        self._dgrad(4, d["z5"], d["p2"], 2, None)
        _native.call("omb_unet_avgpool", _p(d["p2"]), _p(d["a4"]), X2, Y2, Z2, B, 32, 1, st)
        _native.call("omb_unet_relu_mask", _p(d["a4"]), _p(a["a4"]), d["a4"].numel(), st)
        self._grads(3, a["a3"], d["a4"], 1)
        self._dgrad(3, d["a4"], d["z3"], 1, a["a3"])
        self._grads(2, a["p1"], d["z3"], 1)
        self._dgrad(2, d["z3"], d["p1"], 1, None)
        _native.call("omb_unet_avgpool", _p(d["p1"]), _p(d["a2"]), X, Y, Z, B, 16, 1, st)
        _native.call("omb_unet_relu_mask", _p(d["a2"]), _p(a["a2"]), d["a2"].numel(), st)
        self._grads(1, a["a1"], d["a2"], 0)
        self._dgrad(1, d["a2"], d["z1"], 0, a["a1"])
        self._grads(0, a["x0"], d["z1"], 0)

    def adam_step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step_count += 1
        st, k = self._stream(), self.step_count
        for (ci, co), p in zip(LAYERS, self.params):
            _native.call("omb_unet_adam", _p(p["w"]), _p(p["mw"]), _p(p["vw"]), _p(p["gw"]), _p(p["wb"]),
                         p["w"].numel(), lr, beta1, beta2, k, eps, st)
            _native.call("omb_unet_adam", _p(p["b"]), _p(p["mb"]), _p(p["vb"]), _p(p["gb"]), None, p["b"].numel(),
                         lr, beta1, beta2, k, eps, st)
            _native.call("omb_unet_flip_weights", _p(p["wb"]), _p(p["wf"]), ci, co, st)
        m, v, mb, vb = self.head_state
        _native.call("omb_unet_adam", _p(self.head_w), _p(m), _p(v), _p(self.gw_head), None, 16, lr, beta1, beta2,
                     k, eps, st)
        _native.call("omb_unet_adam", _p(self.head_b), _p(mb), _p(vb), _p(self.gb_head), None, 1, lr, beta1, beta2,
                     k, eps, st)
