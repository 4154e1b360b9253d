"""Learned warm start for the MBS loop: a 3-D convolutional encoder-decoder.

No counterpart in the reference.  The network predicts the field psi0 of a
solve from the medium and the source; the MBS loop then starts from it
(``WaveSim.exec(source, warm_start=model)``) and iterates to the same energy
tolerance, so the loop, not the network, decides the answer.

Architecture (channels-last activations in bf16, 3x3x3 convolutions with zero
padding 1, ReLU after every convolution except the head):

    level 1 (full)  : 8 -> 32 -> 32          } skip 1
    level 2 (1/2)   : 32 -> 64 -> 64         } skip 2     2x2x2 average pooling
    level 3 (1/4)   : 64 -> 96 -> 96         } skip 3     between levels
    bottom  (1/8)   : 96 -> 128 -> 128
    up 3 (1/4)      : [128 up, 96 skip] -> 96 -> 96       nearest x2 upsampling
    up 2 (1/2)      : [96 up, 64 skip] -> 64 -> 64        and channel concat
    up 1 (full)     : [64 up, 32 skip] -> 32 -> 32
    head            : 32 -> 2 (Re, Im), fp32

about 2.7 million parameters.  Inputs per voxel (ws_net_features): (n - n_bg)
/ 0.2, the source amplitude, cos / sin of the straight-ray phase k0 sum_z
(n - n_bg), zeros.  Output: the envelope of the field, E / (a exp(i k0 n_bg
z)) with a the amplitude of a unit plane source.  Voxels are in the ROI's
column-major order, i.e. the network sees a (z, x, y) volume.

Every arithmetic step is a kernel of this package (include/wavesim_b200_net.h):
the forward convolutions and the input gradients are implicit GEMMs on the
tcgen05 tensor cores (ws_conv3_fwd_bf16 / ws_conv3_upcat_fwd_bf16, the input
gradient with tap-flipped weights), the weight gradients explicit GEMMs
(ws_gemm_bf16) of transposed im2col matrices; Adam keeps fp32 master
weights and a bf16 copy for the GEMMs.  PyTorch only allocates and clears
device memory.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib

P = C.c_void_p
I64 = C.c_int64
INT = C.c_int


def _bind():
    L = _lib.lib
    sig = {
        "ws_conv3_fwd_bf16": [P, P, P, P, P] + [INT] * 8 + [P, P],
        "ws_conv3_upcat_fwd_bf16": [P, P, P, P, P, P] + [INT] * 9 + [P, P],
        "ws_net_features": [P, P, INT, INT, INT, C.c_float, C.c_float, P, P],
        "ws_net_envelope_to_field": [P, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64), C.c_float, C.c_float, INT, P,
                                     P],
        "ws_net_space_to_depth": [P, P, INT, INT, INT, INT, INT, P],
        "ws_net_flip_weights": [P, INT, INT, INT, P, INT, INT, P],
        "ws_net_relu_grad_bf16": [P, P, I64, INT, P, INT, P],
        "ws_net_im2col3": [P, P, INT, INT, INT, INT, INT, INT, P],
        "ws_net_col2im3": [P, P, INT, INT, INT, INT, INT, INT, P],
        "ws_net_transpose_f32_bf16": [P, P, I64, I64, I64, P],
        "ws_net_transpose_bf16": [P, P, I64, I64, I64, I64, P],
        "ws_net_avgpool2": [P, P, INT, INT, INT, INT, INT, P],
        "ws_net_avgpool2_grad": [P, P, INT, INT, INT, INT, INT, P],
        "ws_net_upcat": [P, P, P, INT, INT, INT, INT, INT, INT, P],
        "ws_net_upcat_grad": [P, P, P, INT, INT, INT, INT, INT, INT, P],
        "ws_net_relu_grad": [P, P, I64, P],
        "ws_net_bias_grad": [P, P, I64, INT, P],
        "ws_net_adam": [P, P, P, P, P, I64, C.c_float, C.c_float, C.c_float, C.c_float, INT, P],
        "ws_net_mse": [P, P, P, P, I64, INT, I64, P],
        "ws_net_f32_to_bf16": [P, P, I64, P],
        "ws_net_add": [P, P, I64, P],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = INT
    return L


_L = None


def lib():
    global _L
    if _L is None:
        _L = _bind()
    return _L


def _ck(rc, what):
    if rc != 0:
        raise _lib.WaveSimError(rc, f"{what}: {_lib.lib.ws_net_last_error().decode(errors='replace')}")


def _ptr(t):
    return None if t is None else t.data_ptr()


def pad64(n):
    return (n + 63) // 64 * 64


def pad8(n):
    return (n + 7) // 8 * 8


class Conv3:
    """3x3x3 convolution Cin -> Cout: fp32 master weights w [Cout][kp] (K =
    27 Cin padded to kp, a multiple of 64), bias b, bf16 copy wb."""

    def __init__(self, cin, cout, relu, rng, torch, dev):
        self.cin, self.cout, self.relu = cin, cout, relu
        self.k = 27 * cin
        self.kp = pad64(self.k)
        self.cpad = pad8(cout)  # channels of the output gradient fed to the input-gradient convolution
        self.kpf = pad64(27 * self.cpad)
        std = math.sqrt(2.0 / self.k) if relu else math.sqrt(1.0 / self.k)
        w = np.zeros((cout, self.kp), np.float32)
        w[:, :self.k] = rng.standard_normal((cout, self.k)) * std
        self.w = torch.from_numpy(w).to(dev)
        self.b = torch.zeros(cout, device=dev)
        self.wb = torch.empty(cout, self.kp, device=dev, dtype=torch.bfloat16)
        self.mw, self.vw = torch.zeros_like(self.w), torch.zeros_like(self.w)
        self.mb, self.vb = torch.zeros_like(self.b), torch.zeros_like(self.b)
        self.gw, self.gb = torch.zeros_like(self.w), torch.zeros_like(self.b)
        self.torch = torch
        self.record = None  # a list: backward appends (x, y, dy, dx) copies (for tests)
        self.refresh()

    def refresh(self):
        _ck(lib().ws_net_f32_to_bf16(self.w.data_ptr(), self.wb.data_ptr(), self.w.numel(), None), "f32_to_bf16")

    @property
    def nparams(self):
        return self.cout * self.k + self.cout

    def forward(self, x, vol, out_f32=False, err=None):
        """x: bf16 [vox][cin]; returns bf16 [vox][cout] (ReLU) or fp32 [vox][cout] (head)."""
        torch = self.torch
        b, d, h, w = vol
        y = torch.empty(b * d * h * w, self.cout, device=x.device, dtype=torch.float32 if out_f32 else torch.bfloat16)
        mode = 3 if out_f32 else (1 if self.relu else 2)
        _ck(lib().ws_conv3_fwd_bf16(x.data_ptr(), self.wb.data_ptr(), self.b.data_ptr(), _ptr(y) if out_f32 else None,
                                    None if out_f32 else _ptr(y), b, d, h, w, self.cin, self.cout, self.kp, mode,
                                    _ptr(err), None), "conv fwd")
        return y

    def forward_upcat_fused(self, u, skip, vol, cu, cs, err=None):
        """The layer on [nearest x2 upsampling of u (cu channels), skip (cs
        channels)] at the resolution `vol`, without writing the concat (the
        kernel computes the upsampled coordinates per tap: slower than
        writing the concat first, see forward_upcat)."""
        torch = self.torch
        b, d, h, w = vol
        y = torch.empty(b * d * h * w, self.cout, device=skip.device, dtype=torch.bfloat16)
        mode = 1 if self.relu else 2
        _ck(lib().ws_conv3_upcat_fwd_bf16(u.data_ptr(), skip.data_ptr(), self.wb.data_ptr(), self.b.data_ptr(), None,
                                          y.data_ptr(), b, d, h, w, cu, cs, self.cout, self.kp, mode, _ptr(err), None),
            "conv upcat fwd")
        return y

    def forward_upcat(self, u, skip, vol, cu, cs, err=None):
        """The layer on [nearest x2 upsampling of u (cu channels), skip (cs
        channels)]: the concat is written once (ws_net_upcat) and read by the
        plain convolution, whose gather is cheaper than the fused one's.
        Returns (output, concat)."""
        torch = self.torch
        b, d, h, w = vol
        cat = torch.empty(b * d * h * w, cu + cs, device=skip.device, dtype=torch.bfloat16)
        _ck(lib().ws_net_upcat(u.data_ptr(), skip.data_ptr(), cat.data_ptr(), b, d, h, w, cu, cs, None), "upcat")
        return self.forward(cat, vol, err=err), cat

    def backward(self, x, y, dy, vol, need_dx=True, err=None):
        """x: layer input (bf16 [vox][cin]); y: its ReLU output (bf16) or None
        for the head; dy: fp32 [vox][cout] gradient of the output (masked in
        place).  Accumulates gw / gb; returns dx fp32 [vox][cin] or None."""
        torch = self.torch
        b, d, h, w = vol
        nvox = b * d * h * w
        L = lib()
        dy_in = dy.clone() if self.record is not None else None
        dyb = torch.empty(nvox, self.cpad, device=dy.device, dtype=torch.bfloat16)
        _ck(L.ws_net_relu_grad_bf16(dy.data_ptr(), _ptr(y) if self.relu else None, nvox, self.cout, dyb.data_ptr(),
                                    self.cpad, None), "relu grad")
        gb = torch.empty(self.cout, device=dy.device)
        _ck(L.ws_net_bias_grad(dy.data_ptr(), gb.data_ptr(), nvox, self.cout, None), "bias grad")
        _ck(L.ws_net_add(self.gb.data_ptr(), gb.data_ptr(), self.cout, None), "add")
        # weight gradient: dW[co][k] = sum_vox dy[vox][co] im2col(x)[vox][k]
        voxp = pad64(nvox)
        col = torch.empty(nvox, self.kp, device=dy.device, dtype=torch.bfloat16)
        _ck(L.ws_net_im2col3(x.data_ptr(), col.data_ptr(), b, d, h, w, self.cin, self.kp, None), "im2col")
        colT = torch.empty(self.kp, voxp, device=dy.device, dtype=torch.bfloat16)
        _ck(L.ws_net_transpose_bf16(col.data_ptr(), colT.data_ptr(), nvox, self.kp, self.kp, voxp, None), "transpose")
        del col
        dyT = torch.empty(self.cout, voxp, device=dy.device, dtype=torch.bfloat16)
        _ck(L.ws_net_transpose_f32_bf16(dy.data_ptr(), dyT.data_ptr(), nvox, self.cout, voxp, None), "transpose")
        gw = torch.empty(self.cout, self.kp, device=dy.device)
        _ck(_lib.lib.ws_gemm_bf16(dyT.data_ptr(), colT.data_ptr(), gw.data_ptr(), None, None, self.cout, self.kp,
                                  voxp, voxp, voxp, self.kp, 0, _ptr(err), None), "gemm wgrad")
        _ck(L.ws_net_add(self.gw.data_ptr(), gw.data_ptr(), gw.numel(), None), "add")
        del colT, dyT
        dx = None
        if need_dx:
            # input gradient: the convolution of dy with the tap-flipped, transposed weights
            wf = torch.empty(self.cin, self.kpf, device=dy.device, dtype=torch.bfloat16)
            _ck(L.ws_net_flip_weights(self.wb.data_ptr(), self.cin, self.cout, self.kp, wf.data_ptr(), self.cpad,
                                      self.kpf, None), "flip weights")
            dx = torch.empty(nvox, self.cin, device=dy.device)
            _ck(L.ws_conv3_fwd_bf16(dyb.data_ptr(), wf.data_ptr(), None, dx.data_ptr(), None, b, d, h, w, self.cpad,
                                    self.cin, self.kpf, 0, _ptr(err), None), "conv dgrad")
        if self.record is not None:
            self.record.append((x.clone(), None if y is None else y.clone(), dy_in, None if dx is None else dx.clone()))
        return dx

    def zero_grad(self):
        self.gw.zero_()
        self.gb.zero_()

    def adam(self, lr, step, b1=0.9, b2=0.999, eps=1e-8):
        L = lib()
        _ck(L.ws_net_adam(self.w.data_ptr(), self.gw.data_ptr(), self.mw.data_ptr(), self.vw.data_ptr(),
                          self.wb.data_ptr(), self.w.numel(), lr, b1, b2, eps, step, None), "adam")
        _ck(L.ws_net_adam(self.b.data_ptr(), self.gb.data_ptr(), self.mb.data_ptr(), self.vb.data_ptr(), None,
                          self.b.numel(), lr, b1, b2, eps, step, None), "adam")


class WarmStartNet:
    """A 4-level encoder-decoder of 3x3x3 convolutions (see the module
    docstring) from in_ch to out_ch channels."""

    def __init__(self, widths=(32, 64, 96, 128), device=0, seed=0, in_ch=8, out_ch=2):
        import torch
        self.IN_CH, self.OUT_CH = in_ch, out_ch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        rng = np.random.default_rng(seed)
        w1, w2, w3, w4 = widths
        mk = lambda ci, co, relu=True: Conv3(ci, co, relu, rng, torch, self.dev)  # noqa: E731
        self.c1a, self.c1b = mk(self.IN_CH, w1), mk(w1, w1)
        self.c2a, self.c2b = mk(w1, w2), mk(w2, w2)
        self.c3a, self.c3b = mk(w2, w3), mk(w3, w3)
        self.c4a, self.c4b = mk(w3, w4), mk(w4, w4)
        self.d3a, self.d3b = mk(w4 + w3, w3), mk(w3, w3)
        self.d2a, self.d2b = mk(w3 + w2, w2), mk(w2, w2)
        self.d1a, self.d1b = mk(w2 + w1, w1), mk(w1, w1)
        self.head = mk(w1, self.OUT_CH, relu=False)
        self.widths = widths
        self.step_count = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=self.dev)  # set by a timed-out tensor-core wait

    @property
    def layers(self):
        return [self.c1a, self.c1b, self.c2a, self.c2b, self.c3a, self.c3b, self.c4a, self.c4b,
                self.d3a, self.d3b, self.d2a, self.d2b, self.d1a, self.d1b, self.head]

    @property
    def nparams(self):
        return sum(l.nparams for l in self.layers)

    def _pool(self, x, vol, c):
        b, d, h, w = vol
        y = self.torch.empty(b * (d // 2) * (h // 2) * (w // 2), c, device=self.dev, dtype=self.torch.bfloat16)
        _ck(lib().ws_net_avgpool2(x.data_ptr(), y.data_ptr(), b, d, h, w, c, None), "pool")
        return y

    def _upcat(self, a, skip, vol, ca, cs):
        b, d, h, w = vol
        y = self.torch.empty(b * d * h * w, ca + cs, device=self.dev, dtype=self.torch.bfloat16)
        _ck(lib().ws_net_upcat(a.data_ptr(), skip.data_ptr(), y.data_ptr(), b, d, h, w, ca, cs, None), "upcat")
        return y

    def _check_err(self):
        if int(self.err.item()):
            self.err.zero_()
            raise _lib.WaveSimError(_lib.WS_ERR_CUDA, "warm-start network: a tensor-core wait timed out")

    def forward(self, x, vol, keep=False):
        """x: bf16 [vox][8] for a volume (b, d, h, w) with d, h, w multiples of 8.
        Returns fp32 [vox][2]; with keep=True also the activations for backward
        (including the decoder concats, which the forward pass reads in place)."""
        w1, w2, w3, w4 = self.widths
        b, d, h, w = vol
        if d % 8 or h % 8 or w % 8:
            raise ValueError("the volume sides must be multiples of 8")
        v1, v2, v3, v4 = vol, (b, d // 2, h // 2, w // 2), (b, d // 4, h // 4, w // 4), (b, d // 8, h // 8, w // 8)
        err = self.err
        a = {"x": x}
        a["e1a"] = self.c1a.forward(x, v1, err=err)
        a["e1"] = self.c1b.forward(a["e1a"], v1, err=err)
        a["p1"] = self._pool(a["e1"], v1, w1)
        a["e2a"] = self.c2a.forward(a["p1"], v2, err=err)
        a["e2"] = self.c2b.forward(a["e2a"], v2, err=err)
        a["p2"] = self._pool(a["e2"], v2, w2)
        a["e3a"] = self.c3a.forward(a["p2"], v3, err=err)
        a["e3"] = self.c3b.forward(a["e3a"], v3, err=err)
        a["p3"] = self._pool(a["e3"], v3, w3)
        a["b4a"] = self.c4a.forward(a["p3"], v4, err=err)
        a["b4"] = self.c4b.forward(a["b4a"], v4, err=err)
        a["d3a"], a["u3"] = self.d3a.forward_upcat(a["b4"], a["e3"], v3, w4, w3, err=err)
        a["d3"] = self.d3b.forward(a["d3a"], v3, err=err)
        a["d2a"], a["u2"] = self.d2a.forward_upcat(a["d3"], a["e2"], v2, w3, w2, err=err)
        a["d2"] = self.d2b.forward(a["d2a"], v2, err=err)
        a["d1a"], a["u1"] = self.d1a.forward_upcat(a["d2"], a["e1"], v1, w2, w1, err=err)
        a["d1"] = self.d1b.forward(a["d1a"], v1, err=err)
        out = self.head.forward(a["d1"], v1, out_f32=True, err=err)
        if keep:
            return out, a
        return out

    def backward(self, a, dout, vol):
        """Back-propagates dout (fp32 [vox][2]) through the activations `a` of forward(keep=True)."""
        torch = self.torch
        L = lib()
        err = self.err
        w1, w2, w3, w4 = self.widths
        b, d, h, w = vol
        v1, v2, v3, v4 = vol, (b, d // 2, h // 2, w // 2), (b, d // 4, h // 4, w // 4), (b, d // 8, h // 8, w // 8)
        n = lambda v: v[0] * v[1] * v[2] * v[3]  # noqa: E731

        def upcat_grad(g, v, ca, cs):
            da = torch.empty(n(v) // 8, ca, device=self.dev)
            ds = torch.empty(n(v), cs, device=self.dev)
            _ck(L.ws_net_upcat_grad(g.data_ptr(), da.data_ptr(), ds.data_ptr(), v[0], v[1], v[2], v[3], ca, cs, None),
                "upcat grad")
            return da, ds

        def pool_grad(g, v, c, skip):
            """gradient through the pooling, plus the skip path's gradient"""
            dx = torch.empty(n(v), c, device=self.dev)
            _ck(L.ws_net_avgpool2_grad(g.data_ptr(), dx.data_ptr(), v[0], v[1], v[2], v[3], c, None), "pool grad")
            _ck(L.ws_net_add(dx.data_ptr(), skip.data_ptr(), dx.numel(), None), "add")
            return dx

        g = self.head.backward(a["d1"], None, dout.clone(), v1, err=err)
        g = self.d1b.backward(a["d1a"], a["d1"], g, v1, err=err)
        g = self.d1a.backward(a["u1"], a["d1a"], g, v1, err=err)
        g_d2, g_e1 = upcat_grad(g, v1, w2, w1)
        g = self.d2b.backward(a["d2a"], a["d2"], g_d2, v2, err=err)
        g = self.d2a.backward(a["u2"], a["d2a"], g, v2, err=err)
        g_d3, g_e2 = upcat_grad(g, v2, w3, w2)
        g = self.d3b.backward(a["d3a"], a["d3"], g_d3, v3, err=err)
        g = self.d3a.backward(a["u3"], a["d3a"], g, v3, err=err)
        g_b4, g_e3 = upcat_grad(g, v3, w4, w3)
        g = self.c4b.backward(a["b4a"], a["b4"], g_b4, v4, err=err)
        g = self.c4a.backward(a["p3"], a["b4a"], g, v4, err=err)
        g = pool_grad(g, v3, w3, g_e3)
        g = self.c3b.backward(a["e3a"], a["e3"], g, v3, err=err)
        g = self.c3a.backward(a["p2"], a["e3a"], g, v3, err=err)
        g = pool_grad(g, v2, w2, g_e2)
        g = self.c2b.backward(a["e2a"], a["e2"], g, v2, err=err)
        g = self.c2a.backward(a["p1"], a["e2a"], g, v2, err=err)
        g = pool_grad(g, v1, w1, g_e1)
        g = self.c1b.backward(a["e1a"], a["e1"], g, v1, err=err)
        self.c1a.backward(a["x"], a["e1a"], g, v1, need_dx=False, err=err)

    def train_step(self, x, target, vol, lr):
        """One Adam step on (x, target fp32 [vox][2]); returns the mean squared error."""
        torch = self.torch
        for l in self.layers:
            l.zero_grad()
        out, a = self.forward(x, vol, keep=True)
        grad = torch.empty_like(out)
        loss = torch.zeros(1, dtype=torch.float64, device=self.dev)
        _ck(lib().ws_net_mse(out.data_ptr(), target.data_ptr(), grad.data_ptr(), loss.data_ptr(), out.shape[0],
                             self.OUT_CH, self.OUT_CH, None), "mse")
        self.backward(a, grad, vol)
        self.step_count += 1
        for l in self.layers:
            l.adam(lr, self.step_count)
        value = float(loss.item())
        self._check_err()
        return value

    def state(self):
        return {f"l{i}.{k}": getattr(l, k).detach().cpu().numpy() for i, l in enumerate(self.layers) for k in ("w", "b")}

    def load(self, state):
        torch = self.torch
        for i, l in enumerate(self.layers):
            l.w.copy_(torch.from_numpy(state[f"l{i}.w"]))
            l.b.copy_(torch.from_numpy(state[f"l{i}.b"]))
            l.refresh()


# ----------------------------------------------------------------------------
# inputs and outputs
# ----------------------------------------------------------------------------
def roi_volume(shape, half=False):
    """Network volume (b, d, h, w) of a ROI (Ny, Nx, Nz): voxels in the ROI's
    column-major order, i.e. (z, x, y) with y fastest; half=True: the
    half-resolution volume after space to depth."""
    Ny, Nx, Nz = shape
    return (1, Nz // 2, Nx // 2, Ny // 2) if half else (1, Nz, Nx, Ny)


def _shape(n_roi):
    return tuple(n_roi.shape) if hasattr(n_roi, "data_ptr") else tuple(np.shape(n_roi))


def features(n_roi, k0, n_bg, torch, dev, src=None):
    """Network input of a ROI (Ny, Nx, Nz; z the propagation direction):
    bf16 [vox][8] from ws_net_features; n_roi a host array or a device tensor
    (real fp32, column-major flat memory), src (optional, ROI-sized) the
    source amplitude, by default a plane of ones at z = 0."""
    Ny, Nx, Nz = _shape(n_roi)
    if hasattr(n_roi, "data_ptr"):
        nd = n_roi
    else:
        nd = torch.from_numpy(np.ascontiguousarray(np.real(np.asarray(n_roi)).astype(np.float32).ravel(order="F")))
        nd = nd.to(dev)
    sd = None
    if src is not None:
        sd = torch.from_numpy(np.ascontiguousarray(np.asarray(src, np.float32).ravel(order="F"))).to(dev)
    out = torch.empty(Ny * Nx * Nz, 8, device=dev, dtype=torch.bfloat16)
    _ck(lib().ws_net_features(nd.data_ptr(), _ptr(sd), Ny, Nx, Nz, n_bg, k0, out.data_ptr(), None), "features")
    return out


def space_to_depth(x, shape, torch):
    """[vox][C] bf16 of a ROI volume -> [hvox][8C] at half resolution (ws_net_space_to_depth)."""
    b, d, h, w = roi_volume(shape)
    C = x.shape[1]
    y = torch.empty(x.shape[0] // 8, 8 * C, device=x.device, dtype=torch.bfloat16)
    _ck(lib().ws_net_space_to_depth(x.data_ptr(), y.data_ptr(), b, d, h, w, C, None), "space to depth")
    return y


def carrier(shape, k0, n_bg):
    """exp(i k0 n_bg z) on a (y, x, z) ROI, z counted from the source plane."""
    z = np.arange(shape[2])
    return np.broadcast_to(np.exp(1j * k0 * n_bg * z)[None, None, :], shape)


def field_to_target(env_roi, scale, half=False):
    """Training target from the ROI envelope (y, x, z): fp32 [vox][2] in the
    ROI's column-major order, or (half=True) [hvox][16] in the
    space-to-depth layout (sub-voxel s of the (z, x, y) volume at columns 2s,
    2s + 1)."""
    e = np.asarray(env_roi) / scale
    if not half:
        e = e.ravel(order="F")
        return np.stack([e.real, e.imag], axis=-1).astype(np.float32)
    Ny, Nx, Nz = e.shape
    v = np.transpose(e, (2, 1, 0)).reshape(Nz // 2, 2, Nx // 2, 2, Ny // 2, 2)
    v = np.transpose(v, (0, 2, 4, 1, 3, 5)).reshape(-1, 8)
    return np.ascontiguousarray(np.stack([v.real, v.imag], axis=-1).reshape(-1, 16).astype(np.float32))


def target_to_field(pred, shape, scale, half=False):
    p = np.asarray(pred)
    if not half:
        p = p.reshape(-1, 2)
        return (p[:, 0] + 1j * p[:, 1]).reshape(shape, order="F") * scale
    Ny, Nx, Nz = shape
    c = p.reshape(-1, 8, 2)
    c = (c[..., 0] + 1j * c[..., 1]).reshape(Nz // 2, Nx // 2, Ny // 2, 2, 2, 2)
    c = np.transpose(c, (0, 3, 1, 4, 2, 5)).reshape(Nz, Nx, Ny)
    return np.transpose(c, (2, 1, 0)) * scale


def field_scale(pixel_size, lam, n_bg):
    """Amplitude of the field of a unit plane source (the 1-D Green's function
    i h / (2 k), utilities/homogeneous_medium_analytic_solution.m:28)."""
    return pixel_size / (2 * (2 * np.pi / lam) * n_bg)


# ----------------------------------------------------------------------------
# training data, training, prediction
# ----------------------------------------------------------------------------
def make_training_set(count, roi=48, bw=8, seed=0, n_bg=1.33, tol=1e-4, pixel_size=0.25, lam=1.0):
    """MBS solutions (this package's solver) of `count` seeded media of the
    c3 sphere distribution with a plane-wave source on the z = 1 face.
    `roi` is one cube side or a sequence of sides (each sample draws one:
    crops of several sizes).  Returns a list of (n_roi, E_roi)."""
    from .problem import Source
    from .simulation import WaveSim
    from .workloads import sphere_medium
    rng = np.random.default_rng(seed)
    sides = [int(roi)] if np.ndim(roi) == 0 else [int(v) for v in roi]
    out = []
    opt = {"lambda": lam, "pixel_size": pixel_size, "boundary_widths": [bw, bw, bw], "energy_threshold": tol,
           "device_setup": True}
    for _ in range(count):
        side = sides[int(rng.integers(len(sides)))]
        n = sphere_medium(side, rng, n_bg=n_bg)
        sim = WaveSim(n, opt)
        E, st = sim.exec(Source(np.ones((side, side)), [1, 1, 1]))
        sim.close()
        out.append((n, E))
    return out


class WarmStart:
    """A trained network plus the normalisation of its inputs and outputs.

    Media and fields are on the ROI, (Ny, Nx, Nz), z the propagation
    direction, the source a plane of ones at z = 1 (the c3 benchmark's).  The
    network works at half resolution: the 8 input channels of 2x2x2 voxels
    go in as 64 channels (space to depth), the 2 x 8 output channels come out
    as the envelope of those 8 voxels, so no convolution runs on the full
    grid.  ROI sides must be multiples of 16."""

    HALF_WIDTHS = (32, 64, 96, 128)

    def __init__(self, net=None, n_bg=1.33, pixel_size=0.25, lam=1.0, device=0, seed=0):
        self.net = net or WarmStartNet(widths=self.HALF_WIDTHS, device=device, seed=seed, in_ch=64, out_ch=16)
        self.half = self.net.IN_CH == 64
        self.n_bg, self.pixel_size, self.lam = n_bg, pixel_size, lam
        self.k0 = 2 * np.pi / lam * pixel_size  # wavenumber per pixel
        self.scale = field_scale(pixel_size, lam, n_bg)

    def _check(self, shape):
        m = 16 if self.half else 8
        if len(shape) != 3 or any(v % m for v in shape):
            raise ValueError(f"the ROI sides must be multiples of {m}, got {tuple(shape)}")

    def _input(self, n_roi):
        shape = _shape(n_roi)
        x = features(n_roi, self.k0, self.n_bg, self.net.torch, self.net.dev)
        if self.half:
            x = space_to_depth(x, shape, self.net.torch)
        return x, roi_volume(shape, self.half)

    def train(self, data, steps, lr=2e-3, lr_end=2e-4, log=None):
        torch = self.net.torch
        prepared = []
        for n, E in data:
            self._check(np.shape(n))
            x, vol = self._input(n)
            env = np.asarray(E) / carrier(np.shape(E), self.k0, self.n_bg)  # the field's envelope
            t = torch.from_numpy(field_to_target(env, self.scale, self.half)).to(self.net.dev)
            prepared.append((x, t, vol))
        losses = []
        for s in range(steps):
            x, t, vol = prepared[s % len(prepared)]
            lr_s = lr * (lr_end / lr) ** (s / max(1, steps - 1))
            losses.append(self.net.train_step(x, t, vol, lr_s))
            if log and (s % 100 == 0 or s == steps - 1):
                log(s, losses[-1])
        return losses

    def envelope(self, n_roi):
        """The network output (fp32 device tensor) for a ROI medium."""
        self._check(_shape(n_roi))
        x, vol = self._input(n_roi)
        return self.net.forward(x, vol)

    def predict(self, n_roi):
        """psi0 on the ROI (y, x, z) as a host array."""
        shape = _shape(n_roi)
        env = target_to_field(self.envelope(n_roi).cpu().numpy(), shape, self.scale, self.half)
        self.net._check_err()
        return env * carrier(shape, self.k0, self.n_bg)

    def predict_grid(self, sim, n_roi=None):
        """psi0 on the full grid of the scalar WaveSim `sim` (boundary layers
        included, ws_net_envelope_to_field) as a flat complex64 device tensor
        in column-major order, the form WaveSim.exec takes as a warm start
        without a host round trip.  n_roi defaults to sim's medium."""
        torch = self.net.torch
        if n_roi is None:
            n_roi = sim.roi_medium()
        shape = _shape(n_roi)
        pred = self.envelope(n_roi)
        N = (I64 * 3)(*[int(v) for v in sim.N[:3]])
        r0 = (I64 * 3)(*[int(sim.roi[0, d]) - 1 for d in range(3)])
        rn = (I64 * 3)(*[int(v) for v in shape])
        psi = torch.empty(int(np.prod(sim.N[:3])), dtype=torch.complex64, device=self.net.dev)
        _ck(lib().ws_net_envelope_to_field(pred.data_ptr(), N, r0, rn, self.scale, self.k0 * self.n_bg,
                                           1 if self.half else 0, psi.data_ptr(), None), "envelope to field")
        self.net._check_err()
        return psi

    def save(self, path, bf16=False, provenance=None):
        """Weights and normalisation to an .npz; bf16=True stores the weights
        as bfloat16 bit patterns (uint16), the precision the kernels use.
        provenance: a dict (e.g. the training command and its results),
        stored as JSON text."""
        st = self.net.state()
        if bf16:
            st = {k: _to_bf16_bits(v) for k, v in st.items()}
        st["meta"] = np.array([self.n_bg, self.pixel_size, self.lam] + list(self.net.widths) +
                              [self.net.IN_CH, self.net.OUT_CH], np.float64)
        if provenance is not None:
            import json
            st["provenance"] = np.array(json.dumps(provenance))
        np.savez_compressed(path, **st)

    @staticmethod
    def provenance(path):
        """The provenance dict stored with a checkpoint (None if absent)."""
        import json
        st = np.load(path)
        return json.loads(str(st["provenance"])) if "provenance" in st.files else None

    @classmethod
    def load(cls, path, device=0):
        st = dict(np.load(path))
        meta = st.pop("meta")
        st.pop("provenance", None)
        st = {k: (_from_bf16_bits(v) if v.dtype == np.uint16 else v) for k, v in st.items()}
        in_ch, out_ch = (int(meta[7]), int(meta[8])) if meta.size > 7 else (8, 2)
        net = WarmStartNet(widths=tuple(int(v) for v in meta[3:7]), device=device, in_ch=in_ch, out_ch=out_ch)
        net.load(st)
        return cls(net, n_bg=float(meta[0]), pixel_size=float(meta[1]), lam=float(meta[2]), device=device)


def _to_bf16_bits(a):
    """fp32 -> bfloat16 bit patterns, round to nearest even."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def _from_bf16_bits(b):
    return (b.astype(np.uint32) << 16).view(np.float32)
