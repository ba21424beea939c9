"""Residual MLP of the learned warm start, run by the library's BF16 kernels.

Architecture (4 layers of width 256): x[128 padded inputs] -> h0 = relu(W0 x
+ b0) -> three residual blocks h_l = h_{l-1} + relu(W_l h_{l-1} + b_l) ->
y = W4 h3 + b4 + base, where ``base`` is the IDW interpolation in normalised
primitives, so the network predicts the correction. W4 starts at zero: the
untrained model is exactly IDW.

PyTorch only holds the device buffers (parameters, Adam moments,
activations) and the stream; every forward, backward, loss and optimizer
step is a kernel of ``libeulersr.so`` (esr_gemm_bf16 on the tcgen05 tensor cores,
head/loss/AdamW/reduction kernels).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from .. import _ffi as F

K_IN = 128      # padded input width (13 features used)
H = 256
N_OUT = 4
ROW_TILE = 128  # the GEMM tiles rows by 128


def _p(t):
    """Device address of a CUDA tensor for a kernel argument. A tensor in host
    memory is refused here: the kernels would dereference its address."""
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError(f"expected a CUDA tensor, got one on {t.device}")
    return C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class MLP:
    # parameter layout in the flat vectors
    SHAPES = [("W0", (H, K_IN)), ("b0", (H,)), ("W1", (H, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)),
              ("W3", (H, H)), ("b3", (H,)), ("W4", (N_OUT, H)), ("b4", (N_OUT,))]

    def __init__(self, device="cuda", seed=0, n_features=13, gemm="tcgen05"):
        if torch.device(device).type != "cuda":
            raise ValueError(f"the MLP runs on the library's CUDA kernels; device must be a CUDA device, not {device!r}")
        self.L = F.lib()
        # the 256-wide layers: tcgen05 kernel, or the mma.sync kernel kept as its cross-check
        self.gemm = {"tcgen05": self.L.esr_gemm_bf16, "mma_sync": self.L.esr_gemm_bf16_mma_sync}[gemm]
        self.device = device
        self.launches = 0          # library kernels launched by forward()
        self.n_features = n_features
        self.offsets = {}
        off = 0
        for name, shp in self.SHAPES:
            self.offsets[name] = (off, shp)
            off += int(np.prod(shp))
        self.n_params = off
        g = torch.Generator().manual_seed(seed)
        p = torch.zeros(off, dtype=torch.float32)
        for name, shp in self.SHAPES:
            o, _ = self.offsets[name]
            n = int(np.prod(shp))
            if name.startswith("W") and name != "W4":
                fan_in = shp[1] if name != "W0" else n_features
                w = torch.randn(shp, generator=g) * math.sqrt(2.0 / fan_in)
                if name == "W0":
                    w[:, n_features:] = 0.0
                elif name != "W0":
                    w *= 0.5        # residual branches start small
                p[o:o + n] = w.reshape(-1)
        self.p = p.to(device)
        self.pb = self.p.to(torch.bfloat16)
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.step_count = 0
        self._ws = {}

    # ------------------------------------------------------------ helpers
    def view(self, name, bf16=False):
        o, shp = self.offsets[name]
        t = self.pb if bf16 else self.p
        return t[o:o + int(np.prod(shp))].view(*shp)

    def gview(self, name):
        o, shp = self.offsets[name]
        return self.g[o:o + int(np.prod(shp))].view(*shp)

    def _buf(self, key, shape, dtype):
        t = self._ws.get(key)
        if t is None or t.shape != torch.Size(shape) or t.dtype != dtype:
            t = torch.empty(shape, dtype=dtype, device=self.device)
            self._ws[key] = t
        return t

    def state_dict(self):
        return {"p": self.p.detach().cpu().numpy(), "n_features": self.n_features}

    def load_state_dict(self, d):
        self.p.copy_(torch.from_numpy(np.asarray(d["p"], np.float32)).to(self.device))
        self.pb.copy_(self.p.to(torch.bfloat16))

    # ------------------------------------------------------------ forward
    def forward(self, X, base=None, keep=False):
        """X: BF16 [rows x 128] (rows a multiple of 128); base: FP32 [rows x 4]."""
        rows = X.shape[0]
        assert rows % ROW_TILE == 0 and X.shape[1] == K_IN and X.dtype == torch.bfloat16
        st = _stream()
        tag = "k" if keep else "f"
        h = [self._buf(f"{tag}h{l}", (rows, H), torch.bfloat16) for l in range(4)]
        z = [self._buf(f"{tag}z{l}", (rows, H), torch.bfloat16) for l in range(4)]
        F.check(self.gemm(0, 0, rows, H, K_IN, _p(X), K_IN, _p(self.view("W0", True)), K_IN, 1,
                                     _p(self.view("b0")), None, None, _p(h[0]), _p(z[0]), H, 1, st))
        for l in range(1, 4):
            F.check(self.gemm(0, 0, rows, H, H, _p(h[l - 1]), H, _p(self.view(f"W{l}", True)), H, 1,
                                         _p(self.view(f"b{l}")), _p(h[l - 1]), None, _p(h[l]), _p(z[l]), H, 1, st))
        y = self._buf(f"{tag}y", (rows, N_OUT), torch.float32)
        F.check(self.L.esr_mlp_head_fwd(_p(h[3]), rows, H, _p(self.view("W4")), _p(self.view("b4")),
                                        _p(base) if base is not None else None, _p(y), st))
        self.launches += 5
        if keep:
            return y, dict(X=X, h=h, z=z)
        return y

    # ----------------------------------------------------------- backward
    def backward(self, acts, dY, splits=None):
        """Fill self.g from dL/dy (FP32 [rows x 4])."""
        X, h, z = acts["X"], acts["h"], acts["z"]
        rows = X.shape[0]
        st = _stream()
        if splits is None:
            splits = 1
            while splits < 64 and rows % (64 * splits * 2) == 0 and rows // (splits * 2) >= 1024:
                splits *= 2
        rpb = 256
        nblk = (rows + rpb - 1) // rpb
        part_head = self._buf("part_head", (nblk, 4 * H + 4), torch.float32)
        dh = self._buf("dh3", (rows, H), torch.bfloat16)
        dz = self._buf("dz3", (rows, H), torch.bfloat16)
        F.check(self.L.esr_mlp_head_bwd(_p(dY), _p(h[3]), _p(z[3]), rows, H, _p(self.view("W4")), _p(dh), _p(dz),
                                        _p(part_head), rpb, st))
        # W4 and b4 are contiguous in the flat layout, as in the partials
        F.check(self.L.esr_reduce_splits(_p(part_head), nblk, 4 * H + 4, 4 * H + 4, _p(self.gview("W4")), st))
        part = self._buf("part_w", (splits, H, H), torch.float32)
        cpart = self._buf("part_c", (nblk, H), torch.float32)
        for l in (3, 2, 1, 0):
            kin = K_IN if l == 0 else H
            src = X if l == 0 else h[l - 1]
            # weight gradient dW_l = dz_l^T src (split-K over rows, fixed-order reduction)
            F.check(self.gemm(1, 1, H, kin, rows, _p(dz), H, _p(src), kin, 0, None, None, None,
                                         _p(part), None, kin, splits, st))
            F.check(self.L.esr_reduce_splits(_p(part), splits, H * kin, H * kin, _p(self.gview(f"W{l}")), st))
            F.check(self.L.esr_colsum_bf16(_p(dz), rows, H, rpb, _p(cpart), st))
            F.check(self.L.esr_reduce_splits(_p(cpart), nblk, H, H, _p(self.gview(f"b{l}")), st))
            if l > 0:
                dh_prev = self._buf(f"dh{l - 1}", (rows, H), torch.bfloat16)
                dz_prev = self._buf(f"dz{l - 1}", (rows, H), torch.bfloat16)
                F.check(self.gemm(0, 1, rows, H, H, _p(dz), H, _p(self.view(f"W{l}", True)), H, 2,
                                             None, _p(dh), _p(z[l - 1]), _p(dh_prev), _p(dz_prev), H, 1, st))
                dh, dz = dh_prev, dz_prev

    def loss(self, y, tgt, w, inv_den):
        rows = y.shape[0]
        st = _stream()
        dpred = self._buf("dpred", (rows, N_OUT), torch.float32)
        nb = (rows + 255) // 256
        part = self._buf("lpart", (nb,), torch.float32)
        F.check(self.L.esr_mlp_loss(_p(y), _p(tgt), _p(w), rows, _p(inv_den), _p(dpred), _p(part), st))
        out = self._buf("lsum", (1,), torch.float32)
        F.check(self.L.esr_reduce_splits(_p(part.view(nb, 1)), nb, 1, 1, _p(out), st))
        return out, dpred

    def adamw(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, wd=1e-4):
        self.step_count += 1
        F.check(self.L.esr_adamw(_p(self.p), _p(self.g), _p(self.m), _p(self.v), self.n_params, lr, b1, b2, eps, wd,
                                 self.step_count, _p(self.pb), _stream()))

    def params_numpy(self):
        out = {}
        for name, _ in self.SHAPES:
            out[name] = self.view(name).detach().cpu().numpy().astype(np.float64)
        return out

    def grads_numpy(self):
        return {name: self.gview(name).detach().cpu().numpy().astype(np.float64) for name, _ in self.SHAPES}
