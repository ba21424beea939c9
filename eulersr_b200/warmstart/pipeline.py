"""Learned warm start end to end: IDW of the LR solution plus a residual MLP.

1. cases: (Mach ~ U[0.7, 3], alpha ~ U[-5, 5] deg) from default_rng(seed);
   the first n_train draws train, the next n_eval draws are held out;
2. data: every case is solved on the LR and HR meshes by the batched solver
   (retire/refill); the LR solution and its LSQ pressure gradient are
   interpolated to the HR cells by IDW (k=6, p=2) on the GPU;
3. model: the residual MLP predicts the normalised HR primitives as IDW +
   correction; loss = shock-weighted relative MSE with weights
   min(1 + |grad p_HR| / mean|grad p_HR|, 5) (preprocessing/dataset.py:168-170,
   loss.py:20-23); trained by the library's BF16 kernels with AdamW;
4. evaluation (eval/convergence_case.py:30-142, driven by ``run.py``): for
   each held-out case the HR FVM runs from freestream (cold), from IDW and
   from IDW+MLP to the same stop rule; reported: iterations, wall time of the
   whole pipeline (LR solve + inference + warm HR solve) and the CD error
   against a long reference solve.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass

import numpy as np
import torch

from .. import _ffi as F
from ..solver import FlowCase, Solver
from .features import AOA_SCALE, MACH_MID, MACH_SCALE, MeshPair
from .mlp import K_IN, MLP, ROW_TILE


def draw_cases(n_train, n_eval, seed=3):
    rng = np.random.default_rng(seed)
    mach = rng.uniform(0.7, 3.0, n_train + n_eval)
    aoa = rng.uniform(-5.0, 5.0, n_train + n_eval)
    return (mach[:n_train], aoa[:n_train]), (mach[n_train:], aoa[n_train:])


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


def pressure_gradients(mesh, dm, states, machs, aoas, device=0):
    """LSQ pressure gradient of each state, from the library's gradient kernel."""
    s = Solver(dm, 1, precision="f64", device=device)
    out = []
    for W, m, a in zip(states, machs, aoas):
        s.set_case(0, FlowCase(mach=float(m), aoa_deg=float(a), tf=1.0), W_init=W)
        out.append(s.gradients(0)[:, 3, :].astype(np.float32))
    s.close()
    return out


def primitives(W, gamma=1.4):
    rho = W[:, 0]
    u, v = W[:, 1] / rho, W[:, 2] / rho
    p = (W[:, 3] - 0.5 * rho * (u * u + v * v)) * (gamma - 1)
    return np.stack([rho, u, v, p], -1)


class WarmStart:
    """IDW (+ MLP) prediction of an HR initial field from an LR solution."""

    def __init__(self, pair: MeshPair, mu=None, sig=None, mlp: MLP | None = None, device="cuda"):
        if torch.device(device).type != "cuda":
            raise ValueError(f"the warm start runs on the library's CUDA kernels; device must be a CUDA device, not {device!r}")
        self.pair = pair
        self.L = F.lib()
        self.device = device
        self.mlp = mlp
        self.mu = torch.tensor(mu if mu is not None else [1.0, 1.0, 0.0, 1.0], dtype=torch.float32, device=device)
        self.sig = torch.tensor(sig if sig is not None else [1.0, 1.0, 1.0, 1.0], dtype=torch.float32, device=device)
        self.n_hr = pair.hr.n_cells
        self.rows = ((self.n_hr + ROW_TILE - 1) // ROW_TILE) * ROW_TILE
        self.launches = 0          # library kernels launched by inputs() and predict_state()
        self.idx = torch.from_numpy(pair.knn_idx).to(device)
        self.dist = torch.from_numpy(pair.knn_dist).to(device)
        self.stat = torch.from_numpy(pair.static5).to(device)

    def inputs(self, lr_prim, lr_gradp, mach, aoa):
        """Feature rows X (BF16, rows padded) and the normalised IDW base for one case."""
        st = _stream()
        n_lr = lr_prim.shape[0]
        lp = torch.as_tensor(lr_prim, dtype=torch.float32, device=self.device).contiguous()
        lg = torch.as_tensor(lr_gradp, dtype=torch.float32, device=self.device).contiguous()
        idw = torch.empty((self.n_hr, 4), dtype=torch.float32, device=self.device)
        idg = torch.empty((self.n_hr, 2), dtype=torch.float32, device=self.device)
        F.check(self.L.esr_idw_apply(_p(lp), n_lr, 4, _p(self.idx), _p(self.dist), self.n_hr, 6, _p(idw), st))
        F.check(self.L.esr_idw_apply(_p(lg), n_lr, 2, _p(self.idx), _p(self.dist), self.n_hr, 6, _p(idg), st))
        X = torch.zeros((self.rows, K_IN), dtype=torch.bfloat16, device=self.device)
        base = torch.zeros((self.rows, 4), dtype=torch.float32, device=self.device)
        F.check(self.L.esr_mlp_features(_p(self.stat), _p(idw), _p(idg), self.n_hr, (mach - MACH_MID) / MACH_SCALE,
                                        aoa / AOA_SCALE, _p(self.mu), _p(self.sig), K_IN, _p(X), _p(base), st))
        self.launches += 3
        return X, base

    def predict_state(self, lr_prim, lr_gradp, mach, aoa, use_mlp=True, gamma=1.4):
        """Conserved HR initial field (float64, HR cell order)."""
        X, base = self.inputs(lr_prim, lr_gradp, mach, aoa)
        pred = self.mlp.forward(X, base) if (use_mlp and self.mlp is not None) else base
        W = torch.empty((self.n_hr, 4), dtype=torch.float64, device=self.device)
        F.check(self.L.esr_mlp_decode(_p(pred), self.n_hr, _p(self.mu), _p(self.sig), gamma, 0.05, 0.05, _p(W),
                                      _stream()))
        self.launches += 1
        return W.cpu().numpy()


@dataclass
class TrainData:
    X: torch.Tensor
    base: torch.Tensor
    tgt: torch.Tensor
    w: torch.Tensor
    inv_den: torch.Tensor


def loss_weights(hr_gradp, factor=1.0):
    """Shock weights of one case's rows (preprocessing/dataset.py:168-170,
    shock_weight_factor 1 by default): min(1 + factor |grad p| / mean |grad p|, 5)."""
    gp = np.sqrt((np.asarray(hr_gradp) ** 2).sum(-1))
    return np.minimum(1.0 + factor * gp / (gp.mean() + 1e-8), 5.0).astype(np.float32)


def build_training_set(ws: WarmStart, lr_states, lr_gradp, hr_states, hr_gradp, machs, aoas, gamma=1.4):
    """Stack every training case's rows on the GPU; sets ws.mu/ws.sig from the HR targets."""
    hr_prims = [primitives(W, gamma).astype(np.float32) for W in hr_states]
    allp = np.concatenate(hr_prims)
    mu = allp.mean(0)
    sig = allp.std(0) + 1e-6
    ws.mu = torch.tensor(mu, device=ws.device)
    ws.sig = torch.tensor(sig, device=ws.device)
    Xs, bs, ts, wts = [], [], [], []
    n = ws.n_hr
    for i in range(len(hr_states)):
        X, base = ws.inputs(primitives(lr_states[i], gamma).astype(np.float32), lr_gradp[i], machs[i], aoas[i])
        Xs.append(X[:n])
        bs.append(base[:n])
        t = (hr_prims[i] - mu) / sig
        ts.append(torch.from_numpy(t.astype(np.float32)).to(ws.device))
        wts.append(torch.from_numpy(loss_weights(hr_gradp[i])).to(ws.device))
    tgt = torch.cat(ts)
    inv_den = (1.0 / ((tgt.double() ** 2).mean(0) + 1e-8)).float()
    return TrainData(torch.cat(Xs), torch.cat(bs), tgt, torch.cat(wts), inv_den.contiguous()), mu, sig


def train(mlp: MLP, data: TrainData, steps=1500, batch=32768, lr=2e-3, seed=0, log_every=250, world=1, rank=0):
    """AdamW on shock-weighted relative MSE. With ``world`` > 1 (one process
    per GPU, torch.distributed initialised) each rank draws batch/world rows
    of its own and the gradients are averaged over ranks before the step."""
    from ..parallel import allreduce_mean_, rank_batch
    local = rank_batch(batch, world, rank)
    g = torch.Generator(device=data.X.device).manual_seed(seed * 1009 + rank)
    R = data.X.shape[0]
    hist = []
    t0 = time.perf_counter()
    for it in range(steps):
        idx = torch.randint(0, R, (local,), generator=g, device=data.X.device)
        X, base, tgt, w = data.X[idx], data.base[idx], data.tgt[idx], data.w[idx]
        y, acts = mlp.forward(X, base, keep=True)
        L, dpred = mlp.loss(y, tgt, w, data.inv_den)
        mlp.backward(acts, dpred)
        allreduce_mean_(mlp.g, world)
        cur = lr * 0.5 * (1 + math.cos(math.pi * it / steps))
        mlp.adamw(lr=cur, wd=1e-5)
        if it % log_every == 0 or it == steps - 1:
            hist.append((it, float(L.item())))
    torch.cuda.synchronize()
    return hist, time.perf_counter() - t0


def eval_loss(mlp: MLP | None, data: TrainData, batch=32768):
    """Weighted relative MSE of IDW (mlp None) or IDW+MLP over a dataset."""
    R = data.X.shape[0]
    tot = 0.0
    for s in range(0, R - R % ROW_TILE, batch):
        e = min(R - R % ROW_TILE, s + batch)
        y = mlp.forward(data.X[s:e], data.base[s:e]) if mlp is not None else data.base[s:e]
        d = (y - data.tgt[s:e]) ** 2 * data.w[s:e, None] * data.inv_den[None, :]
        tot += float(d.sum().item())
    return tot / (4 * (R - R % ROW_TILE))
