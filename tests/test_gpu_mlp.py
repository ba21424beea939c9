"""BF16 MLP kernels against the CPU oracle (oracle/mlp_oracle.py): forward,
loss gradient and every parameter gradient; a training smoke test; the IDW
kernel against eval/core.py's formula."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(rows=512, seed=0):
    import torch
    from eulersr_b200.warmstart.mlp import MLP, K_IN
    m = MLP(seed=seed)
    g = torch.Generator().manual_seed(seed + 1)
    # non-zero head so gradients reach every layer
    m.view("W4").copy_((torch.randn(4, 256, generator=g) * 0.05).cuda())
    m.view("b4").copy_((torch.randn(4, generator=g) * 0.1).cuda())
    m.pb.copy_(m.p.to(torch.bfloat16))
    X = torch.zeros(rows, K_IN)
    X[:, :13] = torch.randn(rows, 13, generator=g)
    X = X.to(torch.bfloat16).cuda()
    base = (torch.randn(rows, 4, generator=g) * 0.5).cuda()
    tgt = (torch.randn(rows, 4, generator=g) * 0.5).cuda()
    w = (1 + torch.rand(rows, generator=g) * 4).cuda()
    inv_den = torch.tensor([1.3, 0.7, 2.0, 1.1]).cuda()
    return m, X, base, tgt, w, inv_den


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_forward_backward_match_oracle():
    import torch
    from oracle import mlp_oracle as MO
    m, X, base, tgt, w, inv_den = _setup()
    y, acts = m.forward(X, base, keep=True)
    L, dpred = m.loss(y, tgt, w, inv_den)
    m.backward(acts, dpred)
    torch.cuda.synchronize()
    P = m.params_numpy()
    Xn = X.float().cpu().numpy()
    yo, ao = MO.forward(P, Xn, base.cpu().numpy())
    assert _rel(y.cpu().numpy(), yo) < 1e-3
    Lo, dyo = MO.loss_and_grad(yo, tgt.cpu().numpy(), w.cpu().numpy(), inv_den.cpu().numpy())
    assert abs(float(L.item()) - Lo) <= 1e-3 * Lo
    go = MO.backward(P, ao, dpred.cpu().numpy().astype(np.float64))
    gg = m.grads_numpy()
    for k in ("W4", "b4", "W3", "b3", "W2", "b2", "W1", "b1", "W0", "b0"):
        assert _rel(gg[k], go[k]) < 2e-2, (k, _rel(gg[k], go[k]))
    # the BF16 gradients also track exact float64 backpropagation
    y64, a64 = MO.forward(P, Xn, base.cpu().numpy(), bf16=False)
    _, dy64 = MO.loss_and_grad(y64, tgt.cpu().numpy(), w.cpu().numpy(), inv_den.cpu().numpy())
    g64 = MO.backward(P, a64, dy64, bf16=False)
    for k in ("W3", "W1", "W0"):
        assert _rel(gg[k], g64[k]) < 6e-2, (k, _rel(gg[k], g64[k]))


def test_training_reduces_loss():
    import torch
    m, X, base, tgt, w, inv_den = _setup(rows=2048, seed=3)
    # a learnable target: a smooth function of the inputs
    Xf = X.float()
    tgt = torch.stack([torch.tanh(Xf[:, 0] + 0.5 * Xf[:, 1]), Xf[:, 2] * 0.3, torch.sin(Xf[:, 3]),
                       0.2 * Xf[:, 4] ** 2], 1).contiguous()
    base = torch.zeros_like(tgt)
    losses = []
    for it in range(300):
        y, acts = m.forward(X, base, keep=True)
        L, dpred = m.loss(y, tgt, w, inv_den)
        m.backward(acts, dpred)
        m.adamw(lr=2e-3)
        losses.append(float(L.item()))
    assert losses[-1] < 0.2 * losses[0], (losses[0], losses[-1])


def test_idw_kernel_matches_formula():
    import torch
    from eulersr_b200 import _ffi as F
    from oracle import euler_oracle as O
    rng = np.random.default_rng(0)
    src = rng.standard_normal((300, 4)).astype(np.float32)
    idx = rng.integers(0, 300, (1000, 6)).astype(np.int32)
    dist = rng.uniform(1e-3, 0.5, (1000, 6)).astype(np.float32)
    ds, di, dd = (torch.from_numpy(a).cuda() for a in (src, idx, dist))
    out = torch.empty((1000, 4), dtype=torch.float32, device="cuda")
    F.check(F.lib().esr_idw_apply(C.c_void_p(ds.data_ptr()), 300, 4, C.c_void_p(di.data_ptr()),
                                  C.c_void_p(dd.data_ptr()), 1000, 6, C.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    ref = O.idw_predict(src, idx, dist)
    assert np.max(np.abs(out.cpu().numpy() - ref)) <= 2e-6 * max(1.0, np.abs(ref).max())
