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
    bad = C.c_int32(7)
    F.check(F.lib().esr_idw_status(C.byref(bad)))
    assert bad.value == 0


def test_idw_kernel_refuses_out_of_range_indices():
    """A neighbour index outside [0, n_src) is never dereferenced: its row
    comes out NaN, the other rows are unchanged, and the status flag reports
    it once (reading it clears it)."""
    import torch
    from eulersr_b200 import _ffi as F
    from oracle import euler_oracle as O
    rng = np.random.default_rng(1)
    src = rng.standard_normal((50, 4)).astype(np.float32)
    idx = rng.integers(0, 50, (64, 6)).astype(np.int32)
    idx[5, 2] = 50          # one past the end
    idx[9, 0] = -1          # negative
    dist = rng.uniform(1e-3, 0.5, (64, 6)).astype(np.float32)
    ds, di, dd = (torch.from_numpy(a).cuda() for a in (src, idx, dist))
    out = torch.empty((64, 4), dtype=torch.float32, device="cuda")
    F.check(F.lib().esr_idw_apply(C.c_void_p(ds.data_ptr()), 50, 4, C.c_void_p(di.data_ptr()),
                                  C.c_void_p(dd.data_ptr()), 64, 6, C.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.isnan(got[[5, 9]]).all()
    good = np.setdiff1d(np.arange(64), [5, 9])
    ref = O.idw_predict(src, idx[good], dist[good])
    assert np.max(np.abs(got[good] - ref)) <= 2e-6 * max(1.0, np.abs(ref).max())
    bad = C.c_int32(0)
    F.check(F.lib().esr_idw_status(C.byref(bad)))
    assert bad.value == 1
    F.check(F.lib().esr_idw_status(C.byref(bad)))
    assert bad.value == 0


def test_feature_and_decode_kernels_match_formula():
    """esr_mlp_features builds the 13 inputs of preprocessing/dataset.py:140-176
    (geometry statics, IDW primitives normalised by mu/sig, asinh of the IDW
    pressure gradient over sig_p, normalised Mach and alpha; zero padding) in
    BF16 plus the float32 IDW base; esr_mlp_decode turns normalised primitives
    back into conserved rows with the density/pressure floors."""
    import torch
    from eulersr_b200 import _ffi as F
    rng = np.random.default_rng(5)
    rows, ld = 777, 128
    stat5 = rng.standard_normal((rows, 5)).astype(np.float32)
    prim = (rng.standard_normal((rows, 4)) * [0.3, 0.5, 0.2, 0.4] + [1.0, 2.0, 0.1, 1.0]).astype(np.float32)
    gradp = (rng.standard_normal((rows, 2)) * 5.0).astype(np.float32)
    mu = np.array([1.1, 1.9, 0.05, 0.9], np.float32)
    sig = np.array([0.25, 0.6, 0.3, 0.5], np.float32)
    mach_n, aoa_n = np.float32(0.37), np.float32(-0.6)
    d = {k: torch.from_numpy(v).cuda() for k, v in dict(stat5=stat5, prim=prim, gradp=gradp, mu=mu, sig=sig).items()}
    X = torch.full((rows, ld), 7.0, dtype=torch.bfloat16, device="cuda")
    base = torch.empty((rows, 4), dtype=torch.float32, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())   # noqa: E731
    F.check(F.lib().esr_mlp_features(p(d["stat5"]), p(d["prim"]), p(d["gradp"]), rows, float(mach_n), float(aoa_n),
                                     p(d["mu"]), p(d["sig"]), ld, p(X), p(base), None))
    torch.cuda.synchronize()
    q = (prim - mu) / sig                                  # float32, correctly rounded on both sides
    assert np.array_equal(base.cpu().numpy(), q)
    want = np.zeros((rows, ld), np.float32)
    want[:, :5] = stat5
    want[:, 5:9] = q
    want[:, 9:11] = np.arcsinh(gradp / (sig[3] + np.float32(1e-8)))
    want[:, 11], want[:, 12] = mach_n, aoa_n
    got = X.float().cpu().numpy()
    bf = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(torch.bfloat16).float().numpy()   # noqa: E731
    assert np.array_equal(got[:, :9], bf(want[:, :9]))
    assert np.array_equal(got[:, 11:], bf(want[:, 11:]))
    # asinh may differ from numpy's in the last float32 bit: one BF16 step at most
    assert np.all(np.abs(got[:, 9:11] - bf(want[:, 9:11])) <= np.abs(bf(want[:, 9:11])) * 2.0 ** -7 + 1e-30)
    # decode: rho = max(q0 sig0 + mu0, floor), u, v, p = max(q3 sig3 + mu3, floor) -> conserved float64
    pred = rng.standard_normal((rows, 4)).astype(np.float32)
    pred[:5, 0] = -10.0                                    # density below the floor
    pred[5:10, 3] = -10.0                                  # pressure below the floor
    W = torch.empty((rows, 4), dtype=torch.float64, device="cuda")
    dp = torch.from_numpy(pred).cuda()
    F.check(F.lib().esr_mlp_decode(p(dp), rows, p(d["mu"]), p(d["sig"]), 1.4, 0.05, 0.05, p(W), None))
    torch.cuda.synchronize()
    r = np.maximum(pred[:, 0].astype(np.float64) * sig[0] + mu[0], 0.05)
    u = pred[:, 1].astype(np.float64) * sig[1] + mu[1]
    v = pred[:, 2].astype(np.float64) * sig[2] + mu[2]
    pr = np.maximum(pred[:, 3].astype(np.float64) * sig[3] + mu[3], 0.05)
    ref = np.stack([r, r * u, r * v, pr / 0.4 + 0.5 * r * (u * u + v * v)], 1)
    assert np.allclose(W.cpu().numpy(), ref, rtol=2e-6, atol=1e-6)
    assert np.all(W.cpu().numpy()[:5, 0] == np.float32(0.05))


@pytest.mark.parametrize("ta,tb,epi,M,N,K,splits", [
    (0, 0, 1, 256, 256, 256, 1),     # forward: z = X W^T + b, h = res + relu(z)
    (0, 0, 1, 128, 256, 128, 1),     # input layer (K = 128)
    (0, 1, 2, 256, 128, 256, 1),     # backward dX with the relu mask
    (1, 1, 0, 256, 128, 512, 2),     # weight gradient, split-K partials
    (1, 1, 0, 128, 256, 2048, 4),    # long K: the stage barriers wrap several times
    (0, 0, 0, 256, 256, 192, 1),     # K-blocks = stages
    (0, 1, 0, 128, 256, 64, 1),      # a single K-block
    (0, 0, 2, 128, 128, 320, 1),
])
def test_tcgen05_gemm_matches_mma_sync(ta, tb, epi, M, N, K, splits):
    """The tcgen05 GEMM (operands in swizzled shared memory, accumulators in
    tensor memory) against the mma.sync kernel and a float64 product of the
    same BF16 operands, for every layout/epilogue the MLP uses."""
    import torch
    from eulersr_b200 import _ffi as F
    L = F.lib()
    g = torch.Generator().manual_seed(M + N + K + 7 * epi)
    A = torch.randn((K, M) if ta else (M, K), generator=g).to(torch.bfloat16).cuda()
    B = torch.randn((K, N) if tb else (N, K), generator=g).to(torch.bfloat16).cuda()
    bias = torch.randn(N, generator=g).cuda()
    res = torch.randn(M, N, generator=g).to(torch.bfloat16).cuda()
    aux = torch.randn(M, N, generator=g).to(torch.bfloat16).cuda()
    lda = M if ta else K
    ldb = N if tb else K
    p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None

    def run(fn):
        if epi == 0:
            o0, o1 = torch.zeros(splits, M, N, device="cuda"), None
        else:
            o0, o1 = torch.zeros(M, N, dtype=torch.bfloat16, device="cuda"), torch.zeros(M, N, dtype=torch.bfloat16, device="cuda")
        F.check(fn(ta, tb, M, N, K, p(A), lda, p(B), ldb, epi, p(bias) if epi == 1 else None,
                   p(res) if epi else None, p(aux) if epi == 2 else None, p(o0), p(o1), N, splits, None))
        torch.cuda.synchronize()
        return o0, o1

    t0, t1 = run(L.esr_gemm_bf16)
    r0, r1 = run(L.esr_gemm_bf16_mma_sync)
    flag = C.c_int32(-1)
    F.check(L.esr_gemm_tc_status(C.byref(flag)))
    assert flag.value == 0
    Ad = A.double().cpu()
    Bd = B.double().cpu()
    ref = (Ad.T if ta else Ad) @ (Bd if tb else Bd.T)
    if epi == 0:
        got = t0.double().sum(0).cpu()
        assert _rel(got.numpy(), ref.numpy()) < 1e-5
        assert _rel(got.numpy(), r0.double().sum(0).cpu().numpy()) < 1e-5
    else:
        # BF16 outputs: both paths agree to BF16 rounding
        for a, b in ((t0, r0), (t1, r1)):
            assert _rel(a.float().cpu().numpy(), b.float().cpu().numpy()) < 4e-3
        if epi == 1:
            z = ref + bias.double().cpu()
            assert _rel(t1.double().cpu().numpy(), z.numpy()) < 4e-3
