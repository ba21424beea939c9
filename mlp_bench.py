"""Throughput of the warm-start MLP kernels on the GPU.

    python mlp_bench.py [--rows 32768] [--reps 20]

Times, with CUDA events on the current stream after warm-up, for the tcgen05
GEMM and the mma.sync GEMM it replaced: one 256-wide forward layer
(rows x 256 x 256 with the bias/ReLU/residual epilogue), the weight-gradient
GEMM (256 x 256 x rows, split-K), a full training step (forward, loss,
backward, AdamW) and the inference of one HR case (25,968 cells padded to
128). TFLOP/s count 2 M N K per GEMM; the peak is the measured dense BF16
GEMM rate of the GPU when MEASURED_PEAKS.json is present.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import sys
from pathlib import Path

import torch

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from eulersr_b200 import _ffi as F  # noqa: E402
from eulersr_b200.warmstart.mlp import H, K_IN, MLP  # noqa: E402


def _time(fn, reps):
    for _ in range(3):
        fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=32768)
    ap.add_argument("--reps", type=int, default=20)
    a = ap.parse_args(argv)
    L = F.lib()
    rows = a.rows
    g = torch.Generator().manual_seed(0)
    X = torch.randn(rows, H, generator=g).to(torch.bfloat16).cuda()
    W = (torch.randn(H, H, generator=g) * 0.06).to(torch.bfloat16).cuda()
    bias = torch.zeros(H).cuda()
    h = torch.empty(rows, H, dtype=torch.bfloat16, device="cuda")
    z = torch.empty_like(h)
    splits = 32
    part = torch.empty(splits, H, H, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    peak = None
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peak = float(json.loads(pk.read_text())["bf16_tflops"])
    out = {"rows": rows, "peak_bf16_tflops": peak}
    for name, fn in (("tcgen05", L.esr_gemm_bf16), ("mma_sync", L.esr_gemm_bf16_mma_sync)):
        fwd = lambda: F.check(fn(0, 0, rows, H, H, p(X), H, p(W), H, 1, p(bias), p(X), None, p(h), p(z), H, 1, st))
        dw = lambda: F.check(fn(1, 1, H, H, rows, p(X), H, p(X), H, 0, None, None, None, p(part), None, H, splits, st))
        t_fwd, t_dw = _time(fwd, a.reps), _time(dw, a.reps)
        flops = 2.0 * rows * H * H
        m = MLP(seed=0, gemm=name)
        Xi = torch.zeros(rows, K_IN, dtype=torch.bfloat16, device="cuda")
        Xi[:, :13] = torch.randn(rows, 13, generator=g).to(torch.bfloat16).cuda()
        base = torch.zeros(rows, 4, device="cuda")
        tgt = torch.randn(rows, 4, generator=g).cuda()
        w = torch.ones(rows, device="cuda")
        inv = torch.ones(4, device="cuda")

        def train_step():
            y, acts = m.forward(Xi, base, keep=True)
            _, dpred = m.loss(y, tgt, w, inv)
            m.backward(acts, dpred)
            m.adamw()
        n_inf = 26112
        Xc = Xi[:n_inf].contiguous()
        bc = base[:n_inf].contiguous()
        t_train = _time(train_step, a.reps)
        t_inf = _time(lambda: m.forward(Xc, bc), a.reps)
        out[name] = {"fwd_layer_ms": t_fwd, "fwd_layer_tflops": flops / t_fwd / 1e9,
                     "wgrad_ms": t_dw, "wgrad_tflops": flops / t_dw / 1e9,
                     "train_step_ms": t_train, "infer_case_ms": t_inf}
        if peak:
            out[name]["fwd_layer_frac"] = flops / t_fwd / 1e9 / peak
    ok = C.c_int32(-1)
    F.check(L.esr_gemm_tc_status(C.byref(ok)))
    out["tcgen05_waits_gave_up"] = int(ok.value)
    print(json.dumps(out))
    return out


if __name__ == "__main__":
    main()
