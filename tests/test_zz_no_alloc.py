"""The allocation-free entry point esr_rel_change_noalloc.

It serves callers that cannot allocate device memory at the moment they need
the stop-rule statistic (their own allocator owns the whole device budget, or
allocation is forbidden after start-up): its partial sums live in a fixed
array inside the library instead of a solver buffer. The result must agree
with the existing esr_residual_probe, which computes the same quantity
||step(W) - W|| / (||W|| + 1e-16) with the solver's own reduction, on two
calls in a row. This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12   # both sum float32 data in float64; only the summation order differs


def test_rel_change_noalloc_matches_probe(diamond02):
    import torch
    from eulersr_b200 import _ffi as F
    from eulersr_b200.solver import Solver, FlowCase
    L = F.lib()
    N = diamond02.n_cells
    case = FlowCase(mach=2.5, aoa_deg=5.0, cfl=0.6, tf=100.0, dtype=np.float32)
    a = Solver(diamond02, 1, precision='f32')
    b = Solver(diamond02, 1, precision='f32')
    a.set_case(0, case)
    b.set_case(0, case)
    W = torch.empty((N, 4), dtype=torch.float32, device='cuda')
    W_next = torch.empty_like(W)
    out = torch.zeros(1, dtype=torch.float64, device='cuda')
    for call in range(2):
        probe = float(a.residual_probe()[0])          # existing entry point
        a.get_state_device(0, W.data_ptr())
        b.step(1)                                     # b holds step(W)
        b.get_state_device(0, W_next.data_ptr())
        a.synchronize()
        b.synchronize()
        F.check(L.esr_rel_change_noalloc(C.c_void_p(W_next.data_ptr()), C.c_void_p(W.data_ptr()), N, 0,
                                         C.c_void_p(out.data_ptr()), None))
        torch.cuda.synchronize()
        got = float(out.item())
        assert probe > 0
        assert abs(got - probe) <= TOL * probe, (call, got, probe)
        a.step(1)                                     # both now at the same next state
    a.close()
    b.close()


def test_rel_change_noalloc_rejects_oversize():
    import torch
    from eulersr_b200 import _ffi as F
    L = F.lib()
    buf = torch.zeros((8, 4), dtype=torch.float32, device='cuda')
    out = torch.zeros(1, dtype=torch.float64, device='cuda')
    rc = L.esr_rel_change_noalloc(C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()), 2 ** 21 + 1, 0,
                                  C.c_void_p(out.data_ptr()), None)
    assert rc == F.ESR_ERR_ARG
    assert b"exceeds the maximum" in L.esr_last_error()


def test_rel_change_noalloc_rejects_host_and_misaligned_pointers():
    """Addresses its kernels could not read are refused before any launch:
    plain and pinned host memory, and device rows or an output that are not
    aligned for the vector loads and the double store."""
    import torch
    from eulersr_b200 import _ffi as F
    L = F.lib()
    dev = torch.zeros((64, 4), dtype=torch.float32, device='cuda')
    out = torch.zeros(4, dtype=torch.float64, device='cuda')
    host = np.zeros((64, 4), dtype=np.float32)
    pinned = torch.zeros((64, 4), dtype=torch.float32, pin_memory=True)
    vp = lambda a: C.c_void_p(a)
    cases = [
        (host.ctypes.data, dev.data_ptr(), out.data_ptr(), b"d_A"),
        (dev.data_ptr(), pinned.data_ptr(), out.data_ptr(), b"d_B"),
        (dev.data_ptr(), dev.data_ptr(), host.ctypes.data, b"d_out"),
        (dev.data_ptr() + 4, dev.data_ptr(), out.data_ptr(), b"aligned"),
        (dev.data_ptr(), dev.data_ptr(), out.data_ptr() + 4, b"aligned"),
    ]
    for a, b, o, what in cases:
        rc = L.esr_rel_change_noalloc(vp(a), vp(b), 16, 0, vp(o), None)
        assert rc == F.ESR_ERR_ARG, (what, rc)
        assert what in L.esr_last_error(), L.esr_last_error()
    torch.cuda.synchronize()
    assert float(out.abs().sum().item()) == 0.0      # nothing was launched


def test_rel_change_noalloc_at_its_maximum_size():
    """At the largest accepted size (2,097,152 rows, every block of the fixed
    array in use) the float64 and float32 forms agree with the same statistic
    computed by torch in float64, on two calls in a row."""
    import torch
    from eulersr_b200 import _ffi as F
    L = F.lib()
    n = 2 ** 21
    g = torch.Generator(device='cuda').manual_seed(11)
    out = torch.zeros(1, dtype=torch.float64, device='cuda')
    for prec, dt in ((1, torch.float64), (0, torch.float32)):
        A = torch.rand((n, 4), generator=g, device='cuda', dtype=torch.float64).to(dt)
        B = torch.rand((n, 4), generator=g, device='cuda', dtype=torch.float64).to(dt)
        want = float(torch.linalg.norm((A.double() - B.double()).flatten()) /
                     (torch.linalg.norm(B.double().flatten()) + 1e-16))
        for call in range(2):
            F.check(L.esr_rel_change_noalloc(C.c_void_p(A.data_ptr()), C.c_void_p(B.data_ptr()), n, prec,
                                             C.c_void_p(out.data_ptr()), None))
            torch.cuda.synchronize()
            assert abs(float(out.item()) - want) <= TOL * want, (prec, call)
