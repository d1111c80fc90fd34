"""fmm_evaluate_noalloc: FMM evaluation that allocates no device memory.

Some callers cannot allocate device memory when they evaluate: an
application that has already reserved the whole GPU for its own memory pool
(so cudaMalloc would fail), or a time-critical loop that must not enter the
allocator.  For them the library offers fmm_evaluate_noalloc, which runs the
same evaluation as fmm_evaluate with its scratch in a static array inside the
library.  This file checks, through the C ABI, that it returns what
fmm_evaluate returns on two calls in a row (the second with different,
fewer targets, so stale scratch from the first call would show), for target
and source evaluation, and that oversized requests are refused.  It is named
to run last, after every other test.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12   # the parity tolerance used by the other GPU tests


def _eval(lib, fn, plan, tx, ty, check):
    import torch
    out = torch.full_like(tx, float("nan"))
    rc = getattr(lib, fn)(plan, ctypes.c_void_p(tx.data_ptr()), ctypes.c_void_p(ty.data_ptr()),
                          tx.numel(), check, ctypes.c_void_p(out.data_ptr()),
                          ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, lib.fmm_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_matches_fmm_evaluate_twice(built_lib):
    import torch
    from flexmm_b200 import KI_FMM, KI_Helper, _lib, workloads
    lib = _lib.load()
    d = workloads.clustered(n=100_000, n_grid=10, seed=31)
    F = KI_FMM(d["x"], d["y"], "Laplace_Eval", 64, 32, bbox=d["bbox"], helper=KI_Helper())
    F.build_expansions(d["tau"])
    rng = np.random.default_rng(7)
    calls = [(rng.uniform(-1, 1, 60_000), rng.uniform(-1, 1, 60_000), 0),
             (rng.uniform(-1, 1, 25_000), rng.uniform(-1, 1, 25_000), 0),
             (d["x"][:40_000], d["y"][:40_000], 1)]
    for tx, ty, check in calls:
        txd = torch.from_numpy(tx).cuda()
        tyd = torch.from_numpy(ty).cuda()
        want = _eval(lib, "fmm_evaluate", F._plan, txd, tyd, check)
        got = _eval(lib, "fmm_evaluate_noalloc", F._plan, txd, tyd, check)
        assert np.isfinite(got).all()
        assert rel_l2(got, want) < TOL


def test_noalloc_modified_helmholtz_and_refused_forms(built_lib):
    """Every FP64 KIFMM kernel goes through the allocation-free route (here
    the modified Helmholtz kernel, two calls in a row); a mixed-precision plan
    is refused before any work, with status 5 (unsupported)."""
    import torch
    from flexmm_b200 import KI_FMM, KI_Helper, _lib, workloads
    lib = _lib.load()
    d = workloads.uniform(n=30_000, n_grid=10, seed=33)
    F = KI_FMM(d["x"], d["y"], "Modified_Helmholtz_Eval", 64, 24, bbox=d["bbox"],
               helper=KI_Helper(), helmholtz_k=5.0)
    F.build_expansions(d["tau"])
    rng = np.random.default_rng(8)
    for n in (20_000, 7_000):
        txd = torch.from_numpy(rng.uniform(-1, 1, n)).cuda()
        tyd = torch.from_numpy(rng.uniform(-1, 1, n)).cuda()
        want = _eval(lib, "fmm_evaluate", F._plan, txd, tyd, 0)
        got = _eval(lib, "fmm_evaluate_noalloc", F._plan, txd, tyd, 0)
        assert np.isfinite(got).all()
        assert rel_l2(got, want) < TOL
    M = KI_FMM(d["x"], d["y"], "Laplace_Eval", 64, 24, bbox=d["bbox"], helper=KI_Helper(),
               precision="mixed")
    M.build_expansions(d["tau"])
    t = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = lib.fmm_evaluate_noalloc(M._plan, ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(t.data_ptr()),
                                  4, 0, ctypes.c_void_p(t.data_ptr()), None)
    assert rc == 5 and b"FP64" in lib.fmm_last_error()


def test_noalloc_refuses_oversized_requests(built_lib):
    import torch
    from flexmm_b200 import KI_FMM, KI_Helper, _lib, workloads
    lib = _lib.load()
    d = workloads.uniform(n=5000, n_grid=10, seed=32)
    F = KI_FMM(d["x"], d["y"], "Laplace_Eval", 32, 16, bbox=d["bbox"], helper=KI_Helper())
    F.build_expansions(d["tau"])
    t = torch.zeros(4, dtype=torch.float64, device="cuda")
    too_many = 262144 + 1   # FMM_NOALLOC_MAX_TARGETS + 1: refused before any work
    rc = lib.fmm_evaluate_noalloc(F._plan, ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(t.data_ptr()),
                                  too_many, 0, ctypes.c_void_p(t.data_ptr()), None)
    assert rc == 6 and b"FMM_NOALLOC_MAX_TARGETS" in lib.fmm_last_error()
