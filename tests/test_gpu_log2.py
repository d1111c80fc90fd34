"""The FP64 passes' table-driven log2 (Laplace kernel) against CUDA's log2.

Bar: absolute error at most 2 ulp of max(1, |log2 x|) -- the Laplace kernel
-log(d^2)/(4 pi) sums these values times charges, so an absolute bound is
what reaches the potential -- over normal arguments spanning the whole
exponent range, values next to every table point, powers of two, and the
special arguments (0, subnormal, inf) that take the library path.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(x):
    import torch
    from flexmm_b200 import _lib
    lib = _lib.load()
    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()
    a, b = torch.empty_like(xd), torch.empty_like(xd)
    rc = lib.fmm_diag_log2(ctypes.c_void_p(xd.data_ptr()), xd.numel(), ctypes.c_void_p(a.data_ptr()),
                           ctypes.c_void_p(b.data_ptr()), None)
    assert rc == 0, lib.fmm_last_error()
    torch.cuda.synchronize()
    return a.cpu().numpy(), b.cpu().numpy()


def test_table_log2_matches_library_log2(built_lib):
    rng = np.random.default_rng(5)
    wide = np.exp2(rng.uniform(-1020, 1020, 400_000))
    near_one = 1.0 + rng.uniform(-2 ** -6, 2 ** -6, 200_000)
    # next to every table point 1 + j/256 and the midpoints between them
    j = np.arange(0, 257)
    pts = np.concatenate([1 + j / 256.0, 1 + (j[:-1] + 0.5) / 256.0])
    around = np.concatenate([np.nextafter(pts, 0), pts, np.nextafter(pts, 3)])
    around = np.concatenate([around * s for s in (1.0, 2.0 ** -30, 2.0 ** 17, 0.5)])
    pow2 = np.exp2(np.arange(-1022, 1023, dtype=np.float64))
    x = np.concatenate([wide, near_one, around, pow2])
    got, lib = _run(x)
    scale = np.maximum(1.0, np.abs(lib))
    err = np.abs(got - lib) / (np.spacing(scale))
    assert err.max() <= 2.0, (err.max(), x[np.argmax(err)])
    # powers of two are exact
    got_p, _ = _run(pow2)
    assert np.array_equal(got_p, np.arange(-1022, 1023, dtype=np.float64))


def test_table_log2_special_arguments(built_lib):
    x = np.array([0.0, 5e-324, 2.5e-310, np.inf, 1.0, 2.0])
    got, lib = _run(x)
    assert got[0] == -np.inf and got[3] == np.inf
    assert np.allclose(got[1:3], lib[1:3], rtol=1e-15, atol=0)
    assert got[4] == 0.0 and got[5] == 1.0
