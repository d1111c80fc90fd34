"""Gradient evaluator (potential + gradient in the target position).

The fixtures come from the reference's own gradient path: kifmm2d FMM with
the evaluator pair of examples/pure_kifmm_laplace_gradient.py registered as
'gradient' (3 outputs) and evaluate_to_points.  CPU tests pin the direct-sum
oracle against those reference outputs; GPU tests hold the FP64 form to the
reference (1e-12 relative L2 per output row) and the mixed form to the FP64
form at the same Nequiv.
"""
import numpy as np
import pytest

from conftest import golden_cases, golden_inputs, kernel_of, load_golden, rel_l2

GRAD_CASES = golden_cases(gradient=True)
PARITY = 1e-12


def _direct_grad(meta, *args):
    from oracle.direct import direct_laplace_grad, direct_mod_helmholtz_grad
    if meta.get("kernel", "laplace") == "laplace":
        return direct_laplace_grad(*args)
    sx, sy, tau, tx, ty, check = args
    return direct_mod_helmholtz_grad(sx, sy, tau, tx, ty, meta["k"], check)


@pytest.mark.parametrize("case", GRAD_CASES)
def test_direct_gradient_oracle_agrees_with_reference_fmm(case):
    """The stored direct sums regenerate (first 500 points), and the reference
    FMM's gradients agree with them to its own truncation error (Nequiv 16:
    ~1e-4; 24-32: <=1e-5)."""
    g = load_golden(case)
    meta = g["meta"]
    d = golden_inputs(meta)
    ds = _direct_grad(meta, d["x"], d["y"], d["tau"], d["x"][:500], d["y"][:500], True)
    np.testing.assert_allclose(ds, g["direct_src"][:, :500], rtol=1e-12, atol=1e-12)
    bar = 3e-4 if meta["neq"] <= 16 else 3e-5
    for r in range(3):
        assert rel_l2(g["src_val"][r], g["direct_src"][r]) < bar
        assert rel_l2(g["tgt_val"][r], g["direct_tgt"][r]) < bar


def test_oracle_gradient_matches_finite_differences():
    """The oracle's gradient is the derivative of its potential (central
    differences, h = 1e-6 on targets away from the sources)."""
    from oracle.direct import direct_laplace, direct_laplace_grad
    rng = np.random.default_rng(3)
    sx, sy, tau = rng.uniform(-1, 1, 300), rng.uniform(-1, 1, 300), rng.standard_normal(300)
    tx, ty = rng.uniform(1.5, 2.0, 20), rng.uniform(1.5, 2.0, 20)
    g = direct_laplace_grad(sx, sy, tau, tx, ty, False)
    h = 1e-6
    fx = (direct_laplace(sx, sy, tau, tx + h, ty, False) - direct_laplace(sx, sy, tau, tx - h, ty, False)) / (2 * h)
    fy = (direct_laplace(sx, sy, tau, tx, ty + h, False) - direct_laplace(sx, sy, tau, tx, ty - h, False)) / (2 * h)
    np.testing.assert_allclose(g[0], direct_laplace(sx, sy, tau, tx, ty, False), rtol=1e-14)
    np.testing.assert_allclose(g[1], fx, rtol=1e-6, atol=1e-8)
    np.testing.assert_allclose(g[2], fy, rtol=1e-6, atol=1e-8)


def _fmm(d, meta, precision="fp64", x=None, y=None):
    from flexmm_b200 import KI_FMM, KI_Helper
    name, params = kernel_of(meta)
    F = KI_FMM(d["x"] if x is None else x, d["y"] if y is None else y, name, meta["ncut"],
               meta["neq"], bbox=d["bbox"], helper=KI_Helper(), precision=precision, **params)
    F.register_evaluator(None, None, "gradient", 3)
    return F


@pytest.mark.gpu
@pytest.mark.parametrize("case", GRAD_CASES)
def test_gradient_matches_reference(built_lib, case):
    g = load_golden(case)
    meta = g["meta"]
    d = golden_inputs(meta)
    F = _fmm(d, meta)
    assert np.array_equal(np.array(F.bbox), g["bbox_used"])
    F.build_expansions(d["tau"])
    us = F.evaluate_to_points(d["x"], d["y"], "gradient", True)
    ut = F.evaluate_to_points(d["tx"], d["ty"], "gradient", False)
    F.status()
    assert us.shape == (3, d["x"].size) and ut.shape == (3, d["tx"].size)
    for r in range(3):
        es, et = rel_l2(us[r], g["src_val"][r]), rel_l2(ut[r], g["tgt_val"][r])
        assert es < PARITY and et < PARITY, (r, es, et)
    # the potential row equals the plain evaluation
    np.testing.assert_allclose(us[0], F.source_evaluation(d["x"], d["y"]), rtol=1e-13, atol=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gradient_on_own_sources_equals_general_path(built_lib, precision):
    """Own torch source tensors take fmm_evaluate_sources_outputs (the tree's
    sorted copy); copies take fmm_evaluate_outputs."""
    import torch
    g = load_golden("grad_clustered_20k_q32")
    meta = g["meta"]
    d = golden_inputs(meta)
    x, y = torch.from_numpy(d["x"]).cuda(), torch.from_numpy(d["y"]).cuda()
    F = _fmm(d, meta, precision, x, y)
    F.build_expansions(torch.from_numpy(d["tau"]).cuda())
    a = F.evaluate_to_points(x, y, "gradient", True).cpu().numpy()
    b = F.evaluate_to_points(x.clone(), y.clone(), "gradient", True).cpu().numpy()
    F.status()
    # mixed: the own-source sweep's FP32 partial sums leave each target's own
    # point out instead of zeroing it in place (a different FP32 order)
    for r in range(3):
        assert rel_l2(a[r], b[r]) < (1e-14 if precision == "fp64" else 1e-7)
    if precision == "fp64":
        for r in range(3):
            assert rel_l2(a[r], g["src_val"][r]) < PARITY


@pytest.mark.gpu
@pytest.mark.parametrize("case", [c for c in GRAD_CASES if "_mh_" not in c])
def test_mixed_gradient_against_fp64_form(built_lib, case):
    """Mixed form vs FP64 form at the same Nequiv: the arithmetic difference
    only (the FMM truncation error is common to both), <= 1e-6 per row,
    coincident sources (duplicates case) skipped exactly."""
    g = load_golden(case)
    meta = g["meta"]
    d = golden_inputs(meta)
    res = {}
    for precision in ("fp64", "mixed"):
        F = _fmm(d, meta, precision)
        F.build_expansions(d["tau"])
        res[precision] = (F.evaluate_to_points(d["x"], d["y"], "gradient", True),
                          F.evaluate_to_points(d["tx"], d["ty"], "gradient", False))
        F.status()
    for k in range(2):
        for r in range(3):
            e = rel_l2(res["mixed"][k][r], res["fp64"][k][r])
            assert np.all(np.isfinite(res["mixed"][k][r])) and e < 1e-6, (k, r, e)


@pytest.mark.gpu
def test_unknown_evaluator_and_bad_leading_dimension(built_lib):
    import ctypes
    from flexmm_b200 import _lib
    g = load_golden("grad_uniform_3k_q16")
    d = golden_inputs(g["meta"])
    F = _fmm(d, g["meta"])
    F.build_expansions(d["tau"])
    with pytest.raises(KeyError):
        F.evaluate_to_points(d["x"], d["y"], "hessian", True)
    with pytest.raises(NotImplementedError):
        F.register_evaluator(None, None, "hessian", 6)
    rc = _lib.load().fmm_evaluate_sources_outputs(F._plan, 7, 1, ctypes.c_void_p(0), 0, None)
    assert rc == 1  # invalid evaluator id
