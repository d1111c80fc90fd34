"""Stokes FMM (flexmm/kifmm2d/vector/stokes_fmm.py) against the reference.

Fixtures: the reference's Stokes FMM run on seeded inputs (rows u, v, p for
source evaluation with check_self and for grid targets) and FP64 direct sums.
The reference's own accuracy is modest (Nequiv 16: ~1e-2, 32: ~1e-5 vs the
direct sum); the bar for this library is agreement with the reference's
outputs: 1e-12 relative L2 per row.
"""
import numpy as np
import pytest

from conftest import golden_cases, golden_inputs, load_golden, rel_l2

CASES = golden_cases(stokes=True)
PARITY = 1e-12


@pytest.mark.parametrize("case", CASES)
def test_direct_stokes_oracle_regenerates_and_bounds_reference(case):
    from oracle.direct import direct_stokes
    g = load_golden(case)
    meta = g["meta"]
    d = golden_inputs(meta)
    ds = direct_stokes(d["x"], d["y"], d["tau"], d["tau2"], d["x"][:300], d["y"][:300], True)
    np.testing.assert_allclose(ds, g["direct_src"][:, :300], rtol=1e-12, atol=1e-12)
    bar = {16: 3e-2, 24: 3e-3, 32: 1e-4}[meta["neq"]]
    for r in range(3):
        assert rel_l2(g["src_val"][r], g["direct_src"][r]) < bar
        assert rel_l2(g["tgt_val"][r], g["direct_tgt"][r]) < bar


def test_stokes_forms_match_definitions():
    """Host operator formation: the corrected form is the plain form with the
    pressure row mirrored into an extra column."""
    from flexmm_b200.stokes import circles, stokes_form
    th = np.linspace(0, 2 * np.pi, 8, endpoint=False)
    sx, sy, lx, ly = circles(0.5, th)
    G = stokes_form(sx, sy, lx, ly)
    C = stokes_form(sx, sy, lx, ly, corrected=True)
    assert G.shape == (17, 16) and C.shape == (17, 17)
    np.testing.assert_array_equal(C[:, :-1], G)
    np.testing.assert_array_equal(C[:-1, -1], G[-1])
    assert C[-1, -1] == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_stokes_matches_reference(built_lib, case):
    from flexmm_b200.stokes import FMM
    g = load_golden(case)
    meta = g["meta"]
    d = golden_inputs(meta)
    F = FMM(d["x"], d["y"], meta["neq"], meta["ncut"], bbox=d["bbox"])
    assert np.array_equal(np.array(F.bbox), g["bbox_used"])
    F.precompute()
    F.build_expansions(d["tau"], d["tau2"])
    us = F.evaluate_to_points(d["x"], d["y"], True)
    ut = F.evaluate_to_points(d["tx"], d["ty"], False)
    F.status()
    for r in range(3):
        es, et = rel_l2(us[r], g["src_val"][r]), rel_l2(ut[r], g["tgt_val"][r])
        assert es < PARITY and et < PARITY, (r, es, et)


@pytest.mark.gpu
def test_stokes_plan_rejects_scalar_calls(built_lib):
    import ctypes
    from flexmm_b200 import _lib
    from flexmm_b200.stokes import FMM
    g = load_golden("stokes_uniform_3k_q16")
    d = golden_inputs(g["meta"])
    F = FMM(d["x"], d["y"], 16, 16, bbox=d["bbox"])
    F.build_expansions(d["tau"], d["tau2"])
    lib = _lib.load()
    assert lib.fmm_evaluate_sources(F._plan, 1, ctypes.c_void_p(0), None) == 1
    assert lib.fmm_build_expansions(F._plan, ctypes.c_void_p(1), None) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("case", golden_cases(stresslet=True))
def test_stresslets_match_reference(built_lib, case):
    """Forces plus stresslets (build_expansions_dipole /
    evaluate_to_points_dipole, stokes_fmm.py:738-858) against the reference's
    own outputs, rows (u, v, p).  The reference's stresslet far field is
    itself 20-30% from the direct sum in u, v at these Nequiv (its pressure
    is close; the fixture records both): the stresslets' check velocities
    are matched by large, cancelling equivalent forces, which amplifies FP64
    rounding, so the bar is 1e-11 here (1e-12 for every other path)."""
    from flexmm_b200.stokes import FMM
    g = load_golden(case)
    meta = g["meta"]
    d = golden_inputs(meta)
    F = FMM(d["x"], d["y"], meta["neq"], meta["ncut"], bbox=d["bbox"])
    assert np.array_equal(np.array(F.bbox), g["bbox_used"])
    F.precompute()
    F.build_expansions_dipole(d["tau"], d["tau2"], d["sgx"], d["sgy"], d["nx"], d["ny"])
    us = np.array([np.asarray(r) for r in F.evaluate_to_points_dipole(d["x"], d["y"], True)])
    ut = np.array([np.asarray(r) for r in F.evaluate_to_points_dipole(d["tx"], d["ty"], False)])
    F.status()
    for r in range(3):
        assert rel_l2(us[r], g["src_val"][r]) < 1e-11, ("src", r)
        assert rel_l2(ut[r], g["tgt_val"][r]) < 1e-11, ("tgt", r)
