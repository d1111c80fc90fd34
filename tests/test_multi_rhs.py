"""Several charge columns on one tree (multi-RHS; the batching form's first
part): every column equals the single-column FMM with that column, for the
Laplace and modified Helmholtz kernels, and matches the FP64 direct sum."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["clustered_20k_q32", "mh_circle_20k_q40_k10"])
def test_column_matches_reference(built_lib, case):
    """A charge column inside a multi-column build reproduces the reference's
    single-column outputs (golden fixture) to the FP64 parity bar."""
    import torch
    from conftest import golden_inputs, kernel_of, load_golden
    from flexmm_b200 import KI_FMM, KI_Helper
    g = load_golden(case)
    meta = g["meta"]
    d = golden_inputs(meta)
    name, params = kernel_of(meta)
    rng = np.random.default_rng(9)
    tau = np.vstack([rng.standard_normal(d["x"].size), d["tau"], rng.standard_normal(d["x"].size)])
    xt, yt = torch.from_numpy(d["x"]).cuda(), torch.from_numpy(d["y"]).cuda()
    F = KI_FMM(xt, yt, name, meta["ncut"], meta["neq"], bbox=d["bbox"], helper=KI_Helper(), **params)
    F.build_expansions(tau)
    us = F.source_evaluation(xt, yt).cpu().numpy()
    ut = F.target_evaluation(d["tx"], d["ty"])
    F.status()
    assert us.shape == (3, d["x"].size) and ut.shape == (3, d["tx"].size)
    assert rel_l2(us[1][g["src_idx"]], g["src_val"]) < 1e-12
    assert rel_l2(ut[1][g["tgt_idx"]], g["tgt_val"]) < 1e-12


def test_multi_rhs_against_direct_sum(built_lib):
    from flexmm_b200 import KI_FMM, KI_Helper, workloads
    from oracle.direct import direct_mod_helmholtz
    d = workloads.circle(n=20000, n_rhs=3, seed=6)
    F = KI_FMM(d["x"], d["y"], "Modified_Helmholtz_Eval", 64, 40, helper=KI_Helper(), helmholtz_k=10.0)
    F.build_expansions(d["tau"])
    u = F.source_evaluation(d["x"], d["y"])
    idx = np.arange(0, 20000, 97)
    for r in range(3):
        ref = direct_mod_helmholtz(d["x"], d["y"], d["tau"][r], d["x"][idx], d["y"][idx], 10.0, True)
        assert rel_l2(u[r][idx], ref) < 1e-9


def test_sixty_four_columns_in_one_pass_per_level(built_lib):
    """64 charge columns (the multi-RHS configuration's width) built with one
    launch per level for all columns: sampled columns equal single-column
    builds on the same tree (1e-13) and the direct sum."""
    import torch
    from flexmm_b200 import KI_FMM, KI_Helper, workloads
    from oracle.direct import direct_mod_helmholtz
    d = workloads.circle(n=30000, n_rhs=64, seed=7)
    x, y = torch.from_numpy(d["x"]).cuda(), torch.from_numpy(d["y"]).cuda()
    # one box for every object, each with a fresh helper: a helper that has
    # cached widths snaps a box to them (the reference's get_bbox), which
    # would give a different tree
    bb = [-0.51, 0.51, -0.51, 0.51]
    F = KI_FMM(x, y, "Modified_Helmholtz_Eval", 64, 40, bbox=bb, helper=KI_Helper(),
               helmholtz_k=10.0)
    F.build_expansions(d["tau"])
    u = F.source_evaluation(x, y).cpu().numpy()
    F.status()
    assert u.shape == (64, 30000) and np.isfinite(u).all()
    idx = np.arange(0, 30000, 151)
    for r in (0, 17, 40, 63):
        S = KI_FMM(x, y, "Modified_Helmholtz_Eval", 64, 40, bbox=bb, helper=KI_Helper(),
                   helmholtz_k=10.0)
        assert S.bbox == F.bbox
        S.build_expansions(d["tau"][r])
        one = S.source_evaluation(x, y).cpu().numpy()
        assert rel_l2(u[r], one) < 1e-13, r
        ref = direct_mod_helmholtz(d["x"], d["y"], d["tau"][r], d["x"][idx], d["y"][idx], 10.0, True)
        assert rel_l2(u[r][idx], ref) < 1e-9, r
