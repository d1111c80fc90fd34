"""Mixed-precision form: error against FP64 direct summation (bar: 1e-6 relative L2)."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

BAR = 1e-6


def _run(d, ncut, neq, precision, tx, ty):
    from flexmm_b200 import KI_FMM, KI_Helper
    F = KI_FMM(d["x"], d["y"], "Laplace_Eval", ncut, neq, bbox=d["bbox"], helper=KI_Helper(),
               precision=precision)
    F.build_expansions(d["tau"])
    return F, F.source_evaluation(d["x"], d["y"]), F.target_evaluation(tx, ty)


@pytest.mark.parametrize("recipe,n,neq", [("clustered", 200_000, 24), ("uniform", 100_000, 24),
                                          ("clustered", 100_000, 32)])
def test_mixed_error_vs_direct_sum(built_lib, recipe, n, neq):
    from flexmm_b200 import direct_evaluation, workloads
    d = getattr(workloads, recipe)(n=n, n_grid=300, seed=41)
    F, us, ut = _run(d, 64, neq, "mixed", d["tx"], d["ty"])
    rng = np.random.default_rng(1)
    si = rng.choice(d["x"].size, 2000, replace=False)
    ti = rng.choice(d["tx"].size, 2000, replace=False)
    ds = direct_evaluation("Laplace_Eval", d["x"], d["y"], d["tau"], d["x"][si], d["y"][si], check=True)
    dt = direct_evaluation("Laplace_Eval", d["x"], d["y"], d["tau"], d["tx"][ti], d["ty"][ti])
    es, et = rel_l2(us[si], ds), rel_l2(ut[ti], dt)
    assert es < BAR and et < BAR, (es, et)


def test_mixed_headline_config_vs_direct_sum(built_lib):
    """The headline configuration: 1M sources in 20 Gaussian clusters plus a
    1000^2 grid, Nequiv 24, mixed form -- against the FP64 direct sums at the
    fixture's 2,000 sampled sources and 2,000 grid targets (bar 1e-6), and
    against the reference's own FP64 Nequiv-24 outputs there."""
    from conftest import golden_inputs, load_golden
    g = load_golden("clustered_1M_q24")
    meta = g["meta"]
    d = golden_inputs(meta)
    F, us, ut = _run(d, meta["ncut"], meta["neq"], "mixed", d["tx"], d["ty"])
    F.status()
    assert np.isfinite(us).all() and np.isfinite(ut).all()
    es = rel_l2(us[g["src_idx"]], g["direct_src"])
    et = rel_l2(ut[g["tgt_idx"]], g["direct_tgt"])
    assert es < BAR and et < BAR, (es, et)
    # the reference at Nequiv 24 is itself ~2e-7 from the direct sum
    assert rel_l2(us[g["src_idx"]], g["src_val"]) < BAR
    assert rel_l2(ut[g["tgt_idx"]], g["tgt_val"]) < BAR


def test_mixed_coincident_points_are_skipped_exactly(built_lib):
    """Duplicated sources: the FP32 path must still skip exactly the coincident pairs."""
    from conftest import golden_inputs, load_golden
    g = load_golden("duplicates_5k_q24")
    d = golden_inputs(g["meta"])
    F, us, ut = _run(d, g["meta"]["ncut"], g["meta"]["neq"], "mixed", d["tx"], d["ty"])
    assert np.isfinite(us).all() and np.isfinite(ut).all()
    assert rel_l2(us, g["direct_src"]) < BAR
    assert rel_l2(ut, g["direct_tgt"]) < BAR


@pytest.mark.parametrize("k,recipe", [(10.0, "clustered"), (0.5, "clustered"), (10.0, "uniform")])
def test_mixed_modified_helmholtz_vs_direct_sum(built_lib, k, recipe):
    """K0(k r) / (2 pi) in the mixed form (FP32 K0 from the Abramowitz-Stegun
    polynomials, box-centred coordinates, 3xTF32 translations) against the
    FP64 direct sum (bar 1e-6), sources (own points skipped) and targets."""
    from flexmm_b200 import KI_FMM, KI_Helper, direct_evaluation, workloads
    d = getattr(workloads, recipe)(n=150_000, n_grid=300, seed=47)
    F = KI_FMM(d["x"], d["y"], "Modified_Helmholtz_Eval", 64, 32, bbox=d["bbox"],
               helper=KI_Helper(), precision="mixed", helmholtz_k=k)
    F.build_expansions(d["tau"])
    us, ut = F.source_evaluation(d["x"], d["y"]), F.target_evaluation(d["tx"], d["ty"])
    F.status()
    rng = np.random.default_rng(3)
    si = rng.choice(d["x"].size, 2000, replace=False)
    ti = rng.choice(d["tx"].size, 2000, replace=False)
    kw = dict(helmholtz_k=k)
    ds = direct_evaluation("Modified_Helmholtz_Eval", d["x"], d["y"], d["tau"], d["x"][si], d["y"][si],
                           check=True, **kw)
    dt = direct_evaluation("Modified_Helmholtz_Eval", d["x"], d["y"], d["tau"], d["tx"][ti], d["ty"][ti], **kw)
    es, et = rel_l2(us[si], ds), rel_l2(ut[ti], dt)
    assert es < BAR and et < BAR, (es, et)


def test_mixed_charge_columns_vs_single_columns_and_direct_sum(built_lib):
    """Charge columns [k, N] in the mixed form (each column's expansions formed
    in turn on one tree), on the multi-RHS workload's kernel and points at a
    smaller size: every row equals the single-column mixed result bit for bit
    (sources and targets), and is within 1e-6 of the FP64 direct sum at 2,000
    sampled sources (the aggregate bar of the mixed form; see the FP32 pair
    sweep's close-pair limit in the design notes)."""
    import torch
    from flexmm_b200 import KI_FMM, KI_Helper, direct_evaluation, workloads
    d = workloads.circle(n=100_000, n_rhs=3, seed=9)
    x, y = torch.from_numpy(d["x"]).cuda(), torch.from_numpy(d["y"]).cuda()
    tau = torch.from_numpy(d["tau"]).cuda()
    rng = np.random.default_rng(2)
    tx = torch.from_numpy(rng.uniform(-0.6, 0.6, 3000)).cuda()
    ty = torch.from_numpy(rng.uniform(-0.6, 0.6, 3000)).cuda()
    # a helper of its own per plan: a shared one snaps later bboxes to its cached widths
    kw = dict(precision="mixed", helmholtz_k=10.0)
    F = KI_FMM(x, y, "Modified_Helmholtz_Eval", 64, 40, helper=KI_Helper(), **kw)
    F.build_expansions(tau)
    us, ut = F.source_evaluation(x, y).cpu().numpy(), F.target_evaluation(tx, ty).cpu().numpy()
    assert us.shape == (3, 100_000) and ut.shape == (3, 3000)
    si = rng.choice(100_000, 2000, replace=False)
    for c in range(3):
        G = KI_FMM(x, y, "Modified_Helmholtz_Eval", 64, 40, helper=KI_Helper(), **kw)
        G.build_expansions(tau[c].contiguous())
        assert np.array_equal(G.source_evaluation(x, y).cpu().numpy(), us[c])
        assert np.array_equal(G.target_evaluation(tx, ty).cpu().numpy(), ut[c])
        ds = direct_evaluation("Modified_Helmholtz_Eval", d["x"], d["y"], d["tau"][c], d["x"][si],
                               d["y"][si], check=True, helmholtz_k=10.0)
        assert rel_l2(us[c][si], ds) < BAR


def test_mixed_modified_helmholtz_refuses_gradients(built_lib):
    from flexmm_b200 import KI_FMM, KI_Helper, workloads
    d = workloads.uniform(n=20_000, n_grid=30, seed=5)
    F = KI_FMM(d["x"], d["y"], "Modified_Helmholtz_Eval", 64, 24, bbox=d["bbox"], helper=KI_Helper(),
               precision="mixed", helmholtz_k=5.0)
    F.build_expansions(d["tau"])
    F.register_evaluator(None, None, "grad", 3)
    with pytest.raises(RuntimeError, match="potential only"):
        F.evaluate_to_points(d["tx"], d["ty"], "grad", False)


_SYNC_SCRIPT = r"""
import sys, numpy as np
sys.path.insert(0, {repo!r})
from flexmm_b200 import KI_FMM, KI_Helper, workloads
d = workloads.clustered(n=150_000, n_grid=200, seed=43)
F = KI_FMM(d["x"], d["y"], "Laplace_Eval", 64, 24, bbox=d["bbox"], helper=KI_Helper(), precision="mixed")
F.build_expansions(d["tau"])
np.save({out!r}, F.target_evaluation(d["tx"], d["ty"]))
"""


def test_tcgen05_m2l_matches_warp_mma_m2l(built_lib, tmp_path):
    """The tcgen05 M2L (default for Nequiv <= 32) and the warp-level mma.sync
    M2L (diagnostic switch FLEXMM_B200_M2L=mma_sync) give the same far field."""
    import os
    import subprocess
    import sys
    from conftest import REPO
    from flexmm_b200 import KI_FMM, KI_Helper, workloads
    d = workloads.clustered(n=150_000, n_grid=200, seed=43)
    F = KI_FMM(d["x"], d["y"], "Laplace_Eval", 64, 24, bbox=d["bbox"], helper=KI_Helper(),
               precision="mixed")
    F.build_expansions(d["tau"])
    ut = F.target_evaluation(d["tx"], d["ty"])
    F.status()   # no bounded wait ran out
    out = str(tmp_path / "sync.npy")
    env = dict(os.environ, FLEXMM_B200_M2L="mma_sync")
    subprocess.run([sys.executable, "-c", _SYNC_SCRIPT.format(repo=REPO, out=out)], env=env,
                   check=True, timeout=600)
    us = np.load(out)
    # both are FP32-rounded forms of the same translation (the tcgen05 path
    # adds its k-step slots in FP32): ~1e-8 apart, against ~1e-7 form error
    assert rel_l2(ut, us) < 3e-8
