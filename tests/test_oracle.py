"""The CPU oracle against the golden fixtures made by running the reference."""
import hashlib

import numpy as np
import pytest

from conftest import golden_cases, golden_inputs, load_golden, oracle_kernel, rel_l2
import canon
from oracle.kifmm import KIFMM
from oracle.kernels import laplace
from oracle.tree import Tree
from oracle.direct import direct_laplace


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(np.asarray(a, dtype=np.int64)).tobytes()).hexdigest()


SMALL = [c for c in golden_cases() if "sample" not in load_golden(c)["meta"]]


@pytest.mark.parametrize("case", SMALL)
def test_oracle_tree_matches_reference_tree(case):
    g = load_golden(case)
    d = golden_inputs(g["meta"])
    t = Tree(d["x"], d["y"], g["meta"]["ncut"], list(g["bbox_used"]))
    assert t.levels == int(g["levels"])
    c = canon.canonical(t)
    got = {k: sha(v) for k, v in c.items()}
    bad = [k for k in g["tree_sha"] if got.get(k) != g["tree_sha"][k]]
    assert not bad, f"canonical tree fields differ from the reference: {bad}"


LARGE = [c for c in golden_cases() if "tree_sha_nonempty" in load_golden(c)]


@pytest.mark.parametrize("case", LARGE)
def test_oracle_tree_matches_reference_tree_at_scale(case):
    """100k uniform and 1M clustered: the oracle's tree against the digests
    of the reference's own tree (interactions from empty boxes left out)."""
    g = load_golden(case)
    d = golden_inputs(g["meta"])
    t = Tree(d["x"], d["y"], g["meta"]["ncut"], list(g["bbox_used"]))
    assert t.levels == int(g["levels"])
    got = {k: sha(v) for k, v in canon.canonical(t, nonempty_sources=True).items()}
    ref = g["tree_sha_nonempty"]
    assert set(got) == set(ref)
    bad = [k for k in ref if got[k] != ref[k]]
    assert not bad, f"canonical tree fields differ from the reference: {bad}"


@pytest.mark.parametrize("case", [c for c in SMALL if load_golden(c)["meta"].get("method") != "bb"])
def test_oracle_results_match_reference(case):
    g = load_golden(case)
    meta = g["meta"]
    d = golden_inputs(meta)
    F = KIFMM(d["x"], d["y"], oracle_kernel(meta), meta["ncut"], meta["neq"], bbox=d["bbox"])
    assert np.allclose(F.bbox, g["bbox_used"], rtol=0, atol=0)
    F.build_expansions(d["tau"])
    us = F.source_evaluation(d["x"], d["y"])
    ut = F.target_evaluation(d["tx"], d["ty"])
    assert rel_l2(us[g["src_idx"]], g["src_val"]) < 1e-13
    assert rel_l2(ut[g["tgt_idx"]], g["tgt_val"]) < 1e-13


def test_golden_inputs_regenerate_bitwise():
    import make_golden
    for case in (golden_cases() + golden_cases(gradient=True) + golden_cases(stokes=True)
                 + golden_cases(local=True)):
        g = load_golden(case)
        d = golden_inputs(g["meta"])
        assert make_golden.sha(d["x"], d["y"], d["tau"], d["tx"], d["ty"]) == str(g["inputs_sha"]), case
    for case in golden_cases(stresslet=True):
        g = load_golden(case)
        d = golden_inputs(g["meta"])
        assert make_golden.sha(d["x"], d["y"], d["tau"], d["tx"], d["ty"]) == str(g["inputs_sha"]), case
    for case in golden_cases(dipole=True):
        g = load_golden(case)
        d = golden_inputs(g["meta"])
        got = make_golden.sha(d["x"], d["y"], d["tau"], d["tx"], d["ty"], d["dlp"], d["nx"], d["ny"])
        assert got == str(g["inputs_sha"]), case


@pytest.mark.parametrize("case", golden_cases(dipole=True))
def test_dipole_fixtures_against_direct_sum(case):
    """The reference's single + double layer FMM (kifmm2d upwardor) is close
    to the oracle's direct sum at its Nequiv (a check of the fixture)."""
    g = load_golden(case)
    assert rel_l2(g["src_val"], g["direct_src"]) < 1e-5
    assert rel_l2(g["tgt_val"], g["direct_tgt"]) < 1e-5


def test_direct_sum_oracle_small():
    rng = np.random.default_rng(3)
    sx, sy, tau = rng.uniform(-1, 1, 300), rng.uniform(-1, 1, 300), rng.standard_normal(300)
    tx, ty = rng.uniform(-1, 1, 50), rng.uniform(-1, 1, 50)
    ref = (-np.log((tx[:, None] - sx) ** 2 + (ty[:, None] - sy) ** 2) / (4 * np.pi) * tau).sum(1)
    assert rel_l2(direct_laplace(sx, sy, tau, tx, ty, False), ref) < 1e-14
    # check=True drops the coincident pair only
    got = direct_laplace(sx, sy, tau, sx[:5], sy[:5], True)
    with np.errstate(divide="ignore"):
        k = -np.log((sx[:5, None] - sx) ** 2 + (sy[:5, None] - sy) ** 2) / (4 * np.pi)
    k[np.arange(5), np.arange(5)] = 0
    assert rel_l2(got, (k * tau).sum(1)) < 1e-14


@pytest.mark.parametrize("case", SMALL)
def test_reference_accuracy_recorded(case):
    """The stored reference outputs agree with FP64 direct sums to the FMM's own accuracy."""
    g = load_golden(case)
    neq = g["meta"]["neq"]
    if g["meta"].get("method") == "bb":  # black-box FMM: p^2 coefficients
        tol = {64: 1e-6, 100: 1e-7, 144: 1e-9, 256: 1e-12}[neq]
    else:
        tol = {16: 1e-4, 24: 1e-6, 32: 1e-8, 40: 1e-9, 60: 1e-13}[neq]
    assert rel_l2(g["src_val"], g["direct_src"]) < tol
    assert rel_l2(g["tgt_val"], g["direct_tgt"]) < tol
