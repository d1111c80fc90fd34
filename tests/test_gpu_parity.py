"""CUDA path against the reference (golden fixtures) and the CPU oracle.

Bar: FP64 results within 1e-12 relative L2 of the reference's own outputs
on the same inputs; the tree equal to the reference's box for box.
"""
import numpy as np
import pytest

from conftest import golden_cases, golden_inputs, kernel_of, load_golden, make_fmm, oracle_direct, rel_l2
import canon

pytestmark = pytest.mark.gpu

PARITY = 1e-12


def _fmm(d, meta, helper=None):
    return make_fmm(d, meta, helper)


@pytest.mark.parametrize("case", golden_cases())
def test_results_match_reference(built_lib, case):
    g = load_golden(case)
    meta = g["meta"]
    d = golden_inputs(meta)
    F = _fmm(d, meta)
    assert np.array_equal(np.array(F.bbox), g["bbox_used"])
    F.build_expansions(d["tau"])
    us = F.source_evaluation(d["x"], d["y"])
    ut = F.target_evaluation(d["tx"], d["ty"])
    es = rel_l2(us[g["src_idx"]], g["src_val"])
    et = rel_l2(ut[g["tgt_idx"]], g["tgt_val"])
    assert es < PARITY and et < PARITY, (es, et)


@pytest.mark.parametrize("case", [c for c in golden_cases() if "sample" not in load_golden(c)["meta"]])
def test_tree_matches_oracle(built_lib, case):
    from oracle.tree import Tree
    g = load_golden(case)
    meta = g["meta"]
    d = golden_inputs(meta)
    F = _fmm(d, meta)
    ot = Tree(d["x"], d["y"], meta["ncut"], F.bbox)
    a = canon.canonical(F.tree, triples_fn=canon.gpu_triples, nonempty_sources=True)
    b = canon.canonical(ot, nonempty_sources=True)
    assert canon.compare(a, b) == []


@pytest.mark.parametrize("case", [c for c in golden_cases() if "tree_sha_nonempty" in load_golden(c)])
def test_tree_matches_reference_at_scale(built_lib, case):
    """100k uniform and 1M clustered sources: the device tree, canonically,
    against digests of the reference's own tree (flexmm/tree.py:451-518) --
    box positions and flags, the leaf of every source, colleague sets and
    interaction lists, level by level."""
    import hashlib
    g = load_golden(case)
    meta = g["meta"]
    d = golden_inputs(meta)
    F = _fmm(d, meta)
    assert np.array_equal(np.array(F.bbox), g["bbox_used"])
    assert F.tree.levels == int(g["levels"])
    c = canon.canonical(F.tree, triples_fn=canon.gpu_triples, nonempty_sources=True)
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(np.asarray(a, dtype=np.int64)).tobytes()).hexdigest()
    got = {k: sha(v) for k, v in c.items()}
    ref = g["tree_sha_nonempty"]
    assert set(got) == set(ref)
    bad = [k for k in ref if got[k] != ref[k]]
    assert not bad, f"device tree differs from the reference's: {bad}"


def test_direct_sum_matches_c_oracle(built_lib):
    """The library's FP64 direct sum (the accuracy yardstick of the mixed
    tests) against the oracle's C direct sum, with and without the
    coincident-pair check, on clustered points with duplicates."""
    from flexmm_b200 import direct_evaluation, workloads
    from oracle.direct import direct_laplace
    d = workloads.clustered(n=30000, n_grid=40, seed=8)
    x, y, tau = d["x"].copy(), d["y"].copy(), d["tau"]
    x[1::7], y[1::7] = x[0::7][: x[1::7].size], y[0::7][: y[1::7].size]
    rng = np.random.default_rng(2)
    si = rng.choice(x.size, 1500, replace=False)
    for tx, ty, check in ((x[si], y[si], True), (d["tx"], d["ty"], False)):
        got = np.asarray(direct_evaluation("Laplace_Eval", x, y, tau, tx, ty, check=check))
        ref = direct_laplace(x, y, tau, tx, ty, check)
        assert np.isfinite(got).all()
        assert rel_l2(got, ref) < 1e-13


def _descent_lines(p, x0, w0, levels):
    """The midpoints the reference's descent compares point p with, level by
    level (FP64, the same recurrence: xm = xmin + w/2)."""
    out, xmin, w = [], x0, w0
    for _ in range(levels):
        hw = 0.5 * w
        xm = xmin + hw
        out.append(xm)
        xmin = xm if p > xm else xm - hw
        w = hw
    return out


def test_tree_with_points_on_split_lines_matches_oracle(built_lib):
    """Points exactly on the descent's midpoints and one ulp either side, in
    a box away from the origin (the midpoints carry FP64 rounding): the
    device's fixed-point keys fall back to the descent there, so every point
    lands in the reference's leaf."""
    from flexmm_b200 import KI_FMM, KI_Helper
    from oracle.tree import Tree
    rng = np.random.default_rng(77)
    bbox = [1000.3, 1000.3 + 0.9, -3.7, -3.7 + 0.9]
    n = 12000
    x = bbox[0] + 0.9 * rng.random(n)
    y = bbox[2] + 0.9 * rng.random(n)
    F0 = KI_FMM(x, y, "Laplace_Eval", 24, 16, bbox=bbox, helper=KI_Helper())
    bb = F0.bbox
    w0 = bb[1] - bb[0]
    xs, ys = [x], [y]
    for i in range(300):
        lx = _descent_lines(x[i], bb[0], w0, 14)
        ly = _descent_lines(y[i], bb[2], w0, 14)
        for a, b in zip(lx, ly):
            for v in (a, np.nextafter(a, -np.inf), np.nextafter(a, np.inf)):
                xs.append(np.array([v, v, x[i]]))
                ys.append(np.array([y[i], b, b]))
    # coarse midpoints are shared by many base points: keep each point once
    xy = np.unique(np.stack([np.concatenate(xs), np.concatenate(ys)], axis=1), axis=0)
    x, y = xy[:, 0].copy(), xy[:, 1].copy()
    F = KI_FMM(x, y, "Laplace_Eval", 24, 16, bbox=bbox, helper=KI_Helper())
    assert list(F.bbox) == list(bb)   # the same box as the lines were drawn in
    ot = Tree(x, y, 24, F.bbox)
    a = canon.canonical(F.tree, triples_fn=canon.gpu_triples, nonempty_sources=True)
    b = canon.canonical(ot, nonempty_sources=True)
    assert canon.compare(a, b) == []


def _direct(d, tx, ty, check):
    from oracle.direct import direct_laplace
    return direct_laplace(d["x"], d["y"], d["tau"], tx, ty, check)


@pytest.mark.parametrize("n,ncut", [(40, 64), (64, 64), (200, 64), (300, 100)])
def test_shallow_trees_equal_direct_sum(built_lib, n, ncut):
    """Trees of 1-2 levels (where the reference itself fails) reduce to the direct sum."""
    from flexmm_b200 import KI_FMM, KI_Helper
    rng = np.random.default_rng(n)
    d = dict(x=rng.uniform(-1, 1, n), y=rng.uniform(-1, 1, n), tau=rng.standard_normal(n))
    F = KI_FMM(d["x"], d["y"], "Laplace_Eval", ncut, 16, bbox=[-1, 1, -1, 1], helper=KI_Helper())
    F.build_expansions(d["tau"])
    tx, ty = rng.uniform(-1, 1, 77), rng.uniform(-1, 1, 77)
    if F.tree.levels < 3:
        assert rel_l2(F.target_evaluation(tx, ty), _direct(d, tx, ty, False)) < 1e-13
        assert rel_l2(F.source_evaluation(d["x"], d["y"]), _direct(d, d["x"], d["y"], True)) < 1e-13


def test_matches_oracle_midsize_and_torch_inputs(built_lib):
    import torch
    from flexmm_b200 import workloads
    from oracle.kifmm import KIFMM
    from oracle.kernels import laplace
    d = workloads.clustered(n=60000, n_grid=120, seed=21)
    meta = dict(ncut=40, neq=40)
    O = KIFMM(d["x"], d["y"], laplace, 40, 40, bbox=d["bbox"])
    O.build_expansions(d["tau"])
    F = _fmm(d, meta)
    F.build_expansions(torch.from_numpy(d["tau"]).cuda())
    ut = F.target_evaluation(torch.from_numpy(d["tx"]).cuda(), torch.from_numpy(d["ty"]).cuda())
    assert isinstance(ut, torch.Tensor) and ut.is_cuda
    assert rel_l2(ut.cpu().numpy(), O.target_evaluation(d["tx"], d["ty"])) < PARITY
    us = F.source_evaluation(d["x"], d["y"])
    assert rel_l2(us, O.source_evaluation(d["x"], d["y"])) < PARITY


def test_targets_outside_bbox_follow_reference_descent(built_lib):
    from flexmm_b200 import workloads
    from oracle.kifmm import KIFMM
    from oracle.kernels import laplace
    d = workloads.uniform(n=20000, n_grid=10, seed=5)
    rng = np.random.default_rng(9)
    tx = rng.uniform(-1.3, 1.3, 3000)
    ty = rng.uniform(-1.3, 1.3, 3000)
    O = KIFMM(d["x"], d["y"], laplace, 32, 24, bbox=d["bbox"])
    O.build_expansions(d["tau"])
    F = _fmm(d, dict(ncut=32, neq=24))
    F.build_expansions(d["tau"])
    assert rel_l2(F.target_evaluation(tx, ty), O.target_evaluation(tx, ty)) < PARITY


def test_helper_reuse_snaps_bbox_like_reference(built_lib):
    from flexmm_b200 import KI_FMM, KI_Helper, workloads
    from oracle.kifmm import snap_bbox
    d = workloads.uniform(n=5000, n_grid=10, seed=6)
    h = KI_Helper()
    F1 = KI_FMM(d["x"], d["y"], "Laplace_Eval", 32, 16, bbox=[-1, 1, -1, 1], helper=h)
    widths = h.collect_widths()
    F2 = KI_FMM(d["x"] * 0.3, d["y"] * 0.3, "Laplace_Eval", 32, 16, bbox=None, helper=h)
    bb = [np.min(d["x"] * 0.3), np.max(d["x"] * 0.3), np.min(d["y"] * 0.3), np.max(d["y"] * 0.3)]
    assert np.allclose(F2.bbox, snap_bbox(None, None, bb, widths), rtol=0, atol=0)
    with pytest.raises(ValueError):
        KI_FMM(d["x"], d["y"], "Laplace_Eval", 32, 24, bbox=[-1, 1, -1, 1], helper=h)


def test_empty_evaluation_and_errors(built_lib):
    from flexmm_b200 import KI_FMM, KI_Helper, workloads
    from flexmm_b200._lib import FMMError
    d = workloads.uniform(n=3000, n_grid=10, seed=7)
    F = KI_FMM(d["x"], d["y"], "Laplace_Eval", 32, 16, bbox=[-1, 1, -1, 1], helper=KI_Helper())
    with pytest.raises(FMMError):
        F.target_evaluation(d["tx"], d["ty"])     # before build_expansions
    F.build_expansions(d["tau"])
    assert F.target_evaluation(np.zeros(0), np.zeros(0)).shape == (0,)
    # more than Ncutoff coincident points cannot be split: clean error, no hang
    x = np.zeros(100)
    with pytest.raises(FMMError):
        KI_FMM(x, x, "Laplace_Eval", 16, 16, bbox=[-1, 1, -1, 1], helper=KI_Helper())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_own_source_evaluation_equals_general_path(built_lib, precision):
    """source_evaluation on the FMM's own tensors runs fmm_evaluate_sources
    (the tree's sorted copy); copies of the same points take the general path
    (upload, locate, sort).  Both give the same potentials, and an in-place
    change of the inputs turns the shortcut off."""
    import torch
    from flexmm_b200 import KI_FMM, KI_Helper
    g = load_golden("clustered_20k_q32")
    meta = g["meta"]
    d = golden_inputs(meta)
    x, y = torch.from_numpy(d["x"]).cuda(), torch.from_numpy(d["y"]).cuda()
    F = KI_FMM(x, y, "Laplace_Eval", meta["ncut"], meta["neq"], bbox=d["bbox"], helper=KI_Helper(),
               precision=precision)
    F.build_expansions(torch.from_numpy(d["tau"]).cuda())
    assert F._own_sources(x, y)
    u_own = F.source_evaluation(x, y).cpu().numpy()
    u_gen = F.source_evaluation(x.clone(), y.clone()).cpu().numpy()
    F.status()
    # FP64: the same arithmetic.  Mixed: the own-source sweep leaves each
    # target's own point out of its FP32 partial sums while the general path
    # zeroes it in place, so the FP32 summation order differs (~1e-9 here,
    # against the form's ~1e-7 error)
    assert rel_l2(u_own, u_gen) < (1e-14 if precision == "fp64" else 1e-8)
    if precision == "fp64":
        assert rel_l2(u_own[g["src_idx"]], g["src_val"]) < PARITY
    x.add_(0.0)
    assert not F._own_sources(x, y)


@pytest.mark.parametrize("k", [0.5, 5.0, 10.0, 200.0])
def test_mod_helmholtz_direct_sum_matches_scipy(built_lib, k):
    """The device K0 (series below 1, per-octave Chebyshev tables above) in the
    FP64 direct sum, against scipy's K0, with k r spanning 1e-7 .. ~600."""
    from flexmm_b200 import direct_evaluation
    from oracle.direct import direct_mod_helmholtz
    rng = np.random.default_rng(int(k * 10))
    r = np.geomspace(1e-7, 600.0, 3000)  # k * distance from a fixed source at 0
    th = rng.uniform(0, 2 * np.pi, r.size)
    sx, sy, tau = np.zeros(1), np.zeros(1), np.ones(1)
    tx, ty = r * np.cos(th) / k, r * np.sin(th) / k
    got = direct_evaluation("Modified_Helmholtz_Eval", sx, sy, tau, tx, ty, helmholtz_k=k)
    ref = direct_mod_helmholtz(sx, sy, tau, tx, ty, k, False)
    nz = ref > 1e-300
    # K0(x) has relative condition number ~x: one rounding of the distance
    # (the device contracts dx*dx + dy*dy into an FMA) moves it by ~x * 1e-16
    assert np.max(np.abs(got[nz] / ref[nz] - 1) / (1.0 + r[nz])) < 2e-14
    assert np.all(np.abs(got[~nz]) < 1e-290)


def test_mixed_form_rejects_kernels_without_fp32_form(built_lib):
    """A tabulated radial kernel has no FP32 form: its mixed form is refused."""
    from flexmm_b200 import KI_FMM, KI_Helper, kernels
    rng = np.random.default_rng(5)
    x, y = rng.uniform(-1, 1, 2000), rng.uniform(-1, 1, 2000)
    kern = kernels.radial(lambda r: np.exp(-r) / (1.0 + r), 1e-6, 4.0, name="ExpDecay")
    with pytest.raises(RuntimeError, match="FP32 form"):
        KI_FMM(x, y, kern, 32, 16, bbox=[-1, 1, -1, 1], helper=KI_Helper(), precision="mixed")


def test_radial_table_kernel_device_matches_host_table(built_lib):
    """The tabulated radial kernel on the device (direct sum) against the same
    table evaluated on the host and against the function it was fitted to."""
    from conftest import struve_kernel
    from flexmm_b200 import direct_evaluation
    from oracle.direct import struve_gf
    k = struve_kernel()
    r = np.geomspace(1e-6, 200.0, 4000)
    th = np.linspace(0, 2 * np.pi, r.size)
    tx, ty = r * np.cos(th), r * np.sin(th)
    got = direct_evaluation(k, np.zeros(1), np.zeros(1), np.ones(1), tx, ty)
    np.testing.assert_allclose(got, k.table(r), rtol=1e-13)
    near = r < 10
    np.testing.assert_allclose(got[near], struve_gf(r[near]), rtol=5e-12)


def test_split_source_evaluation_equals_one_pass(built_lib):
    """Own-source evaluation split in two -- the near field on a side stream
    from the moment the charges are sorted, the far field on the plan stream
    adding it -- equals the one-pass evaluation up to the order of the two
    sums, in both forms (fmm_set_split_evaluation on, then off)."""
    import torch
    from flexmm_b200 import KI_FMM, KI_Helper, set_split_evaluation, workloads
    d = workloads.clustered(n=120_000, n_grid=10, seed=44)
    x, y = torch.from_numpy(d["x"]).cuda(), torch.from_numpy(d["y"]).cuda()
    try:
        for prec, neq in (("fp64", 40), ("mixed", 24)):
            got = {}
            for mode in (True, False):
                set_split_evaluation(mode)
                F = KI_FMM(x, y, "Laplace_Eval", 64, neq, bbox=d["bbox"], helper=KI_Helper(),
                           precision=prec)
                F.build_expansions(d["tau"])
                got[mode] = F.source_evaluation(x, y).cpu().numpy()
                F.status()
                assert np.isfinite(got[mode]).all()
            # mixed: FP32 partial sums grouped differently (L2T and P2P apart),
            # ~1e-9 apart, against the form's ~1e-7 error
            assert rel_l2(got[True], got[False]) < (1e-14 if prec == "fp64" else 2e-8), prec
    finally:
        set_split_evaluation(None)


@pytest.mark.parametrize("case", golden_cases(dipole=True))
def test_dipoles_match_reference(built_lib, case):
    """Charges and dipoles (the Laplace single plus double layer) driven as
    the reference's example drives kifmm2d (register_upwardor /
    register_evaluator with Laplace_Both_Eval, build_expansions(tau,
    'slp+dlp', normals)): within 1e-12 of the reference's own outputs."""
    import torch
    from flexmm_b200 import KI_FMM, KI_Helper
    g = load_golden(case)
    meta = g["meta"]
    d = golden_inputs(meta)

    def Laplace_Both_Eval(sx, sy, tx, ty, tau, extras):   # matched by its name
        raise AssertionError("the device form is built in")
    x, y = torch.from_numpy(d["x"]).cuda(), torch.from_numpy(d["y"]).cuda()
    F = KI_FMM(x, y, "Laplace_Eval", meta["ncut"], meta["neq"], bbox=d["bbox"], helper=KI_Helper())
    F.register_upwardor(Laplace_Both_Eval, "slp+dlp")
    F.register_evaluator(F.helper.functions["kernel_app"], Laplace_Both_Eval, "slp+dlp->u", 1)
    F.build_expansions(np.vstack([d["tau"], d["dlp"]]), "slp+dlp", np.vstack([d["nx"], d["ny"]]))
    us = F.evaluate_to_points(x, y, "slp+dlp->u", True)[0]      # own sources (split near field)
    ut = F.evaluate_to_points(d["tx"], d["ty"], "slp+dlp->u", False)[0]
    us2 = F.evaluate_to_points(d["x"], d["y"], "slp+dlp->u", True)[0]   # located afresh
    F.status()
    assert rel_l2(us.cpu().numpy(), g["src_val"]) < PARITY
    assert rel_l2(ut, g["tgt_val"]) < PARITY
    assert rel_l2(us2, g["src_val"]) < PARITY


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_results_are_bitwise_reproducible(built_lib, precision):
    """Two builds and evaluations of the same problem give the same bits:
    the tree's sorts are stable, its prefix sums (split counts, charge sums)
    group their additions by a fixed layout, and no result depends on
    timing."""
    import torch
    from flexmm_b200 import KI_FMM, KI_Helper, workloads
    d = workloads.clustered(n=300_000, n_grid=300, seed=9)
    x, y = torch.from_numpy(d["x"]).cuda(), torch.from_numpy(d["y"]).cuda()
    tx, ty = torch.from_numpy(d["tx"]).cuda(), torch.from_numpy(d["ty"]).cuda()
    helper = KI_Helper()
    outs = []
    for _ in range(2):
        F = KI_FMM(x, y, "Laplace_Eval", 64, 24 if precision == "mixed" else 40, bbox=d["bbox"],
                   helper=helper, precision=precision)
        F.build_expansions(d["tau"])
        outs.append((F.source_evaluation(x, y).cpu(), F.target_evaluation(tx, ty).cpu()))
        F.status()
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pinned_host_charges_equal_device_charges(built_lib, precision):
    """Charges given as a pinned host tensor are copied on a stream of their
    own, beside the tree's last kernels: the results equal those of the same
    charges given on the device, bit for bit, over repeated builds."""
    import torch
    from flexmm_b200 import KI_FMM, workloads
    d = workloads.clustered(n=200_000, n_grid=100)
    x, y = (torch.from_numpy(d[k]).cuda() for k in ("x", "y"))
    tau_h = torch.from_numpy(d["tau"]).pin_memory()
    neq = {"fp64": 60, "mixed": 24}[precision]

    def run(tau):
        F = KI_FMM(x, y, "Laplace_Eval", 64, neq, bbox=d["bbox"], precision=precision)
        F.build_expansions(tau)
        return F.source_evaluation(x, y).cpu()

    ref = run(tau_h.cuda())
    for _ in range(3):
        assert torch.equal(run(tau_h), ref)


def test_binned_targets_match_sorted_targets(built_lib):
    """Targets are binned into their leaves (a descent along each key's
    digits) by fmm_evaluate and sorted by fmm_evaluate_noalloc: every target
    must land in the same leaf, so the two agree point by point to rounding --
    including targets exactly on dyadic split lines, outside the bbox, and
    at the sources themselves.  A target in another leaf would differ at the
    FMM's truncation level (~1e-8 here)."""
    import ctypes
    import torch
    from flexmm_b200 import KI_FMM, KI_Helper, _lib
    lib = _lib.load()
    rng = np.random.default_rng(23)
    x, y = rng.uniform(-1, 1, 50_000), rng.uniform(-1, 1, 50_000)
    F = KI_FMM(x, y, "Laplace_Eval", 32, 24, bbox=[-1, 1, -1, 1], helper=KI_Helper())
    F.build_expansions(rng.standard_normal(50_000))
    g = -1 + np.arange(65) / 32.0                      # split lines of levels <= 5
    gx, gy = np.meshgrid(g, g)
    ox, oy = rng.uniform(-1.5, 1.5, 8000), rng.uniform(-1.5, 1.5, 8000)
    out = (np.abs(ox) > 1) | (np.abs(oy) > 1)
    cases = [(np.concatenate([gx.ravel(), rng.uniform(-1, 1, 20_000), ox[out]]),
              np.concatenate([gy.ravel(), rng.uniform(-1, 1, 20_000), oy[out]]), 0),
             (x[:20_000], y[:20_000], 1)]
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for tx, ty, check in cases:
        txd, tyd = torch.from_numpy(tx).cuda(), torch.from_numpy(ty).cuda()
        res = []
        for fn in ("fmm_evaluate", "fmm_evaluate_noalloc"):
            o = torch.full_like(txd, float("nan"))
            rc = getattr(lib, fn)(F._plan, ctypes.c_void_p(txd.data_ptr()), ctypes.c_void_p(tyd.data_ptr()),
                                  txd.numel(), check, ctypes.c_void_p(o.data_ptr()), stream)
            assert rc == 0, lib.fmm_last_error()
            torch.cuda.synchronize()
            res.append(o.cpu().numpy())
        binned, sorted_ = res
        assert np.isfinite(binned).all()
        scale = np.sqrt(np.mean(sorted_ ** 2))
        assert np.max(np.abs(binned - sorted_)) < 1e-12 * scale
