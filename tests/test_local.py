"""Near-field-only evaluation (the LocalEvaluator family): the GPU tree with
the width floor and the colleague sums, against the reference's own
LocalEvaluator, category LocalEvaluator and PeriodicLocalEvaluator outputs
(golden fixtures; bar 1e-12) and the FP64 direct sum of the compactly
supported test kernel (whose support the colleagues cover)."""
import numpy as np
import pytest

from conftest import golden_cases, golden_inputs, load_golden, rel_l2

_KERNELS = {}


def bump_kernel(delta):
    """(1 - r^2/delta^2)^3 for r < delta, else 0, as a tabulated radial kernel."""
    if delta not in _KERNELS:
        from make_golden import local_bump
        from flexmm_b200.kernels import radial
        _KERNELS[delta] = radial(local_bump(delta), 1e-30, 4.0, tol=1e-6, name="LocalBump")
    return _KERNELS[delta]


def test_periodic_images_match_reference_rule():
    """The image set of the periodic evaluator: every source near a side
    repeated across it, corners across both sides and the diagonal."""
    from flexmm_b200.periodic_local_evaluator_category import periodic_images
    x = np.array([0.0, -0.99, 0.99, -0.99, 0.99, 0.5])
    y = np.array([0.0, 0.0, 0.98, -0.995, -0.97, 0.99])
    c = np.arange(6)
    px, py, pc, pi = periodic_images(x, y, c, [-1, 1, -1, 1], 0.05)
    got = sorted(zip(np.round(px, 12), np.round(py, 12), pi))
    want = [(0.0, 0.0, 0), (-0.99, 0.0, 1), (1.01, 0.0, 1), (0.99, 0.98, 2), (-1.01, 0.98, 2),
            (0.99, -1.02, 2), (-1.01, -1.02, 2), (-0.99, -0.995, 3), (1.01, -0.995, 3),
            (-0.99, 1.005, 3), (1.01, 1.005, 3), (0.99, -0.97, 4), (-1.01, -0.97, 4),
            (0.99, 1.03, 4), (-1.01, 1.03, 4), (0.5, 0.99, 5), (0.5, -1.01, 5)]
    assert got == sorted((round(a, 12), round(b, 12), i) for a, b, i in want)
    assert np.array_equal(pc, c[pi])


@pytest.mark.gpu
@pytest.mark.parametrize("case", golden_cases(local=True))
def test_local_evaluators_match_reference(built_lib, case):
    g = load_golden(case)
    meta = g["meta"]
    d = golden_inputs(meta)
    K = bump_kernel(meta["delta"])
    n, m = d["x"].size, d["tx"].size
    out_s, out_t = np.zeros((n, 1)), np.zeros((m, 1))
    if meta["local"] == "plain":
        from flexmm_b200.local_evaluator import LocalEvaluator
        E = LocalEvaluator(d["x"], d["y"], K, meta["delta"], ncutoff=meta["ncut"])
        assert E.bbox == list(g["bbox_used"])
        E.load_tau(d["tau"])
        E.source_evaluation(d["x"], d["y"], out_s)
        E.target_evaluation(d["tx"], d["ty"], out_t)
    elif meta["local"] == "category":
        from flexmm_b200.local_evaluator_category import LocalEvaluator
        E = LocalEvaluator(d["x"], d["y"], d["cat"], K, meta["delta"], ncutoff=meta["ncut"])
        E.load_tau(d["tau"])
        E.target_evaluation(d["x"], d["y"], d["cat"], out_s)
        E.target_evaluation(d["tx"], d["ty"], d["tcat"], out_t)
    else:
        from flexmm_b200.periodic_local_evaluator_category import PeriodicLocalEvaluator
        E = PeriodicLocalEvaluator(d["x"], d["y"], d["cat"], K, meta["delta"], [-1, 1, -1, 1],
                                   ncutoff=meta["ncut"])
        assert E.bbox == list(g["bbox_used"])
        E.load_tau(d["tau"])
        E.target_evaluation(d["x"], d["y"], d["cat"], out_s)
        E.target_evaluation(d["tx"], d["ty"], d["tcat"], out_t)
    es, et = rel_l2(out_s[:, 0], g["src_val"]), rel_l2(out_t[:, 0], g["tgt_val"])
    assert es < 1e-12 and et < 1e-12, (es, et)
    assert rel_l2(out_s[:, 0], g["direct_src"]) < 1e-12
    assert rel_l2(out_t[:, 0], g["direct_tgt"]) < 1e-12
