"""Batched independent Stokes problems (StokesBatch): forward and charge adjoint.

The batch runs each problem's own FP64 Stokes FMM (pinned to the reference's
Stokes FMM at 1e-12 in test_stokes.py), spread over CUDA streams.  Bars:
every problem's batch result equals the same problem run alone with the same
box and operators (1e-12); the forward and the adjoint agree with FP64 direct
sums to the method's accuracy at Nequiv 32 (the reference itself is ~1e-4
there); the adjoint's construction (Stokes velocity of (gu, gv) plus the
Laplace gradient of gp) is exact on direct sums (1e-12, CPU).
"""
import numpy as np
import pytest

from conftest import rel_l2

SIZES = [300, 1500, 4000, 800, 2500, 2000]


def _problems(seed=7):
    rng = np.random.default_rng(seed)
    probs, forces, cots = [], [], []
    for n in SIZES:
        probs.append((rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)))
        forces.append((rng.standard_normal(n), rng.standard_normal(n)))
        cots.append((rng.standard_normal(n), rng.standard_normal(n), rng.standard_normal(n)))
    return probs, forces, cots


def _adjoint_direct(x, y, gu, gv, gp):
    from oracle.direct import direct_laplace_grad, direct_stokes
    vel = direct_stokes(x, y, gu, gv, x, y, True)
    grad = direct_laplace_grad(x, y, gp, x, y, True)
    return vel[0] + grad[1], vel[1] + grad[2]


def test_stokes_adjoint_construction_on_direct_sums():
    """<g, A f> = <A^T g, f> with A the Stokeslet self-interaction (u, v, p)
    and A^T g = Stokes velocity of (gu, gv) + Laplace gradient of gp."""
    from oracle.direct import direct_stokes
    rng = np.random.default_rng(3)
    n = 400
    x, y = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    fx, fy = rng.standard_normal(n), rng.standard_normal(n)
    gu, gv, gp = rng.standard_normal(n), rng.standard_normal(n), rng.standard_normal(n)
    u, v, p = direct_stokes(x, y, fx, fy, x, y, True)
    dfx, dfy = _adjoint_direct(x, y, gu, gv, gp)
    lhs = gu @ u + gv @ v + gp @ p
    rhs = dfx @ fx + dfy @ fy
    assert abs(lhs - rhs) <= 1e-12 * (abs(lhs) + abs(rhs))


@pytest.mark.gpu
def test_stokes_batch_forward_equals_single_problems_and_direct(built_lib):
    import torch
    from flexmm_b200.batch import StokesBatch
    from flexmm_b200.stokes import FMM
    from oracle.direct import direct_stokes
    probs, forces, _ = _problems()
    B = StokesBatch(probs, Nequiv=32, Ncutoff=64, n_streams=4)
    outs = B.forward(forces)
    torch.cuda.synchronize()
    B.status()
    for k, ((x, y), (fx, fy)) in enumerate(zip(probs, forces)):
        got = [t.cpu().numpy() for t in outs[k]]
        # the same problem alone, with the operators it was created with
        F = FMM(x, y, 32, 64, None, precomputations=B._stokes[k].input_precomputations)
        assert list(F.bbox) == list(B._stokes[k].bbox)
        F.build_expansions(fx, fy)
        alone = F.evaluate_to_points(x, y, True)
        ds = direct_stokes(x, y, fx, fy, x, y, True)
        for r in range(3):
            assert rel_l2(got[r], alone[r]) < 1e-12, (k, r)
            assert rel_l2(got[r], ds[r]) < 1e-3, (k, r)


@pytest.mark.gpu
def test_stokes_batch_adjoint_matches_direct_adjoint(built_lib):
    import torch
    from flexmm_b200.batch import StokesBatch
    probs, forces, cots = _problems(seed=11)
    B = StokesBatch(probs, Nequiv=32, Ncutoff=64, n_streams=3)
    outs = B.adjoint(cots)
    torch.cuda.synchronize()
    B.status()
    for k, ((x, y), (gu, gv, gp)) in enumerate(zip(probs, cots)):
        dfx, dfy = (t.cpu().numpy() for t in outs[k])
        ex, ey = _adjoint_direct(x, y, gu, gv, gp)
        assert rel_l2(dfx, ex) < 1e-3 and rel_l2(dfy, ey) < 1e-3, k
    # a second forward after the adjoint reuses the same plans
    again = B.forward(forces)
    torch.cuda.synchronize()
    assert all(np.isfinite(t.cpu().numpy()).all() for tup in again for t in tup)


@pytest.mark.gpu
def test_stokes_batch_reads_forces_made_on_the_callers_stream(built_lib):
    """Forces produced by GPU kernels on the caller's stream immediately before
    the call (and dropped right after it): the batch streams wait for them."""
    import torch
    from flexmm_b200.batch import StokesBatch
    probs, forces, _ = _problems(seed=5)
    B = StokesBatch(probs, Nequiv=32, Ncutoff=64, n_streams=4)
    ref = B.forward(forces)
    torch.cuda.synchronize()
    ref = [[t.cpu().numpy() for t in tup] for tup in ref]
    big = torch.empty(64 * 1024 * 1024, dtype=torch.float64, device="cuda")
    dev = []
    for fx, fy in forces:
        big.normal_()  # keeps the caller's stream busy ahead of the copies below
        a = torch.from_numpy(fx).cuda(non_blocking=True) * 2.0 - torch.from_numpy(fx).cuda()
        b = torch.from_numpy(fy).cuda() + 0.0
        dev.append((a, b))
    outs = B.forward(dev)
    del dev
    torch.cuda.synchronize()
    for k in range(len(probs)):
        for r in range(3):
            assert rel_l2(outs[k][r].cpu().numpy(), ref[k][r]) < 1e-14, (k, r)


@pytest.mark.gpu
def test_stokes_batch_graph_replay_equals_eager(built_lib):
    """The whole batch captured as one CUDA graph (forward and adjoint):
    replays with new inputs equal the eager calls."""
    import torch
    from flexmm_b200.batch import StokesBatch
    probs, forces, cots = _problems(seed=21)
    B = StokesBatch(probs, Nequiv=24, Ncutoff=64, n_streams=4)
    gf = B.graph("forward")
    ga = B.graph("adjoint")
    for seed in (1, 2):
        rng = np.random.default_rng(seed)
        f = [(rng.standard_normal(x.size), rng.standard_normal(x.size)) for x, _ in probs]
        c = [tuple(rng.standard_normal(x.size) for _ in range(3)) for x, _ in probs]
        want_f = [[t.cpu().numpy() for t in tup] for tup in B.forward(f)]
        want_a = [[t.cpu().numpy() for t in tup] for tup in B.adjoint(c)]
        dev = lambda a: torch.from_numpy(a).cuda()
        got_f = gf.replay([tuple(dev(v) for v in tup) for tup in f])
        got_f = [[t.cpu().numpy() for t in tup] for tup in got_f]
        got_a = ga.replay([tuple(dev(v) for v in tup) for tup in c])
        got_a = [[t.cpu().numpy() for t in tup] for tup in got_a]
        torch.cuda.synchronize()
        B.status()
        for k in range(len(probs)):
            for r in range(3):
                assert rel_l2(got_f[k][r], want_f[k][r]) < 1e-14, (seed, k, r)
            for r in range(2):
                assert rel_l2(got_a[k][r], want_a[k][r]) < 1e-14, (seed, k, r)
