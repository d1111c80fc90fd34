"""Differentiation form: gradients of L = 0.5 ||u - u_ref||^2 through the
transposed FMM, against FP64 direct-sum gradients and central differences
(the configuration: Laplace black-box FMM, Chebyshev order 16)."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _problem(n=6000, m=2500, seed=3):
    rng = np.random.default_rng(seed)
    return (rng.uniform(-1, 1, n), rng.uniform(-1, 1, n), rng.standard_normal(n),
            rng.uniform(-1, 1, m), rng.uniform(-1, 1, m), rng.standard_normal(m))


@pytest.mark.parametrize("method", ["bb", "kifmm"])
def test_adjoint_gradients_match_direct_sum(built_lib, method):
    """N = 20,000 sources, 10,000 targets: every gradient against its FP64
    direct-sum value (bar 1e-8 relative L2)."""
    import torch
    from flexmm_b200.autograd import fmm_potential
    from oracle.direct import direct_laplace, direct_laplace_grad
    sx, sy, tau, tx, ty, uref = _problem(n=20_000, m=10_000)
    T = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda", requires_grad=True)
    vs = [T(a) for a in (sx, sy, tau, tx, ty)]
    kw = dict(method=method, Ncutoff=64, p=16, Nequiv=60, bbox=[-1, 1, -1, 1])
    u = fmm_potential(*vs, **kw)
    loss = 0.5 * ((u - torch.tensor(uref, device="cuda")) ** 2).sum()
    loss.backward()
    got = [v.grad.cpu().numpy() for v in vs]
    # FP64 direct sums
    ud = direct_laplace(sx, sy, tau, tx, ty, False)
    r = ud - uref
    Gs = direct_laplace_grad(tx, ty, r, sx, sy, False)   # field of charges r at the sources
    Gt = direct_laplace_grad(sx, sy, tau, tx, ty, False)  # forward field's gradient at the targets
    ref = [tau * Gs[1], tau * Gs[2], Gs[0], r * Gt[1], r * Gt[2]]
    assert rel_l2(u.detach().cpu().numpy(), ud) < 1e-11
    for name, a, b in zip(["sx", "sy", "tau", "tx", "ty"], got, ref):
        assert rel_l2(a, b) < 1e-8, (name, rel_l2(a, b))


def test_adjoint_matches_central_differences_frozen_tree(built_lib):
    """Central differences h = 1e-6 on 50 random coordinates (sources,
    charges, targets), the trees frozen (FMMPotential: perturbed points are
    moved inside the trees built at the start).  The loss difference is
    formed as L+ - L- = 0.5 sum (u+ - u-)(u+ + u- - 2 u_ref), an identity
    that avoids cancelling two losses of ~1e6, and the central differences
    at h and 2h are Richardson-extrapolated, (4 D(h) - D(2h)) / 3: a target
    a distance d from a source has a central-difference error ~h^2 / d^3,
    1e-4 relative at d ~ 1e-3, which the extrapolation removes.  Bar per
    coordinate: 1e-5 max(1, |g|)."""
    import torch
    from flexmm_b200.autograd import FMMPotential
    sx, sy, tau, tx, ty, uref = _problem(n=20_000, m=10_000, seed=4)
    kw = dict(method="bb", Ncutoff=64, p=16, bbox=[-1, 1, -1, 1])
    ur = torch.tensor(uref, device="cuda")
    D = lambda a, g=False: torch.tensor(a, dtype=torch.float64, device="cuda", requires_grad=g)
    P = FMMPotential(D(sx), D(sy), D(tx), D(ty), **kw)

    def u_of(a):
        with torch.no_grad():
            return P(*[D(v) for v in a])
    vs = [D(v, True) for v in (sx, sy, tau, tx, ty)]
    u = P(*vs)
    (0.5 * ((u - ur) ** 2).sum()).backward()
    rng = np.random.default_rng(0)
    h = 1e-6
    base = [v.copy() for v in (sx, sy, tau, tx, ty)]
    picks = [(int(w), int(rng.integers(base[w].size))) for w in rng.integers(0, 5, 50)]
    assert len(picks) == 50
    def central(which, k, step):
        plus = [v.copy() for v in base]
        minus = [v.copy() for v in base]
        plus[which][k] += step
        minus[which][k] -= step
        up, um = u_of(plus), u_of(minus)
        return float((0.5 * (up - um) * (up + um - 2 * ur)).sum()) / (2 * step)
    for which, k in picks:
        fd = (4 * central(which, k, h) - central(which, k, 2 * h)) / 3
        an = float(vs[which].grad[k])
        assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (which, k, fd, an)


def test_backward_recomputes_expansions(built_lib):
    """The forward FMM keeps its tree and releases its expansions; the
    backward forms them again (the gradients stay those of the direct sum)."""
    import torch
    from flexmm_b200.autograd import _FMMPotential, _Trees, _make
    sx, sy, tau, tx, ty, uref = _problem(n=5000, m=2000, seed=6)
    T = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda", requires_grad=True)
    vs = [T(a) for a in (sx, sy, tau, tx, ty)]
    trees = _Trees(_make("bb", "Laplace_Eval", 64, 32, 16, [-1, 1, -1, 1], {}))
    u = _FMMPotential.apply(*vs, trees)
    assert trees.F is not None and not trees.F._expanded   # tree kept, expansions released
    assert trees.A is None                                 # the adjoint tree comes in backward
    (u * torch.tensor(uref, device="cuda")).sum().backward()
    assert not trees.F._expanded and not trees.A._expanded
    from oracle.direct import direct_laplace_grad
    Gt = direct_laplace_grad(sx, sy, tau, tx, ty, False)
    assert rel_l2(vs[3].grad.cpu().numpy(), uref * Gt[1]) < 1e-8
