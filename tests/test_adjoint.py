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
    import torch
    from flexmm_b200.autograd import fmm_potential
    from oracle.direct import direct_laplace, direct_laplace_grad
    sx, sy, tau, tx, ty, uref = _problem()
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


def test_adjoint_matches_central_differences(built_lib):
    """Central differences h = 1e-6 on a few source and target coordinates
    (the tree is rebuilt at each perturbed point; no point crosses a box
    boundary at this h for this seed)."""
    import torch
    from flexmm_b200.autograd import fmm_potential
    sx, sy, tau, tx, ty, uref = _problem(n=3000, m=1000, seed=4)
    kw = dict(method="bb", Ncutoff=64, p=16, bbox=[-1, 1, -1, 1])
    ur = torch.tensor(uref, device="cuda")

    def loss_of(a):
        u = fmm_potential(*[torch.tensor(v, dtype=torch.float64, device="cuda") for v in a], **kw)
        return 0.5 * float(((u - ur) ** 2).sum())
    vs = [torch.tensor(v, dtype=torch.float64, device="cuda", requires_grad=True) for v in (sx, sy, tau, tx, ty)]
    u = fmm_potential(*vs, **kw)
    (0.5 * ((u - ur) ** 2).sum()).backward()
    rng = np.random.default_rng(0)
    h = 1e-6
    for which in (0, 1, 2, 3, 4):
        base = [v.copy() for v in (sx, sy, tau, tx, ty)]
        for k in rng.choice(base[which].size, 4, replace=False):
            plus = [v.copy() for v in base]
            minus = [v.copy() for v in base]
            plus[which][k] += h
            minus[which][k] -= h
            fd = (loss_of(plus) - loss_of(minus)) / (2 * h)
            an = float(vs[which].grad[k])
            assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (which, k, fd, an)
