"""Host-side logic of flexmm_b200 (no GPU): kernel registry, operators, bbox snapping."""
import numpy as np
import pytest

from flexmm_b200 import helpers, kernels
from oracle.kifmm import Precomputation, snap_bbox
from oracle.kernels import laplace


def test_kernel_registry_accepts_reference_style_functions():
    def Laplace_Eval(sx, sy, tx, ty):  # a user's own function, like the reference's examples
        return 0.0
    k = kernels.resolve(Laplace_Eval)
    assert k.name == "Laplace_Eval" and k.kernel_id == 0
    assert kernels.resolve("Laplace_Eval").key == k.key
    with pytest.raises(ValueError):
        kernels.resolve("NotAKernel")


@pytest.mark.parametrize("neq", [16, 24, 32, 40, 60])
def test_operators_match_oracle_precomputation(neq):
    k = kernels.Laplace()
    w = 2.0 / 2 ** 5
    P = helpers.KIPrecomputation(w, neq, k)
    O = Precomputation(w, neq, laplace)
    assert np.array_equal(P.large_x, O.large_x) and np.array_equal(P.large_y, O.large_y)
    assert np.array_equal(P.m2mc, O.M2MC)
    # same compression decision and factors as M2L_Evaluator, offset by offset
    for o, (ox, oy) in enumerate(helpers.offsets()):
        op = O.M2LF[(ox + 3, oy + 3)]
        r = P.m2l_rank[o]
        if op.kind == "dense":
            assert r == -1 and np.array_equal(P.m2l_a[o], op.m2l)
        elif op.kind == "svd":
            assert r == op.rank
            assert np.array_equal(P.m2l_a[o], op.M2) and np.array_equal(P.m2l_b[o], op.M1)
        else:
            assert r == 0
    # the factored check-to-equivalent solve and LU give the same far field
    # for the check potential of sources inside the box
    import scipy.linalg
    rng = np.random.default_rng(0)
    sx, sy = rng.uniform(-w / 2, w / 2, (2, 50))
    tau = rng.standard_normal(50)
    b = laplace(sx[None, :], sy[None, :], O.large_x[:, None], O.large_y[:, None]) @ tau
    x_lu = scipy.linalg.lu_solve(O.S2L_LU, b)
    x_svd = P.c2e_vh.T @ (P.c2e_sinv * (P.c2e_u.T @ b))
    th = rng.uniform(0, 2 * np.pi, 40)
    fx, fy = 3 * w * np.cos(th), 3 * w * np.sin(th)
    far = lambda x: laplace(O.small_x[None, :], O.small_y[None, :], fx[:, None], fy[:, None]) @ x
    exact = laplace(sx[None, :], sy[None, :], fx[:, None], fy[:, None]) @ tau
    assert np.linalg.norm(far(x_svd) - far(x_lu)) / np.linalg.norm(exact) < 1e-12


def test_offsets_order_is_ox_major():
    offs = helpers.offsets()
    assert len(offs) == 40 and offs[0] == (-3, -3) and offs[-1] == (3, 3)
    assert all(max(abs(a), abs(b)) >= 2 for a, b in offs)


@pytest.mark.parametrize("bbox,widths", [
    ([-1, 1, -1, 1], []),
    ([-0.3, 0.2, -0.1, 0.35], [2.0, 1.0, 0.5, 0.25]),
    ([0, 3, 0, 1], [0.125]),
])
def test_bbox_snapping_matches_reference_rule(bbox, widths):
    h = helpers.KI_Helper()
    for w in widths:
        h.precomputations[helpers.width_key(w)] = object()
    got = h.get_bbox(None, None, bbox)
    want = snap_bbox(None, None, bbox, np.array(widths, dtype=float))
    assert np.array_equal(np.array(got), np.array(want))


def test_helper_rejects_other_kernel_or_nequiv():
    h = helpers.KI_Helper()
    h.attach(kernels.Laplace(), 24)
    h.attach(kernels.Laplace(), 24)
    with pytest.raises(ValueError):
        h.attach(kernels.Laplace(), 32)


def test_registered_kernel_names_of_the_reference():
    """Every kernel of the reference's examples resolves by its name:
    Laplace_Eval, Modified_Helmholtz_Eval, the Struve example's Kernel, and
    the Stokeslet (whose FMM is the Stokes FMM class)."""
    import numpy as np
    from flexmm_b200.kernels import KERNEL_STOKES, _BY_NAME, resolve, struve_gf
    assert resolve("Laplace_Eval").name == "Laplace_Eval"
    assert resolve("Modified_Helmholtz_Eval", helmholtz_k=10.0).params[0] == 10.0
    assert {"Laplace_Eval", "Modified_Helmholtz_Eval", "Kernel", "Stokes"} <= set(_BY_NAME)
    st = resolve("Stokes")
    assert st.vector and st.kernel_id == KERNEL_STOKES
    # the Stokeslet's host rows against the reference's formulas at one pair
    dx, dy = 0.3, -0.7
    d2 = dx * dx + dy * dy
    rows = st.host(0.0, 0.0, dx, dy)
    assert np.isclose(rows[0, 0], (-0.5 * np.log(d2) + dx * dx / d2) / (4 * np.pi))
    assert np.isclose(rows[2, 1], dy / d2 / (2 * np.pi))
    # GF through scipy bridges scipy's NaN intervals
    r = np.array([0.5, 25.8463, 27.329, 28.995, 100.0])
    assert np.all(np.isfinite(struve_gf(r)))
