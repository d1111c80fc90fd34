"""Generate the golden fixtures by running the reference flexmm itself.

Run in a container that has the reference checkout (it is copied into
``oracle/_ref`` and imported with host shims by ``oracle.refimport``):

    python tests/golden/make_golden.py            # all cases
    python tests/golden/make_golden.py small      # only the quick ones
    python tests/golden/make_golden.py tree-digests   # reference tree digests of the large cases

For every case the inputs are regenerated from ``flexmm_b200.workloads``
recipes (seeded numpy), the reference ``KI_FMM`` is built with a fresh
``KI_Helper`` (never the shared default helper), and the fixture stores:

* ``meta``      the case description (recipe, seed, sizes, Ncutoff, Nequiv, bbox)
* ``inputs_sha`` sha256 of the input arrays, so drift of the generator is caught
* ``src_idx`` / ``src_val``  source-evaluation results (all, or a seeded sample)
* ``tgt_idx`` / ``tgt_val``  target-evaluation results (all, or a seeded sample)
* ``direct_src`` / ``direct_tgt`` FP64 direct sums at the sampled points
* ``tree_sha``  sha256 of every canonical tree array of the reference tree
  (``tests/canon.py``), for cases small enough to canonicalise quickly
* ``tree_sha_nonempty`` (the sampled 100k / 1M cases) the same digests of the
  reference's tree with interactions from empty source boxes left out

Gradient cases (``grad_*``) run the reference's kifmm2d FMM with the
gradient evaluator of examples/pure_kifmm_laplace_gradient.py
(``register_evaluator(..., 'gradient', 3)`` + ``evaluate_to_points``) and store
``src_val`` / ``tgt_val`` as [3, n] rows (u, du/dx, du/dy), with the FP64
direct sums ``direct_src`` / ``direct_tgt`` likewise.
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.dirname(HERE))

from flexmm_b200 import workloads  # noqa: E402
from oracle import refimport  # noqa: E402
from oracle.direct import (direct_laplace, direct_laplace_grad, direct_mod_helmholtz,  # noqa: E402
                           direct_mod_helmholtz_grad, direct_radial, direct_stokes, struve_gf)
import canon  # noqa: E402


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def case_inputs(meta):
    kind = meta["recipe"]
    if kind == "uniform":
        d = workloads.uniform(n=meta["n"], n_grid=meta["n_grid"], seed=meta["seed"])
    elif kind == "clustered":
        d = workloads.clustered(n=meta["n"], n_grid=meta["n_grid"], seed=meta["seed"])
    elif kind == "circle":
        d = workloads.circle(n=meta["n"], n_rhs=1, seed=meta["seed"])
        d["tau"] = d["tau"][0]
        g = np.linspace(-0.45, 0.45, meta["n_grid"])
        gx, gy = np.meshgrid(g, g)
        d["tx"], d["ty"] = gx.ravel(), gy.ravel()
    elif kind == "square100":  # the Struve example's layout, examples/bbfmm_struve.py:48-53
        rng = np.random.default_rng(meta["seed"])
        n = meta["n"]
        x, y = rng.uniform(0, 100, n), rng.uniform(0, 100, n)
        tau = rng.uniform(0, 1, n)
        g = np.linspace(0, 100, meta["n_grid"])
        gx, gy = np.meshgrid(g, g)
        d = dict(x=x, y=y, tau=tau, tx=gx.ravel(), ty=gy.ravel(), bbox=[-10.0, 110.0, -10.0, 110.0])
    elif kind == "duplicates":
        rng = np.random.default_rng(meta["seed"])
        n = meta["n"]
        x = rng.uniform(-1, 1, n)
        y = rng.uniform(-1, 1, n)
        # every fifth point is repeated once: coincident sources
        x[1::5] = x[0::5][: x[1::5].size]
        y[1::5] = y[0::5][: y[1::5].size]
        tau = rng.standard_normal(n)
        tx, ty = workloads.grid(meta["n_grid"])
        d = dict(x=x, y=y, tau=tau, tx=tx, ty=ty, bbox=[-1.0, 1.0, -1.0, 1.0])
    else:
        raise ValueError(kind)
    if meta.get("bbox", "given") == "none":
        d["bbox"] = None
    if meta.get("method") == "stokes":  # second force component
        d["tau2"] = np.random.default_rng(meta["seed"] + 1000).standard_normal(d["x"].size)
    if meta.get("stresslet"):  # double-layer strengths and unit normals of the Stokes FMM
        r4 = np.random.default_rng(meta["seed"] + 4000)
        d["sgx"], d["sgy"] = r4.standard_normal(d["x"].size), r4.standard_normal(d["x"].size)
        th = r4.uniform(0, 2 * np.pi, d["x"].size)
        d["nx"], d["ny"] = np.cos(th), np.sin(th)
    if meta.get("local") in ("category", "periodic"):  # source and target categories
        r3 = np.random.default_rng(meta["seed"] + 3000)
        d["cat"] = r3.integers(0, meta["ncat"], d["x"].size)
        d["tcat"] = r3.integers(0, meta["ncat"], d["tx"].size)
    if meta.get("dipole"):  # double-layer strengths and unit normals
        r2 = np.random.default_rng(meta["seed"] + 2000)
        d["dlp"] = r2.standard_normal(d["x"].size)
        th = r2.uniform(0, 2 * np.pi, d["x"].size)
        d["nx"], d["ny"] = np.cos(th), np.sin(th)
    return d


CASES = {
    # name: (meta, small)
    "uniform_3k_q16": (dict(recipe="uniform", seed=10, n=3000, n_grid=41, ncut=16, neq=16), True),
    "uniform_100_q16": (dict(recipe="uniform", seed=11, n=100, n_grid=9, ncut=16, neq=16), True),
    "clustered_20k_q32": (dict(recipe="clustered", seed=12, n=20000, n_grid=64, ncut=32, neq=32), True),
    "clustered_20k_q60": (dict(recipe="clustered", seed=13, n=20000, n_grid=64, ncut=64, neq=60), True),
    "circle_20k_q24_nobbox": (dict(recipe="circle", seed=14, n=20000, n_grid=50, ncut=32, neq=24,
                                   bbox="none"), True),
    "duplicates_5k_q24": (dict(recipe="duplicates", seed=15, n=5000, n_grid=33, ncut=16, neq=24), True),
    "grad_uniform_3k_q16": (dict(recipe="uniform", seed=16, n=3000, n_grid=41, ncut=16, neq=16,
                                 gradient=True), True),
    "grad_clustered_20k_q32": (dict(recipe="clustered", seed=17, n=20000, n_grid=64, ncut=32,
                                    neq=32, gradient=True), True),
    "grad_duplicates_5k_q24": (dict(recipe="duplicates", seed=18, n=5000, n_grid=33, ncut=16,
                                    neq=24, gradient=True), True),
    "mh_uniform_3k_q24_k5": (dict(recipe="uniform", seed=19, n=3000, n_grid=41, ncut=16, neq=24,
                                  kernel="mh", k=5.0), True),
    "mh_circle_20k_q40_k10": (dict(recipe="circle", seed=20, n=20000, n_grid=50, ncut=64, neq=40,
                                   kernel="mh", k=10.0, bbox="none"), True),
    "mh_duplicates_5k_q24_k5": (dict(recipe="duplicates", seed=21, n=5000, n_grid=33, ncut=16,
                                     neq=24, kernel="mh", k=5.0), True),
    "grad_mh_clustered_20k_q32_k5": (dict(recipe="clustered", seed=22, n=20000, n_grid=64, ncut=32,
                                          neq=32, kernel="mh", k=5.0, gradient=True), True),
    "bb_uniform_3k_p8": (dict(recipe="uniform", seed=23, n=3000, n_grid=41, ncut=32, neq=64,
                              method="bb", p=8), True),
    "bb_clustered_20k_p12": (dict(recipe="clustered", seed=24, n=20000, n_grid=64, ncut=64, neq=144,
                                  method="bb", p=12), True),
    "bb_uniform_10k_p16": (dict(recipe="uniform", seed=25, n=10000, n_grid=50, ncut=64, neq=256,
                                method="bb", p=16), True),
    "bb_mh_duplicates_5k_p10_k5": (dict(recipe="duplicates", seed=26, n=5000, n_grid=33, ncut=32,
                                        neq=100, method="bb", p=10, kernel="mh", k=5.0), True),
    "bb_struve_square_5k_p12": (dict(recipe="square100", seed=27, n=5000, n_grid=41, ncut=30,
                                     neq=144, method="bb", p=12, kernel="struve"), True),
    "stokes_uniform_3k_q16": (dict(recipe="uniform", seed=28, n=3000, n_grid=41, ncut=16, neq=16,
                                   method="stokes"), True),
    "stokes_clustered_20k_q32": (dict(recipe="clustered", seed=29, n=20000, n_grid=64, ncut=64,
                                      neq=32, method="stokes"), True),
    "stokes_duplicates_5k_q24": (dict(recipe="duplicates", seed=30, n=5000, n_grid=33, ncut=16,
                                      neq=24, method="stokes"), True),
    "dip_uniform_5k_q24": (dict(recipe="uniform", seed=31, n=5000, n_grid=41, ncut=32, neq=24,
                                dipole=True), True),
    "dip_clustered_20k_q32": (dict(recipe="clustered", seed=32, n=20000, n_grid=64, ncut=64,
                                   neq=32, dipole=True), True),
    "dip_duplicates_5k_q24": (dict(recipe="duplicates", seed=33, n=5000, n_grid=33, ncut=16,
                                   neq=24, dipole=True), True),
    "local_uniform_20k": (dict(recipe="uniform", seed=34, n=20000, n_grid=64, ncut=20,
                               local="plain", delta=2.0 ** -5), True),
    "local_cat_clustered_20k": (dict(recipe="clustered", seed=35, n=20000, n_grid=64, ncut=20,
                                     local="category", delta=2.0 ** -5, ncat=7), True),
    "local_periodic_10k": (dict(recipe="uniform", seed=36, n=10000, n_grid=50, ncut=20,
                                local="periodic", delta=2.0 ** -4, ncat=5), True),
    "sdip_uniform_3k_q16": (dict(recipe="uniform", seed=37, n=3000, n_grid=41, ncut=16, neq=16,
                                 method="stokes", stresslet=True), True),
    "sdip_clustered_20k_q32": (dict(recipe="clustered", seed=38, n=20000, n_grid=64, ncut=64,
                                    neq=32, method="stokes", stresslet=True), True),
    "uniform_100k_q32": (dict(recipe="uniform", seed=0, n=100000, n_grid=316, ncut=64, neq=32,
                              sample=2000), False),
    "clustered_1M_q60": (dict(recipe="clustered", seed=1, n=1000000, n_grid=1000, ncut=64, neq=60,
                              sample=2000), False),
    "clustered_1M_q24": (dict(recipe="clustered", seed=1, n=1000000, n_grid=1000, ncut=64, neq=24,
                              sample=2000), False),
}


def scipy_bessel():
    """numba-callable K0, K1 from scipy.special.cython_special (the reference's
    examples tabulate the same functions with function_generator, which is
    not installed)."""
    import ctypes
    from numba.extending import get_cython_function_address
    f = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.c_double)
    return (f(get_cython_function_address("scipy.special.cython_special", "k0")),
            f(get_cython_function_address("scipy.special.cython_special", "k1")))


def reference_kernel(meta):
    """The reference example's scalar kernel for the case (numba)."""
    import numba
    if meta.get("kernel", "laplace") == "laplace":
        @numba.njit(fastmath=True)
        def Laplace_Eval(sx, sy, tx, ty):
            dx = tx - sx
            dy = ty - sy
            d2 = dx**2 + dy**2
            return -np.log(d2) / (4 * np.pi)
        return Laplace_Eval
    if meta["kernel"] == "struve":
        import ctypes
        from numba.extending import get_cython_function_address
        st = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.c_double, ctypes.c_double)(
            get_cython_function_address("scipy.special.cython_special", "struve"))
        y1 = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.c_double)(
            get_cython_function_address("scipy.special.cython_special", "y1"))

        # examples/bbfmm_struve.py:29-46, GF from scipy instead of function_generator
        @numba.njit(fastmath=True)
        def Kernel(sx, sy, tx, ty):
            dx = tx - sx
            dy = ty - sy
            d = np.sqrt(dx**2 + dy**2)
            return (d * (y1(d) - st(-3.0, d)) - 4 * st(-2.0, d)) / d**2
        return Kernel
    k0c, _ = scipy_bessel()
    hk = float(meta["k"])

    # examples/kifmm_modified_helmholtz.py:33-39
    @numba.njit(fastmath=True)
    def Modified_Helmholtz_Eval(sx, sy, tx, ty):
        dx = tx - sx
        dy = ty - sy
        d = np.sqrt(dx**2 + dy**2)
        return k0c(hk * d) / (2 * np.pi)
    return Modified_Helmholtz_Eval


def direct(meta, grad, *args):
    if meta.get("kernel", "laplace") == "laplace":
        return (direct_laplace_grad if grad else direct_laplace)(*args)
    if meta["kernel"] == "struve":
        return direct_radial(struve_gf, *args)
    sx, sy, tau, tx, ty, check = args
    f = direct_mod_helmholtz_grad if grad else direct_mod_helmholtz
    return f(sx, sy, tau, tx, ty, meta["k"], check)


def run_case(name, meta, ref):
    from flexmm.flexmm2d.kifmm import KI_FMM, KI_Helper
    Laplace_Eval = reference_kernel(meta)
    if meta.get("method") == "bb":  # black-box FMM, flexmm/flexmm2d/bbfmm.py:212-231
        from flexmm.flexmm2d.bbfmm import BB_FMM, BB_Helper

        def KI_FMM(x, y, kernel, ncut, neq, bbox, helper):  # noqa: F811
            return BB_FMM(x, y, kernel, ncut, meta["p"], bbox=bbox, helper=BB_Helper())
        KI_Helper = type(None)  # noqa: F811

    d = case_inputs(meta)
    t0 = time.time()
    F = KI_FMM(d["x"], d["y"], Laplace_Eval, meta["ncut"], meta["neq"], bbox=d["bbox"],
               helper=KI_Helper())
    F.build_expansions(d["tau"])
    us = F.source_evaluation(d["x"], d["y"])
    ut = F.target_evaluation(d["tx"], d["ty"])
    t1 = time.time()
    rng = np.random.default_rng(12345)
    if "sample" in meta:
        si = np.sort(rng.choice(d["x"].size, meta["sample"], replace=False))
        ti = np.sort(rng.choice(d["tx"].size, meta["sample"], replace=False))
    else:
        si = np.arange(d["x"].size)
        ti = np.arange(d["tx"].size)
    ds = direct(meta, False, d["x"], d["y"], d["tau"], d["x"][si], d["y"][si], True)
    dt = direct(meta, False, d["x"], d["y"], d["tau"], d["tx"][ti], d["ty"][ti], False)
    out = dict(
        meta=json.dumps(meta),
        inputs_sha=sha(d["x"], d["y"], d["tau"], d["tx"], d["ty"]),
        bbox_used=np.array(F.bbox, dtype=np.float64),
        levels=np.int64(F.tree.levels),
        src_idx=si, src_val=us[si], tgt_idx=ti, tgt_val=ut[ti],
        direct_src=ds, direct_tgt=dt,
    )
    if "sample" not in meta:
        c = canon.canonical(F.tree)
        out["tree_sha"] = json.dumps({k: sha(np.asarray(v, dtype=np.int64)) for k, v in c.items()})
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    rel = lambda a, b: np.linalg.norm(a - b) / np.linalg.norm(b)
    print(f"{name}: levels {F.tree.levels} ref {t1 - t0:.1f}s  err vs direct src {rel(us[si], ds):.2e} "
          f"tgt {rel(ut[ti], dt):.2e}", flush=True)


def run_gradient_case(name, meta, ref):
    import numba
    from flexmm.kifmm2d.scalar.fmm import FMM

    Eval = reference_kernel(meta)
    if meta.get("kernel", "laplace") == "laplace":
        # examples/pure_kifmm_laplace_gradient.py:32-55
        @numba.njit(fastmath=True)
        def Gradient_Eval1(sx, sy, tx, ty, tau, extras):
            dx = tx - sx
            dy = ty - sy
            d2 = dx * dx + dy * dy
            id2 = 1.0 / d2
            scale = -1.0 / (2 * np.pi)
            return -np.log(d2) / (4 * np.pi) * tau, scale * dx * id2 * tau, scale * dy * id2 * tau

        @numba.njit(fastmath=True)
        def Gradient_Eval2(sx, sy, tx, ty, tau, extras):
            dx = tx - sx
            dy = ty - sy
            d2 = dx * dx + dy * dy
            id2 = 1.0 / d2
            scale = -1.0 / (2 * np.pi)
            return (-np.log(d2) / (4 * np.pi) * tau[0], scale * dx * id2 * tau[0],
                    scale * dy * id2 * tau[0])
    else:
        k0c, k1c = scipy_bessel()
        hk = float(meta["k"])

        # examples/pure_kifmm_modified_helmholtz_gradient.py:45-70
        @numba.njit(fastmath=True)
        def Gradient_Eval1(sx, sy, tx, ty, tau, extras):
            dx = tx - sx
            dy = ty - sy
            d = np.sqrt(dx**2 + dy**2)
            scale = 1.0 / (2 * np.pi)
            g = -hk * k1c(hk * d) * scale / d * tau
            return k0c(hk * d) * scale * tau, dx * g, dy * g

        @numba.njit(fastmath=True)
        def Gradient_Eval2(sx, sy, tx, ty, tau, extras):
            dx = tx - sx
            dy = ty - sy
            d = np.sqrt(dx**2 + dy**2)
            scale = 1.0 / (2 * np.pi)
            g = -hk * k1c(hk * d) * scale / d * tau[0]
            return k0c(hk * d) * scale * tau[0], dx * g, dy * g

    d = case_inputs(meta)
    t0 = time.time()
    F = FMM(d["x"], d["y"], Eval, meta["ncut"], meta["neq"], bbox=d["bbox"])
    F.build_expansions(d["tau"])
    F.register_evaluator(Gradient_Eval1, Gradient_Eval2, "gradient", 3)
    us = F.evaluate_to_points(d["x"], d["y"], "gradient", True)
    ut = F.evaluate_to_points(d["tx"], d["ty"], "gradient", False)
    t1 = time.time()
    si = np.arange(d["x"].size)
    ti = np.arange(d["tx"].size)
    ds = direct(meta, True, d["x"], d["y"], d["tau"], d["x"], d["y"], True)
    dt = direct(meta, True, d["x"], d["y"], d["tau"], d["tx"], d["ty"], False)
    out = dict(
        meta=json.dumps(meta),
        inputs_sha=sha(d["x"], d["y"], d["tau"], d["tx"], d["ty"]),
        bbox_used=np.array(F.bbox, dtype=np.float64),
        levels=np.int64(F.tree.levels),
        src_idx=si, src_val=us, tgt_idx=ti, tgt_val=ut,
        direct_src=ds, direct_tgt=dt,
    )
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    rel = lambda a, b: np.linalg.norm(a - b) / np.linalg.norm(b)
    print(f"{name}: levels {F.tree.levels} ref {t1 - t0:.1f}s  err vs direct "
          + " ".join(f"src[{r}] {rel(us[r], ds[r]):.2e} tgt[{r}] {rel(ut[r], dt[r]):.2e}" for r in range(3)),
          flush=True)


def run_dipole_case(name, meta, ref):
    """Single plus double layer through the reference's kifmm2d FMM, as
    examples/pure_kifmm_laplace_dipoles.py:94-98 drives it: the upwardor and
    the evaluator Laplace_Both_Eval, tau = [slp, dlp], extras = normals."""
    import numba
    from flexmm.kifmm2d.scalar.fmm import FMM
    Laplace_Eval = reference_kernel(meta)

    # examples/pure_kifmm_laplace_dipoles.py:31-40
    @numba.njit(fastmath=True)
    def Laplace_Both_Eval(sx, sy, tx, ty, tau, extras):
        nx = extras[0]
        ny = extras[1]
        dx = tx - sx
        dy = ty - sy
        n_dot_d = nx * dx + ny * dy
        d2 = dx * dx + dy * dy
        return (-np.log(d2) / (4 * np.pi) * tau[0] + n_dot_d / d2 / (2 * np.pi) * tau[1],)

    d = case_inputs(meta)
    tau = np.vstack([d["tau"], d["dlp"]])
    dipvec = np.vstack([d["nx"], d["ny"]])
    t0 = time.time()
    F = FMM(d["x"], d["y"], Laplace_Eval, meta["ncut"], meta["neq"], bbox=d["bbox"])
    F.register_upwardor(Laplace_Both_Eval, "slp+dlp")
    F.register_evaluator(F.helper.functions["kernel_app"], Laplace_Both_Eval, "slp+dlp->u", 1)
    F.build_expansions(tau, "slp+dlp", dipvec)
    us = F.evaluate_to_points(d["x"], d["y"], "slp+dlp->u", True)[0]
    ut = F.evaluate_to_points(d["tx"], d["ty"], "slp+dlp->u", False)[0]
    t1 = time.time()
    from oracle.direct import direct_laplace_dipole
    ds = direct_laplace_dipole(d["x"], d["y"], d["tau"], d["dlp"], d["nx"], d["ny"], d["x"], d["y"], True)
    dt = direct_laplace_dipole(d["x"], d["y"], d["tau"], d["dlp"], d["nx"], d["ny"], d["tx"], d["ty"],
                               False)
    out = dict(
        meta=json.dumps(meta),
        inputs_sha=sha(d["x"], d["y"], d["tau"], d["tx"], d["ty"], d["dlp"], d["nx"], d["ny"]),
        bbox_used=np.array(F.bbox, dtype=np.float64),
        levels=np.int64(F.tree.levels),
        src_idx=np.arange(d["x"].size), src_val=us, tgt_idx=np.arange(d["tx"].size), tgt_val=ut,
        direct_src=ds, direct_tgt=dt,
    )
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    rel = lambda a, b: np.linalg.norm(a - b) / np.linalg.norm(b)
    print(f"{name}: levels {F.tree.levels} ref {t1 - t0:.1f}s  err vs direct src {rel(us, ds):.2e} "
          f"tgt {rel(ut, dt):.2e}", flush=True)


def local_bump(delta):
    """The test kernel of the local evaluators: (1 - r^2/delta^2)^3 for
    r < delta, else 0 (compact support of radius delta)."""
    def f(r):
        r = np.asarray(r, dtype=np.float64)
        q = 1.0 - (r / delta) ** 2
        return np.where(r < delta, q * q * q, 0.0)
    return f


def local_direct(meta, sx, sy, tau, tx, ty, check, scat=None, tcat=None):
    """FP64 direct sum of the compact bump (numpy): every source within delta."""
    f = local_bump(meta["delta"])
    out = np.zeros(tx.size)
    step = max(1, 2_000_000 // max(sx.size, 1))
    for a in range(0, tx.size, step):
        b = min(tx.size, a + step)
        dx = tx[a:b, None] - sx[None, :]
        dy = ty[a:b, None] - sy[None, :]
        w = f(np.sqrt(dx * dx + dy * dy)) * tau[None, :]
        if check:
            w = np.where((dx == 0) & (dy == 0), 0.0, w)
        if scat is not None:
            w = np.where(scat[None, :] == tcat[a:b, None], 0.0, w)
        out[a:b] = w.sum(1)
    return out


def run_local_case(name, meta, ref):
    """The reference's local evaluators (flexmm/flexmm2d/local_evaluator.py,
    local_evaluator_category.py, periodic_local_evaluator_category.py) with
    the compact bump as Kernel_Add, ncutoff and min_distance from meta."""
    import numba
    D2 = float(meta["delta"]) ** 2

    @numba.njit(fastmath=True)
    def Kernel_Add(sx, sy, tx, ty, tau, out):
        dx = tx - sx
        dy = ty - sy
        d2 = dx * dx + dy * dy
        if d2 < D2:
            q = 1.0 - d2 / D2
            out[0] += q * q * q * tau

    d = case_inputs(meta)
    n, m = d["x"].size, d["tx"].size
    kind = meta["local"]
    out_s = np.zeros((n, 1))
    out_t = np.zeros((m, 1))
    t0 = time.time()
    if kind == "plain":
        from flexmm.flexmm2d.local_evaluator import LocalEvaluator
        E = LocalEvaluator(d["x"], d["y"], Kernel_Add, meta["delta"], ncutoff=meta["ncut"])
        E.load_tau(d["tau"])
        E.source_evaluation(d["x"], d["y"], out_s)
        E.target_evaluation(d["tx"], d["ty"], out_t)
        ds = local_direct(meta, d["x"], d["y"], d["tau"], d["x"], d["y"], True)
        dt = local_direct(meta, d["x"], d["y"], d["tau"], d["tx"], d["ty"], False)
    elif kind == "category":
        from flexmm.flexmm2d.local_evaluator_category import LocalEvaluator
        E = LocalEvaluator(d["x"], d["y"], d["cat"], Kernel_Add, meta["delta"], ncutoff=meta["ncut"])
        E.load_tau(d["tau"])
        E.target_evaluation(d["x"], d["y"], d["cat"], out_s)
        E.target_evaluation(d["tx"], d["ty"], d["tcat"], out_t)
        ds = local_direct(meta, d["x"], d["y"], d["tau"], d["x"], d["y"], False, d["cat"], d["cat"])
        dt = local_direct(meta, d["x"], d["y"], d["tau"], d["tx"], d["ty"], False, d["cat"], d["tcat"])
    else:
        from flexmm.flexmm2d.periodic_local_evaluator_category import PeriodicLocalEvaluator
        bounds = [-1.0, 1.0, -1.0, 1.0]
        E = PeriodicLocalEvaluator(d["x"], d["y"], d["cat"], Kernel_Add, meta["delta"], bounds,
                                   ncutoff=meta["ncut"])
        E.load_tau(d["tau"])
        E.target_evaluation(d["x"], d["y"], d["cat"], out_s)
        E.target_evaluation(d["tx"], d["ty"], d["tcat"], out_t)
        # direct sum over the 3 x 3 periodic copies of the sources
        sx = np.concatenate([d["x"] + 2 * a for a in (-1, 0, 1) for b in (-1, 0, 1)])
        sy = np.concatenate([d["y"] + 2 * b for a in (-1, 0, 1) for b in (-1, 0, 1)])
        st, sc = np.tile(d["tau"], 9), np.tile(d["cat"], 9)
        ds = local_direct(meta, sx, sy, st, d["x"], d["y"], False, sc, d["cat"])
        dt = local_direct(meta, sx, sy, st, d["tx"], d["ty"], False, sc, d["tcat"])
    t1 = time.time()
    out = dict(
        meta=json.dumps(meta),
        inputs_sha=sha(d["x"], d["y"], d["tau"], d["tx"], d["ty"]),
        bbox_used=np.array(E.bbox, dtype=np.float64),
        levels=np.int64(getattr(getattr(E, "tree", None), "levels", 0)),
        src_idx=np.arange(n), src_val=out_s[:, 0], tgt_idx=np.arange(m), tgt_val=out_t[:, 0],
        direct_src=ds, direct_tgt=dt,
    )
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    rel = lambda a, b: np.linalg.norm(a - b) / np.linalg.norm(b)
    print(f"{name}: ref {t1 - t0:.1f}s  vs direct src {rel(out_s[:, 0], ds):.2e} "
          f"tgt {rel(out_t[:, 0], dt):.2e}", flush=True)


def run_stokes_case(name, meta, ref):
    """The reference's Stokes FMM (flexmm/kifmm2d/vector/stokes_fmm.py:592-858):
    src_val / tgt_val are [3, n] rows (u, v, p)."""
    from flexmm.kifmm2d.vector.stokes_fmm import FMM
    d = case_inputs(meta)
    t0 = time.time()
    F = FMM(d["x"], d["y"], meta["neq"], meta["ncut"], bbox=d["bbox"])
    F.precompute()
    if meta.get("stresslet"):  # build_expansions_dipole / evaluate_to_points_dipole
        from oracle.direct import direct_stokes_dipole
        F.build_expansions_dipole(d["tau"], d["tau2"], d["sgx"], d["sgy"], d["nx"], d["ny"])
        us = np.array(F.evaluate_to_points_dipole(d["x"], d["y"], True))
        ut = np.array(F.evaluate_to_points_dipole(d["tx"], d["ty"], False))
        t1 = time.time()
        srcs = (d["x"], d["y"], d["tau"], d["tau2"], d["sgx"], d["sgy"], d["nx"], d["ny"])
        ds = direct_stokes_dipole(*srcs, d["x"], d["y"], True)
        dt = direct_stokes_dipole(*srcs, d["tx"], d["ty"], False)
    else:
        F.build_expansions(d["tau"], d["tau2"])
        us = np.array(F.evaluate_to_points(d["x"], d["y"], True))
        ut = np.array(F.evaluate_to_points(d["tx"], d["ty"], False))
        t1 = time.time()
        ds = direct_stokes(d["x"], d["y"], d["tau"], d["tau2"], d["x"], d["y"], True)
        dt = direct_stokes(d["x"], d["y"], d["tau"], d["tau2"], d["tx"], d["ty"], False)
    out = dict(
        meta=json.dumps(meta),
        inputs_sha=sha(d["x"], d["y"], d["tau"], d["tx"], d["ty"]),
        bbox_used=np.array(F.bbox, dtype=np.float64),
        levels=np.int64(F.tree.levels),
        src_idx=np.arange(d["x"].size), src_val=us, tgt_idx=np.arange(d["tx"].size), tgt_val=ut,
        direct_src=ds, direct_tgt=dt,
    )
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    rel = lambda a, b: np.linalg.norm(a - b) / np.linalg.norm(b)
    print(f"{name}: levels {F.tree.levels} ref {t1 - t0:.1f}s  err vs direct "
          + " ".join(f"src[{r}] {rel(us[r], ds[r]):.2e} tgt[{r}] {rel(ut[r], dt[r]):.2e}" for r in range(3)),
          flush=True)


def add_tree_digests(name, meta, ref):
    """Canonical digests of the reference's own tree for a large (sampled)
    case, added to its existing fixture: the reference Tree alone
    (flexmm/tree.py:451-518) on the case's inputs and the bbox the reference
    FMM used.  ``tree_sha_nonempty`` keeps only interactions whose source box
    holds points (the form the device tree's lists take)."""
    from flexmm.tree import Tree
    path = os.path.join(HERE, name + ".npz")
    old = dict(np.load(path, allow_pickle=False))
    d = case_inputs(meta)
    t0 = time.time()
    T = Tree(d["x"], d["y"], meta["ncut"], list(old["bbox_used"]))
    t1 = time.time()
    assert T.levels == int(old["levels"])
    c = canon.canonical(T, nonempty_sources=True)
    old["tree_sha_nonempty"] = json.dumps({k: sha(np.asarray(v, dtype=np.int64)) for k, v in c.items()})
    np.savez_compressed(path, **old)
    print(f"{name}: reference tree {t1 - t0:.1f}s, {T.levels} levels, digests added", flush=True)


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "tree-digests":
        refimport.build_ref()
        ref = refimport.load_reference()
        for name, (meta, small) in CASES.items():
            if "sample" in meta and meta.get("method") is None:
                add_tree_digests(name, meta, ref)
        return
    only_small = len(sys.argv) > 1 and sys.argv[1] == "small"
    names = [a for a in sys.argv[1:] if a in CASES]
    refimport.build_ref()
    ref = refimport.load_reference()
    for name, (meta, small) in CASES.items():
        if names and name not in names:
            continue
        if only_small and not small:
            continue
        if meta.get("method") == "stokes":
            run_stokes_case(name, meta, ref)
        elif meta.get("dipole"):
            run_dipole_case(name, meta, ref)
        elif meta.get("local"):
            run_local_case(name, meta, ref)
        else:
            (run_gradient_case if meta.get("gradient") else run_case)(name, meta, ref)


if __name__ == "__main__":
    main()
