import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))
for p in (REPO, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(HERE, "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def golden_cases(gradient=False, stokes=False, dipole=False, local=False, stresslet=False):
    """Fixture names: potential cases; (gradient=True) the grad_* cases whose
    results are [3, n] rows (u, du/dx, du/dy); (stokes=True) the stokes_*
    cases, rows (u, v, p); (dipole=True) the dip_* cases (single plus
    double layer through kifmm2d's upwardor / evaluator)."""
    names = sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))
    if stokes:
        return [n for n in names if n.startswith("stokes_")]
    if dipole:
        return [n for n in names if n.startswith("dip_")]
    if local:   # the local evaluators (near field only)
        return [n for n in names if n.startswith("local_")]
    if stresslet:  # the Stokes FMM with stresslets (build_expansions_dipole)
        return [n for n in names if n.startswith("sdip_")]
    return [n for n in names if n.startswith("grad_") == gradient
            and not n.startswith(("stokes_", "dip_", "local_", "sdip_"))]


def load_golden(name):
    import json
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False))
    d["meta"] = json.loads(str(d["meta"]))
    for k in ("tree_sha", "tree_sha_nonempty"):
        if k in d:
            d[k] = json.loads(str(d[k]))
    return d


def golden_inputs(meta):
    sys.path.insert(0, GOLDEN)
    from make_golden import case_inputs
    return case_inputs(meta)


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="session")
def built_lib():
    """Path of the built CUDA library (built here with nvcc when missing)."""
    from flexmm_b200 import build
    return build.build()


_STRUVE = {}


def struve_kernel():
    """The Struve example's kernel as a tabulated radial kernel (one per process)."""
    if "k" not in _STRUVE:
        from flexmm_b200.kernels import radial
        from oracle.direct import struve_gf
        # scipy's GF loses relative accuracy to cancellation at large r
        # (~1e-12 below r = 10, ~1e-6 at 256): the fit tolerance follows it
        _STRUVE["k"] = radial(struve_gf, 1e-30, 256.0, tol=1e-5, name="Kernel")
    return _STRUVE["k"]


def kernel_of(meta):
    """(kernel: registered name or Kernel, kernel keyword parameters) of a golden case."""
    kind = meta.get("kernel", "laplace")
    if kind == "laplace":
        return "Laplace_Eval", {}
    if kind == "struve":   # the Struve example's kernel, by its name
        return "Kernel", {}
    return "Modified_Helmholtz_Eval", {"helmholtz_k": meta["k"]}


def oracle_kernel(meta):
    from oracle.kernels import laplace, mod_helmholtz
    if meta.get("kernel", "laplace") == "struve":
        from oracle.direct import struve_gf
        return lambda sx, sy, tx, ty: struve_gf(np.sqrt((tx - sx) ** 2 + (ty - sy) ** 2))
    return laplace if meta.get("kernel", "laplace") == "laplace" else mod_helmholtz(meta["k"])


def oracle_direct(meta, sx, sy, tau, tx, ty, check):
    from oracle.direct import direct_laplace, direct_mod_helmholtz
    if meta.get("kernel", "laplace") == "laplace":
        return direct_laplace(sx, sy, tau, tx, ty, check)
    return direct_mod_helmholtz(sx, sy, tau, tx, ty, meta["k"], check)


def make_fmm(d, meta, helper=None, precision="fp64", x=None, y=None):
    """Our FMM object for a golden case: KI_FMM, or BB_FMM for black-box cases."""
    from flexmm_b200 import BB_FMM, BB_Helper, KI_FMM, KI_Helper
    name, params = kernel_of(meta)
    x = d["x"] if x is None else x
    y = d["y"] if y is None else y
    if meta.get("method") == "bb":
        return BB_FMM(x, y, name, meta["ncut"], meta["p"], bbox=d["bbox"],
                      helper=helper if helper is not None else BB_Helper(), **params)
    return KI_FMM(x, y, name, meta["ncut"], meta["neq"], bbox=d["bbox"],
                  helper=helper if helper is not None else KI_Helper(), precision=precision, **params)
