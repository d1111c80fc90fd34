"""Seeded synthetic point sets for the five benchmark configurations.

No public dataset is involved: every input is drawn from
``numpy.random.default_rng(seed)`` in the order written below, so the same
arrays are produced on every machine with the same numpy.  ``scale``
shrinks the point counts for tests (the distributions stay the same).

* ``uniform``    100,000 sources U[-1,1]^2, charges N(0,1), 316^2 grid targets
* ``clustered``  1,000,000 sources in 20 Gaussian clusters (centres
                 U[-0.9,0.9]^2, sigma 0.01, equal weights), charges N(0,1),
                 1000^2 grid targets
* ``circle``     1,000,000 sources at uniform angles on a circle of radius 0.5
                 with radial jitter U(-1e-3,1e-3), ``n_rhs`` charge columns
* ``bbfmm``      500,000 sources and 250,000 targets U[-1,1]^2, charges and a
                 per-target reference field N(0,1)
* ``stokes``     256 problems, sizes log-uniform in [2,000, 200,000], sources
                 U[-1,1]^2, forces (fx, fy) N(0,1)
"""
import numpy as np

SEEDS = {"uniform": 0, "clustered": 1, "circle": 2, "bbfmm": 3, "stokes": 4}


def grid(n):
    g = np.linspace(-1, 1, n)
    gx, gy = np.meshgrid(g, g)
    return gx.ravel(), gy.ravel()


def uniform(n=100_000, n_grid=316, seed=SEEDS["uniform"]):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, n)
    y = rng.uniform(-1, 1, n)
    tau = rng.standard_normal(n)
    tx, ty = grid(n_grid)
    return dict(x=x, y=y, tau=tau, tx=tx, ty=ty, bbox=[-1.0, 1.0, -1.0, 1.0])


def clustered(n=1_000_000, n_grid=1000, n_clusters=20, sigma=0.01, seed=SEEDS["clustered"]):
    rng = np.random.default_rng(seed)
    per = n // n_clusters
    c = rng.uniform(-0.9, 0.9, (n_clusters, 2))
    m = per * n_clusters
    x = np.repeat(c[:, 0], per) + sigma * rng.standard_normal(m)
    y = np.repeat(c[:, 1], per) + sigma * rng.standard_normal(m)
    tau = rng.standard_normal(m)
    tx, ty = grid(n_grid)
    return dict(x=x, y=y, tau=tau, tx=tx, ty=ty, bbox=[-1.0, 1.0, -1.0, 1.0])


def circle(n=1_000_000, n_rhs=64, seed=SEEDS["circle"]):
    rng = np.random.default_rng(seed)
    th = rng.uniform(0, 2 * np.pi, n)
    r = 0.5 + rng.uniform(-1e-3, 1e-3, n)
    x = r * np.cos(th)
    y = r * np.sin(th)
    tau = rng.standard_normal((n_rhs, n))
    return dict(x=x, y=y, tau=tau, bbox=None)


def bbfmm(n=500_000, m=250_000, seed=SEEDS["bbfmm"]):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, n)
    y = rng.uniform(-1, 1, n)
    tau = rng.standard_normal(n)
    tx = rng.uniform(-1, 1, m)
    ty = rng.uniform(-1, 1, m)
    u_ref = rng.standard_normal(m)
    return dict(x=x, y=y, tau=tau, tx=tx, ty=ty, u_ref=u_ref, bbox=[-1.0, 1.0, -1.0, 1.0])


def stokes(n_problems=256, nmin=2000, nmax=200_000, seed=SEEDS["stokes"]):
    rng = np.random.default_rng(seed)
    sizes = np.round(np.exp(rng.uniform(np.log(nmin), np.log(nmax), n_problems))).astype(np.int64)
    probs = []
    for n in sizes:
        x = rng.uniform(-1, 1, n)
        y = rng.uniform(-1, 1, n)
        fx = rng.standard_normal(n)
        fy = rng.standard_normal(n)
        probs.append(dict(x=x, y=y, fx=fx, fy=fy, bbox=[-1.0, 1.0, -1.0, 1.0]))
    return probs
