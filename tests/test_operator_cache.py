"""On-disk operator cache of KI_Helper (the reference's operator cache,
flexmm/flexmm2d/helpers.py:36-84 and float_dict.py, kept across processes).
Host only: the cache holds the FP64 host operators, formed before upload."""
import os

import numpy as np

from flexmm_b200.helpers import KI_Helper, KIPrecomputation, width_key
from flexmm_b200.kernels import resolve


def _same(a, b):
    assert a.width == b.width
    for name in ("c2e_sinv", "c2e_u", "c2e_vh", "m2mc", "small_x", "small_y", "large_x", "large_y",
                 "m2l_rank"):
        np.testing.assert_array_equal(getattr(a, name), getattr(b, name))
    for xa, xb in zip(a.m2l_a + a.m2l_b, b.m2l_a + b.m2l_b):
        assert (xa is None) == (xb is None)
        if xa is not None:
            np.testing.assert_array_equal(xa, xb)


def test_precomputation_array_round_trip():
    k = resolve("Laplace_Eval")
    pre = KIPrecomputation(0.125, 40, k)   # Nequiv 40: SVD-compressed M2L offsets too
    assert (pre.m2l_rank > 0).any()
    _same(pre, KIPrecomputation.from_arrays(pre.to_arrays()))


def test_disk_cache_is_written_and_loaded_by_a_new_helper(tmp_path):
    k = resolve("Laplace_Eval")
    h1 = KI_Helper(cache_dir=str(tmp_path))
    h1.attach(k, 24)
    widths = [2.0 / 2 ** l for l in range(2, 6)]
    formed = [h1.precomputation(w) for w in widths]
    files = [f for d in os.listdir(tmp_path) for f in os.listdir(tmp_path / d)]
    assert len(files) == len(widths) and all(f.endswith(".npz") for f in files)
    # a new helper (a new process, say) snaps a bbox like a fresh reference
    # helper -- the widths on disk play no part -- and reads a width from
    # disk when it needs it, without forming it
    h2 = KI_Helper(cache_dir=str(tmp_path))
    h2.attach(k, 24)
    assert h2.precomputations == {}
    bb = [-0.9, 0.8, -0.7, 0.95]
    assert h2.get_bbox(None, None, bb) == KI_Helper().get_bbox(None, None, bb)
    real_init = KIPrecomputation.__init__

    def refuse(*args, **kwargs):
        raise AssertionError("formed again instead of read from the cache")
    KIPrecomputation.__init__ = refuse
    try:
        for w, pre in zip(widths, formed):
            _same(h2.precomputation(w), pre)
    finally:
        KIPrecomputation.__init__ = real_init
    assert sorted(h2.precomputations) == sorted(width_key(w) for w in widths)
    # and then snaps like the helper that formed them
    assert h2.get_bbox(None, None, bb) == h1.get_bbox(None, None, bb)


def test_disk_cache_skips_temporary_and_truncated_files(tmp_path):
    """A writer's temporary file, or a truncated cache file left by a crash,
    never breaks a helper: the width is formed again."""
    k = resolve("Laplace_Eval")
    h1 = KI_Helper(cache_dir=str(tmp_path))
    h1.attach(k, 24)
    good = h1.precomputation(0.25)
    d = next(tmp_path.iterdir())
    f = next(p for p in d.iterdir() if p.name.endswith(".npz"))
    data = f.read_bytes()
    (d / ".w_123.tmp").write_bytes(data[: len(data) // 2])
    f.write_bytes(data[: len(data) // 3])   # a truncated zip
    h2 = KI_Helper(cache_dir=str(tmp_path))
    h2.attach(k, 24)
    _same(h2.precomputation(0.25), good)
    # the width formed again is written back whole
    h3 = KI_Helper(cache_dir=str(tmp_path))
    h3.attach(k, 24)
    assert h3._load_disk(width_key(0.25)) is not None


def test_disk_cache_keeps_kernels_and_nequiv_apart(tmp_path):
    lap, mh = resolve("Laplace_Eval"), resolve("Modified_Helmholtz_Eval", helmholtz_k=10.0)
    a = KI_Helper(cache_dir=str(tmp_path))
    a.attach(lap, 24)
    a.precomputation(0.25)
    for kern, neq in ((lap, 32), (mh, 24)):
        b = KI_Helper(cache_dir=str(tmp_path))
        b.attach(kern, neq)
        assert b._load_disk(width_key(0.25)) is None
    # a damaged file is skipped, and that width is formed again
    d = next(tmp_path.iterdir())
    f = next(d.iterdir())
    f.write_bytes(b"not an npz file")
    c = KI_Helper(cache_dir=str(tmp_path))
    c.attach(lap, 24)
    assert c._load_disk(width_key(0.25)) is None
    _same(c.precomputation(0.25), KIPrecomputation(0.25, 24, lap))


def test_stokes_operators_round_trip_and_disk_cache(tmp_path, monkeypatch):
    from flexmm_b200 import stokes
    pre = stokes.StokesPrecomputation(0.25, 16)
    back = stokes.StokesPrecomputation.from_arrays(pre.to_arrays())
    for name in ("small_x", "small_y", "large_x", "large_y", "m2mc", "l2lc", "m2l_rank"):
        np.testing.assert_array_equal(getattr(pre, name), getattr(back, name))
    for name in ("e2c", "c2e"):
        for part in ("U", "SI", "VH"):
            np.testing.assert_array_equal(getattr(getattr(pre, name), part),
                                          getattr(getattr(back, name), part))
    for xa, xb in zip(pre.m2l_a + pre.m2l_b, back.m2l_a + back.m2l_b):
        assert (xa is None) == (xb is None)
        if xa is not None:
            np.testing.assert_array_equal(xa, xb)
    # formed once, then read back from disk without being formed again
    first = stokes.stokes_precomputation(0.5, 16, cache_dir=str(tmp_path))
    assert any(f.endswith(".npz") for d in tmp_path.iterdir() for f in os.listdir(d))

    def refuse(*args, **kwargs):
        raise AssertionError("formed again instead of read from the cache")
    monkeypatch.setattr(stokes.StokesPrecomputation, "__init__", refuse)
    again = stokes.stokes_precomputation(0.5, 16, cache_dir=str(tmp_path))
    np.testing.assert_array_equal(again.m2mc, first.m2mc)
    np.testing.assert_array_equal(again.c2e.U, first.c2e.U)
