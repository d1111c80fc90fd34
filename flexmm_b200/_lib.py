"""ctypes binding of ``libflexmm_b200.so`` (include/flexmm_b200.h).

The library is built in-tree by ``python -m flexmm_b200.build``.  There is
no CPU fallback: constructing an FMM without the library, or without a CUDA
device, raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libflexmm_b200.so")

N_OFFSETS = 40
PRECISION = {"fp64": 0, "mixed": 1}
EVALUATORS = {"potential": (0, 1), "gradient": (1, 3), "stokes": (2, 3)}   # id, outputs
N_PHASES = 12
PHASES = ["tree", "targets", "upward", "m2l", "downward", "evaluate", "direct", "tree_splits",
          "tree_balance", "tree_nodes", "prep", "spare"]
MAX_LEVELS = 30
MAX_NEQUIV = 64

STATUS = {
    0: "OK", 1: "INVALID_ARGUMENT", 2: "CUDA", 3: "TREE_TOO_DEEP",
    4: "NOT_READY", 5: "UNSUPPORTED", 6: "CAPACITY",
}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p


class LevelOps(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_double),
        ("large_x", _dp), ("large_y", _dp),
        ("c2e_u", _dp), ("c2e_sinv", _dp), ("c2e_vh", _dp),
        ("m2mc", _dp),
        ("m2l_rank", _ip),
        ("m2l_a", ctypes.POINTER(_dp)),
        ("m2l_b", ctypes.POINTER(_dp)),
    ]


class BBLevelOps(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_double),
        ("m2l_rank", _ip),
        ("m2l_a", ctypes.POINTER(_dp)),
        ("m2l_b", ctypes.POINTER(_dp)),
    ]


BB_MAX_P = 16


class StokesLevelOps(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_double),
        ("large_x", _dp), ("large_y", _dp),
        ("e2c_u", _dp), ("e2c_sinv", _dp), ("e2c_vh", _dp),
        ("c2e_u", _dp), ("c2e_sinv", _dp), ("c2e_vh", _dp),
        ("m2mc", _dp), ("l2lc", _dp),
        ("m2l_rank", _ip),
        ("m2l_a", ctypes.POINTER(_dp)),
        ("m2l_b", ctypes.POINTER(_dp)),
    ]

# (name, restype, argtypes) of every exported entry point
SIGNATURES = [
    ("fmm_ops_create", ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_int, ctypes.POINTER(_vp)]),
    ("fmm_ops_add", ctypes.c_int, [_vp, ctypes.POINTER(LevelOps), _ip]),
    ("fmm_ops_destroy", ctypes.c_int, [_vp]),
    ("fmm_build_expansions_multi", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int64, _vp]),
    ("fmm_evaluate_multi", ctypes.c_int,
     [_vp, _vp, _vp, ctypes.c_int64, ctypes.c_int, _vp, ctypes.c_int64, _vp]),
    ("fmm_evaluate_sources_multi", ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int64, _vp]),
    ("fmm_stokes_ops_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    ("fmm_stokes_ops_add", ctypes.c_int, [_vp, ctypes.POINTER(StokesLevelOps), _ip]),
    ("fmm_build_expansions2", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("fmm_kernel_table_create", ctypes.c_int, [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip]),
    ("fmm_bb_ops_create", ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.POINTER(_vp)]),
    ("fmm_bb_ops_add", ctypes.c_int, [_vp, ctypes.POINTER(BBLevelOps), _ip]),
    ("fmm_plan_create", ctypes.c_int,
     [_vp, _vp, _vp, ctypes.c_int64, ctypes.c_int, _dp, _vp, ctypes.POINTER(_vp)]),
    ("fmm_plan_info", ctypes.c_int, [_vp, _ip, _dp, _ip]),
    ("fmm_plan_bind", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    ("fmm_plan_bind_levels", ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    ("fmm_plan_set_precision", ctypes.c_int, [_vp, ctypes.c_int]),
    ("fmm_build_expansions", ctypes.c_int, [_vp, _vp, _vp]),
    ("fmm_evaluate", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int64, ctypes.c_int, _vp, _vp]),
    ("fmm_evaluate_sources", ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp]),
    ("fmm_evaluate_outputs", ctypes.c_int,
     [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int64, ctypes.c_int, _vp, ctypes.c_int64, _vp]),
    ("fmm_evaluate_sources_outputs", ctypes.c_int,
     [_vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int64, _vp]),
    ("fmm_build_expansions_dipole", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    ("fmm_plan_create_local", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int64, ctypes.c_int,
                                             ctypes.c_double, _dp, _vp, ctypes.POINTER(_vp)]),
    ("fmm_local_evaluate", ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int64, ctypes.c_int, _vp,
                                          _vp, _vp, _vp]),
    ("fmm_build_expansions2_dipole", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("fmm_plan_destroy", ctypes.c_int, [_vp]),
    ("fmm_plan_drop_expansions", ctypes.c_int, [_vp]),
    ("fmm_plan_move_sources", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("fmm_plan_status", ctypes.c_int, [_vp]),
    ("fmm_tree_export", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("fmm_direct", ctypes.c_int, [ctypes.c_int, _dp, _vp, _vp, _vp, ctypes.c_int64, _vp, _vp,
                                  ctypes.c_int64, ctypes.c_int, _vp, _vp]),
    ("fmm_diag_log2", ctypes.c_int, [_vp, ctypes.c_int64, _vp, _vp, _vp]),
    ("fmm_timing_enable", ctypes.c_int, [ctypes.c_int]),
    ("fmm_set_split_evaluation", ctypes.c_int, [ctypes.c_int]),
    ("fmm_timing_read", ctypes.c_int, [_dp, ctypes.POINTER(ctypes.c_int64)]),
    ("fmm_evaluate_noalloc", ctypes.c_int,
     [_vp, _vp, _vp, ctypes.c_int64, ctypes.c_int, _vp, _vp]),
    ("fmm_last_error", ctypes.c_char_p, []),
]

_LIB = None


class FMMError(RuntimeError):
    def __init__(self, fn, code, msg):
        super().__init__(f"{fn} failed ({STATUS.get(code, code)}): {msg}")
        self.code = code


def load(path=LIB_PATH):
    """Load the CUDA library (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise ImportError(f"flexmm_b200 CUDA library not built: {path} is missing "
                          "(run `python -m flexmm_b200.build`)")
    lib = ctypes.CDLL(path)
    for name, res, args in SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _LIB = lib
    return lib


def call(name, *args):
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != 0:
        raise FMMError(name, rc, lib.fmm_last_error().decode(errors="replace"))
    return rc
