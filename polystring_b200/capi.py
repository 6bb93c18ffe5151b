"""ctypes binding of libpolystring_b200.so (include/polystring_b200.h).

The library is built in-tree (polystring_b200/_build/); importing this module
never falls back to anything else: a missing library raises ImportError.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libpolystring_b200.so")

PS_OK = 0
PS_ERR_INVALID = -1
PS_ERR_UNSUPPORTED = -2
PS_ERR_CUDA = -3
PS_ERR_QUADRATURE = -4
PS_ERR_STATE = -6
# contour points the fixed table of ps_density_solve_device_noalloc holds
PS_DENSITY_NOALLOC_MAX_LEN = 8192

MDE = {"RQM4": 0, "OS4": 0, "OS2": 1, "PSEUDOSPECTRAL": 1, "ETDRK4": 2}
SCFT = {"EM": 0, "ANDERSON": 1}
CONTOUR = {"TRAPEZOID": 0, "TRAPEZOIDAL": 0, "SIMPSON": 1}
RULES = {"trapezoid": 0, "simpson": 1, "quad4_closed": 2, "quad4_open": 3,
         "quad4_semiopen_left": 4, "quad4_semiopen_right": 5}
CELL = {"LAMELLAR": 0, "SQUARE": 1, "RECTANGULAR": 2, "RECT": 2, "HEXAGONAL2": 3, "OBLIQUE": 4,
        "CUBIC": 5, "TETRAGONAL": 6, "ORTHORHOMBIC": 7, "HEXAGONAL3": 8, "TRIGONAL": 9,
        "MONOCLINIC": 10, "TRICLINIC": 11}
FIELDS = {"wA": 0, "wB": 1, "phiA": 2, "phiB": 3, "yita": 4, "qA": 5, "qB": 6, "qAc": 7, "qBc": 8}

# exported symbols and their signatures: (name, restype, argtypes)
_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p


class UnitCellC(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("system", ctypes.c_int),
                ("a", ctypes.c_double), ("b", ctypes.c_double), ("c", ctypes.c_double),
                ("alpha", ctypes.c_double), ("beta", ctypes.c_double), ("gamma", ctypes.c_double)]


class ModelABParamsC(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("Lx", ctypes.c_int), ("Ly", ctypes.c_int), ("Lz", ctypes.c_int),
                ("cell", UnitCellC), ("sA", ctypes.c_int), ("sB", ctypes.c_int),
                ("chiN", ctypes.c_double), ("lamA", ctypes.c_double), ("lamB", ctypes.c_double),
                ("lamYita", ctypes.c_double), ("mde", ctypes.c_int), ("scft", ctypes.c_int),
                ("n_anderson", ctypes.c_int), ("compressible", ctypes.c_int), ("contour", ctypes.c_int),
                ("etdrk4_M", ctypes.c_int)]


class ModelABCParamsC(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("Lx", ctypes.c_int), ("Ly", ctypes.c_int), ("Lz", ctypes.c_int),
                ("cell", UnitCellC), ("sA", ctypes.c_int), ("sB", ctypes.c_int), ("sC", ctypes.c_int),
                ("chiAB", ctypes.c_double), ("chiBC", ctypes.c_double), ("chiAC", ctypes.c_double),
                ("lamA", ctypes.c_double), ("lamB", ctypes.c_double), ("lamC", ctypes.c_double),
                ("lamYita", ctypes.c_double), ("scft", ctypes.c_int), ("n_anderson", ctypes.c_int),
                ("contour", ctypes.c_int)]


SIGNATURES = [
    ("ps_version", ctypes.c_char_p, []),
    ("ps_tuning_log", ctypes.c_char_p, []),
    ("ps_last_error", ctypes.c_char_p, []),
    ("ps_measure_fp64_peak", ctypes.c_int, [_dp]),
    ("ps_updater_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(UnitCellC), ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_double, ctypes.POINTER(_vp)]),
    ("ps_updater_create_etdrk4", ctypes.c_int, [ctypes.POINTER(UnitCellC), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_double, ctypes.c_int, ctypes.POINTER(_vp)]),
    ("ps_updater_clone", ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    ("ps_updater_destroy", None, [_vp]),
    ("ps_updater_solve", ctypes.c_int, [_vp, _dp, _dp, ctypes.c_int]),
    ("ps_updater_solve_device", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _vp]),
    ("ps_density_solve", ctypes.c_int, [ctypes.c_int, _dp, _dp, ctypes.c_int, ctypes.c_longlong,
                                        ctypes.c_double, ctypes.c_double, _dp]),
    ("ps_density_solve_device", ctypes.c_int, [ctypes.c_int, _vp, _vp, ctypes.c_int, ctypes.c_longlong,
                                               ctypes.c_double, ctypes.c_double, _vp, _vp]),
    ("ps_density_solve_device_noalloc", ctypes.c_int, [ctypes.c_int, _vp, _vp, ctypes.c_int, ctypes.c_longlong,
                                                       ctypes.c_double, ctypes.c_double, _vp, _vp]),
    ("ps_grid_mean_device", ctypes.c_int, [_vp, ctypes.c_longlong, _dp, _vp]),
    ("ps_model_ab_create", ctypes.c_int, [ctypes.POINTER(ModelABParamsC), ctypes.POINTER(_vp)]),
    ("ps_model_ab_destroy", None, [_vp]),
    ("ps_model_ab_set_fields", ctypes.c_int, [_vp, _dp, _dp]),
    ("ps_model_ab_set_fields_device", ctypes.c_int, [_vp, _vp, _vp]),
    ("ps_model_ab_update", ctypes.c_int, [_vp, ctypes.c_int]),
    ("ps_model_ab_update_timed", ctypes.c_int, [_vp, ctypes.c_int, _dp, _dp]),
    ("ps_model_ab_propagate", ctypes.c_int, [_vp, ctypes.c_int]),
    ("ps_model_ab_H", ctypes.c_int, [_vp, _dp, _dp, _dp]),
    ("ps_model_ab_residual", ctypes.c_int, [_vp, _dp]),
    ("ps_model_ab_Q", ctypes.c_int, [_vp, _dp]),
    ("ps_model_ab_forward", ctypes.c_int, [_vp]),
    ("ps_model_ab_grad_w", ctypes.c_int, [_vp, _dp, _dp, ctypes.c_double, _dp, _dp]),
    ("ps_model_ab_stress", ctypes.c_int, [_vp, _dp]),
    ("ps_model_ab_stress_checkpointed", ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    ("ps_model_ab_get", ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    ("ps_model_ab_device_ptr", ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_vp)]),
    ("ps_model_ab_synchronize", ctypes.c_int, [_vp]),
    ("ps_model_abc_create", ctypes.c_int, [ctypes.POINTER(ModelABCParamsC), ctypes.POINTER(_vp)]),
    ("ps_model_abc_destroy", None, [_vp]),
    ("ps_model_abc_set_fields", ctypes.c_int, [_vp, _dp, _dp, _dp]),
    ("ps_model_abc_update", ctypes.c_int, [_vp, ctypes.c_int]),
    ("ps_model_abc_Q", ctypes.c_int, [_vp, _dp]),
    ("ps_model_abc_H", ctypes.c_int, [_vp, _dp, _dp, _dp]),
    ("ps_model_abc_residual", ctypes.c_int, [_vp, _dp]),
    ("ps_model_abc_get", ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    ("ps_model_abc_synchronize", ctypes.c_int, [_vp]),
    ("ps_model_ab_launches_per_iteration", ctypes.c_int, [_vp]),
    ("ps_model_ab_launches_per_propagate", ctypes.c_int, [_vp]),
    ("ps_model_ab_stream", _vp, [_vp]),
    ("ps_string_ab_create", ctypes.c_int, [ctypes.POINTER(ModelABParamsC), ctypes.c_int, ctypes.c_int,
                                           ctypes.POINTER(_vp)]),
    ("ps_string_ab_destroy", None, [_vp]),
    ("ps_string_ab_set_images", ctypes.c_int, [_vp, _dp, _dp]),
    ("ps_string_ab_iterate", ctypes.c_int, [_vp, ctypes.c_int]),
    ("ps_string_ab_H", ctypes.c_int, [_vp, _dp]),
    ("ps_string_ab_S", ctypes.c_int, [_vp, _dp]),
    ("ps_string_ab_get", ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    ("ps_string_ab_synchronize", ctypes.c_int, [_vp]),
    ("ps_string_ab_launches_per_iteration", ctypes.c_int, [_vp]),
    ("ps_string_ab_create_shard", ctypes.c_int, [ctypes.POINTER(ModelABParamsC), ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_int, ctypes.c_int, ctypes.POINTER(_vp)]),
    ("ps_string_ab_relax", ctypes.c_int, [_vp]),
    ("ps_string_ab_reparameterize", ctypes.c_int, [_vp]),
    ("ps_string_ab_device_ptr", ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_vp)]),
    ("ps_string_ab_stream", _vp, [_vp]),
    ("ps_batch_ab_create", ctypes.c_int, [ctypes.POINTER(ModelABParamsC), ctypes.c_int, ctypes.POINTER(_vp)]),
    ("ps_batch_ab_create_mixed", ctypes.c_int, [ctypes.POINTER(ModelABParamsC), ctypes.c_int,
                                                ctypes.POINTER(ModelABCParamsC), ctypes.c_int, ctypes.POINTER(_vp)]),
    ("ps_batch_ab_set_fields_abc", ctypes.c_int, [_vp, ctypes.c_int, _dp, _dp, _dp]),
    ("ps_batch_ab_destroy", None, [_vp]),
    ("ps_batch_ab_set_fields", ctypes.c_int, [_vp, ctypes.c_int, _dp, _dp]),
    ("ps_batch_ab_update", ctypes.c_int, [_vp, ctypes.c_int]),
    ("ps_batch_ab_update_timed", ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    ("ps_batch_ab_H", ctypes.c_int, [_vp, ctypes.c_int, _dp, _dp, _dp]),
    ("ps_batch_ab_residual", ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    ("ps_batch_ab_get", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _dp]),
    ("ps_batch_ab_synchronize", ctypes.c_int, [_vp]),
    ("ps_batch_ab_launches_per_iteration", ctypes.c_int, [_vp]),
    ("ps_batch_ab_launches_per_propagate", ctypes.c_int, [_vp]),
    ("ps_batch_ab_gridpoint_steps", ctypes.c_int, [_vp, _dp]),
]

_lib = None


class PSError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("polystring_b200 error %d: %s" % (code, msg))
        self.code = code


def load():
    """Load the in-tree library (raises ImportError when it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libpolystring_b200.so is not built (run python -m polystring_b200.build)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != PS_OK:
        raise PSError(rc, load().ps_last_error().decode())
    return rc


def dptr(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def make_cell(dim, system, a, b=0.0, c=0.0, alpha=0.0, beta=0.0, gamma=0.0):
    if isinstance(system, str):
        system = CELL[system.upper()]
    return UnitCellC(dim, system, a, b, c, alpha, beta, gamma)
