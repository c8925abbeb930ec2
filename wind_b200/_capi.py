"""ctypes mirror of include/wind.h (structs, enums, prototypes).

Only plain C types cross this boundary: pointers, sizes and enums.  The same
struct definitions are used for every library that speaks the wind_network
layout.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import networks as _nets

# wind_status
WIND_OK = 0
WIND_ERR_ARGUMENT = 1
WIND_ERR_UNSUPPORTED = 2
WIND_ERR_CUDA = 3
WIND_ERR_NOMEM = 4
WIND_ERR_TIMEOUT = 5
WIND_ERR_BUSY = 6
WIND_ERR_NOT_FOUND = 7

# per-system status bits
SYS_OK = 0
SYS_NONFINITE = 1
SYS_MAX_ATTEMPTS = 2
SYS_STALLED = 4
SYS_REFINE_FALLBACK = 8
SYS_TIMEOUT = 16
SYS_BAD_INPUT = 32

METHOD_SIE = 0
METHOD_RK2 = 1
METHOD_SIM = 2
CTRL_DEVICE = 0
CTRL_GOLD = 1
SOLVER_GJE_F64 = 0
SOLVER_LU_F64 = 1
SOLVER_MIXED = 2
SOLVER_MIXED_TC = 4
MEM_HOST = 0
MEM_DEVICE = 1

METHODS = {"sie": METHOD_SIE, "rk2": METHOD_RK2, "sim": METHOD_SIM}
CONTROLLERS = {"device": CTRL_DEVICE, "gold": CTRL_GOLD}
SOLVER_AUTO = 3
SOLVERS = {"gje_f64": SOLVER_GJE_F64, "lu_f64": SOLVER_LU_F64, "mixed": SOLVER_MIXED,
           "auto": SOLVER_AUTO, "mixed_tc": SOLVER_MIXED_TC}


class WindNetwork(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("n_eq", C.c_int32),
        ("n_const", C.c_int32),
        ("n_react", C.c_int32),
        ("constants", C.c_void_p),
        ("rates", C.c_void_p),
        ("species", C.c_void_p),
        ("linear", C.c_void_p),
    ]


class WindOptions(C.Structure):
    _fields_ = [
        ("method", C.c_int32),
        ("solver", C.c_int32),
        ("controller", C.c_int32),
        ("spec_width", C.c_int32),
        ("max_attempts", C.c_int64),
        ("timeout_s", C.c_double),
    ]


NOALLOC_MAX_GROUPS = 256


class WindGroup(C.Structure):
    _fields_ = [
        ("net", WindNetwork),
        ("y", C.c_void_p),
        ("nsys", C.c_int64),
        ("tnow", C.c_double),
        ("tend", C.c_double),
        ("n_integration_steps", C.c_int32),
        ("pad_", C.c_int32),
        ("atol", C.c_double),
        ("rtol", C.c_double),
        ("sys_status", C.c_void_p),
        ("sys_nsteps", C.c_void_p),
    ]


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"], "arrays crossing the C ABI must be contiguous"
        return a.ctypes.data
    # torch tensor (device or host)
    return int(a.data_ptr())


def network_struct(net: "_nets.Network", arrays=None) -> WindNetwork:
    """Build a WindNetwork.  ``arrays`` optionally overrides the four data
    arrays (e.g. device tensors); by default the Network's host arrays are
    used.  The caller keeps the arrays alive for the duration of the call."""
    a = arrays or {}
    cst = a.get("constants", net.constants)
    rts = a.get("rates", net.rates)
    spc = a.get("species", net.species)
    lin = a.get("linear", net.linear)
    return WindNetwork(net.kind, net.n_eq, net.n_const, net.n_react,
                       _ptr(cst), _ptr(rts), _ptr(spc), _ptr(lin))


def declare_api(lib: C.CDLL) -> C.CDLL:
    """Attach prototypes of include/wind.h to a loaded library."""
    P = C.c_void_p
    lib.wind_default_options.argtypes = [C.POINTER(WindOptions)]
    lib.wind_default_options.restype = None
    lib.wind_integrate.argtypes = [
        C.POINTER(WindOptions), C.POINTER(WindNetwork), C.c_double, C.c_double,
        C.c_int32, P, C.c_int64, C.c_double, C.c_double, P, P, P, C.c_int32, P]
    lib.wind_integrate.restype = C.c_int
    lib.wind_integrate_batch.argtypes = [C.POINTER(WindOptions), C.POINTER(WindGroup),
                                         C.c_int32, P]
    lib.wind_integrate_batch.restype = C.c_int
    lib.wind_integrate_batch_noalloc.argtypes = [C.POINTER(WindOptions), C.POINTER(WindGroup),
                                                 C.c_int32, P]
    lib.wind_integrate_batch_noalloc.restype = C.c_int
    lib.wind_integrate_output_steps.argtypes = [
        C.POINTER(WindOptions), C.POINTER(WindNetwork), C.c_double, C.c_double,
        C.c_int32, C.c_int32, P, C.c_int64, C.c_double, C.c_double, P, P,
        C.c_int32, P]
    lib.wind_integrate_output_steps.restype = C.c_int
    lib.wind_integrate_global.argtypes = [
        C.POINTER(WindOptions), C.POINTER(WindNetwork), C.c_double, C.c_double,
        C.c_int32, P, C.c_int64, C.c_double, C.c_double, P, P, C.c_int32, P]
    lib.wind_integrate_global.restype = C.c_int
    lib.wind_plugin_create.argtypes = [C.c_char_p, C.c_int32, C.c_int32, C.c_char_p,
                                       C.POINTER(C.c_void_p), C.c_char_p, C.c_int64]
    lib.wind_plugin_create.restype = C.c_int
    lib.wind_plugin_destroy.argtypes = [C.c_void_p]
    lib.wind_plugin_destroy.restype = C.c_int
    lib.wind_integrate_plugin.argtypes = [
        C.POINTER(WindOptions), C.c_void_p, C.c_double, C.c_double, C.c_int32, C.c_void_p,
        C.c_void_p, C.c_int64, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
        C.c_int32, C.c_void_p]
    lib.wind_integrate_plugin.restype = C.c_int
    lib.wind_version.restype = C.c_char_p
    lib.wind_status_string.argtypes = [C.c_int]
    lib.wind_status_string.restype = C.c_char_p
    lib.wind_launch_count.restype = C.c_int64
    lib.wind_last_error.restype = C.c_char_p
    return lib
