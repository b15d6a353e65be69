"""ctypes binding of libbafqmc_b200.so (declarations in include/bafqmc_b200.h).

The library is the only compute path: if it is missing or fails to load,
importing the solver raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libbafqmc_b200.so"

OK = 0
ERRORS = {-1: "BAFQMC_EARG", -2: "BAFQMC_ECUDA", -3: "BAFQMC_EUNSUPPORTED", -4: "BAFQMC_ESTATE",
          -5: "BAFQMC_ENUMERIC", -6: "BAFQMC_ETIMEOUT"}
OBS_SCALARS = 32
COUNTERS = 14
POLE_SCALARS = 5
NUM_CLASSES = 7
PRECISION = {"fp64": 0, "mixed": 1, "wait_test": 2}


class BafqmcError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Point(C.Structure):
    """bafqmc_point: one paramC_sets.txt parameter set."""
    _fields_ = [
        ("sector", C.c_int), ("Lx", C.c_int), ("Ly", C.c_int), ("Ltrot", C.c_int),
        ("beta", C.c_double), ("U1", C.c_double), ("U2", C.c_double), ("mu", C.c_double),
        ("delta", C.c_double), ("Nwrap", C.c_int), ("shiftLoc", C.c_double), ("iniType", C.c_int),
        ("iniAmpl", C.c_double), ("iniBias1", C.c_double), ("iniBias2", C.c_double),
        ("LxTherm", C.c_int), ("LyTherm", C.c_int), ("LtrotTherm", C.c_int),
    ]


# name -> (restype, argtypes); every symbol declared in include/bafqmc_b200.h
_P = C.c_void_p
_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int32)
_FP = C.POINTER(C.c_float)
SIGNATURES = {
    "bafqmc_create": (C.c_int, [C.POINTER(Point), C.c_int, _IP, C.c_int, C.c_int, C.POINTER(_P)]),
    "bafqmc_create_tuned": (C.c_int, [C.POINTER(Point), C.c_int, _IP, C.c_int, C.c_int, _IP, C.POINTER(_P)]),
    "bafqmc_autotune": (C.c_int, [C.POINTER(Point), C.c_int, C.c_int, C.c_int, _IP, _DP]),
    "bafqmc_destroy": (None, [_P]),
    "bafqmc_last_error": (C.c_char_p, []),
    "bafqmc_point_dim": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                   C.POINTER(C.c_int)]),
    "bafqmc_obs_stride": (C.c_int, [_P]),
    "bafqmc_num_chains": (C.c_int, [_P]),
    "bafqmc_fields_from_seeds": (C.c_int, [_P, _IP]),
    "bafqmc_set_state": (C.c_int, [_P, _IP, _DP]),
    "bafqmc_get_state": (C.c_int, [_P, _IP, _DP]),
    "bafqmc_warmup_prior": (C.c_int, [_P, C.c_int]),
    "bafqmc_pre": (C.c_int, [_P]),
    "bafqmc_sweep": (C.c_int, [_P, C.c_int]),
    "bafqmc_bin_chain_obs": (C.c_int, [_P, _DP]),
    "bafqmc_bin_point_obs": (C.c_int, [_P, _DP]),
    "bafqmc_get_green": (C.c_int, [_P, C.c_int, _DP]),
    "bafqmc_log_weight": (C.c_int, [_P, _DP]),
    "bafqmc_pole_diagnostics": (C.c_int, [_P, _DP, C.c_int, _DP]),
    "bafqmc_set_precision": (C.c_int, [_P, C.c_int]),
    "bafqmc_set_time_displaced": (C.c_int, [_P, C.c_int, C.c_int]),
    "bafqmc_time_displaced_stats": (C.c_int, [_P, _DP, C.c_int]),
    "bafqmc_time_displaced_probe": (C.c_int, [_P, C.c_int, _DP]),
    "bafqmc_stats_reset": (C.c_int, [_P, C.c_int, C.c_int]),
    "bafqmc_global_shift": (C.c_int, [_P, _DP, _IP]),
    "bafqmc_stats": (C.c_int, [_P, _DP, _DP, _IP]),
    "bafqmc_counters": (C.c_int, [_P, _DP]),
    "bafqmc_phase_timers": (C.c_int, [_P, C.c_int, _DP]),
    "bafqmc_synchronize": (C.c_int, [_P]),
    "bafqmc_stream": (_P, [_P]),
    "bafqmc_sweep_noalloc": (C.c_int, [C.POINTER(Point), C.c_int, _P, _P, C.c_int, _P, _P]),
    "bafqmc_net_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(_P)]),
    "bafqmc_net_destroy": (None, [_P]),
    "bafqmc_net_num_params": (C.c_longlong, [_P]),
    "bafqmc_net_set_params": (C.c_int, [_P, _FP]),
    "bafqmc_net_get_params": (C.c_int, [_P, _FP]),
    "bafqmc_net_set_tensor_cores": (C.c_int, [_P, C.c_int]),
    "bafqmc_net_forward": (C.c_int, [_P, C.c_int, _DP, _FP]),
    "bafqmc_net_loss_grad": (C.c_int, [_P, C.c_int, _DP, _DP, _DP, _FP]),
    "bafqmc_net_reserve_data": (C.c_int, [_P, C.c_int, C.c_int]),
    "bafqmc_net_collect": (C.c_int, [_P, _P]),
    "bafqmc_net_train": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_double, C.c_ulonglong, _DP]),
    "bafqmc_net_status": (C.c_int, [_P, _IP]),
    "bafqmc_net_set_wait_test": (C.c_int, [_P, C.c_int]),
    "bafqmc_net_time_layers": (C.c_int, [_P, C.c_int, C.c_int, _DP]),
    "bafqmc_learned_move": (C.c_int, [_P, _P, _IP, _DP]),
}

_lib = None


def load(path: Path | None = None) -> C.CDLL:
    """Load the library once; raises if it is missing (no fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"{p} is missing: build it with `python -m bafqmc_b200.build`")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != OK:
        msg = load().bafqmc_last_error()
        raise BafqmcError(rc, msg.decode() if msg else "")
