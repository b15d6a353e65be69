"""B200 implementation of the BAFQMC finite-temperature auxiliary-field sweep.

The compute path is libbafqmc_b200.so (hand-written sm_100a CUDA behind the C
ABI in include/bafqmc_b200.h); this package is its host side: parameter files,
run-directory driver and result decoding.
"""
from .params import SolverParams, ParamError, conf_transfer
from .observables import decode, FILE_ORDER

__all__ = ["SolverParams", "ParamError", "conf_transfer", "decode", "FILE_ORDER", "Ensemble",
           "run_directory"]


def __getattr__(name):
    if name in ("Ensemble", "run_directory", "pole_diagnostics"):
        from . import solver
        return getattr(solver, name)
    raise AttributeError(name)
