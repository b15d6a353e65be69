"""ctypes binding of the C++ restatement of the number-conserving sweep
(oracle/csweep.cpp, built by oracle/Makefile into oracle/libcsweep.so).

Test infrastructure, like oracle.py: it is the timed CPU baseline of bench.py
and a second restatement that tests/test_oracle_cport.py checks against
oracle.py.  The set-up quantities (e^{-+dtau K}, HS couplings, lattice bonds,
K-point phases, initial fields) come from oracle.py, so both restatements start
from the same inputs.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import oracle as O

LIB = Path(__file__).resolve().parent / "libcsweep.so"
NOBS = 15
OBS_NAMES = ("density_total", "energy_density", "kinetic", "doubleOcc", "numsquare_up", "sf_K_re", "sf_K_im",
             "dw_K_re", "dw_K_im", "psf_Gamma_re", "psf_Gamma_im", "accepted_0", "accepted_1", "proposals_0",
             "Xmaxm")
_lib = None


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise FileNotFoundError(f"{LIB} is not built (make -C oracle)")
        lib = C.CDLL(str(LIB))
        D, I = C.POINTER(C.c_double), C.POINTER(C.c_int)
        lib.csweep_run.restype = C.c_int
        lib.csweep_run.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, D, I,
                                   D, D, D, C.c_int, I, C.c_int, C.POINTER(C.c_int32), D, C.c_int, C.c_int, D, D, D]
        _lib = lib
    return _lib


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def inputs(p: O.Params) -> dict:
    """The point's set-up quantities from oracle.py."""
    latt = O.Lattice(p)
    opT = O.OperatorKinetic(p, latt)
    ops = [O.OperatorHubbard(p.U1, p.Dtau, O.CHANNEL_RELATIVE), O.OperatorHubbard(p.U2, p.Dtau, O.CHANNEL_TOTAL)]
    n = p.Ndim
    phase = (np.exp(1j * latt.k_dot_r[latt.indexK, latt.imj]) if latt.hasK else np.zeros((n, n))).astype(complex)
    return {
        "latt": latt,
        "expP": np.ascontiguousarray(opT.expT_P, dtype=complex),
        "expM": np.ascontiguousarray(opT.expT_M, dtype=complex),
        "alpha": np.array([[o.alpha.real, o.alpha.imag] for o in ops], dtype=float),
        "active": np.array([1 if o.active else 0 for o in ops], dtype=np.int32),
        "phase": np.ascontiguousarray(phase),
        "hasK": int(latt.hasK),
        "bonds": np.ascontiguousarray(latt.bonds[:, 1:4], dtype=np.int32),
    }


def run(p: O.Params, seeds: np.ndarray, phi: np.ndarray, nsweep: int, nthreads: int = 1, want_green: bool = False,
        setup: dict | None = None) -> dict:
    """bafqmc_pre's work and nsweep sweeps for each chain (seeds [nchains],
    phi [nchains][Ltrot][Ns][2], both updated in place).  Returns the last
    sweep's averaged observables per chain, the final G (optional) and the
    longest time a thread spent in sweeps."""
    if p.pairing:
        raise ValueError("the C++ restatement covers the number-conserving sweep")
    lib = load()
    s = setup or inputs(p)
    nch = seeds.size
    assert seeds.dtype == np.int32 and phi.dtype == np.float64 and phi.flags.c_contiguous
    obs = np.zeros((nch, NOBS))
    G = np.zeros((nch, p.Ndim, p.Ndim), dtype=complex) if want_green else None
    secs = np.zeros(1)
    rc = lib.csweep_run(p.Ndim, p.Ltrot, p.Nwrap, p.shiftLoc, p.RT, p.U1, p.U2, _d(s["alpha"]), _i(s["active"]),
                        _d(s["expP"].view(np.float64)), _d(s["expM"].view(np.float64)),
                        _d(s["phase"].view(np.float64)), s["hasK"], _i(s["bonds"]), nch,
                        seeds.ctypes.data_as(C.POINTER(C.c_int32)), _d(phi), int(nsweep), int(nthreads), _d(obs),
                        _d(G.view(np.float64)) if G is not None else None, _d(secs))
    if rc != 0:
        raise RuntimeError(f"csweep_run returned {rc}")
    return {"obs": obs, "G": G, "sweep_seconds": float(secs[0])}
