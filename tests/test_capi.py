"""CPU checks of the drop-in boundary: the library loads and exports every
symbol that include/bafqmc_b200.h declares; parameter parsing mirrors
calc_basic.f90:48-106.  No compute call is made without a GPU."""
import ctypes
import re

import numpy as np
import pytest

from bafqmc_b200 import _lib, build
from bafqmc_b200.params import ParamError, SolverParams, conf_transfer


def _declared(root):
    text = (root / "include" / "bafqmc_b200.h").read_text()
    return sorted(set(re.findall(r"\b(bafqmc_[a-z_]+)\s*\(", text)))


def test_header_and_binding_agree(root):
    assert sorted(_lib.SIGNATURES) == _declared(root)


def test_library_exports_every_declared_symbol(root):
    lib = ctypes.CDLL(str(build.build()))
    for name in _declared(root):
        assert hasattr(lib, name), name


def test_error_path_without_device(root):
    lib = _lib.load(build.build())
    h = ctypes.c_void_p()
    pt = _lib.Point(sector=0, Lx=3, Ly=3, Ltrot=7, beta=1.0, U1=1.0, U2=0.0, mu=-5.0, delta=0.0, Nwrap=2,
                    shiftLoc=1.5, iniType=2, iniAmpl=1.0, iniBias1=0.0, iniBias2=0.0, LxTherm=3, LyTherm=3,
                    LtrotTherm=7)
    cp = np.zeros(1, dtype=np.int32)
    rc = lib.bafqmc_create(ctypes.byref(pt), 1, cp.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), 1, 0,
                           ctypes.byref(h))
    assert rc == -1 and b"multiple of Nwrap" in lib.bafqmc_last_error()
    pt.Ltrot, pt.LtrotTherm, pt.U2 = 8, 8, 0.5
    rc = lib.bafqmc_create(ctypes.byref(pt), 1, cp.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), 1, 0,
                           ctypes.byref(h))
    assert rc == -1 and b"U2 must be non-positive" in lib.bafqmc_last_error()


def test_params_reference_example(root):
    text = """1.0         -0.6        -7.0
3           3           100         1.0
3           3           100
10          1000        1           1.5
.false.     0
.true.      500         1.0         1.0
2           1.0         0.0         0.0
"""
    p = SolverParams.from_text(text)
    assert (p.U1, p.U2, p.mu, p.Nwarm, p.is_warm, p.Nst) == (1.0, -0.6, -7.0, 500, True, 10)
    assert SolverParams.from_text(p.to_text()) == p
    with pytest.raises(ParamError):
        SolverParams.from_text(text.replace("1.0         -0.6", "1.0         0.6"))


def test_conf_transfer_tiles_like_reference():
    from oracle import oracle as O
    op = O.Params(U1=1, U2=0, mu=-5, Nlx=6, Nly=3, Ltrot=8, Beta=1, NlxTherm=3, NlyTherm=3, LtrotTherm=4,
                  Nwrap=2, Nbin=1, Nsweep=1, shiftLoc=1.0)
    p = SolverParams(U1=1, U2=0, mu=-5, Nlx=6, Nly=3, Ltrot=8, Beta=1, NlxTherm=3, NlyTherm=3, LtrotTherm=4,
                     Nwrap=2, Nbin=1, Nsweep=1, shiftLoc=1.0)
    therm = np.random.default_rng(1).standard_normal((4, 9, 2))
    np.testing.assert_array_equal(conf_transfer(p, therm), O.conf_transfer(op, therm))
