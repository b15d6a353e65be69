"""paramC_sets.txt contract of the reference solvers (calc_basic.f90:48-106;
the pairing program reads RDelta as a fourth value on line 1,
src/pairing/src/calc_basic.f90:51-52).

Seven positional lines, Fortran list-directed values; anything after line 7 is
ignored, as the reference reads exactly seven records.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

ZERO = 1.0e-10   # calc_basic.f90:5
NAUX = 2


def _tok(t: str):
    s = t.strip().strip(",")
    low = s.lower()
    if low in (".true.", "t", ".t.", "true"):
        return True
    if low in (".false.", "f", ".f.", "false"):
        return False
    return s


def _f(t) -> float:
    return float(str(t).replace("D", "E").replace("d", "e"))


class ParamError(ValueError):
    """Mirrors the reference's `stop` on invalid input."""


@dataclass
class SolverParams:
    U1: float
    U2: float
    mu: float
    Nlx: int
    Nly: int
    Ltrot: int
    Beta: float
    NlxTherm: int
    NlyTherm: int
    LtrotTherm: int
    Nwrap: int
    Nbin: int
    Nsweep: int
    shiftLoc: float
    is_tau: bool = False
    Nthermal: int = 0
    is_warm: bool = False
    Nwarm: int = 0
    shiftWarm: tuple = (0.0, 0.0)
    iniType: int = 2
    iniAmpl: float = 1.0
    iniBias: tuple = (0.0, 0.0)
    delta: float = 0.0
    sector: int = 0

    @property
    def Lq(self) -> int:
        return self.Nlx * self.Nly

    @property
    def Nsite(self) -> int:
        return self.Lq

    @property
    def Ndim(self) -> int:
        """The reference's matrix dimension: Ns, or 4Ns for the Nambu solver
        (src/pairing/src/calc_basic.f90:99-101)."""
        return 4 * self.Lq if self.sector == 1 else self.Lq

    @property
    def block_dim(self) -> int:
        """Dimension of the Green's function the device propagates: Ns, or the
        {b, c^dagger} block 2Ns of a Nambu chain."""
        return 2 * self.Lq if self.sector == 1 else self.Lq

    @property
    def Dtau(self) -> float:
        return self.Beta / float(self.Ltrot)

    @property
    def Nst(self) -> int:
        return self.Ltrot // self.Nwrap

    def validate(self) -> "SolverParams":
        if self.U1 < -ZERO:
            raise ParamError("U1 must be non-negative (relative-density channel)")
        if self.U2 > ZERO:
            raise ParamError("U2 must be non-positive (total-density channel)")
        if self.Ltrot % self.Nwrap != 0:
            raise ParamError("Ltrot is not a multiple of Nwrap")
        if self.iniType not in (1, 2, 3):
            raise ParamError(f"incorrect initype input {self.iniType}")
        return self

    @classmethod
    def from_text(cls, text: str, pairing: bool = False) -> "SolverParams":
        rows = [ln.replace(",", " ").split() for ln in text.splitlines()]
        if len(rows) < 7 or any(len(r) == 0 for r in rows[:7]):
            raise ParamError("paramC_sets.txt needs seven non-empty lines")
        r = [[_tok(t) for t in row] for row in rows[:7]]
        p = cls(
            U1=_f(r[0][0]), U2=_f(r[0][1]), mu=_f(r[0][2]),
            delta=_f(r[0][3]) if pairing else 0.0, sector=1 if pairing else 0,
            Nlx=int(r[1][0]), Nly=int(r[1][1]), Ltrot=int(r[1][2]), Beta=_f(r[1][3]),
            NlxTherm=int(r[2][0]), NlyTherm=int(r[2][1]), LtrotTherm=int(r[2][2]),
            Nwrap=int(r[3][0]), Nbin=int(r[3][1]), Nsweep=int(r[3][2]), shiftLoc=_f(r[3][3]),
            is_tau=bool(r[4][0]), Nthermal=int(r[4][1]),
            is_warm=bool(r[5][0]), Nwarm=int(r[5][1]), shiftWarm=(_f(r[5][2]), _f(r[5][3])),
            iniType=int(r[6][0]), iniAmpl=_f(r[6][1]), iniBias=(_f(r[6][2]), _f(r[6][3])),
        )
        return p.validate()

    @classmethod
    def from_file(cls, path, pairing: bool = False) -> "SolverParams":
        return cls.from_text(Path(path).read_text(), pairing=pairing)

    def to_text(self) -> str:
        b = lambda v: ".true." if v else ".false."
        first = f"{self.U1!r} {self.U2!r} {self.mu!r}" + (f" {self.delta!r}" if self.sector == 1 else "")
        return "\n".join([
            first,
            f"{self.Nlx} {self.Nly} {self.Ltrot} {self.Beta!r}",
            f"{self.NlxTherm} {self.NlyTherm} {self.LtrotTherm}",
            f"{self.Nwrap} {self.Nbin} {self.Nsweep} {self.shiftLoc!r}",
            f"{b(self.is_tau)} {self.Nthermal}",
            f"{b(self.is_warm)} {self.Nwarm} {self.shiftWarm[0]!r} {self.shiftWarm[1]!r}",
            f"{self.iniType} {self.iniAmpl!r} {self.iniBias[0]!r} {self.iniBias[1]!r}",
        ]) + "\n"


def conf_transfer(p: SolverParams, phi_therm: np.ndarray) -> np.ndarray:
    """Tile a (LtrotTherm, NlxTherm*NlyTherm, 2) field onto (Ltrot, Nlx*Nly, 2) (fields.f90:156-234)."""
    phi_therm = np.asarray(phi_therm, dtype=np.float64).reshape(p.LtrotTherm, p.NlxTherm * p.NlyTherm, NAUX)
    out = np.zeros((p.Ltrot, p.Lq, NAUX))
    ny, nx = np.meshgrid(np.arange(1, p.Nly + 1), np.arange(1, p.Nlx + 1), indexing="ij")
    tx = np.where(nx > p.NlxTherm, nx - p.NlxTherm, nx)
    ty = np.where(ny > p.NlyTherm, ny - p.NlyTherm, ny)
    iit = ((ty - 1) * p.NlxTherm + (tx - 1)).ravel()
    ii = ((ny - 1) * p.Nlx + (nx - 1)).ravel()
    out[: p.LtrotTherm, ii, :] = phi_therm[:, iit, :]
    for nt in range(p.LtrotTherm, p.Ltrot):
        out[nt] = out[nt - p.LtrotTherm]
    return out
