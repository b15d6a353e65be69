"""CPU oracle for the BAFQMC finite-temperature sweep (number-conserving solver).

TEST INFRASTRUCTURE ONLY.  This module is the parity checker for the CUDA
path in ``bafqmc_b200``.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline / reference legs of ``bench.py`` may import it; the product path
never does, and it must not be used as a fallback.

It restates, call for call, the reference Fortran solver of YinkaiYu/BAFQMC
(files cited as ``src/number_conserving/src/<file>.f90:<line>``) in NumPy,
with SciPy's LAPACK wrappers (ZGEQP3, ZUNGQR, ZUNMQR, ZTRSM, ZTRMM) standing
in for the reference's own LAPACK calls so the stabilisation follows the same
factorisation sequence.  Fortran arrays are 1-based column-major; here every
matrix keeps the same (row, column) meaning with 0-based indices.

Parity pins (checked in ``tests/test_oracle.py``):
  * the RNG known-answer test of ``src/common/test_numerics.f90:177-189``;
  * the dense fixed-field reference of ``tests/physics/test_fixed_field_solver.py``
    (golden vectors in ``tests/golden/fixed_field.json``, generated by importing
    that file), tolerance 2e-10;
  * the Gaussian closed forms of ``tests/physics/test_gaussian_solvers.py:44-77``
    (golden vectors in ``tests/golden/gaussian.json``), tolerances 2e-9 / 2e-8.
Bitwise parity with the reference's LAPACK is not pinned (no Fortran, MPI or
LAPACK toolchain exists to run the reference); the reference tests themselves
pin the LAPACK boundary only through invariants at 2e-10.
"""

from __future__ import annotations

import cmath
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
from scipy.linalg import blas, lapack

# --------------------------------------------------------------------------
# constants (calc_basic.f90:5-13)
ZERO = 1.0e-10
PI = math.acos(-1.0)
NAUX = 2
NBOND = 3
LCG_A = 48828125
LCG_M = 2147483648


# --------------------------------------------------------------------------
# RNG (src/common/random.f90:1-11; fields.f90:280-288)
def ranf(seed: int) -> tuple[int, float]:
    """One LCG step: seed <- 48828125*seed mod 2^31, u = seed/2^31."""
    seed = (LCG_A * seed) % LCG_M
    return seed, seed / LCG_M


def rng_gaussian(seed: int) -> tuple[int, float]:
    """Box-Muller cosine branch, two draws (fields.f90:280-288)."""
    seed, x1 = ranf(seed)
    seed, x2 = ranf(seed)
    return seed, math.sqrt(-2.0 * math.log(x1)) * math.cos(2.0 * PI * x2)


# --------------------------------------------------------------------------
# parameters (calc_basic.f90:48-106)
def _fortran_token(tok: str):
    t = tok.strip().strip(",")
    low = t.lower()
    if low in (".true.", "t", ".t.", "true"):
        return True
    if low in (".false.", "f", ".f.", "false"):
        return False
    return t


def _float(tok) -> float:
    return float(str(tok).replace("D", "E").replace("d", "e"))


@dataclass
class Params:
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
    RT: float = 1.0

    @property
    def Lq(self) -> int:
        return self.Nlx * self.Nly

    @property
    def Ndim(self) -> int:
        return self.Lq

    @property
    def Dtau(self) -> float:
        return self.Beta / float(self.Ltrot)

    @property
    def Nst(self) -> int:
        if self.Ltrot % self.Nwrap != 0:
            raise ValueError("Ltrot is not a multiple of Nwrap")
        return self.Ltrot // self.Nwrap

    @classmethod
    def from_text(cls, text: str) -> "Params":
        rows = [ln.replace(",", " ").split() for ln in text.splitlines()]
        rows = [r for r in rows][:7]
        r = [[_fortran_token(t) for t in row] for row in rows]
        p = cls(
            U1=_float(r[0][0]), U2=_float(r[0][1]), mu=_float(r[0][2]),
            Nlx=int(r[1][0]), Nly=int(r[1][1]), Ltrot=int(r[1][2]), Beta=_float(r[1][3]),
            NlxTherm=int(r[2][0]), NlyTherm=int(r[2][1]), LtrotTherm=int(r[2][2]),
            Nwrap=int(r[3][0]), Nbin=int(r[3][1]), Nsweep=int(r[3][2]), shiftLoc=_float(r[3][3]),
            is_tau=bool(r[4][0]), Nthermal=int(r[4][1]),
            is_warm=bool(r[5][0]), Nwarm=int(r[5][1]),
            shiftWarm=(_float(r[5][2]), _float(r[5][3])),
            iniType=int(r[6][0]), iniAmpl=_float(r[6][1]),
            iniBias=(_float(r[6][2]), _float(r[6][3])),
        )
        if p.U1 < -ZERO:
            raise ValueError("U1 must be non-negative (relative-density channel)")
        if p.U2 > ZERO:
            raise ValueError("U2 must be non-positive (total-density channel)")
        _ = p.Nst
        return p


# --------------------------------------------------------------------------
# lattice (lattice.f90:21-125)
class Lattice:
    def __init__(self, p: Params):
        nlx, nly = p.Nlx, p.Nly
        lq = nlx * nly
        self.Lq = lq
        # cell_list / inv_cell_list (lattice.f90:38-47): index = (ny-1)*Nlx + (nx-1)
        self.cell = np.zeros((lq, 2), dtype=np.int64)
        self.inv_cell = np.zeros((nlx + 1, nly + 1), dtype=np.int64)
        nc = 0
        for ny in range(1, nly + 1):
            for nx in range(1, nlx + 1):
                self.cell[nc] = (nx, ny)
                self.inv_cell[nx, ny] = nc
                nc += 1

        def npbc(nr, L):
            if nr > L:
                return nr - L
            if nr < 1:
                return nr + L
            return nr

        # imj (lattice.f90:59-70)
        self.imj = np.zeros((lq, lq), dtype=np.int64)
        for jj in range(lq):
            for ii in range(lq):
                ix, iy = self.cell[ii]
                jx, jy = self.cell[jj]
                self.imj[ii, jj] = self.inv_cell[(ix - jx) % nlx + 1, (iy - jy) % nly + 1]
        # vectors (lattice.f90:72-90)
        a1 = (1.0, 0.0)
        a2 = (0.5, math.sqrt(3.0) / 2.0)
        b1 = (2.0 * PI, -2.0 * PI / math.sqrt(3.0))
        b2 = (0.0, 4.0 * PI / math.sqrt(3.0))
        self.aimj = np.zeros((lq, 2))
        self.xk = np.zeros((lq, 2))
        for ii in range(lq):
            ix, iy = self.cell[ii]
            self.aimj[ii, 0] = (ix - 1) * a1[0] + (iy - 1) * a2[0]
            self.aimj[ii, 1] = (ix - 1) * a1[1] + (iy - 1) * a2[1]
            self.xk[ii, 0] = (ix - 1) * b1[0] / nlx + (iy - 1) * b2[0] / nly
            self.xk[ii, 1] = (ix - 1) * b1[1] / nlx + (iy - 1) * b2[1] / nly
        self.k_dot_r = self.xk[:, 0:1] * self.aimj[None, :, 0] + self.xk[:, 1:2] * self.aimj[None, :, 1]
        # bonds (lattice.f90:98-111)
        self.bonds = np.zeros((lq, NBOND + 1), dtype=np.int64)
        for iy in range(1, nly + 1):
            for ix in range(1, nlx + 1):
                i = self.inv_cell[ix, iy]
                self.bonds[i, 0] = i
                self.bonds[i, 1] = self.inv_cell[npbc(ix + 1, nlx), npbc(iy, nly)]
                self.bonds[i, 2] = self.inv_cell[npbc(ix, nlx), npbc(iy + 1, nly)]
                self.bonds[i, 3] = self.inv_cell[npbc(ix - 1, nlx), npbc(iy + 1, nly)]
        # K point (obser_equal.f90:121-125)
        self.hasK = (nlx % 3 == 0) and (nly % 3 == 0)
        self.indexK = self.inv_cell[2 * nlx // 3 + 1, nly // 3 + 1] if self.hasK else 0
        self.indexzero = self.inv_cell[1, 1]


# --------------------------------------------------------------------------
# kinetic propagator (non_interact.f90:33-109)
def ham_T(p: Params, latt: Lattice) -> np.ndarray:
    n = p.Ndim
    H = np.zeros((n, n), dtype=complex)
    z = complex(p.RT, 0.0)
    for ii in range(n):
        for nb in range(1, NBOND + 1):
            jj = latt.bonds[ii, nb]
            H[ii, jj] += z
            H[jj, ii] += z.conjugate()
    for ii in range(n):
        H[ii, ii] -= complex(p.mu, 0.0)
    return H


class OperatorKinetic:
    def __init__(self, p: Params, latt: Lattice):
        H = ham_T(p, latt)
        w, U = np.linalg.eigh(H)
        self.energy_min = float(w.min())
        self.energy_max = float(w.max())
        self.bandwidth = self.energy_max - self.energy_min
        Ud = U.conj().T
        self.expT_P = (U * np.exp(-p.Dtau * w)) @ Ud
        self.expT_M = (U * np.exp(p.Dtau * w)) @ Ud


# --------------------------------------------------------------------------
# HS operator (operator_Hubbard.f90:36-68)
class OperatorHubbard:
    def __init__(self, U: float, dtau: float):
        self.alpha = 0j
        if U < -ZERO:
            self.alpha = complex(math.sqrt(-2.0 * U * dtau), 0.0)
        if U > ZERO:
            self.alpha = complex(0.0, math.sqrt(2.0 * U * dtau))
        self.active = abs(U) > ZERO
        self.acc_local = 0.0
        self.acc_therm = 0.0
        self.nc = 0
        self.nacc = 0

    def get_exp(self, phi: float, nflag: int) -> tuple[complex, complex]:
        gaussian = complex(math.exp(-0.5 * phi * phi), 0.0)
        expalpha = cmath.exp(self.alpha * phi * nflag)
        return gaussian, expalpha

    def get_delta(self, phi_old: float, phi_new: float) -> tuple[complex, complex]:
        g_old, e_old = self.get_exp(phi_old, 1)
        g_new, e_new = self.get_exp(phi_new, 1)
        return g_new / g_old, e_new / e_old - 1.0

    def reset(self):
        self.nc = 0
        self.nacc = 0

    def count(self, toggle: bool):
        self.nc += 1
        if toggle:
            self.nacc += 1


# --------------------------------------------------------------------------
# field initialisation (fields.f90:115-154, 156-234)
def conf_set(p: Params, seed: int) -> tuple[int, np.ndarray]:
    """Returns (advanced seed, phi_therm[LtrotTherm, NdimTherm, Naux])."""
    nd = p.NlxTherm * p.NlyTherm
    phi = np.zeros((p.LtrotTherm, nd, NAUX))
    for nt in range(p.LtrotTherm):
        for ii in range(nd):
            for ns in range(NAUX):
                if p.iniType == 1:
                    seed, x = ranf(seed)
                    phi[nt, ii, ns] = p.iniBias[ns] + p.iniAmpl * (x - 0.5)
                elif p.iniType == 2:
                    seed, x = rng_gaussian(seed)
                    phi[nt, ii, ns] = p.iniBias[ns] + p.iniAmpl * x
                elif p.iniType == 3:
                    seed, x = rng_gaussian(seed)
                    phi[nt, ii, ns] = p.iniBias[ns] + p.iniAmpl * abs(x)
                else:
                    raise ValueError(f"incorrect initype input {p.iniType}")
    return seed, phi


def conf_transfer(p: Params, phi_therm: np.ndarray) -> np.ndarray:
    """Tile a (LtrotTherm, NlxTherm*NlyTherm) configuration onto (Ltrot, Nlx*Nly)."""
    phi = np.zeros((p.Ltrot, p.Lq, NAUX))
    for nt in range(p.LtrotTherm):
        for ny in range(1, p.Nly + 1):
            for nx in range(1, p.Nlx + 1):
                tx = nx - p.NlxTherm if nx > p.NlxTherm else nx
                ty = ny - p.NlyTherm if ny > p.NlyTherm else ny
                iit = (ty - 1) * p.NlxTherm + (tx - 1)
                ii = (ny - 1) * p.Nlx + (nx - 1)
                phi[nt, ii, :] = phi_therm[nt, iit, :]
    for nt in range(p.LtrotTherm, p.Ltrot):
        phi[nt] = phi[nt - p.LtrotTherm]
    return phi


# --------------------------------------------------------------------------
# stabilisation (stabilization.f90:41-190)
def qdrp_decompose(mat: np.ndarray):
    """ZGEQP3 with free pivots, then split D=|diag R| off R (stabilization.f90:41-67).

    Returns (qr, d, jpvt0, tau) with jpvt0 0-based: (mat*P)[:, j] = mat[:, jpvt0[j]].
    """
    n = mat.shape[0]
    qr, jpvt, tau, _, info = lapack.zgeqp3(np.asfortranarray(mat), lwork=max(1, 64 * n))
    if info != 0:
        raise RuntimeError(f"zgeqp3 info={info}")
    d = np.zeros(n, dtype=complex)
    for i in range(n):
        x = abs(qr[i, i])
        d[i] = x
        qr[i, i:] = qr[i, i:] / x
    return qr, d, jpvt - 1, tau


def _ungqr(qr, tau):
    q, _, info = lapack.zungqr(qr, tau, lwork=max(1, 64 * qr.shape[0]))
    if info != 0:
        raise RuntimeError(f"zungqr info={info}")
    return q


@dataclass
class Propagator:
    """process_matrix.f90:6-15, 37-47."""
    n: int
    UUR: np.ndarray = None
    VUR: np.ndarray = None
    DUR: np.ndarray = None
    UUL: np.ndarray = None
    VUL: np.ndarray = None
    DUL: np.ndarray = None
    Gr: np.ndarray = None
    Xmaxm: float = 0.0
    Xmeanm: float = 0.0

    def __post_init__(self):
        n = self.n
        eye = np.eye(n, dtype=complex)
        self.UUR = eye.copy(); self.VUR = eye.copy(); self.DUR = np.ones(n, dtype=complex)
        self.UUL = eye.copy(); self.VUL = eye.copy(); self.DUL = np.ones(n, dtype=complex)
        self.Gr = eye.copy()


def stab_UR(prop: Propagator):
    """stabilization.f90:69-93."""
    mat = prop.UUR * prop.DUR[None, :]
    qr, d, piv, tau = qdrp_decompose(mat)
    prop.DUR = d
    v = prop.VUR[piv, :]                       # ZLAPMR forward: P^T V
    v = blas.ztrmm(1.0, qr, v, side=0, lower=0, trans_a=0, diag=0)
    prop.VUR = np.array(v)
    prop.UUR = _ungqr(qr, tau)


def stab_UL(prop: Propagator):
    """stabilization.f90:95-119."""
    mat = prop.UUL.conj().T * prop.DUL[None, :]
    qr, d, piv, tau = qdrp_decompose(mat)
    prop.DUL = d
    v = prop.VUL[:, piv]                       # ZLAPMT forward: V P
    v = blas.ztrmm(1.0, qr, v, side=1, lower=0, trans_a=2, diag=0)
    prop.VUL = np.array(v)
    prop.UUL = _ungqr(qr, tau).conj().T


def stab_green(prop: Propagator, nt: int, ltrot: int, want_logdet: bool = False):
    """G = (I - B)^-1 from the right and left UDV factors (stabilization.f90:121-190).

    With want_logdet, also returns sum(log D) of the final pivoted QR, so that
    log|det G| = -sum(log D) (the U factors are unitary).
    """
    n = prop.n
    vrvl = prop.VUR @ prop.VUL
    inv_ulur = prop.UUR.conj().T @ prop.UUL.conj().T
    temp = vrvl * prop.DUL[None, :]
    vrvl = prop.DUR[:, None] * temp
    mat = inv_ulur - vrvl
    if nt > ltrot // 2:
        mat = mat.conj().T
    qr, dup, piv, tau = qdrp_decompose(mat)
    lw = max(1, 64 * n)
    if nt < ltrot // 2 + 1:
        temp = np.asfortranarray(prop.UUR.conj().T)
        temp, _, info = lapack.zunmqr(b"L", b"C", qr, tau, temp, lw)
        if info != 0:
            raise RuntimeError("zunmqr")
        temp = temp / dup[:, None]
        temp = blas.ztrsm(1.0, qr, temp, side=0, lower=0, trans_a=0, diag=0)
        out = np.empty_like(temp)
        out[piv, :] = temp                      # ZLAPMR backward: P X
        gr = prop.UUL.conj().T @ out
    else:
        temp = np.asfortranarray(prop.UUL.conj().T)
        temp, _, info = lapack.zunmqr(b"R", b"N", qr, tau, temp, lw)
        if info != 0:
            raise RuntimeError("zunmqr")
        temp = temp / dup[None, :]
        temp = blas.ztrsm(1.0, qr, temp, side=1, lower=0, trans_a=2, diag=0)
        out = np.empty_like(temp)
        out[:, piv] = temp                      # ZLAPMT backward: X P^T
        gr = out @ prop.UUR.conj().T
    gr = np.array(gr)
    if want_logdet:
        return gr, float(np.sum(np.log(dup.real)))
    return gr


def compare_mat(a: np.ndarray, b: np.ndarray) -> float:
    """stabilization.f90:256-266 (L1 distance)."""
    return float(np.sum(np.abs(a - b)))


@dataclass
class WrapList:
    """process_matrix.f90:26-33, 94-101: slots 0..Nst of the left and right UDV factors."""
    n: int
    nst: int

    def __post_init__(self):
        n, m = self.n, self.nst + 1
        self.UR = np.zeros((m, n, n), dtype=complex)
        self.VR = np.zeros((m, n, n), dtype=complex)
        self.DR = np.zeros((m, n), dtype=complex)
        self.UL = np.zeros((m, n, n), dtype=complex)
        self.VL = np.zeros((m, n, n), dtype=complex)
        self.DL = np.zeros((m, n), dtype=complex)


# --------------------------------------------------------------------------
# equal-time observables (obser_equal.f90:6-198)
OBS_REAL = ("density_up", "density_do", "density_total", "kinetic", "doubleOcc", "squareOcc",
            "num_up", "num_do", "numsquare_up", "numsquare_do", "onsite_n2_up", "onsite_n2_do",
            "interaction_energy_density", "energy_density")
OBS_CPLX = ("sf_K", "psf_Gamma", "dw_K")


class ObserEqual:
    def __init__(self, lq: int):
        self.lq = lq
        self.reset()

    def reset(self):
        for k in OBS_REAL:
            setattr(self, k, 0.0)
        for k in OBS_CPLX:
            setattr(self, k, 0j)
        self.den_corr_up = np.zeros(self.lq, dtype=complex)
        self.den_corr_do = np.zeros(self.lq, dtype=complex)
        self.den_corr_updo = np.zeros(self.lq, dtype=complex)
        self.density_site_total = np.zeros(self.lq)

    def ave(self, nobs: int):
        z = 1.0 / float(nobs)
        for k in OBS_REAL:
            setattr(self, k, getattr(self, k) * z)
        for k in OBS_CPLX:
            setattr(self, k, getattr(self, k) * complex(z, 0.0))
        self.den_corr_up *= z
        self.den_corr_do *= z
        self.den_corr_updo *= z
        self.density_site_total *= z

    def calc(self, G: np.ndarray, p: Params, latt: Lattice):
        """obser_equal.f90:95-198."""
        n = p.Ndim
        lq = float(p.Lq)
        eye = np.eye(n)
        grup = G
        grupc = grup.T - eye
        grdo = G.conj()
        grdoc = grdo.T - eye
        du = np.diag(grupc)
        dd = np.diag(grdoc)
        dens_local = (du + dd).real
        self.density_up += float(np.sum(du.real / lq))
        self.density_do += float(np.sum(dd.real / lq))
        self.doubleOcc += float(np.sum((du * dd).real / lq))
        self.squareOcc += float(np.sum((du * du + dd * dd).real / lq))
        self.num_up += float(np.sum(du.real))
        self.num_do += float(np.sum(dd.real))
        self.density_total += float(np.sum(dens_local / lq))
        self.density_site_total += dens_local
        onsite_up = float(np.sum((2.0 * du * du + du).real))
        onsite_do = float(np.sum((2.0 * dd * dd + dd).real))
        double_s = float(np.sum((du * dd).real / lq))
        self.numsquare_up += float(np.sum((du[:, None] * du[None, :] + grupc * grup).real))
        self.numsquare_do += float(np.sum((dd[:, None] * dd[None, :] + grdoc * grdo).real))
        lq2 = complex(lq * lq, 0.0)
        psf = np.sum(grupc * grdoc) / lq2
        sfk = 0j
        dwk = 0j
        if latt.hasK:
            phase = np.exp(1j * latt.k_dot_r[latt.indexK, latt.imj])
            sfk = np.sum(phase * (grupc + grdoc)) / lq2
            term = (du[:, None] * du[None, :] + grupc * grup + dd[:, None] * dd[None, :] + grdoc * grdo
                    + du[:, None] * dd[None, :] + dd[:, None] * du[None, :])
            dwk = np.sum(phase * term) / lq2
        up_term = (du[:, None] * du[None, :] + grupc * grup) / complex(lq, 0.0)
        do_term = (dd[:, None] * dd[None, :] + grdoc * grdo) / complex(lq, 0.0)
        ud_term = (du[:, None] * dd[None, :]) / complex(lq, 0.0)
        np.add.at(self.den_corr_up, latt.imj.ravel(), up_term.ravel())
        np.add.at(self.den_corr_do, latt.imj.ravel(), do_term.ravel())
        np.add.at(self.den_corr_updo, latt.imj.ravel(), ud_term.ravel())
        kin = 0.0
        for nb in range(1, NBOND + 1):
            jj = latt.bonds[:, nb]
            ii = np.arange(n)
            kin += float(np.sum(p.RT * (grupc[ii, jj] + grupc[jj, ii] + grdoc[ii, jj] + grdoc[jj, ii]).real / lq))
        inter = (p.U1 + p.U2) * (onsite_up + onsite_do) / lq + 2.0 * (p.U2 - p.U1) * double_s
        self.kinetic += kin
        self.onsite_n2_up += onsite_up
        self.onsite_n2_do += onsite_do
        self.interaction_energy_density += inter
        self.energy_density += kin + inter
        self.sf_K += complex(sfk)
        self.psf_Gamma += complex(psf)
        self.dw_K += complex(dwk)

    def as_dict(self, latt: Lattice) -> dict:
        """The values the bin writer emits (fourier_trans.f90:250-348)."""
        out = {k: getattr(self, k) for k in OBS_REAL}
        for k in OBS_CPLX:
            out[k] = getattr(self, k)
        out["density_site_total"] = self.density_site_total.copy()
        # FFT_RtoK at momentum index "indexzero" (k = 0): exp(0) = 1 for every r
        lq = float(self.lq)
        out["den_upup_sub11"] = complex(np.sum(self.den_corr_up) / lq)
        out["den_dodo_sub11"] = complex(np.sum(self.den_corr_do) / lq)
        out["den_updo"] = complex(np.sum(self.den_corr_updo) / lq)
        return out


# --------------------------------------------------------------------------
# one Markov chain (one MPI rank of the reference)
class Chain:
    def __init__(self, p: Params, latt: Lattice, opT: OperatorKinetic, seed: int, phi: np.ndarray):
        self.p = p
        self.latt = latt
        self.opT = opT
        self.seed = int(seed)
        self.phi = np.array(phi, dtype=float)           # [Ltrot, Ns, Naux]
        self.op = [OperatorHubbard(p.U1, p.Dtau), OperatorHubbard(p.U2, p.Dtau)]
        self.prop = Propagator(p.Ndim)
        self.wr = WrapList(p.Ndim, p.Nst)
        self.obs = ObserEqual(p.Lq)
        self.nobs = 0
        self.acc_sum = [0.0, 0.0]        # sum over bins of per-bin acceptance ratio (AccCounter%acc)
        self.therm_acc_sum = [0.0, 0.0]
        self.last_logdet_M = None

    # ---- local update (localU.f90:31-77)
    def metro(self, nf: int, ii: int, nt: int):
        p, op, G = self.p, self.op[nf], self.prop.Gr
        phi_old = self.phi[nt, ii, nf]
        self.seed, xflip = ranf(self.seed)
        xdif = (xflip - 0.5) * abs(p.shiftLoc)
        phi_new = phi_old + xdif
        ratio_exp, delta = op.get_delta(phi_old, phi_new)
        ratio_det = 1.0 + delta * (1.0 - G[ii, ii])
        ratio_det = 1.0 / ratio_det
        ratio_abs = abs(ratio_exp * ratio_det * ratio_det.conjugate())
        self.seed, rnd = ranf(self.seed)
        if ratio_abs > rnd:
            op.count(True)
            temp_alpha = -ratio_det * delta
            col = G[:, ii].copy()
            vec = -G[ii, :].copy()
            vec[ii] += 1.0
            self.prop.Gr = G + temp_alpha * np.outer(col, vec)
            self.phi[nt, ii, nf] = phi_new
        else:
            op.count(False)

    def _expalpha(self, nf, phi, nflag):
        return self.op[nf].get_exp(phi, nflag)[1]

    def prop_L(self, nf: int, nt: int):
        """LocalU_prop_L (localU.f90:79-95)."""
        n = self.p.Ndim
        for ii in range(n - 1, -1, -1):
            self.metro(nf, ii, nt)
            G = self.prop.Gr
            G[:, ii] *= self._expalpha(nf, self.phi[nt, ii, nf], 1)
            G[ii, :] *= self._expalpha(nf, self.phi[nt, ii, nf], -1)
        for ii in range(n - 1, -1, -1):
            self.prop.UUL[:, ii] *= self._expalpha(nf, self.phi[nt, ii, nf], 1)

    def prop_R(self, nf: int, nt: int):
        """LocalU_prop_R (localU.f90:97-113)."""
        n = self.p.Ndim
        for ii in range(n):
            G = self.prop.Gr
            G[ii, :] *= self._expalpha(nf, self.phi[nt, ii, nf], 1)
            G[:, ii] *= self._expalpha(nf, self.phi[nt, ii, nf], -1)
            self.metro(nf, ii, nt)
        for ii in range(n):
            self.prop.UUR[ii, :] *= self._expalpha(nf, self.phi[nt, ii, nf], 1)

    # ---- prior-only warm-up (localU.f90:115-145; local_sweep.f90:64-78)
    def therm(self):
        p = self.p
        for o in self.op:
            o.reset()
        for nt in range(p.Ltrot):
            for nf in (0, 1):
                o = self.op[nf]
                if not o.active:
                    continue
                for ii in range(p.Ndim):
                    phi_old = self.phi[nt, ii, nf]
                    self.seed, xflip = ranf(self.seed)
                    phi_new = phi_old + (xflip - 0.5) * abs(p.shiftLoc)
                    ratio_exp, _ = o.get_delta(phi_old, phi_new)
                    self.seed, rnd = ranf(self.seed)
                    if abs(ratio_exp) > rnd:
                        o.count(True)
                        self.phi[nt, ii, nf] = phi_new
                    else:
                        o.count(False)
        for nf in (0, 1):
            if self.op[nf].active:
                self.therm_acc_sum[nf] += self.op[nf].nacc / self.op[nf].nc

    # ---- slice propagation (multiply.f90:7-16, 66-86)
    def _scale_rows(self, M, nf, nt, nflag):
        for ii in range(self.p.Ndim):
            M[ii, :] *= self._expalpha(nf, self.phi[nt, ii, nf], nflag)

    def propT_L(self):
        pr, o = self.prop, self.opT
        pr.Gr = pr.Gr @ o.expT_P
        pr.Gr = o.expT_M @ pr.Gr
        pr.UUL = pr.UUL @ o.expT_P

    def propT_R(self):
        pr, o = self.prop, self.opT
        pr.Gr = o.expT_P @ pr.Gr
        pr.Gr = pr.Gr @ o.expT_M
        pr.UUR = o.expT_P @ pr.UUR

    # ---- wraps (stabilization.f90:268-366)
    def wrap_pre(self, nt: int):
        p, pr, wr = self.p, self.prop, self.wr
        st = nt // p.Nwrap
        if nt != 0:
            stab_UR(pr)
        wr.UR[st] = pr.UUR; wr.VR[st] = pr.VUR; wr.DR[st] = pr.DUR
        if nt == p.Ltrot:
            pr.Gr = stab_green(pr, nt, p.Ltrot)

    def _drift(self, gr):
        pr = self.prop
        dif = compare_mat(gr, pr.Gr)
        if dif > pr.Xmaxm:
            pr.Xmaxm = dif
        pr.Xmeanm += dif
        pr.Gr = gr

    def wrap_L(self, nt: int):
        p, pr, wr = self.p, self.prop, self.wr
        st = nt // p.Nwrap
        pr.UUR = wr.UR[st].copy(); pr.VUR = wr.VR[st].copy(); pr.DUR = wr.DR[st].copy()
        if nt == 0:
            wr.UR[:] = 0; wr.VR[:] = 0; wr.DR[:] = 0
        if nt != p.Ltrot:
            stab_UL(pr)
            self._drift(stab_green(pr, nt, p.Ltrot))
        wr.UL[st] = pr.UUL; wr.VL[st] = pr.VUL; wr.DL[st] = pr.DUL

    def wrap_R(self, nt: int):
        p, pr, wr = self.p, self.prop, self.wr
        st = nt // p.Nwrap
        pr.UUL = wr.UL[st].copy(); pr.VUL = wr.VL[st].copy(); pr.DUL = wr.DL[st].copy()
        if nt == p.Ltrot:
            wr.UL[:] = 0; wr.VL[:] = 0; wr.DL[:] = 0
        if nt != 0:
            stab_UR(pr)
            if nt == p.Ltrot:
                gr, self.last_logdet_M = stab_green(pr, nt, p.Ltrot, want_logdet=True)
            else:
                gr = stab_green(pr, nt, p.Ltrot)
            self._drift(gr)
        wr.UR[st] = pr.UUR; wr.VR[st] = pr.VUR; wr.DR[st] = pr.DUR

    # ---- sweep schedule (local_sweep.f90:80-161)
    def pre(self):
        p, pr = self.p, self.prop
        self.wrap_pre(0)
        for nt in range(1, p.Ltrot + 1):
            for nf in (0, 1):
                if self.op[nf].active:
                    self._scale_rows(pr.UUR, nf, nt - 1, 1)
            pr.UUR = self.opT.expT_P @ pr.UUR
            if nt % p.Nwrap == 0:
                self.wrap_pre(nt)

    def measure(self):
        self.obs.calc(self.prop.Gr, self.p, self.latt)
        self.nobs += 1

    def sweep_L(self):
        p = self.p
        for nt in range(p.Ltrot, 0, -1):
            if nt % p.Nwrap == 0:
                self.wrap_L(nt)
            self.measure()
            self.propT_L()
            if self.op[1].active:
                self.prop_L(1, nt - 1)
            if self.op[0].active:
                self.prop_L(0, nt - 1)
        self.wrap_L(0)

    def sweep_R(self):
        p = self.p
        self.wrap_R(0)
        for nt in range(1, p.Ltrot + 1):
            if self.op[0].active:
                self.prop_R(0, nt - 1)
            if self.op[1].active:
                self.prop_R(1, nt - 1)
            self.propT_R()
            if nt % p.Nwrap == 0:
                self.wrap_R(nt)
            self.measure()

    def sweep_bin(self):
        """Local_sweep%sweep with is_beta=.true. (local_sweep.f90:136-161)."""
        for o in self.op:
            o.reset()
        self.obs.reset()
        self.nobs = 0
        for _ in range(self.p.Nsweep):
            self.sweep_L()
            self.sweep_R()
        self.obs.ave(self.nobs)
        for nf in (0, 1):
            if self.op[nf].active:
                self.acc_sum[nf] += self.op[nf].nacc / self.op[nf].nc

    # ---- diagnostics (fields.f90:29-33; pole_diagnostics.f90:91-123)
    def log_weight_fields(self) -> float:
        return float(-0.5 * np.sum(self.phi * self.phi))

    def pole_diagnostics(self):
        G = self.prop.Gr
        small = np.finfo(float).tiny
        ev = np.linalg.eigvals(G)
        sv = np.linalg.svd(G, compute_uv=False)
        z = np.where(np.abs(ev) <= small, complex(1.0 / small, 0.0), 1.0 / np.where(ev == 0, 1, ev))
        pole_distance = max(float(np.min(np.abs(z))), small)
        return {
            "pole_z": z,
            "pole_distance": pole_distance,
            "pole_x": -math.log10(pole_distance),
            "green_spectral_radius": float(np.max(np.abs(ev))),
            "green_smax": float(np.max(sv)),
            "log_weight": self.log_weight_fields() + 2.0 * float(np.sum(np.log(np.maximum(sv, small)))),
        }


# --------------------------------------------------------------------------
# ensemble of chains = the reference's MPI job (main.f90:22-85)
def init_chains(p: Params, seeds: list[int] | None = None, confin: list | None = None):
    """conf_therm_in (fields.f90:47-113): seeds -> fields, or explicit (seed, phi) per chain."""
    latt = Lattice(p)
    opT = OperatorKinetic(p, latt)
    chains = []
    if confin is not None:
        for seed, phi_therm in confin:
            phi = conf_transfer(p, np.asarray(phi_therm).reshape(p.LtrotTherm, -1, NAUX))
            chains.append(Chain(p, latt, opT, seed, phi))
    else:
        for s in seeds:
            s2, phi_therm = conf_set(p, int(s))
            chains.append(Chain(p, latt, opT, s2, conf_transfer(p, phi_therm)))
    return latt, opT, chains


def chain_average(chains: list[Chain]) -> dict:
    """m_process_obs_equal (fourier_trans.f90:350-457): sum over ranks / ISIZE."""
    dicts = [c.obs.as_dict(c.latt) for c in chains]
    out = {}
    for k in dicts[0]:
        vals = [d[k] for d in dicts]
        if isinstance(vals[0], np.ndarray):
            out[k] = np.sum(vals, axis=0) / float(len(vals))
        elif isinstance(vals[0], complex):
            out[k] = complex(sum(vals)) / complex(float(len(vals)), 0.0)
        else:
            out[k] = float(sum(vals)) / float(len(vals))
    return out


def run(p: Params, seeds=None, confin=None, want_pole=True, callback=None):
    """main.f90 flow for one job; returns (per-bin chain averages, chains)."""
    latt, opT, chains = init_chains(p, seeds, confin)
    if p.is_warm:
        for _ in range(p.Nwarm):
            for c in chains:
                c.therm()
    for c in chains:
        c.pre()
    bins = []
    for nbc in range(p.Nbin):
        for c in chains:
            c.sweep_bin()
        avg = chain_average(chains)
        if want_pole:
            avg["pole"] = [c.pole_diagnostics() for c in chains]
        bins.append(avg)
        if callback is not None:
            callback(nbc, chains, avg)
    return bins, chains


def read_confin(path: Path, p: Params, nchains: int):
    """Parse confin.txt; returns None for a leading 0 (seed-generated fields)."""
    toks = Path(path).read_text().split()
    if int(float(toks[0])) == 0:
        return None
    per = p.LtrotTherm * p.NlxTherm * p.NlyTherm * NAUX
    out = []
    pos = 0
    for _ in range(nchains):
        seed = int(float(toks[pos])); pos += 1
        vals = np.array([_float(t) for t in toks[pos:pos + per]]); pos += per
        out.append((seed, vals))
    return out
