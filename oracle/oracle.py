"""CPU oracle for the BAFQMC finite-temperature sweep (number-conserving and
Nambu pairing solvers).

TEST INFRASTRUCTURE ONLY.  This module is the parity checker for the CUDA
path in ``bafqmc_b200``.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline / reference legs of ``bench.py`` may import it; the product path
never does, and it must not be used as a fallback.

It restates, call for call, the reference Fortran solvers of YinkaiYu/BAFQMC
(files cited as ``src/number_conserving/src/<file>.f90:<line>``; the Nambu
solver's files as ``src/pairing/src/<file>.f90:<line>``) in NumPy,
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
The pairing path is pinned by the same Gaussian closed forms at Delta = 0,
+-0.2 (pair_equal included), by its Delta = 0 agreement with the
number-conserving path, and by a dense fixed-field reference of the Nambu
Green's function and estimators built in ``tests/test_oracle_pairing.py``.
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
NSEC = 4            # pairing sectors b, c, b^dagger, c^dagger (src/pairing/src/calc_basic.f90:13)
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
    RDelta: float = 0.0
    pairing: bool = False
    # Nambu propagator by scipy.linalg.expm instead of the reference's ZGEEV form
    # (an exact exponential, for separating the reference's propagator error from
    # the device's at points where G amplifies it)
    exact_expm: bool = False

    @property
    def Lq(self) -> int:
        return self.Nlx * self.Nly

    @property
    def Nsite(self) -> int:
        return self.Lq

    @property
    def Ndim(self) -> int:
        """Ns, or Nsite*Nsec for the Nambu solver (src/pairing/src/calc_basic.f90:99-101)."""
        return NSEC * self.Lq if self.pairing else self.Lq

    @property
    def Dtau(self) -> float:
        return self.Beta / float(self.Ltrot)

    @property
    def Nst(self) -> int:
        if self.Ltrot % self.Nwrap != 0:
            raise ValueError("Ltrot is not a multiple of Nwrap")
        return self.Ltrot // self.Nwrap

    @classmethod
    def from_text(cls, text: str, pairing: bool = False) -> "Params":
        """read_input (calc_basic.f90:48-59); the pairing solver reads RDelta as the
        fourth value of line 1 (src/pairing/src/calc_basic.f90:51-52)."""
        rows = [ln.replace(",", " ").split() for ln in text.splitlines()]
        rows = [r for r in rows][:7]
        r = [[_fortran_token(t) for t in row] for row in rows]
        p = cls(
            U1=_float(r[0][0]), U2=_float(r[0][1]), mu=_float(r[0][2]),
            RDelta=_float(r[0][3]) if pairing else 0.0, pairing=pairing,
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


def inv_dim(latt_lq: int, site: int, sec: int) -> int:
    """inv_dim_list(site, sec) of the Nambu lattice, 0-based: sector-major order
    b, c, b^dagger, c^dagger (src/pairing/src/lattice.f90:26-35)."""
    return sec * latt_lq + site


def ham_T_pairing(p: Params, latt: Lattice) -> np.ndarray:
    """def_hamT of the Nambu solver (src/pairing/src/non_interact.f90:33-111)."""
    ns = p.Lq
    n = p.Ndim
    H = np.zeros((n, n), dtype=complex)
    z = complex(p.RT, 0.0)
    for i in range(ns):
        i1, i2, i3, i4 = (inv_dim(ns, i, k) for k in range(NSEC))
        for nb in range(1, NBOND + 1):
            j = latt.bonds[i, nb]
            j1, j2, j3, j4 = (inv_dim(ns, j, k) for k in range(NSEC))
            H[i1, j1] += z
            H[i2, j2] += z
            H[j3, i3] -= z
            H[j4, i4] -= z
            H[j1, i1] += z.conjugate()
            H[j2, i2] += z.conjugate()
            H[i3, j3] -= z.conjugate()
            H[i4, j4] -= z.conjugate()
    z = complex(p.RDelta, 0.0)
    for i in range(ns):
        i1, i2, i3, i4 = (inv_dim(ns, i, k) for k in range(NSEC))
        H[i1, i4] += z
        H[i2, i3] += z
        H[i3, i2] -= z
        H[i4, i1] -= z
    z = complex(-p.mu, 0.0)
    for i in range(ns):
        i1, i2, i3, i4 = (inv_dim(ns, i, k) for k in range(NSEC))
        H[i1, i1] += z
        H[i2, i2] += z
        H[i3, i3] -= z
        H[i4, i4] -= z
    return H


def inv_and_det(a: np.ndarray):
    """ZGETRF + ZGETRI with the LU determinant (src/common/mymats.f90:52-77;
    src/pairing/src/localU.f90:194-220)."""
    lu, ipiv, info = lapack.zgetrf(np.asfortranarray(a))
    if info < 0:
        raise RuntimeError(f"zgetrf info={info}")
    det = complex(1.0, 0.0)
    for i in range(a.shape[0]):
        det = det * lu[i, i]
        if ipiv[i] != i:
            det = -det
    ainv, info = lapack.zgetri(lu, ipiv)
    if info != 0:
        raise RuntimeError(f"zgetri info={info}")
    return np.array(ainv), det


class OperatorKinetic:
    def __init__(self, p: Params, latt: Lattice):
        if p.pairing:
            # opT_set + exp_general_matrix (src/pairing/src/non_interact.f90:113-178): the
            # Nambu matrix is not Hermitian, so ZGEEV, the inverse eigenvector matrix and
            # exp(-+dtau w) on the eigenvalues.
            H = ham_T_pairing(p, latt)
            if p.exact_expm:
                from scipy.linalg import expm
                w = np.linalg.eigvals(H)
                self.energy_min = float(np.min(w.real))
                self.energy_max = float(np.max(w.real))
                self.bandwidth = self.energy_max - self.energy_min
                self.expT_P = expm(-p.Dtau * H)
                self.expT_M = expm(p.Dtau * H)
                return
            w, V = np.linalg.eig(H)
            Vinv, _ = inv_and_det(V)
            self.energy_min = float(np.min(w.real))
            self.energy_max = float(np.max(w.real))
            self.bandwidth = self.energy_max - self.energy_min
            self.expT_P = (V * np.exp(-p.Dtau * w)[None, :]) @ Vinv
            self.expT_M = (V * np.exp(p.Dtau * w)[None, :]) @ Vinv
            return
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
CHANNEL_RELATIVE = 1   # U1 (n_b - n_c)^2 (src/pairing/src/operator_Hubbard.f90:10-11)
CHANNEL_TOTAL = 2      # U2 (n_b + n_c)^2
# sign of alpha*phi in the factor of each Nambu sector b, c, b^dagger, c^dagger
# (src/pairing/src/operator_Hubbard.f90:155-166, 186-197)
SECTOR_SIGN = {CHANNEL_RELATIVE: (1, -1, -1, 1), CHANNEL_TOTAL: (1, 1, -1, -1)}


class PhaseCounter:
    """Phase statistics of the Nambu weight ratio (src/pairing/src/operator_Hubbard.f90:228-284)."""

    def __init__(self):
        self.count_proposed = 0.0
        self.count_accepted = 0.0
        self.sum_abs_arg_proposed = 0.0
        self.sum_abs_arg_accepted = 0.0
        self.branch_pi_count = 0.0
        self.reset()

    def reset(self):
        self.nc_prop_bin = 0.0
        self.nc_acc_bin = 0.0
        self.sum_abs_prop_bin = 0.0
        self.sum_abs_acc_bin = 0.0
        self.branch_pi_count_bin = 0.0

    def count(self, phase: float, accepted: bool):
        a = abs(phase)
        self.nc_prop_bin += 1.0
        self.sum_abs_prop_bin += a
        if a > 0.9 * PI:
            self.branch_pi_count_bin += 1.0
        if accepted:
            self.nc_acc_bin += 1.0
            self.sum_abs_acc_bin += a

    def ratio(self):
        self.count_proposed += self.nc_prop_bin
        self.count_accepted += self.nc_acc_bin
        self.sum_abs_arg_proposed += self.sum_abs_prop_bin
        self.sum_abs_arg_accepted += self.sum_abs_acc_bin
        self.branch_pi_count += self.branch_pi_count_bin


class OperatorHubbard:
    def __init__(self, U: float, dtau: float, channel: int = 0):
        self.alpha = 0j
        if U < -ZERO:
            self.alpha = complex(math.sqrt(-2.0 * U * dtau), 0.0)
        if U > ZERO:
            self.alpha = complex(0.0, math.sqrt(2.0 * U * dtau))
        self.active = abs(U) > ZERO
        self.channel = channel
        self.acc_local = 0.0
        self.acc_therm = 0.0
        self.nc = 0
        self.nacc = 0
        self.phase = PhaseCounter()

    def get_delta_pairing(self, phi_old: float, phi_new: float):
        """opU_get_delta of the Nambu solver (src/pairing/src/operator_Hubbard.f90:100-137).

        Returns (ratio_gaussian, ratio_constant, diagonal of the 4x4 Delta)."""
        g_old, e_old = self.get_exp(phi_old, 1)
        g_new, e_new = self.get_exp(phi_new, 1)
        ratio_gaussian = g_new / g_old
        ratio_constant = complex(1.0, 0.0)
        if self.channel == CHANNEL_TOTAL:
            ratio_constant = e_old / e_new
        dphi = phi_new - phi_old
        p = cmath.exp(self.alpha * dphi * 1) - 1.0
        m = cmath.exp(-self.alpha * dphi * 1) - 1.0
        d = tuple(p if sg > 0 else m for sg in SECTOR_SIGN[self.channel])
        return ratio_gaussian, ratio_constant, np.array(d, dtype=complex)

    def sector_factors(self, phi: float, nflag: int) -> np.ndarray:
        """exp(+-alpha*phi*nflag) per sector, as opU_mmult_R/L apply them."""
        ep = cmath.exp(self.alpha * phi * nflag)
        em = cmath.exp(-self.alpha * phi * nflag)
        return np.array([ep if sg > 0 else em for sg in SECTOR_SIGN[self.channel]], dtype=complex)

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


@dataclass
class PropGreen:
    """The time-displaced Green's functions (process_matrix.f90:17-24, 62-84):
    Gr00 = G(0,0), Grtt = G(tau,tau), Grt0 = G(tau,0), Gr0t = G(0,tau), and the
    drift maxima / sums of Wrap_tau (index 0: Gr0t, 1: Grt0, 2: Grtt, the order
    Wrap_tau fills them, stabilization.f90:384-398)."""
    n: int

    def __post_init__(self):
        self.Xmaxm = [0.0, 0.0, 0.0]
        self.Xmeanm = [0.0, 0.0, 0.0]

    def reset(self, gr: np.ndarray):
        """Propgr_reset (process_matrix.f90:75-84)."""
        self.Gr00 = gr.copy()
        self.Grtt = gr.copy()
        self.Grt0 = gr.copy()
        self.Gr0t = -(np.eye(self.n, dtype=complex) - gr)


def udv_unpivoted(a: np.ndarray):
    """MyMats udv (src/common/mymats.f90:79-117): A = U diag(D) V by ZGEQRF without
    pivoting, D = |diag R|, V = R / D row-wise, U from ZUNGQR."""
    n = a.shape[0]
    qr, tau, _, info = lapack.zgeqrf(np.asfortranarray(a), lwork=max(1, 64 * n))
    if info != 0:
        raise RuntimeError(f"zgeqrf info={info}")
    d = np.abs(np.diag(qr)).astype(complex)
    v = np.triu(qr) / d[:, None]
    return _ungqr(qr, tau), d, v


def stab_green_big(prop: Propagator, fermion_sign: bool = False):
    """stabilization.f90:192-254: the 2N x 2N inverse whose blocks are G(0,0),
    G(0,tau), G(tau,0), G(tau,tau), from the right factors of B(tau,0) and the left
    factors of B(beta,tau).  Returns (Gr00, Gr0t, Grt0, Grtt).

    The middle matrix is diag(VUL, UUR)^-1 K diag(VUR, UUL)^-1 with
    K = [[I, s B(beta,tau)], [-B(tau,0), I]], whose inverse has top-left block
    (I - s B(beta,0))^-1.  The reference puts +DUL in the top-right block
    (stabilization.f90:206-209), i.e. s = -1, the fermion sign: its G(0,0) block
    is (I + B)^-1, not the bosonic G = (I - B)^-1 of stab_green.  The default
    here is the bosonic s = +1, consistent with the slice-by-slice propagation;
    fermion_sign=True reproduces the reference's matrix."""
    n = prop.n
    inv = np.linalg.inv   # ZGETRF + ZGETRI (MyMats inv)
    inv_ulur = inv(prop.UUL @ prop.UUR)
    inv_vrvl = inv(prop.VUR @ prop.VUL)
    big = np.zeros((2 * n, 2 * n), dtype=complex)
    big[:n, :n] = inv_vrvl
    big[n:, n:] = inv_ulur
    for r in range(n):
        big[r, r + n] = prop.DUL[r] if fermion_sign else -prop.DUL[r]
        big[r + n, r] = -prop.DUR[r]
    bu, bd, bv = udv_unpivoted(big)
    left = np.zeros((2 * n, 2 * n), dtype=complex)
    left[:n, :n] = inv(prop.VUR)
    left[n:, n:] = inv(prop.UUL)
    left = left @ inv(bv)
    right = np.zeros((2 * n, 2 * n), dtype=complex)
    right[:n, :n] = inv(prop.VUL)
    right[n:, n:] = inv(prop.UUR)
    right = inv(bu) @ right
    left = left / bd[None, :]
    tot = left @ right
    return tot[:n, :n], tot[:n, n:], tot[n:, :n], tot[n:, n:]


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
# equal-time observables of the Nambu solver (src/pairing/src/obser_equal.f90)
OBS_REAL_PAIR = ("density_up", "density_do", "density", "density_total", "kinetic", "doubleOcc", "squareOcc",
                 "local_numsquare", "pair_equal", "num_up", "num_do", "numsquare_up", "numsquare_do",
                 "onsite_n2_up", "onsite_n2_do", "interaction_energy_density", "pairing_energy_density",
                 "chemical_energy_density", "grand_energy_density", "energy_density")


class ObserEqualPairing:
    def __init__(self, lq: int):
        self.lq = lq
        self.reset()

    def reset(self):
        """Obs_equal_reset (obser_equal.f90:43-74)."""
        for k in OBS_REAL_PAIR:
            setattr(self, k, 0.0)
        for k in OBS_CPLX:
            setattr(self, k, 0j)
        self.den_corr_up = np.zeros(self.lq, dtype=complex)
        self.den_corr_do = np.zeros(self.lq, dtype=complex)
        self.den_corr_updo = np.zeros(self.lq, dtype=complex)
        self.single_corr = np.zeros(self.lq, dtype=complex)
        self.density_site_total = np.zeros(self.lq)

    def ave(self, nobs: int):
        """Obs_equal_ave (obser_equal.f90:76-110)."""
        z = 1.0 / float(nobs)
        for k in OBS_REAL_PAIR:
            setattr(self, k, getattr(self, k) * z)
        for k in OBS_CPLX:
            setattr(self, k, getattr(self, k) * z)
        self.den_corr_up *= z
        self.den_corr_do *= z
        self.den_corr_updo *= z
        self.single_corr *= z
        self.density_site_total *= z

    def calc(self, G: np.ndarray, p: Params, latt: Lattice):
        """Obs_equal_calc (obser_equal.f90:112-271), Norb = 1."""
        ns = p.Lq
        lq = float(p.Lq)
        blk = lambda r, c: G[r * ns:(r + 1) * ns, c * ns:(c + 1) * ns]
        # rows b, c, b^dagger, c^dagger; the reference names a block by its row
        # operator and the conjugate of its column operator (obser_equal.f90:133-153)
        G_b_bdag, G_b_cdag, G_b_b, G_b_c = blk(0, 0), blk(0, 1), -blk(0, 2), -blk(0, 3)
        G_c_bdag, G_c_cdag, G_c_b, G_c_c = blk(1, 0), blk(1, 1), -blk(1, 2), -blk(1, 3)
        G_bdag_bdag, G_bdag_cdag, G_bdag_b, G_bdag_c = blk(2, 0), blk(2, 1), -blk(2, 2), -blk(2, 3)
        G_cdag_bdag, G_cdag_cdag, G_cdag_b, G_cdag_c = blk(3, 0), blk(3, 1), -blk(3, 2), -blk(3, 3)
        d = np.arange(ns)
        nb = G_bdag_b[d, d]
        nc = G_cdag_c[d, d]
        Dbb = nb * nb + G_bdag_b[d, d] * G_b_bdag[d, d] + G_bdag_bdag[d, d] * G_b_b[d, d]
        Dcc = nc * nc + G_cdag_c[d, d] * G_c_cdag[d, d] + G_cdag_cdag[d, d] * G_c_c[d, d]
        Dbc = nb * nc + G_bdag_cdag[d, d] * G_b_c[d, d] + G_bdag_c[d, d] * G_b_cdag[d, d]
        pair = (G_b_c[d, d] + G_bdag_cdag[d, d]).real
        s_density_total = 0.0
        s_double = 0.0
        s_pair = 0.0
        s_n2_up = 0.0
        s_n2_do = 0.0
        for ii in range(ns):   # site loop (obser_equal.f90:168-192), in the reference's order
            site = ii
            self.density_up += nb[ii].real / float(ns)
            self.density_do += nc[ii].real / float(ns)
            self.density += (nb[ii] + nc[ii]).real / float(ns)
            self.num_up += nb[ii].real
            self.num_do += nc[ii].real
            self.doubleOcc += Dbc[ii].real / float(ns)
            self.squareOcc += (nb[ii] * nb[ii] + nc[ii] * nc[ii]).real / float(ns)
            self.local_numsquare += (Dbb[ii] + Dcc[ii]).real / float(ns)
            self.pair_equal += pair[ii] / float(ns)
            self.density_site_total[site] += (nb[ii] + nc[ii]).real
            s_density_total += (nb[ii] + nc[ii]).real / float(ns)
            s_double += Dbc[ii].real / float(ns)
            s_pair += pair[ii] / float(ns)
            s_n2_up += Dbb[ii].real
            s_n2_do += Dcc[ii].real
        # pair loop (obser_equal.f90:194-233): i = row site ii, j = column site jj
        i = d[:, None]
        j = d[None, :]
        PDbb = G_bdag_b[i, i] * G_bdag_b[j, j] + G_bdag_b * G_b_bdag + G_bdag_bdag * G_b_b
        PDcc = G_cdag_c[i, i] * G_cdag_c[j, j] + G_cdag_c * G_c_cdag + G_cdag_cdag * G_c_c
        PDbc = G_bdag_b[i, i] * G_cdag_c[j, j] + G_bdag_cdag * G_b_c + G_bdag_c * G_b_cdag
        PDcb = G_cdag_c[i, i] * G_bdag_b[j, j] + G_cdag_bdag * G_c_b + G_cdag_b * G_c_bdag
        self.numsquare_up += float(np.sum(PDbb.real))
        self.numsquare_do += float(np.sum(PDcc.real))
        zlq = complex(lq, 0.0)
        np.add.at(self.den_corr_up, latt.imj.ravel(), (PDbb / zlq).ravel())
        np.add.at(self.den_corr_do, latt.imj.ravel(), (PDcc / zlq).ravel())
        np.add.at(self.den_corr_updo, latt.imj.ravel(), (PDbc / zlq).ravel())
        np.add.at(self.single_corr, latt.imj.ravel(), (G_bdag_b / zlq).ravel())
        norm_k = 1.0 / (lq * lq)
        sfk = 0j
        dwk = 0j
        if latt.hasK:
            phase = np.exp(1j * latt.k_dot_r[latt.indexK, latt.imj])
            sfk = complex(np.sum(phase * (G_bdag_b + G_cdag_c) * norm_k))
            dwk = complex(np.sum(phase * (PDbb + PDcc + PDbc + PDcb) * norm_k))
        psf = complex(np.sum((G_bdag_cdag[i, i] * G_c_b[j, j] + G_bdag_c * G_cdag_b + G_bdag_b * G_cdag_c) * norm_k))
        kin = 0.0
        for nbd in range(1, NBOND + 1):   # obser_equal.f90:235-244
            jj = latt.bonds[:, nbd]
            ii = np.arange(ns)
            terms = p.RT * (G_bdag_b[ii, jj] + G_bdag_b[jj, ii] + G_cdag_c[ii, jj] + G_cdag_c[jj, ii]).real / float(ns)
            kin += float(np.sum(terms))
        s_inter = (p.U1 + p.U2) * (s_n2_up + s_n2_do) / float(ns) + 2.0 * (p.U2 - p.U1) * s_double
        s_pairing = p.RDelta * s_pair
        s_chem = -p.mu * s_density_total
        s_energy = kin + s_inter + s_pairing
        self.kinetic += kin
        self.density_total += s_density_total
        self.onsite_n2_up += s_n2_up
        self.onsite_n2_do += s_n2_do
        self.interaction_energy_density += s_inter
        self.pairing_energy_density += s_pairing
        self.chemical_energy_density += s_chem
        self.energy_density += s_energy
        self.grand_energy_density += s_energy + s_chem
        self.sf_K += sfk
        self.dw_K += dwk
        self.psf_Gamma += psf

    def as_dict(self, latt: Lattice) -> dict:
        """The values the pairing bin writer emits (src/pairing/src/fourier_trans.f90:276-405)."""
        out = {k: getattr(self, k) for k in OBS_REAL_PAIR}
        for k in OBS_CPLX:
            out[k] = getattr(self, k)
        out["density_site_total"] = self.density_site_total.copy()
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
        self.op = [OperatorHubbard(p.U1, p.Dtau, CHANNEL_RELATIVE), OperatorHubbard(p.U2, p.Dtau, CHANNEL_TOTAL)]
        self.prop = Propagator(p.Ndim)
        self.wr = WrapList(p.Ndim, p.Nst)
        self.obs = ObserEqualPairing(p.Lq) if p.pairing else ObserEqual(p.Lq)
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

    # ---- Nambu local update (src/pairing/src/localU.f90:33-113)
    def _sec(self, site: int):
        return [inv_dim(self.p.Lq, site, k) for k in range(NSEC)]

    def metro_pairing(self, nf: int, site: int, nt: int):
        p, op, G = self.p, self.op[nf], self.prop.Gr
        phi_old = self.phi[nt, site, nf]
        self.seed, xflip = ranf(self.seed)
        xdif = (xflip - 0.5) * abs(p.shiftLoc)
        phi_new = phi_old + xdif
        ratio_gaussian, ratio_constant, dvec = op.get_delta_pairing(phi_old, phi_new)
        isec = self._sec(site)
        eye = np.eye(NSEC, dtype=complex)
        pblock = eye + dvec[:, None] * (eye - G[np.ix_(isec, isec)])
        pinv, det = inv_and_det(pblock)
        ratio_det = det ** (-0.5)
        ratio_exp = ratio_gaussian * ratio_constant
        ratio_total = ratio_exp * ratio_det
        ratio_phase = math.atan2(ratio_total.imag, ratio_total.real)
        ratio_abs = abs(ratio_total)
        self.seed, rnd = ranf(self.seed)
        if ratio_abs > rnd:
            op.count(True)
            op.phase.count(ratio_phase, True)
            left = G[:, isec]
            mid = pinv * dvec[None, :]
            right = -G[isec, :]
            right[np.arange(NSEC), isec] += 1.0
            self.prop.Gr = G - (left @ mid) @ right
            self.phi[nt, site, nf] = phi_new
        else:
            op.count(False)
            op.phase.count(ratio_phase, False)

    def _mmult_R(self, M, nf, site, phi, nflag):
        """opU_mmult_R: rows of the site's sectors (src/pairing/src/operator_Hubbard.f90:139-168)."""
        f = self.op[nf].sector_factors(phi, nflag)
        for k, r in enumerate(self._sec(site)):
            M[r, :] = f[k] * M[r, :]

    def _mmult_L(self, M, nf, site, phi, nflag):
        """opU_mmult_L: columns of the site's sectors (src/pairing/src/operator_Hubbard.f90:170-199)."""
        f = self.op[nf].sector_factors(phi, nflag)
        for k, c in enumerate(self._sec(site)):
            M[:, c] = M[:, c] * f[k]

    def prop_L_pairing(self, nf: int, nt: int):
        """LocalU_prop_L (src/pairing/src/localU.f90:115-131)."""
        ns = self.p.Lq
        for ii in range(ns - 1, -1, -1):
            self.metro_pairing(nf, ii, nt)
            self._mmult_L(self.prop.Gr, nf, ii, self.phi[nt, ii, nf], 1)
            self._mmult_R(self.prop.Gr, nf, ii, self.phi[nt, ii, nf], -1)
        for ii in range(ns - 1, -1, -1):
            self._mmult_L(self.prop.UUL, nf, ii, self.phi[nt, ii, nf], 1)

    def prop_R_pairing(self, nf: int, nt: int):
        """LocalU_prop_R (src/pairing/src/localU.f90:133-149)."""
        ns = self.p.Lq
        for ii in range(ns):
            self._mmult_R(self.prop.Gr, nf, ii, self.phi[nt, ii, nf], 1)
            self._mmult_L(self.prop.Gr, nf, ii, self.phi[nt, ii, nf], -1)
            self.metro_pairing(nf, ii, nt)
        for ii in range(ns):
            self._mmult_R(self.prop.UUR, nf, ii, self.phi[nt, ii, nf], 1)

    def _expalpha(self, nf, phi, nflag):
        return self.op[nf].get_exp(phi, nflag)[1]

    def prop_L(self, nf: int, nt: int):
        """LocalU_prop_L (localU.f90:79-95)."""
        if self.p.pairing:
            return self.prop_L_pairing(nf, nt)
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
        if self.p.pairing:
            return self.prop_R_pairing(nf, nt)
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
                for ii in range(p.Nsite):
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
        """propU_pre: opU_mmult_R on every site (multiply.f90:7-16)."""
        if self.p.pairing:
            for ii in range(self.p.Nsite):
                self._mmult_R(M, nf, ii, self.phi[nt, ii, nf], nflag)
            return
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

    # ---- time-displaced Green's functions (dynamics.f90:38-58, multiply.f90:48-97,
    # Wrap_tau stabilization.f90:368-404)
    def tau_sweep_R(self, u2_slot_bug: bool = False, fermion_sign: bool = False, on_slice=None):
        """Dyn_reset + Dyn_sweep_R at the start of a right traversal (both solvers;
        the pairing solver's dynamics.f90 is the same code on its 4Ns matrices): G(tau,0),
        G(0,tau) and G(tau,tau) propagated slice by slice from G(0,0), recomputed by
        stab_green_big every Nwrap slices, the drifts recorded in self.pg.
        The reference passes the U1 field slot to the U2 operator
        (dynamics.f90:52); u2_slot_bug=True reproduces that, False uses the U2 slot.
        fermion_sign=True uses the reference's stab_green_big matrix (see there).
        on_slice(nt, pg) is called after each slice's stabilisation (a test hook)."""
        import copy
        p, o = self.p, self.opT
        prop = copy.deepcopy(self.prop)          # Dyn_reset: Prop_d = Prop
        if not hasattr(self, "pg"):
            self.pg = PropGreen(p.Ndim)
        pg = self.pg
        pg.reset(self.prop.Gr)
        for nt in range(1, p.Ltrot + 1):
            for nf in (0, 1):
                if not self.op[nf].active:
                    continue
                slot = 0 if (u2_slot_bug and nf == 1) else nf
                if p.pairing:   # propgrU_R of the pairing solver (src/pairing/src/multiply.f90:48-64)
                    for ii in range(p.Nsite):
                        ph = self.phi[nt - 1, ii, slot]
                        self._mmult_R(pg.Grt0, nf, ii, ph, 1)
                        self._mmult_L(pg.Gr0t, nf, ii, ph, -1)
                        self._mmult_R(pg.Grtt, nf, ii, ph, 1)
                        self._mmult_L(pg.Grtt, nf, ii, ph, -1)
                    for ii in range(p.Nsite):
                        self._mmult_R(prop.UUR, nf, ii, self.phi[nt - 1, ii, slot], 1)
                    continue
                ep = np.array([self._expalpha(nf, self.phi[nt - 1, ii, slot], 1) for ii in range(p.Ndim)])
                em = np.array([self._expalpha(nf, self.phi[nt - 1, ii, slot], -1) for ii in range(p.Ndim)])
                pg.Grt0 = ep[:, None] * pg.Grt0
                pg.Gr0t = pg.Gr0t * em[None, :]
                pg.Grtt = ep[:, None] * pg.Grtt * em[None, :]
                prop.UUR = ep[:, None] * prop.UUR
            pg.Grt0 = o.expT_P @ pg.Grt0
            pg.Gr0t = pg.Gr0t @ o.expT_M
            pg.Grtt = (o.expT_P @ pg.Grtt) @ o.expT_M
            prop.UUR = o.expT_P @ prop.UUR
            if nt % p.Nwrap == 0:
                st = nt // p.Nwrap
                prop.UUL = self.wr.UL[st].copy(); prop.VUL = self.wr.VL[st].copy(); prop.DUL = self.wr.DL[st].copy()
                stab_UR(prop)
                g00, g0t, gt0, gtt = stab_green_big(prop, fermion_sign)
                for k, (new, old) in enumerate(((g0t, pg.Gr0t), (gt0, pg.Grt0), (gtt, pg.Grtt))):
                    dif = compare_mat(new, old)
                    pg.Xmaxm[k] = max(pg.Xmaxm[k], dif)
                    pg.Xmeanm[k] += dif
                pg.Gr00, pg.Gr0t, pg.Grt0, pg.Grtt = g00, g0t, gt0, gtt
            if on_slice is not None:
                on_slice(nt, pg)

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

    def sweep_R(self, tau: bool = False):
        p = self.p
        if tau:   # Local_sweep_R's toggle (local_sweep.f90:119-123)
            self.tau_sweep_R()
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

    def sweep_bin(self, tau: bool = False):
        """Local_sweep%sweep with is_beta=.true. (local_sweep.f90:136-161); tau runs
        the time-displaced pass at the start of each right traversal."""
        for o in self.op:
            o.reset()
            o.phase.reset()
        self.obs.reset()
        self.nobs = 0
        for _ in range(self.p.Nsweep):
            self.sweep_L()
            self.sweep_R(tau)
        self.obs.ave(self.nobs)
        for nf in (0, 1):
            if self.op[nf].active:
                self.acc_sum[nf] += self.op[nf].nacc / self.op[nf].nc
                if self.p.pairing:
                    self.op[nf].phase.ratio()   # src/pairing/src/local_sweep.f90:158-159

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
        if want_pole and not p.pairing:   # the pairing program has no pole diagnostics
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
