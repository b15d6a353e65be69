"""Pins of the Nambu (pairing) oracle, CPU only.

1. Gaussian closed forms of the reference test
   tests/physics/test_gaussian_solvers.py:44-77 (golden vectors in
   tests/golden/gaussian.json) at Delta = 0, +0.2, -0.2 and Nwrap = 10, 2,
   with that test's tolerances (abs 2e-9, rel 2e-8), pair_equal included, and
   the sign symmetry of test_pairing_phase_changes_only_the_anomalous_sign.
2. Delta = 0 with interactions: the Nambu solver samples the same weight as
   the number-conserving solver, so from the same seeds it takes the same
   decisions and measures the same observables (the interacting form of
   test_zero_pairing_matches_number_conserving_solver).
3. Dense fixed-field reference at Delta = 0.3 with both channels: with
   shiftLoc = 0 every proposal leaves the field unchanged, so each bin is the
   average over tau of the estimators of G(tau) = (I - B(tau,0) B(beta,tau))^-1.
   The reference is built here from scratch in the 2Ns block {b, c^dagger} of
   the Nambu matrix with its own Hamiltonian, propagators and estimator
   formulas, independent of the oracle's 4Ns code.
4. After sweeps with moves at Delta = 0.3, the oracle's G equals the dense
   (I - B(beta,0))^-1 of the final fields: the rank-4 Woodbury updates and the
   wraps reproduce the exact Green's function.
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest
from scipy.linalg import expm

from oracle.oracle import Lattice, OperatorKinetic, Params, ham_T_pairing, run

GOLDEN = Path(__file__).resolve().parent / "golden"


def _gauss_params(delta, nwrap):
    return Params(U1=0.0, U2=0.0, mu=-5.0, Nlx=3, Nly=3, Ltrot=100, Beta=1.0, NlxTherm=3, NlyTherm=3,
                  LtrotTherm=100, Nwrap=nwrap, Nbin=1, Nsweep=1, shiftLoc=1.0, iniAmpl=0.1,
                  RDelta=delta, pairing=True)


@pytest.mark.parametrize("nwrap", [10, 2])
@pytest.mark.parametrize("delta", [0.0, 0.2, -0.2])
def test_gaussian_closed_forms(delta, nwrap):
    g = json.loads((GOLDEN / "gaussian.json").read_text())
    tol = dict(abs_tol=g["params"]["abs_tol"], rel_tol=g["params"]["rel_tol"])
    exact = g["expected"]["0.0" if delta == 0.0 else "0.2"]
    bins, _ = run(_gauss_params(delta, nwrap), seeds=[24681357])
    b = bins[0]
    for k, v in exact.items():
        want = -v if (k == "pair_equal" and delta < 0) else v
        got = b[k].real if isinstance(b[k], complex) else b[k]
        assert math.isclose(got, want, **tol), (k, got, want)
    for k in ("sf_K", "dw_K"):
        assert math.isclose(b[k].imag, 0.0, **tol)
    if delta > 0:
        assert b["pair_equal"] < -0.01


def test_zero_pairing_interacting_matches_number_conserving():
    kw = dict(U1=1.0, U2=-0.5, mu=-5.0, Nlx=3, Nly=3, Ltrot=20, Beta=2.0, NlxTherm=3, NlyTherm=3,
              LtrotTherm=20, Nwrap=5, Nbin=2, Nsweep=1, shiftLoc=1.5, iniAmpl=1.0)
    bn, cn = run(Params(**kw), seeds=[4099, 777])
    bp, cp = run(Params(**kw, RDelta=0.0, pairing=True), seeds=[4099, 777])
    for a, b in zip(cn, cp):
        assert a.seed == b.seed
        np.testing.assert_array_equal(a.phi, b.phi)
        assert a.acc_sum == b.acc_sum
        for o in b.op:
            assert o.phase.count_proposed == 720 and o.phase.branch_pi_count == 0
            assert o.phase.sum_abs_arg_proposed < 1e-10
    for x, y in zip(bn, bp):
        for k in ("density_total", "density_up", "energy_density", "kinetic", "doubleOcc", "squareOcc",
                  "numsquare_up", "onsite_n2_up", "interaction_energy_density", "sf_K", "dw_K", "psf_Gamma",
                  "den_upup_sub11", "den_updo"):
            np.testing.assert_allclose(y[k], x[k], rtol=1e-10, atol=1e-16, err_msg=k)
        np.testing.assert_allclose(y["density_site_total"], x["density_site_total"], rtol=1e-10)


# ---------------------------------------------------------------------------
# independent 2Ns block reference
def _block_hamiltonian(lx, ly, mu, delta):
    """H on {b_i, c^dagger_i}: [[A - mu, Delta], [-Delta, -A + mu]], A the
    triangular-lattice adjacency with bonds (x+1,y), (x,y+1), (x-1,y+1)."""
    ns = lx * ly
    A = np.zeros((ns, ns))
    for y in range(ly):
        for x in range(lx):
            i = y * lx + x
            for dx, dy in ((1, 0), (0, 1), (-1, 1)):
                j = ((y + dy) % ly) * lx + (x + dx) % lx
                A[i, j] += 1.0
                A[j, i] += 1.0
    eye = np.eye(ns)
    return np.block([[A - mu * eye, delta * eye], [-delta * eye, -A + mu * eye]]), A


def _block_B(p, phi_slice, expK):
    """One slice of the block: e^{-dtau H} diag(f1 f2); U1 scales b and c^dagger by
    e^{alpha1 phi1}, U2 scales b by e^{alpha2 phi2} and c^dagger by e^{-alpha2 phi2}."""
    ns = p.Lq
    a1 = 1j * math.sqrt(2.0 * p.U1 * p.Dtau) if p.U1 > 1e-10 else 0.0
    a2 = math.sqrt(-2.0 * p.U2 * p.Dtau) if p.U2 < -1e-10 else 0.0
    f = np.ones(2 * ns, dtype=complex)
    f[:ns] *= np.exp(a1 * phi_slice[:, 0]) * np.exp(a2 * phi_slice[:, 1])
    f[ns:] *= np.exp(a1 * phi_slice[:, 0]) * np.exp(-a2 * phi_slice[:, 1])
    return expK * f[None, :]


def _block_green(p, phi, expK, nt):
    n = 2 * p.Lq
    M = np.eye(n, dtype=complex)
    for l in list(range(nt + 1, p.Ltrot + 1)) + list(range(1, nt + 1)):   # B(beta,tau) first, B(tau,0) last
        M = _block_B(p, phi[l - 1], expK) @ M
    return np.linalg.inv(np.eye(n) - M)


def _block_estimators(G1, p, A):
    """Estimators from the {b, c^dagger} block alone: with Ga = G1[b,b],
    Gb = G1[b,c^dagger], Gc = G1[c^dagger,b], Gd = G1[c^dagger,c^dagger],
    n_b(i) = -conj(Gd_ii) and n_c(i) = -Gd_ii; the (c, b^dagger) block is the
    complex conjugate of this one."""
    ns = p.Lq
    Ga, Gb, Gc, Gd = G1[:ns, :ns], G1[:ns, ns:], G1[ns:, :ns], G1[ns:, ns:]
    nb = -np.conj(np.diag(Gd))
    nc = -np.diag(Gd)
    Dbb_s = nb * nb + nb * np.diag(Ga)
    Dbc_s = nb * nc - np.conj(np.diag(Gc)) * np.diag(Gb)
    Dbb = nb[:, None] * nb[None, :] - np.conj(Gd) * Ga
    Dbc = nb[:, None] * nc[None, :] - np.conj(Gc) * Gb
    lat = Lattice(p)
    out = {}
    dens = float(np.sum(2.0 * nb.real)) / ns
    out["density_total"] = dens
    out["density_up"] = float(np.sum(nb.real)) / ns
    out["doubleOcc"] = float(np.sum(Dbc_s.real)) / ns
    out["local_numsquare"] = 2.0 * float(np.sum(Dbb_s.real)) / ns
    pair = float(np.sum(np.diag(Gc).real - np.diag(Gb).real)) / ns
    out["pair_equal"] = pair
    out["numsquare_up"] = float(np.sum(Dbb.real))
    kin = 0.0
    for i in range(ns):
        for j in range(ns):
            if A[i, j] != 0.0:
                kin += A[i, j] * (-2.0 * Gd[i, j].real) / ns
    out["kinetic"] = kin
    onsite = float(np.sum(Dbb_s.real))
    inter = (p.U1 + p.U2) * 2.0 * onsite / ns + 2.0 * (p.U2 - p.U1) * out["doubleOcc"]
    out["interaction_energy_density"] = inter
    out["energy_density"] = kin + inter + p.RDelta * pair
    out["grand_energy_density"] = out["energy_density"] - p.mu * dens
    ph = np.exp(1j * lat.k_dot_r[lat.indexK, lat.imj])
    out["sf_K"] = complex(np.sum(ph * (-2.0 * Gd.real))) / ns ** 2
    out["dw_K"] = complex(np.sum(ph * 2.0 * (Dbb.real + Dbc.real))) / ns ** 2
    out["psf_Gamma"] = complex(-np.conj(np.trace(Gc) * np.trace(Gb)) + np.sum(np.abs(Gd) ** 2)) / ns ** 2
    out["den_updo"] = complex(np.sum(Dbc)) / ns / ns
    out["density_site_total"] = 2.0 * nb.real
    return out


def _fixed_fields(p, seed=11):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((p.Ltrot, p.Lq, 2))


@pytest.mark.parametrize("nwrap", [1, 2, 6])
def test_dense_fixed_field_reference(nwrap):
    p = Params(U1=0.7, U2=-0.1, mu=-5.0, Nlx=3, Nly=3, Ltrot=6, Beta=0.6, NlxTherm=3, NlyTherm=3, LtrotTherm=6,
               Nwrap=nwrap, Nbin=1, Nsweep=1, shiftLoc=0.0, RDelta=0.3, pairing=True)
    phi = _fixed_fields(p)
    bins, chains = run(p, confin=[(12345, phi)])
    np.testing.assert_array_equal(chains[0].phi, phi)
    H1, A = _block_hamiltonian(3, 3, p.mu, p.RDelta)
    expK = expm(-p.Dtau * H1)
    ests = [_block_estimators(_block_green(p, phi, expK, nt), p, A) for nt in range(1, p.Ltrot + 1)]
    got = bins[0]
    for k in ests[0]:
        want = np.mean([e[k] for e in ests], axis=0)
        np.testing.assert_allclose(got[k], want, rtol=2e-10, atol=1e-13, err_msg=k)


def test_green_after_moves_is_exact():
    p = Params(U1=0.7, U2=-0.3, mu=-4.0, Nlx=3, Nly=3, Ltrot=12, Beta=1.2, NlxTherm=3, NlyTherm=3, LtrotTherm=12,
               Nwrap=3, Nbin=1, Nsweep=2, shiftLoc=1.5, RDelta=0.3, pairing=True)
    bins, chains = run(p, seeds=[97531])
    c = chains[0]
    assert 0.0 < c.acc_sum[0] < 1.0 and 0.0 < c.acc_sum[1] < 1.0
    H1, _ = _block_hamiltonian(3, 3, p.mu, p.RDelta)
    G1 = _block_green(p, c.phi, expm(-p.Dtau * H1), p.Ltrot)
    ns = p.Lq
    G = c.prop.Gr
    blk1 = np.ix_(list(range(ns)) + list(range(3 * ns, 4 * ns)), list(range(ns)) + list(range(3 * ns, 4 * ns)))
    blk2 = np.ix_(list(range(ns, 2 * ns)) + list(range(2 * ns, 3 * ns)), list(range(ns, 2 * ns)) + list(range(2 * ns, 3 * ns)))
    scale = np.max(np.abs(G1))
    np.testing.assert_allclose(G[blk1], G1, rtol=0, atol=1e-10 * scale)
    np.testing.assert_allclose(G[blk2], np.conj(G1), rtol=0, atol=1e-10 * scale)
    off = G.copy()
    off[blk1] = 0.0
    off[blk2] = 0.0
    assert np.max(np.abs(off)) < 1e-10 * scale


def test_reference_propagator_fails_on_the_finite_trace_boundary():
    """The reference forms the Nambu e^{-dtau H} from ZGEEV eigenvectors
    (src/pairing/src/non_interact.f90:131-178).  Inside mu < -3t - |Delta| that
    agrees with an exact exponential to ~1e-15; on the boundary (mu = -4,
    Delta = 1) the matrix is nearly defective and the eigenvector form is off
    by more than 1e-3, so a chain's G there depends on the propagator's
    construction, not only on the model.  (The device builds e^{-dtau H} by
    scaling and squaring, which agrees with scipy's expm at both points.)"""
    errs = {}
    for delta, mu in [(0.3, -5.0), (0.5, -4.0), (1.0, -4.0)]:
        p = Params(U1=1.0, U2=-0.5, mu=mu, Nlx=3, Nly=3, Ltrot=40, Beta=2.0, NlxTherm=3, NlyTherm=3,
                     LtrotTherm=40, Nwrap=10, Nbin=1, Nsweep=1, shiftLoc=1.5, iniType=2, iniAmpl=1.0, RDelta=delta,
                     pairing=True)
        latt = Lattice(p)
        kin = OperatorKinetic(p, latt)
        errs[(delta, mu)] = float(np.max(np.abs(kin.expT_P - expm(-p.Dtau * ham_T_pairing(p, latt)))))
    assert errs[(0.3, -5.0)] < 1e-13 and errs[(0.5, -4.0)] < 1e-13
    assert errs[(1.0, -4.0)] > 1e-3
