"""GPU parity of the sweep, called through the C ABI, against the oracle and
the reference's golden vectors.

Tolerances: G, weights and estimators 1e-10 relative (atol 1e-12 for values
that vanish); seeds, accepted fields and acceptance counts bit-exact.
"""
import json

import numpy as np
import pytest

from bafqmc_b200.params import SolverParams
from oracle import oracle as O

pytestmark = pytest.mark.gpu

RTOL = 1e-10
ATOL = 1e-12


@pytest.fixture(scope="module")
def solver_mod():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from bafqmc_b200 import build, solver
    build.build()
    return solver


def both_params(**kw):
    base = dict(U1=1.0, U2=0.0, mu=-5.0, Nlx=3, Nly=3, Ltrot=40, Beta=4.0, NlxTherm=3, NlyTherm=3,
                LtrotTherm=40, Nwrap=10, Nbin=2, Nsweep=1, shiftLoc=1.5, iniType=2, iniAmpl=1.0)
    base.update(kw)
    if "Ltrot" in kw and "LtrotTherm" not in kw:
        base["LtrotTherm"] = kw["Ltrot"]
    if "Nlx" in kw and "NlxTherm" not in kw:
        base["NlxTherm"] = kw["Nlx"]
    if "Nly" in kw and "NlyTherm" not in kw:
        base["NlyTherm"] = kw["Nly"]
    return O.Params(**base), SolverParams(**base)


def compare_bin(gpu: dict, ora: dict, label=""):
    for k in ("density_up", "density_do", "density_total", "kinetic", "doubleOcc", "squareOcc", "num_up", "num_do",
              "numsquare_up", "numsquare_do", "onsite_n2_up", "onsite_n2_do", "interaction_energy_density",
              "energy_density", "sf_K", "psf_Gamma", "dw_K", "den_upup_sub11", "den_dodo_sub11", "den_updo",
              "density_site_total"):
        np.testing.assert_allclose(np.atleast_1d(gpu[k]), np.atleast_1d(ora[k]), rtol=RTOL, atol=ATOL,
                                   err_msg=f"{label} {k}")


def compare_pole(gpu: dict, ora: dict, label=""):
    """Device pole diagnostics against the oracle's (ZGEEV/ZGESVD through NumPy).
    The poles are matched as sets: eigenvalue order is solver-specific."""
    for k in ("log_weight", "pole_distance", "pole_x", "green_spectral_radius", "green_smax"):
        np.testing.assert_allclose(gpu[k], ora[k], rtol=RTOL, atol=ATOL, err_msg=f"{label} {k}")
    zg, zo = list(gpu["pole_z"]), list(ora["pole_z"])
    assert len(zg) == len(zo)
    scale = max(abs(z) for z in zo)
    for z in zg:
        j = int(np.argmin([abs(z - w) for w in zo]))
        assert abs(z - zo[j]) <= RTOL * scale, f"{label} pole {z} vs {zo[j]}"
        zo.pop(j)


def assert_green_close(Gg, Go, label=""):
    err = np.max(np.abs(Gg - Go)) / np.max(np.abs(Go))
    assert err < RTOL, f"{label} G rel err {err:.3e}"


@pytest.mark.parametrize("nwrap", [1, 2, 6])
def test_fixed_field_matches_reference_dense(solver_mod, root, nwrap):
    """tests/physics/test_fixed_field_solver.py through the GPU (tolerance 2e-10)."""
    g = json.loads((root / "tests/golden/fixed_field.json").read_text())
    pp, exp, tol = g["params"], g["expected"], g["params"]["tolerance"]
    fields = np.array(g["fields_t_site_aux"])
    p = SolverParams(U1=pp["U1"], U2=pp["U2"], mu=pp["mu"], Nlx=3, Nly=3, Ltrot=6, Beta=pp["beta"], NlxTherm=3,
                     NlyTherm=3, LtrotTherm=6, Nwrap=nwrap, Nbin=3, Nsweep=1, shiftLoc=0.0, iniType=1,
                     iniAmpl=0.0)
    with solver_mod.Ensemble([p], [0]) as ens:
        ens.set_state([1357911], [fields])
        ens.pre()
        for _ in range(p.Nbin):
            ens.sweep(1)
            b = ens.point_obs()[0]
            for k in ("density_total", "density_site_total", "kinetic", "doubleOcc", "onsite_n2_up",
                      "onsite_n2_do", "interaction_energy_density", "energy_density"):
                np.testing.assert_allclose(np.atleast_1d(b[k]), np.atleast_1d(exp[k]), rtol=tol, atol=tol,
                                           err_msg=k)
            d = ens.pole_diagnostics()[0]
            for k in ("log_weight", "pole_distance", "pole_x", "green_spectral_radius", "green_smax"):
                np.testing.assert_allclose(d[k], exp[k], rtol=tol, atol=tol, err_msg=k)
        seeds, phis = ens.get_state()
        np.testing.assert_array_equal(phis[0], fields)


@pytest.mark.parametrize("nwrap", [10, 2])
def test_gaussian_closed_forms(solver_mod, root, nwrap):
    """tests/physics/test_gaussian_solvers.py number-conserving half (abs 2e-9, rel 2e-8)."""
    g = json.loads((root / "tests/golden/gaussian.json").read_text())
    exp = g["expected"]["0.0"]
    p = SolverParams(U1=0.0, U2=0.0, mu=-5.0, Nlx=3, Nly=3, Ltrot=100, Beta=1.0, NlxTherm=3, NlyTherm=3,
                     LtrotTherm=100, Nwrap=nwrap, Nbin=4, Nsweep=1, shiftLoc=1.0, iniType=2, iniAmpl=0.1)
    with solver_mod.Ensemble([p], [0]) as ens:
        ens.fields_from_seeds([7])
        ens.pre()
        for _ in range(p.Nbin):
            ens.sweep(1)
            b = ens.point_obs()[0]
            for k in ("density_total", "energy_density", "sf_K", "dw_K"):
                a = b[k].real if isinstance(b[k], complex) else b[k]
                assert abs(a - exp[k]) <= g["params"]["abs_tol"] + g["params"]["rel_tol"] * abs(exp[k]), k


def _run_both(op, sp, seeds, nbins, nwarm=0):
    latt, opT, chains = O.init_chains(op, seeds=seeds)
    from bafqmc_b200 import solver
    ens = solver.Ensemble([sp], [0] * len(seeds))
    ens.fields_from_seeds(seeds)
    s0, phi0 = ens.get_state()
    for c, ch in enumerate(chains):
        assert int(s0[c]) == ch.seed
        np.testing.assert_array_equal(phi0[c], ch.phi)
    if nwarm:
        for _ in range(nwarm):
            for ch in chains:
                ch.therm()
        ens.warmup_prior(nwarm)
        s1, phi1 = ens.get_state()
        for c, ch in enumerate(chains):
            assert int(s1[c]) == ch.seed
            np.testing.assert_array_equal(phi1[c], ch.phi)
    for ch in chains:
        ch.pre()
    ens.pre()
    for c, ch in enumerate(chains):
        assert_green_close(ens.green(c), ch.prop.Gr, "pre")
    for b in range(nbins):
        for ch in chains:
            ch.sweep_bin()
        ens.sweep(1)
        seeds_g, phis_g = ens.get_state()
        cobs = ens.chain_obs()
        cnt = ens.counters()
        lw = ens.log_weight()
        pole = ens.pole_diagnostics()
        for c, ch in enumerate(chains):
            assert int(seeds_g[c]) == ch.seed, f"bin {b} chain {c} seed"
            np.testing.assert_array_equal(phis_g[c], ch.phi, err_msg=f"bin {b} chain {c} fields")
            assert_green_close(ens.green(c), ch.prop.Gr, f"bin {b} chain {c}")
            compare_bin(cobs[c], ch.obs.as_dict(latt), f"bin {b} chain {c}")
            np.testing.assert_allclose(cnt[c, 0:2], ch.acc_sum, rtol=0, atol=0)
            np.testing.assert_allclose(lw[c], ch.pole_diagnostics()["log_weight"], rtol=RTOL)
            compare_pole(pole[c], ch.pole_diagnostics(), f"bin {b} chain {c}")
        avg = O.chain_average(chains)
        compare_bin(ens.point_obs()[0], avg, f"bin {b} average")
    ens.close()
    return chains


def test_config1_shape_one_channel(solver_mod):
    """3x3, L=40, beta=4, U1=1, U2=0 (only channel 1 active), Nwrap=10."""
    op, sp = both_params()
    _run_both(op, sp, [1234567], nbins=3)


def test_both_channels_with_prior_warmup(solver_mod):
    op, sp = both_params(U2=-0.5, Ltrot=20, Beta=2.0, Nwrap=5, is_warm=True, Nwarm=3)
    _run_both(op, sp, [99991, 4242, 777], nbins=2, nwarm=3)


def test_nonsquare_no_K_point(solver_mod):
    """4x3 lattice: no K point, sf_K and dw_K stay zero (obser_equal.f90:121-125)."""
    op, sp = both_params(Nlx=4, Nly=3, U2=-0.3, Ltrot=12, Beta=1.2, Nwrap=4)
    _run_both(op, sp, [31337], nbins=2)


def test_6x6_config2_point(solver_mod):
    """6x6, L=160, beta=8, U1=1, U2=-0.5, mu=-5, Nwrap=10 (the batched benchmark point), two chains."""
    op, sp = both_params(Nlx=6, Nly=6, Ltrot=160, Beta=8.0, U2=-0.5)
    _run_both(op, sp, [20240601, 17], nbins=1)


def test_ragged_points_one_handle(solver_mod):
    """Chains of different N, L and Nwrap in one handle and one launch per size class."""
    from bafqmc_b200 import solver
    specs = [dict(), dict(Nlx=4, Nly=4, Ltrot=16, Beta=1.6, Nwrap=4, U2=-0.5),
             dict(Nlx=6, Nly=3, Ltrot=12, Beta=0.6, Nwrap=3, U1=0.5, U2=-0.2, mu=-6.0)]
    pairs = [both_params(**s) for s in specs]
    chain_point = [0, 1, 2, 1, 0]
    seeds = [11, 22, 33, 44, 55]
    ens = solver.Ensemble([sp for _, sp in pairs], chain_point)
    ens.fields_from_seeds(seeds)
    ens.pre()
    ens.sweep(1)
    cobs = ens.chain_obs()
    for c, (pt, seed) in enumerate(zip(chain_point, seeds)):
        op = pairs[pt][0]
        latt, _, chains = O.init_chains(op, seeds=[seed])
        chains[0].pre()
        chains[0].sweep_bin()
        assert_green_close(ens.green(c), chains[0].prop.Gr, f"chain {c}")
        compare_bin(cobs[c], chains[0].obs.as_dict(latt), f"chain {c}")
    ens.close()


@pytest.mark.parametrize("lx,ly", [(8, 8), (6, 7)])
def test_n72_class_against_oracle(solver_mod, lx, ly):
    """N = 64 and 42 sites: the size class with G and U in shared memory and
    the two workspaces in HBM, one CTA per SM; 6x7 has no K point."""
    op, sp = both_params(U2=-0.5, Nlx=lx, Nly=ly, Ltrot=20, Beta=1.0, Nwrap=5)
    _run_both(op, sp, [31, 32], nbins=1)


def test_pole_diagnostics_near_the_band_edge(solver_mod):
    """4x4 (lowest free level at -2) at mu = -2.05, beta = 8 and weak coupling:
    G is far from the identity (largest singular values about 3.2 and 1.6,
    condition numbers 4.8 and 2.5), so the device eigenvalue and
    singular-value routines are checked on a non-trivial spectrum against
    ZGEEV/ZGESVD of the oracle's G."""
    op, sp = both_params(U1=0.2, U2=-0.05, mu=-2.05, Nlx=4, Nly=4, Ltrot=80, Beta=8.0, Nwrap=10)
    chains = _run_both(op, sp, [5, 6], nbins=1)
    assert max(ch.pole_diagnostics()["green_smax"] for ch in chains) > 2.0


def test_run_directory_number_conserving_program(solver_mod, tmp_path):
    """The run-directory contract of src/number_conserving: every per-bin file,
    including the pole files (one row per chain per bin), against the oracle."""
    op, sp = both_params(U2=-0.5, Nlx=4, Nly=4, Ltrot=40, Beta=4.0, Nbin=2)
    (tmp_path / "paramC_sets.txt").write_text(sp.to_text())
    (tmp_path / "confin.txt").write_text("0\n")
    (tmp_path / "seeds.txt").write_text("4099\n777\n")
    solver_mod.run_directory(tmp_path, nchains=2)
    bins, chains = O.run(op, seeds=[4099, 777])
    from bafqmc_b200.observables import FILE_ORDER
    for name in FILE_ORDER:
        rows = [ln.split() for ln in (tmp_path / name).read_text().splitlines() if ln.strip()]
        assert len(rows) == sp.Nbin, name
        for b, row in enumerate(rows):
            got = np.array([float(t) for t in row])
            want = bins[b][name]
            if isinstance(want, complex):
                want = np.array([want.real, want.imag])
            np.testing.assert_allclose(got, np.atleast_1d(want), rtol=1e-9, atol=1e-12, err_msg=f"{name} bin {b}")
    for k in ("pole_distance", "pole_x", "green_spectral_radius", "green_smax", "log_weight"):
        vals = [float(t) for t in (tmp_path / k).read_text().split()]
        want = [bins[b]["pole"][c][k] for b in range(sp.Nbin) for c in range(2)]
        np.testing.assert_allclose(vals, want, rtol=1e-9, err_msg=k)
    rows = [ln.split() for ln in (tmp_path / "pole_z").read_text().splitlines() if ln.strip()]
    assert len(rows) == 2 * sp.Nbin
    for r, row in enumerate(rows):
        v = np.array([float(t) for t in row])
        got = v[0::2] + 1j * v[1::2]
        compare_pole({**bins[r // 2]["pole"][r % 2], "pole_z": got}, bins[r // 2]["pole"][r % 2], f"pole_z row {r}")


def test_bin_graph_replay_and_recapture(solver_mod):
    """A bin is one CUDA graph launch (reset, Nsweep sweeps per kernel class,
    finish), captured on the first bin, replayed on the second and captured
    again when the phase timers change the kernel arguments on the third; every
    bin matches the oracle's Nsweep = 2 bins."""
    op, sp = both_params(U2=-0.5, Nsweep=2)
    latt, opT, chains = O.init_chains(op, seeds=[77, 78])
    with solver_mod.Ensemble([sp], [0, 0]) as ens:
        ens.fields_from_seeds([77, 78])
        ens.pre()
        for ch in chains:
            ch.pre()
        for b in range(3):
            if b == 2:
                ens.phase_timers(True)
            for ch in chains:
                ch.sweep_bin()
            ens.sweep(2)
            seeds, phis = ens.get_state()
            cobs = ens.chain_obs()
            for c, ch in enumerate(chains):
                assert int(seeds[c]) == ch.seed, f"bin {b} chain {c} seed"
                np.testing.assert_array_equal(phis[c], ch.phi, err_msg=f"bin {b} chain {c} fields")
                assert_green_close(ens.green(c), ch.prop.Gr, f"bin {b} chain {c}")
                compare_bin(cobs[c], ch.obs.as_dict(latt), f"bin {b} chain {c}")
        assert ens.phase_timers(False).sum() > 0


@pytest.mark.parametrize("lx,ly", [(12, 12), (9, 9), (10, 11)])
def test_n144_class_against_oracle(solver_mod, lx, ly):
    """N = 144, 81 and 110 sites: the class whose G, U, workspaces and product
    scratch live in a per-chain HBM region (warp-per-column factorisations,
    tiled out-of-place products); 10x11 has no K point."""
    op, sp = both_params(U2=-0.5, Nlx=lx, Nly=ly, Ltrot=20, Beta=1.0, Nwrap=5)
    _run_both(op, sp, [41, 42], nbins=1)


def test_12x12_beta10_point(solver_mod):
    """The 12x12 point: U1 = 1, U2 = -0.5, mu = -5, beta = 10, dtau = 0.05
    (L = 200), Nwrap = 10, one chain, one bin."""
    op, sp = both_params(U2=-0.5, Nlx=12, Nly=12, Ltrot=200, Beta=10.0, Nwrap=10)
    _run_both(op, sp, [20241203], nbins=1)
