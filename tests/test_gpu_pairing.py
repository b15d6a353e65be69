"""GPU parity of the Nambu pairing sweep, called through the C ABI, against the
pairing oracle (a restatement of src/pairing/src/*.f90 in its 4Ns form) and
the reference's Gaussian golden vectors.

The device propagates the {b, c^dagger} block of the 4Ns Green's function; it
is compared with that block of the oracle's matrix.  Tolerances: G and
estimators 1e-10 relative to the largest entry / value (atol 1e-12 for values
that vanish); seeds, accepted fields, acceptance and proposal counts
bit-exact.  The oracle takes e^{-dtau H} from a general eigendecomposition of
the 4Ns matrix, as the reference does; at these points that differs from an
exact exponential by ~1e-15 and is inside the tolerance.  The points are
chosen away from condensation: where I - B(beta,0) approaches singularity
(e.g. 4x4, mu=-4, U2=-0.5 with unit Gaussian fields) a 1e-15 change of the
propagator moves the oracle's own G and bins by 1e-10 to 1e-7 and the chains
run away to unphysical densities, so no two FP64 implementations can agree
there to 1e-10.
"""
import json

import numpy as np
import pytest

from bafqmc_b200.params import SolverParams
from oracle import oracle as O

pytestmark = pytest.mark.gpu

RTOL = 1e-10
ATOL = 1e-12
PAIR_KEYS = ("density_up", "density_do", "density", "density_total", "kinetic", "doubleOcc", "squareOcc",
             "local_numsquare", "pair_equal", "num_up", "num_do", "numsquare_up", "numsquare_do", "onsite_n2_up",
             "onsite_n2_do", "interaction_energy_density", "pairing_energy_density", "chemical_energy_density",
             "grand_energy_density", "energy_density", "sf_K", "dw_K", "psf_Gamma", "den_upup_sub11",
             "den_dodo_sub11", "den_updo", "density_site_total")


@pytest.fixture(scope="module")
def solver_mod():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from bafqmc_b200 import build, solver
    build.build()
    return solver


def pair_params(delta=0.3, **kw):
    base = dict(U1=1.0, U2=-0.5, mu=-5.0, Nlx=3, Nly=3, Ltrot=20, Beta=2.0, Nwrap=5, Nbin=2, Nsweep=1,
                shiftLoc=1.5, iniType=2, iniAmpl=1.0)
    base.update(kw)
    base.setdefault("NlxTherm", base["Nlx"])
    base.setdefault("NlyTherm", base["Nly"])
    base.setdefault("LtrotTherm", base["Ltrot"])
    return O.Params(**base, RDelta=delta, pairing=True), SolverParams(**base, delta=delta, sector=1)


def oracle_block(G4: np.ndarray, ns: int) -> np.ndarray:
    idx = list(range(ns)) + list(range(3 * ns, 4 * ns))
    return G4[np.ix_(idx, idx)]


def compare_bin(gpu: dict, ora: dict, label=""):
    for k in PAIR_KEYS:
        np.testing.assert_allclose(np.atleast_1d(gpu[k]), np.atleast_1d(ora[k]), rtol=RTOL, atol=ATOL,
                                   err_msg=f"{label} {k}")


def assert_green_close(Gg, Go, label=""):
    err = np.max(np.abs(Gg - Go)) / np.max(np.abs(Go))
    assert err < RTOL, f"{label} G rel err {err:.3e}"


@pytest.mark.parametrize("nwrap", [10, 2])
@pytest.mark.parametrize("delta", [0.0, 0.2, -0.2])
def test_gaussian_closed_forms(solver_mod, root, delta, nwrap):
    """tests/physics/test_gaussian_solvers.py pairing half (abs 2e-9, rel 2e-8), all bins."""
    g = json.loads((root / "tests/golden/gaussian.json").read_text())
    exp = g["expected"]["0.0" if delta == 0.0 else "0.2"]
    tol_a, tol_r = g["params"]["abs_tol"], g["params"]["rel_tol"]
    _, p = pair_params(delta, U1=0.0, U2=0.0, Ltrot=100, Beta=1.0, Nwrap=nwrap, Nbin=4, shiftLoc=1.0, iniAmpl=0.1)
    with solver_mod.Ensemble([p], [0]) as ens:
        ens.fields_from_seeds([24681357])
        ens.pre()
        for _ in range(p.Nbin):
            ens.sweep(1)
            b = ens.point_obs()[0]
            for k, v in exp.items():
                want = -v if (k == "pair_equal" and delta < 0) else v
                a = b[k].real if isinstance(b[k], complex) else b[k]
                assert abs(a - want) <= tol_a + tol_r * abs(want), (k, a, want)
            for k in ("sf_K", "dw_K"):
                assert abs(b[k].imag) <= tol_a


def _run_both(ops, sps, chain_point, seeds, nbins, nwarm=0):
    """Oracle chains vs one device handle holding every chain (possibly ragged)."""
    from bafqmc_b200 import solver
    ora = []
    for c, s in enumerate(seeds):
        latt, _, chs = O.init_chains(ops[chain_point[c]], seeds=[s])
        ora.append((latt, chs[0]))
    ens = solver.Ensemble(sps, chain_point)
    ens.fields_from_seeds(seeds)
    s0, phi0 = ens.get_state()
    for c, (_, ch) in enumerate(ora):
        assert int(s0[c]) == ch.seed
        np.testing.assert_array_equal(phi0[c], ch.phi)
    if nwarm:
        for _ in range(nwarm):
            for _, ch in ora:
                ch.therm()
        ens.warmup_prior(nwarm)
        s1, phi1 = ens.get_state()
        for c, (_, ch) in enumerate(ora):
            assert int(s1[c]) == ch.seed
            np.testing.assert_array_equal(phi1[c], ch.phi)
    for _, ch in ora:
        ch.pre()
    ens.pre()

    def ref_green(ch):
        return oracle_block(ch.prop.Gr, ch.p.Lq) if ch.p.pairing else ch.prop.Gr

    for c, (_, ch) in enumerate(ora):
        assert_green_close(ens.green(c), ref_green(ch), f"pre chain {c}")
    for b in range(nbins):
        for _, ch in ora:
            ch.sweep_bin()
        ens.sweep(1)
        seeds_g, phis_g = ens.get_state()
        cobs = ens.chain_obs()
        cnt = ens.counters()
        for c, (latt, ch) in enumerate(ora):
            lab = f"bin {b} chain {c}"
            assert int(seeds_g[c]) == ch.seed, f"{lab} seed"
            np.testing.assert_array_equal(phis_g[c], ch.phi, err_msg=f"{lab} fields")
            assert_green_close(ens.green(c), ref_green(ch), lab)
            np.testing.assert_allclose(cnt[c, 0:2], ch.acc_sum, rtol=0, atol=0)
            if ch.p.pairing:
                compare_bin(cobs[c], ch.obs.as_dict(latt), lab)
                for nf in (0, 1):
                    if ch.op[nf].active:
                        assert cnt[c, 10 + nf] == ch.op[nf].phase.count_proposed
                        assert cnt[c, 12 + nf] == ch.op[nf].phase.count_accepted
            else:
                ref = ch.obs.as_dict(latt)
                for k in ("density_total", "energy_density", "sf_K", "dw_K", "kinetic", "den_updo",
                          "density_site_total"):
                    np.testing.assert_allclose(np.atleast_1d(cobs[c][k]), np.atleast_1d(ref[k]), rtol=RTOL,
                                               atol=ATOL, err_msg=f"{lab} {k}")
    ens.close()
    return ora


def test_both_channels_with_warmup(solver_mod):
    op, sp = pair_params(0.3)
    ora = _run_both([op], [sp], [0, 0, 0], [4099, 777, 31337], nbins=2, nwarm=2)
    for _, ch in ora:
        assert 0.0 < ch.acc_sum[0] < 2.0 and 0.0 < ch.acc_sum[1] < 2.0


def test_relative_channel_only_2x2(solver_mod):
    op, sp = pair_params(0.25, U2=0.0, Nlx=2, Nly=2, Ltrot=16, Beta=1.6, Nwrap=4)
    _run_both([op], [sp], [0, 0], [11, 12], nbins=2)


def test_total_channel_only_4x4_negative_delta(solver_mod):
    op, sp = pair_params(-0.5, U1=0.0, U2=-0.5, mu=-5.0, Nlx=4, Nly=4, Ltrot=20, Beta=1.0, Nwrap=5)
    _run_both([op], [sp], [0, 0], [2024, 2025], nbins=2)


def test_ragged_sectors_and_sizes_in_one_handle(solver_mod):
    """Number-conserving and Nambu points of three sizes in one launch per class."""
    o1, s1 = pair_params(0.5)
    o2, s2 = pair_params(1.0, U2=0.0, mu=-6.0, Nlx=2, Nly=2, Ltrot=10, Beta=0.5, Nwrap=5)
    kw = dict(U1=1.0, U2=-0.5, mu=-5.0, Nlx=3, Nly=3, Ltrot=20, Beta=2.0, NlxTherm=3, NlyTherm=3, LtrotTherm=20,
              Nwrap=5, Nbin=1, Nsweep=1, shiftLoc=1.5, iniType=2, iniAmpl=1.0)
    o3, s3 = O.Params(**kw), SolverParams(**kw)
    _run_both([o1, o2, o3], [s1, s2, s3], [0, 1, 2, 0, 2, 1], [5, 6, 7, 8, 9, 10], nbins=1)


def test_run_directory_pairing_program(solver_mod, tmp_path):
    """The pairing program's run-directory contract: paramC_sets.txt with RDelta,
    seeds.txt, the pairing file set, confout.txt; bins equal the oracle's chain
    averages."""
    op, sp = pair_params(0.3, Nbin=2)
    (tmp_path / "paramC_sets.txt").write_text(sp.to_text())
    (tmp_path / "confin.txt").write_text("0\n")
    (tmp_path / "seeds.txt").write_text("4099\n777\n")
    solver_mod.run_directory(tmp_path, nchains=2, pairing=True)
    bins, chains = O.run(op, seeds=[4099, 777])
    from bafqmc_b200.observables import FILE_ORDER_PAIRING
    for name in FILE_ORDER_PAIRING:
        rows = [ln.split() for ln in (tmp_path / name).read_text().splitlines() if ln.strip()]
        assert len(rows) == sp.Nbin, name
        for b, row in enumerate(rows):
            got = np.array([float(t) for t in row])
            want = bins[b][name]
            if isinstance(want, complex):
                want = np.array([want.real, want.imag])
            np.testing.assert_allclose(got, np.atleast_1d(want), rtol=1e-9, atol=1e-12, err_msg=f"{name} bin {b}")
    assert not (tmp_path / "pole_z").exists()
    info = (tmp_path / "info.txt").read_text()
    assert "pairing Delta" in info and "Phase_U1_local_proposals" in info and "Phase_U2_local_proposals" in info
    toks = (tmp_path / "confout.txt").read_text().split()
    assert int(toks[0]) == chains[0].seed
    np.testing.assert_array_equal(np.array([float(t) for t in toks[1:1 + chains[0].phi.size]]),
                                  chains[0].phi.ravel())


def test_nambu_6x6_in_the_n72_class(solver_mod):
    """2Ns = 72: G and U in shared memory, the two workspaces in HBM."""
    op, sp = pair_params(0.5, mu=-6.0, Nlx=6, Nly=6, Ltrot=20, Beta=1.0, Nwrap=5)
    _run_both([op], [sp], [0, 0], [606, 607], nbins=1)


def test_run_directory_pairing_time_displaced(solver_mod, tmp_path):
    """The pairing program with is_tau = .true. and Nthermal = 1 over 2 bins: the
    pass runs in bin 2 only, info.txt gets Dyn_control_print's six lines after
    the acceptance and phase lines, with the drifts of the 4Ns matrices (twice
    the stored block's), and the checkpoint equals a run without the pass."""
    import dataclasses
    _, sp = pair_params(0.3, Nbin=2)
    out = {}
    for tau in (False, True):
        d = tmp_path / ("tau" if tau else "plain")
        d.mkdir()
        (d / "paramC_sets.txt").write_text(dataclasses.replace(sp, is_tau=tau, Nthermal=1).to_text())
        (d / "confin.txt").write_text("0\n")
        (d / "seeds.txt").write_text("4099\n777\n")
        solver_mod.run_directory(d, nchains=2, pairing=True)
        out[tau] = d
    assert (out[False] / "confout.txt").read_text() == (out[True] / "confout.txt").read_text()
    lines = (out[True] / "info.txt").read_text().splitlines()
    labels = [ln.split(":")[0].strip() for ln in lines]
    i = labels.index("Max diff GRtt")
    assert labels[i:i + 6] == ["Max diff GRtt", "Mean diff GRtt", "Max diff GRt0", "Mean diff GRt0",
                               "Max diff GR0t", "Mean diff GR0t"]
    vals = [float(lines[i + k].split(":")[1]) for k in range(6)]
    assert all(0 < v < 1e-8 for v in vals), vals
    rec = json.loads((out[True] / "run_record.json").read_text())
    assert rec["tau_passes"] == 2 and rec["tau_nonfinite"] == 0
