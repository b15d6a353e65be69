"""Failure detection through the C ABI, with the failure made on the host.

* A NaN field is rejected at the boundary (bafqmc_set_state returns
  BAFQMC_EARG naming the chain); the handle takes a valid state afterwards.
* A finite but absurd field (phi = 1e300 in the U2 channel, whose factor
  e^{alpha phi} overflows) makes that chain's Green's function non-finite in
  bafqmc_pre.  The chain is flagged (status bit 0) and quarantined: sweeps
  skip it, the point average leaves it out, its pole diagnostics are NaN, and
  the other chains run bit-identically to a handle without it.
No device fault, trap or hang is involved: the overflow is ordinary
floating-point arithmetic and every loop of the kernels is bounded.
"""
import json

import numpy as np
import pytest

from bafqmc_b200.params import SolverParams

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver_mod():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from bafqmc_b200 import build, solver
    build.build()
    return solver


def point(nbin=1):
    return SolverParams(U1=1.0, U2=-0.5, mu=-5.0, Nlx=3, Nly=3, Ltrot=40, Beta=4.0, NlxTherm=3, NlyTherm=3,
                        LtrotTherm=40, Nwrap=10, Nbin=nbin, Nsweep=1, shiftLoc=1.5, iniType=2, iniAmpl=1.0)


def test_nan_field_rejected_at_the_boundary(solver_mod):
    from bafqmc_b200 import _lib
    p = point()
    with solver_mod.Ensemble([p], [0, 0]) as ens:
        ens.fields_from_seeds([1, 2])
        seeds, phis = ens.get_state()
        bad = [phis[0].copy(), phis[1].copy()]
        bad[1].ravel()[17] = np.nan
        with pytest.raises(_lib.BafqmcError, match="chain 1"):
            ens.set_state(seeds, bad)
        with pytest.raises(_lib.BafqmcError):
            ens.pre()   # no fields after the rejected state
        ens.set_state(seeds, phis)
        ens.pre()
        ens.sweep(1)
        assert ens.quarantined() == []


def test_overflowing_chain_is_quarantined_and_the_others_are_unaffected(solver_mod):
    p = point()
    seeds = [11, 12, 13]
    with solver_mod.Ensemble([p], [0, 0, 0]) as ens:
        ens.fields_from_seeds(seeds)
        s0, phi0 = ens.get_state()
        phi_bad = [x.copy() for x in phi0]
        phi_bad[1].reshape(p.Ltrot, 9, 2)[5, 4, 1] = 1e300   # U2 channel, slice 5, site 4
        ens.set_state(s0, phi_bad)
        ens.pre()
        assert ens.quarantined() == [1]
        for _ in range(2):
            ens.sweep(1)
        s3, phi3 = ens.get_state()
        obs3 = ens.chain_obs_raw()
        pt3 = ens.point_obs_raw()
        pole = ens.pole_diagnostics()
        assert ens.quarantined() == [1]
    assert int(s3[1]) == int(s0[1])
    np.testing.assert_array_equal(phi3[1], phi_bad[1])      # never swept
    assert np.isnan(pole[1]["pole_distance"]) and np.isfinite(pole[0]["pole_distance"])
    with solver_mod.Ensemble([p], [0, 0]) as two:
        two.set_state([s0[0], s0[2]], [phi0[0], phi0[2]])
        two.pre()
        for _ in range(2):
            two.sweep(1)
        s2, phi2 = two.get_state()
        obs2 = two.chain_obs_raw()
        pt2 = two.point_obs_raw()
    for a, b in ((0, 0), (2, 1)):
        assert int(s3[a]) == int(s2[b])
        np.testing.assert_array_equal(phi3[a], phi2[b])
        np.testing.assert_array_equal(obs3[a], obs2[b])
    np.testing.assert_array_equal(pt3, pt2)


def test_run_directory_reports_a_quarantined_chain(solver_mod, tmp_path):
    p = point(nbin=2)
    with solver_mod.Ensemble([p], [0, 0]) as ens:
        ens.fields_from_seeds([21, 22])
        seeds, phis = ens.get_state()
    phis[0].reshape(p.Ltrot, 9, 2)[0, 0, 1] = 1e300
    (tmp_path / "paramC_sets.txt").write_text(p.to_text())
    with open(tmp_path / "confin.txt", "w") as f:
        for c in range(2):
            f.write(f" {int(seeds[c])}\n" + "".join(f" {float(v)!r}\n" for v in phis[c].ravel()))
    (tmp_path / "seeds.txt").write_text("21\n22\n")
    lines = []
    solver_mod.run_directory(tmp_path, nchains=2, log=lines.append)
    assert any("chain 0 quarantined" in ln for ln in lines)
    assert "chains quarantined: 0" in (tmp_path / "info.txt").read_text()
    rec = json.loads((tmp_path / "run_record.json").read_text())
    assert rec["quarantined_chains"] == [0] and rec["status"][1] == 0
    rows = (tmp_path / "density_total").read_text().split()
    assert len(rows) == 2 and all(np.isfinite(float(v)) for v in rows)   # the healthy chain's average
