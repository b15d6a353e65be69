"""Pins the CPU oracle against the reference's own golden vectors.

* RNG known-answer test: src/common/test_numerics.f90:177-189.
* Dense fixed-field reference: tests/physics/test_fixed_field_solver.py:40-119
  (fixture tests/golden/fixed_field.json), tolerance 2e-10 as in that test.
* Gaussian closed forms: tests/physics/test_gaussian_solvers.py:44-77
  (fixture tests/golden/gaussian.json), abs 2e-9 / rel 2e-8 as in that test.
"""
import json

import numpy as np
import pytest

from oracle import oracle as O


def test_rng_known_answer():
    seed = 1
    seed, _ = O.ranf(seed)
    assert seed == 48828125
    seed, _ = O.ranf(seed)
    assert seed == 52882121
    expected = seed
    for _ in range(10000):
        expected = (48828125 * expected) % 2147483648
        seed, u = O.ranf(seed)
        assert seed == expected
        assert 0.0 <= u < 1.0


def _fixed_params(g, nwrap):
    pp = g["params"]
    return O.Params(U1=pp["U1"], U2=pp["U2"], mu=pp["mu"], Nlx=pp["Lx"], Nly=pp["Ly"],
                    Ltrot=pp["Ltrot"], Beta=pp["beta"], NlxTherm=pp["Lx"], NlyTherm=pp["Ly"],
                    LtrotTherm=pp["Ltrot"], Nwrap=nwrap, Nbin=pp["Nbin"], Nsweep=1,
                    shiftLoc=0.0, iniType=1, iniAmpl=0.0)


@pytest.mark.parametrize("nwrap", [1, 2, 6])
def test_oracle_fixed_field(root, nwrap):
    g = json.loads((root / "tests/golden/fixed_field.json").read_text())
    tol = g["params"]["tolerance"]
    fields = np.array(g["fields_t_site_aux"])
    exp = g["expected"]
    p = _fixed_params(g, nwrap)
    bins, chains = O.run(p, confin=[(1357911, fields.ravel())])
    assert len(bins) == p.Nbin
    for b in bins:
        for k in ("density_total", "density_site_total", "kinetic", "doubleOcc", "onsite_n2_up",
                  "onsite_n2_do", "interaction_energy_density", "energy_density"):
            np.testing.assert_allclose(np.atleast_1d(b[k]), np.atleast_1d(exp[k]), rtol=tol, atol=tol, err_msg=k)
        for k in ("log_weight", "pole_distance", "pole_x", "green_spectral_radius", "green_smax"):
            np.testing.assert_allclose(b["pole"][0][k], exp[k], rtol=tol, atol=tol, err_msg=k)
    np.testing.assert_allclose(chains[0].phi.ravel(), fields.ravel(), rtol=0, atol=2e-15)


@pytest.mark.parametrize("nwrap", [10, 2])
def test_oracle_gaussian(root, nwrap):
    g = json.loads((root / "tests/golden/gaussian.json").read_text())
    exp = g["expected"]["0.0"]
    p = O.Params(U1=0.0, U2=0.0, mu=-5.0, Nlx=3, Nly=3, Ltrot=100, Beta=1.0, NlxTherm=3, NlyTherm=3,
                 LtrotTherm=100, Nwrap=nwrap, Nbin=g["params"]["Nbin"], Nsweep=1, shiftLoc=1.0,
                 iniType=2, iniAmpl=0.1)
    bins, _ = O.run(p, seeds=[7], want_pole=False)
    for b in bins:
        for k in ("density_total", "energy_density", "sf_K", "dw_K"):
            a = b[k].real if isinstance(b[k], complex) else b[k]
            assert abs(a - exp[k]) <= g["params"]["abs_tol"] + g["params"]["rel_tol"] * abs(exp[k]), k


def test_params_roundtrip_reference_format():
    text = """0.0         0.0         -5.0
3           3           100         1.0
3           3           100
10          8           1           1.5
.false.     0
.false.     0           1.0         1.0
2           0.1         0.0         0.0

U1_relative  U2_total    mu
"""
    p = O.Params.from_text(text)
    assert (p.Nlx, p.Nly, p.Ltrot, p.Nwrap, p.Nbin, p.Nsweep) == (3, 3, 100, 10, 8, 1)
    assert p.is_tau is False and p.is_warm is False and p.iniType == 2
    assert p.Nst == 10
    with pytest.raises(ValueError):
        O.Params.from_text(text.replace("10          8", "7           8"))
