"""Chain averages on 3x3 clusters against exact diagonalisation and against the
reference solver's own published runs.

The reference's paper data set (benchmarks/paper/data) holds, for each 3x3
case, the run's paramC_sets.txt, the ED value and the reference's DQMC mean
and standard error of density_total, energy_density, S_SF(K) and S_DW(K); the
last two are the real parts of the sf_K and dw_K files
(benchmarks/paper/analysis.py:14-17).  tests/golden/make_golden.py copies them
into tests/golden/paper_3x3.json.

Each case runs here as an ensemble of independent chains with the case's own
parameters (Ltrot, shiftLoc, prior warm-up, initial fields): prior warm-up,
G(beta), discarded thermalisation sweeps, then measured bins.  The standard
error SE is the spread of the chain means over sqrt(chains).  The bar, per
observable: |mean - DQMC_ref| <= 2 sqrt(SE^2 + SE_ref^2), and |mean - ED| <= 2 SE
for every case whose reference run itself lies within 2 SE_ref of ED on all
four observables.  The Nambu cases at Delta = 0.05 and Delta >= 0.2 do not (the
reference's runs sit 2.6 to 10 SE_ref from ED values computed with at most 3
bosons per site, nmax = 3, ncut = 4); they are checked against the reference's
DQMC only.

The benchmark set's single-chain point (3x3, U1 = 1, U2 = 0, mu = -5, beta = 4,
dtau = 0.1, 1000 warm-up and 10^4 measured sweeps) is the physics point of
the pairing case at Delta = 0, whose ED value it is checked against, with its
own dtau and schedule per chain.
"""
import json
import math
import time

import numpy as np
import pytest

from bafqmc_b200.params import SolverParams

pytestmark = pytest.mark.gpu

FILES = {"density_total": "density_total", "energy_density": "energy_density", "S_SF_K": "sf_K",
         "S_DW_K": "dw_K"}


@pytest.fixture(scope="module")
def solver_mod():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from bafqmc_b200 import build, solver
    build.build()
    return solver


@pytest.fixture(scope="module")
def paper(root):
    return json.loads((root / "tests/golden/paper_3x3.json").read_text())["cases"]


def case_params(case: dict) -> SolverParams:
    text = "\n".join(" ".join(r) for r in case["paramC_sets"]) + "\n"
    return SolverParams.from_text(text, pairing=case["model"] == "pairing")


def ensemble_means(solver, p: SolverParams, nchains: int, ntherm: int, nbins: int, nsweep: int, seed0: int):
    """Per observable: (mean over chains of the chain means, SE of that mean)."""
    seeds = (seed0 + 7919 * np.arange(nchains)).astype(np.int32)
    acc = {k: np.zeros(nchains) for k in FILES}
    t0 = time.time()
    with solver.Ensemble([p], np.zeros(nchains, dtype=np.int32)) as ens:
        ens.fields_from_seeds(seeds)
        if p.is_warm:
            ens.warmup_prior(p.Nwarm)
        ens.pre()
        if ntherm:
            ens.sweep(ntherm)
        for _ in range(nbins):
            ens.sweep(nsweep)
            for c, o in enumerate(ens.chain_obs()):
                for k, f in FILES.items():
                    acc[k][c] += complex(o[f]).real
    out = {}
    for k, v in acc.items():
        m = v / nbins
        out[k] = (float(m.mean()), float(m.std(ddof=1) / math.sqrt(nchains)))
    print(f"  {nchains} chains x {ntherm} + {nbins * nsweep} sweeps in {time.time() - t0:.1f} s")
    return out


def reference_matches_ed(case: dict) -> bool:
    return all(abs(v["dqmc"] - v["ed"]) <= 2.0 * v["stderr"] for v in case["observables"].values())


def check(got: dict, case: dict, against_dqmc: bool, label: str):
    lines, bad = [], []
    against_ed = not against_dqmc or reference_matches_ed(case)
    for k, (m, se) in got.items():
        ref = case["observables"][k]
        z_ed = (m - ref["ed"]) / se
        lines.append(f"{label} {k}: {m:.6e} +- {se:.2e}  ED {ref['ed']:.6e} (z {z_ed:+.2f})")
        if against_ed and abs(z_ed) > 2.0:
            bad.append(f"{k} vs ED z={z_ed:+.2f}")
        if against_dqmc:
            sd = math.sqrt(se ** 2 + ref["stderr"] ** 2)
            z_ref = (m - ref["dqmc"]) / sd
            lines[-1] += f"  ref DQMC {ref['dqmc']:.6e} +- {ref['stderr']:.2e} (z {z_ref:+.2f})"
            if abs(z_ref) > 2.0:
                bad.append(f"{k} vs reference DQMC z={z_ref:+.2f}")
    print("\n".join(lines))
    assert not bad, f"{label}: " + "; ".join(bad)


def test_reference_ed_consistency_rule(paper):
    assert [k for k, c in paper.items() if not reference_matches_ed(c) and c["model"] == "pairing"] == [
        "triangle_pairing_delta_3x3_D0p05_mum5_b4", "triangle_pairing_delta_3x3_D0p2_mum5_b4",
        "triangle_pairing_delta_3x3_D0p25_mum5_b4", "triangle_pairing_delta_3x3_D0p3_mum5_b4"]


@pytest.mark.parametrize("cid,nchains,nbins,nsweep,seed0", [
    ("triangle_3x3_U2_-0.5_mu-7_b1", 256, 10, 100, 1001),
    ("triangle_3x3_U1_0.5_mu-3.5_b4", 256, 10, 100, 2002),
    ("triangle_pairing_delta_3x3_D0p1_mum5_b4", 256, 8, 75, 3003),
    ("triangle_pairing_delta_3x3_D0p15_mum5_b4", 256, 8, 75, 6006),
    ("triangle_pairing_delta_3x3_D0p2_mum5_b4", 256, 8, 75, 4004),
])
def test_paper_case_against_ed_and_reference(solver_mod, paper, cid, nchains, nbins, nsweep, seed0):
    case = paper[cid]
    p = case_params(case)
    got = ensemble_means(solver_mod, p, nchains, ntherm=150, nbins=nbins, nsweep=nsweep, seed0=seed0)
    check(got, case, True, cid)


def test_single_chain_config_against_ed(solver_mod, paper):
    """3x3, U1 = 1, U2 = 0, mu = -5, beta = 4, dtau = 0.1 (L = 40), Nwrap = 10,
    N(0,1) fields: 1000 warm-up and 10^4 measured sweeps per chain, 64 chains."""
    case = paper["triangle_pairing_delta_3x3_D0_mum5_b4"]
    p = SolverParams(U1=1.0, U2=0.0, mu=-5.0, Nlx=3, Nly=3, Ltrot=40, Beta=4.0, NlxTherm=3, NlyTherm=3, LtrotTherm=40,
                     Nwrap=10, Nbin=1, Nsweep=1, shiftLoc=1.5, iniType=2, iniAmpl=1.0)
    got = ensemble_means(solver_mod, p, 64, ntherm=1000, nbins=20, nsweep=500, seed0=5005)
    check(got, case, False, "3x3 U1=1 mu=-5 beta=4 dtau=0.1")


@pytest.mark.parametrize("mu,beta,seed0", [(-5.0, 2.0, 8008), (-4.0, 2.0, 9009), (-4.0, 4.0, 10010)])
def test_ragged_grid_points_against_own_ed(solver_mod, mu, beta, seed0):
    """3x3 points of the ragged grid (U1 = 1, U2 = 0, dtau = 0.05, Nwrap = 10,
    shiftLoc 1.5) that the reference's stored ED does not cover, against
    oracle/ed.py with up to 4 bosons (against 5: 1e-8, 4e-5 and 1e-10 relative
    at these points, far below the standard errors).  U2 = 0: each boson costs
    at least 2 above mu, so the truncated grand-canonical sum converges; at
    U2 < 0 bosons bind on a site and it does not."""
    from oracle import ed
    L = int(round(beta / 0.05))
    p = SolverParams(U1=1.0, U2=0.0, mu=mu, Nlx=3, Nly=3, Ltrot=L, Beta=beta, NlxTherm=3, NlyTherm=3, LtrotTherm=L,
                     Nwrap=10, Nbin=1, Nsweep=1, shiftLoc=1.5, iniType=2, iniAmpl=1.0)
    ref = ed.observables(3, 3, 1.0, 0.0, mu, beta, n_max_total=4)
    case = {"observables": {k: {"ed": v, "dqmc": v, "stderr": 0.0} for k, v in ref.items()}}
    got = ensemble_means(solver_mod, p, 256, ntherm=200, nbins=10, nsweep=100, seed0=seed0)
    check(got, case, False, f"3x3 U1=1 U2=0 mu={mu} beta={beta}")
