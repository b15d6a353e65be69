"""Global shift moves (bafqmc_global_shift) against the oracle.

The move shifts every field of auxiliary channel ns by X_ns = (u - 1/2)|shift|
(the chain's next two draws) and accepts by w'/w >= u' (third draw) with
log w = -sum phi^2 / 2 + 2 log|det G|, the exponent of the weight the local
updates sample.  The oracle recomputes both weights from scratch (its pre and
its pole diagnostics' log_weight), so the decisions, seeds and fields must be
bit-exact, and a chain continues from an accepted proposal exactly as the
oracle does from the shifted fields.  Chain averages with global moves
interleaved stay on the ED value.
"""
import json
import math

import numpy as np
import pytest

from bafqmc_b200.params import SolverParams
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver_mod():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from bafqmc_b200 import build, solver
    build.build()
    return solver


def both(**kw):
    base = dict(U1=1.0, U2=-0.5, mu=-5.0, Nlx=3, Nly=3, Ltrot=20, Beta=1.0, NlxTherm=3, NlyTherm=3, LtrotTherm=20,
                Nwrap=5, Nbin=1, Nsweep=1, shiftLoc=1.5, iniType=2, iniAmpl=1.0)
    base.update(kw)
    return O.Params(**base), SolverParams(**base)


def oracle_log_weight(p, seed, phi):
    _, _, (ch,) = O.init_chains(p, confin=[(seed, phi)])
    ch.pre()
    return ch.pole_diagnostics()["log_weight"], ch


def test_global_shift_decisions_and_continuation_match_the_oracle(solver_mod):
    op, sp = both()
    seeds0 = [11, 12, 13, 14, 15, 16, 17, 18]
    shift = (0.08, 0.08)
    _, _, chains = O.init_chains(op, seeds=seeds0)
    with solver_mod.Ensemble([sp], [0] * len(seeds0)) as ens:
        ens.fields_from_seeds(seeds0)
        ens.pre()
        ens.sweep(1)
        for ch in chains:
            ch.pre()
            ch.sweep_bin()
        acc = ens.global_shift(shift)
        seeds_g, phis_g = ens.get_state()
        ens.sweep(1)
        seeds_2, phis_2 = ens.get_state()
        greens = [ens.green(c) for c in range(len(seeds0))]
    assert 0 < acc.sum() < len(seeds0), acc   # both outcomes occur
    for k, ch in enumerate(chains):
        lw, _ = oracle_log_weight(op, ch.seed, ch.phi)
        seed, x0 = O.ranf(ch.seed)
        seed, x1 = O.ranf(seed)
        prop = ch.phi.copy()
        prop[:, :, 0] += (x0 - 0.5) * shift[0]
        prop[:, :, 1] += (x1 - 0.5) * shift[1]
        lw2, ch2 = oracle_log_weight(op, seed, prop)
        seed, u = O.ranf(seed)
        accept = math.exp(lw2 - lw) >= u
        assert bool(acc[k]) == accept, k
        assert int(seeds_g[k]) == seed
        np.testing.assert_array_equal(phis_g[k], prop if accept else ch.phi)
        nxt = ch2 if accept else ch
        nxt.seed = seed
        if not accept:   # the chain keeps its state; the oracle rebuilds it the same way
            _, nxt = oracle_log_weight(op, seed, ch.phi)
        nxt.sweep_bin()
        assert int(seeds_2[k]) == nxt.seed
        np.testing.assert_array_equal(phis_2[k], nxt.phi)
        assert np.max(np.abs(greens[k] - nxt.prop.Gr)) <= 1e-10 * np.max(np.abs(nxt.prop.Gr))


def test_averages_with_global_moves_stay_on_ed(solver_mod, root):
    """3x3, U1 = 1, U2 = -0.5, mu = -7, beta = 1, dtau = 0.01 (a paper case):
    a global shift after every sweep; chain averages within 2 SE of ED."""
    case = json.loads((root / "tests/golden/paper_3x3.json").read_text())["cases"]["triangle_3x3_U2_-0.5_mu-7_b1"]
    p = SolverParams.from_text("\n".join(" ".join(r) for r in case["paramC_sets"]) + "\n")
    nch, nbins, per = 256, 10, 60
    keys = {"density_total": "density_total", "energy_density": "energy_density", "S_SF_K": "sf_K", "S_DW_K": "dw_K"}
    sums = {k: np.zeros(nch) for k in keys}
    nacc = 0
    with solver_mod.Ensemble([p], np.zeros(nch, dtype=np.int32)) as ens:
        ens.fields_from_seeds(7000 + 13 * np.arange(nch))
        ens.warmup_prior(p.Nwarm)
        ens.pre()
        ens.sweep(150)
        for _ in range(nbins):
            for _ in range(per):   # one bin = per sweeps, each followed by a global move
                ens.sweep(1)
                obs = ens.chain_obs()
                for c in range(nch):
                    for k, f in keys.items():
                        sums[k][c] += complex(obs[c][f]).real / per
                nacc += int(ens.global_shift((0.05, 0.05)).sum())
    print("global acceptance", nacc / (nch * nbins * per))
    assert nacc > 0
    for k in keys:
        m = sums[k] / nbins
        mean, se = m.mean(), m.std(ddof=1) / math.sqrt(nch)
        z = (mean - case["observables"][k]["ed"]) / se
        print(f"{k}: {mean:.6e} +- {se:.2e} (z {z:+.2f})")
        assert abs(z) <= 2.0, k
