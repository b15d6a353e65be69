"""Kernel classes and the autotuner through the C ABI.

A kernel class is one tile configuration of the sweep kernels (threads, CTAs
per SM, GEMM micro-tile, factorisation register layout, workspace placement).
bafqmc_autotune times every class that can hold a point on scratch handles and
picks the fastest; bafqmc_create_tuned runs chains in the chosen classes.  A
point gives the same chain in every class: decisions, seeds and fields bit-
exact, G and estimators within 1e-10 (the classes differ only in the order of
some reductions).
"""
import numpy as np
import pytest

from bafqmc_b200.params import SolverParams

pytestmark = pytest.mark.gpu

# kernel class -> (largest Ndim, Nambu)
HOLDS = {0: (16, 0), 1: (36, 0), 2: (72, 0), 3: (16, 1), 4: (36, 1), 5: (72, 1), 6: (144, 0)}


@pytest.fixture(scope="module")
def solver_mod():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from bafqmc_b200 import build, solver
    build.build()
    return solver


def points():
    kw = dict(U1=1.0, U2=-0.5, Nwrap=10, Nbin=1, Nsweep=1, iniType=2, iniAmpl=1.0)
    return [
        SolverParams(mu=-5.0, Nlx=3, Nly=3, Ltrot=40, Beta=2.0, NlxTherm=3, NlyTherm=3, LtrotTherm=40,
                     shiftLoc=1.5, **kw),
        SolverParams(mu=-6.0, Nlx=4, Nly=4, Ltrot=20, Beta=1.0, NlxTherm=4, NlyTherm=4, LtrotTherm=20,
                     shiftLoc=1.0, delta=0.5, sector=1, **kw),
        SolverParams(mu=-5.0, Nlx=6, Nly=6, Ltrot=40, Beta=2.0, NlxTherm=6, NlyTherm=6, LtrotTherm=40,
                     shiftLoc=1.5, **kw),
    ]


def test_autotune_picks_a_holding_class_per_point(solver_mod):
    pts = points()
    classes, table = solver_mod.autotune(pts, trial_chains=64)
    print("classes", classes.tolist())
    print("ms per chain-sweep\n", np.array2string(table, precision=4))
    for i, p in enumerate(pts):
        nd, pair = p.block_dim, 1 if p.sector == 1 else 0
        ok = [c for c, (nmax, sec) in HOLDS.items() if nd <= nmax and sec == pair]
        assert sorted(np.nonzero(np.isfinite(table[i]))[0].tolist()) == ok
        assert classes[i] in ok and table[i, classes[i]] == np.nanmin(table[i])


def test_chains_agree_across_classes(solver_mod):
    pts = points()
    chain_point = [0, 1, 2, 0, 1, 2]
    seeds = [7, 8, 9, 10, 11, 12]
    runs = []
    for classes in (None, [2, 5, 6]):
        with solver_mod.Ensemble(pts, chain_point, classes=classes) as ens:
            ens.fields_from_seeds(seeds)
            ens.pre()
            ens.sweep(1)
            s, phi = ens.get_state()
            runs.append((s, phi, ens.chain_obs_raw(), [ens.green(c) for c in range(len(seeds))]))
    (s0, p0, o0, g0), (s1, p1, o1, g1) = runs
    np.testing.assert_array_equal(s0, s1)
    for c in range(len(seeds)):
        np.testing.assert_array_equal(p0[c], p1[c])
        assert np.max(np.abs(g0[c] - g1[c])) <= 1e-10 * np.max(np.abs(g0[c]))
        np.testing.assert_allclose(o1[c], o0[c], rtol=1e-10, atol=1e-12)


def test_class_that_cannot_hold_a_point_is_rejected(solver_mod):
    from bafqmc_b200 import _lib
    pts = points()
    with pytest.raises(_lib.BafqmcError, match="cannot run point 2"):
        solver_mod.Ensemble(pts, [0, 1, 2], classes=[0, 4, 0])
