"""The time-displaced pass on the GPU (tau_kernel) against the oracle
(oracle.Chain.tau_sweep_R with the bosonic sign and the U2 field slot).

* 3x3, beta = 1 (well conditioned): G(0,0), G(0,tau), G(tau,0), G(tau,tau)
  of the device at a propagated slice, a wrap slice and the last slice agree
  with the oracle within 1e-10 of each matrix's largest entry; seeds and
  fields stay bit-exact with the oracle's Markov chain.
* The pass does not change the Markov chain: G, seeds, fields and counters
  of an ensemble with the pass on equal those of one without it, bit for bit;
  the bin observables agree to 1e-14 (with the pass the left and right
  traversals run as two launches, whose sums are added to the bin separately).
* 6x6, beta = 8, L = 160, mu = -3.1 (G departs from I by 8e-2): the four
  functions at a wrap slice and a propagated slice within 1e-9 of the largest
  entry, and the drifts Wrap_tau records are rounding-level (below 1e-9 of
  sum |G|; the reference warns at 5.5e-5).
* 8x8 (N = 64, the pass in the larger size class): the four functions within
  1e-9 at a wrap slice and a propagated slice (measured 1.4e-11 and 8e-11).
* A Nambu chain: the {b, c^dagger} block of the oracle's 4Ns functions.
* Refusals: Ndim > 72, a probe slice outside 0..Ltrot, statistics before the
  pass was enabled.
"""
import numpy as np
import pytest

from bafqmc_b200.params import SolverParams
from oracle import oracle as O

pytestmark = pytest.mark.gpu

KW = dict(U1=1.0, U2=-0.5, mu=-3.5, Nlx=3, Nly=3, Ltrot=20, Beta=1.0, NlxTherm=3, NlyTherm=3, LtrotTherm=20,
          Nwrap=5, Nbin=1, Nsweep=1, shiftLoc=1.5, iniType=2, iniAmpl=1.0)


@pytest.fixture(scope="module")
def mods():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from bafqmc_b200 import build
    build.build()
    from bafqmc_b200 import _lib, solver
    return solver, _lib


def _oracle_bin(ch, probe_nt):
    """One oracle bin with the pass; the four functions at slice probe_nt."""
    rec = {}

    def hook(nt, pg):
        if nt == probe_nt:
            rec["g"] = (pg.Gr00.copy(), pg.Gr0t.copy(), pg.Grt0.copy(), pg.Grtt.copy())

    ch.tau_sweep_R = lambda: O.Chain.tau_sweep_R(ch, on_slice=hook)
    ch.sweep_bin(tau=True)
    return rec["g"]


def _compare(dev, ora, tol, what):
    names = ("G(0,0)", "G(0,tau)", "G(tau,0)", "G(tau,tau)")
    worst = 0.0
    for name, d, o in zip(names, dev, ora):
        err = float(np.max(np.abs(d - o)) / max(1e-300, np.max(np.abs(o))))
        worst = max(worst, err)
        assert err <= tol, (what, name, err)
    return worst


def test_time_displaced_functions_match_oracle_3x3(mods):
    solver, _ = mods
    op, sp = O.Params(**KW), SolverParams(**KW)
    seeds = [11, 12, 13]
    _, _, chains = O.init_chains(op, seeds=seeds)
    with solver.Ensemble([sp], [0] * len(seeds)) as ens:
        ens.fields_from_seeds(seeds)
        ens.pre()
        for ch in chains:
            ch.pre()
        for probe in (3, 5, 20):
            ens.set_time_displaced(True, probe)
            ens.sweep(1)
            s, phis = ens.get_state()
            for c, ch in enumerate(chains):
                ora = _oracle_bin(ch, probe)
                worst = _compare(ens.time_displaced_probe(c), ora, 1e-10, (probe, c))
                print(f"slice {probe} chain {c}: max relative error {worst:.2e}")
                assert int(s[c]) == ch.seed
                np.testing.assert_array_equal(phis[c], ch.phi)
                np.testing.assert_allclose(ens.green(c), ch.prop.Gr, rtol=0,
                                           atol=1e-10 * max(1.0, float(np.max(np.abs(ch.prop.Gr)))))
        st = ens.time_displaced_stats()
    for c, ch in enumerate(chains):
        scale = float(np.sum(np.abs(ch.prop.Gr)))
        assert st[c, 6] == 3 and st[c, 7] == 0, st[c]
        assert np.all(st[c, 0:3] > 0) and np.all(st[c, 0:3] < 1e-10 * scale), st[c]
        assert np.all(st[c, 3:6] >= st[c, 0:3])
        # the oracle's drifts are rounding-level too
        assert max(ch.pg.Xmaxm) < 1e-10 * scale


def test_the_pass_leaves_the_markov_chain_unchanged(mods):
    solver, _ = mods
    sp = SolverParams(**KW)
    seeds = [21, 22, 23, 24]
    out = []
    for tau in (False, True):
        with solver.Ensemble([sp], [0] * len(seeds)) as ens:
            ens.fields_from_seeds(seeds)
            ens.pre()
            if tau:
                ens.set_time_displaced(True)
            for _ in range(2):
                ens.sweep(1)
            s, phis = ens.get_state()
            out.append((s, np.stack(phis), [ens.green(c) for c in range(len(seeds))], ens.chain_obs(),
                        ens.counters()))
    (s0, p0, g0, o0, c0), (s1, p1, g1, o1, c1) = out
    np.testing.assert_array_equal(s0, s1)
    np.testing.assert_array_equal(p0, p1)
    for a, b in zip(g0, g1):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(o0, o1):
        for k in a:
            np.testing.assert_allclose(np.asarray(a[k]), np.asarray(b[k]), rtol=1e-14, atol=1e-300, err_msg=k)
    np.testing.assert_array_equal(c0[:, :6], c1[:, :6])


def test_time_displaced_functions_6x6_beta8(mods):
    solver, _ = mods
    kw = dict(KW, mu=-3.1, Nlx=6, Nly=6, NlxTherm=6, NlyTherm=6, Ltrot=160, LtrotTherm=160, Beta=8.0, Nwrap=10)
    op, sp = O.Params(**kw), SolverParams(**kw)
    seeds = [5]
    _, _, (ch,) = O.init_chains(op, seeds=seeds)
    ch.pre()
    with solver.Ensemble([sp], [0]) as ens:
        ens.fields_from_seeds(seeds)
        ens.pre()
        for probe in (80, 85):
            ens.set_time_displaced(True, probe)
            ens.sweep(1)
            ora = _oracle_bin(ch, probe)
            worst = _compare(ens.time_displaced_probe(0), ora, 1e-9, probe)
            print(f"6x6 beta 8 slice {probe}: max relative error {worst:.2e}")
            s, phis = ens.get_state()
            assert int(s[0]) == ch.seed
            np.testing.assert_array_equal(phis[0], ch.phi)
        st = ens.time_displaced_stats(reset=True)
        assert np.all(ens.time_displaced_stats() == 0)
    scale = float(np.sum(np.abs(ch.prop.Gr)))
    print("device drifts", st[0, :3], "oracle", ch.pg.Xmaxm)
    assert st[0, 6] == 2 and st[0, 7] == 0
    assert np.all(st[0, 0:3] < 1e-9 * scale), st[0]


def test_time_displaced_functions_8x8_larger_class(mods):
    """N = 64 (36 < N <= 72): the pass runs in the N <= 144 class's context (2N = 128)."""
    solver, _ = mods
    kw = dict(KW, Nlx=8, Nly=8, NlxTherm=8, NlyTherm=8)
    op, sp = O.Params(**kw), SolverParams(**kw)
    _, _, (ch,) = O.init_chains(op, seeds=[77])
    ch.pre()
    with solver.Ensemble([sp], [0]) as ens:
        ens.fields_from_seeds([77])
        ens.pre()
        for probe in (5, 12):
            ens.set_time_displaced(True, probe)
            ens.sweep(1)
            worst = _compare(ens.time_displaced_probe(0), _oracle_bin(ch, probe), 1e-9, probe)
            print(f"8x8 slice {probe}: max relative error {worst:.2e}")
            s, phis = ens.get_state()
            assert int(s[0]) == ch.seed
            np.testing.assert_array_equal(phis[0], ch.phi)


def test_nambu_time_displaced_functions_match_oracle(mods):
    """A Nambu chain (3x3, Delta = 0.3, beta = 1): the device's pass on the
    {b, c^dagger} block against that block of the oracle's 4Ns functions
    (src/pairing/src/dynamics.f90 restated in oracle.Chain.tau_sweep_R), at a
    propagated slice, a wrap slice and the last slice: within 1e-9 of each
    block's largest entry; seeds and fields bit-exact."""
    solver, _ = mods
    from test_gpu_pairing import oracle_block, pair_params
    op, sp = pair_params(0.3, mu=-5.0, Nlx=3, Nly=3, Ltrot=20, Beta=1.0, Nwrap=5, Nbin=1)
    seeds = [41, 42]
    _, _, chains = O.init_chains(op, seeds=seeds)
    for ch in chains:
        ch.pre()
    with solver.Ensemble([sp], [0] * len(seeds)) as ens:
        ens.fields_from_seeds(seeds)
        ens.pre()
        for probe in (3, 5, 20):
            ens.set_time_displaced(True, probe)
            ens.sweep(1)
            s, phis = ens.get_state()
            for c, ch in enumerate(chains):
                ora = [oracle_block(m, op.Lq) for m in _oracle_bin(ch, probe)]
                worst = _compare(ens.time_displaced_probe(c), ora, 1e-9, (probe, c))
                print(f"Nambu slice {probe} chain {c}: max relative error {worst:.2e}")
                assert int(s[c]) == ch.seed
                np.testing.assert_array_equal(phis[c], ch.phi)
        st = ens.time_displaced_stats()
    assert np.all(st[:, 6] == 3) and np.all(st[:, 7] == 0)


def test_refusals(mods):
    solver, _lib = mods
    big = SolverParams(**dict(KW, Nlx=12, Nly=12, NlxTherm=12, NlyTherm=12))
    with solver.Ensemble([big], [0]) as ens:
        with pytest.raises(_lib.BafqmcError) as ei:
            ens.set_time_displaced(True)
        assert ei.value.code == -3
    with solver.Ensemble([SolverParams(**KW)], [0]) as ens:
        with pytest.raises(_lib.BafqmcError) as ei:
            ens.set_time_displaced(True, KW["Ltrot"] + 1)
        assert ei.value.code == -1
        with pytest.raises(_lib.BafqmcError) as ei:
            ens.time_displaced_stats()
        assert ei.value.code == -4
