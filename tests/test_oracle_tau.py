"""The oracle's time-displaced path (Dyn_sweep_R, dynamics.f90:38-58; Wrap_tau and
stab_green_big, stabilization.f90:192-254, 368-404) against dense products.

At the start of a right traversal the pass copies the propagator state (right
factors of B(0,0) = I, left factors of B(beta,0), G = G(0,0)) and propagates
G(tau,0) = B(tau,0) G, G(0,tau) = -(I - G) B(tau,0)^{-1} and
G(tau,tau) = B(tau,0) G B(tau,0)^{-1} slice by slice, replacing them every
Nwrap slices by the 2N x 2N stabilised inverse.  At beta = 1 the dense
products are well conditioned, so both must agree with the formulas to
1e-10; the stabilised G(0,0) block must reproduce G."""
import numpy as np

from oracle import oracle as O


def _chain(u2=-0.5, seed=321):
    p = O.Params(U1=1.0, U2=u2, mu=-3.5, Nlx=3, Nly=3, Ltrot=20, Beta=1.0, NlxTherm=3, NlyTherm=3, LtrotTherm=20,
                 Nwrap=5, Nbin=1, Nsweep=1, shiftLoc=1.5, iniType=2, iniAmpl=1.0)
    _, opT, (ch,) = O.init_chains(p, seeds=[seed])
    ch.pre()
    ch.sweep_L()
    return p, opT, ch


def _slice_B(ch, opT, nt, slots=(0, 1)):
    """B_nt = e^{-dtau K} D_2 D_1 with D_nf = diag(e^{alpha phi}) from field slot slots[nf]."""
    d = np.ones(ch.p.Ndim, dtype=complex)
    for nf in (0, 1):
        if ch.op[nf].active:
            d = d * np.array([ch._expalpha(nf, ch.phi[nt - 1, i, slots[nf]], 1) for i in range(ch.p.Ndim)])
    return opT.expT_P @ np.diag(d)


def test_time_displaced_green_functions_match_dense_products():
    p, opT, ch = _chain()
    G = ch.prop.Gr.copy()
    eye = np.eye(p.Ndim)
    rec = {}
    ch.tau_sweep_R(on_slice=lambda nt, pg: rec.__setitem__(nt, (pg.Gr00.copy(), pg.Gr0t.copy(), pg.Grt0.copy(),
                                                                   pg.Grtt.copy())))
    B = np.eye(p.Ndim, dtype=complex)
    for nt in range(1, p.Ltrot + 1):
        B = _slice_B(ch, opT, nt) @ B
        g00, g0t, gt0, gtt = rec[nt]
        Binv = np.linalg.inv(B)
        for got, want in ((gt0, B @ G), (g0t, -(eye - G) @ Binv), (gtt, B @ G @ Binv)):
            assert np.max(np.abs(got - want)) <= 1e-10 * max(1.0, np.max(np.abs(want))), nt
        if nt % p.Nwrap == 0:
            assert np.max(np.abs(g00 - G)) <= 1e-10 * max(1.0, np.max(np.abs(G)))
    # the drifts of the stabilisation (L1 distances) are rounding-level
    assert max(ch.pg.Xmaxm) < 1e-10 * np.sum(np.abs(G)) and all(x > 0 for x in ch.pg.Xmeanm)


def test_reference_stab_green_big_has_the_fermion_sign():
    """stabilization.f90:206-209 put +DUL in the top-right block, so the
    reference's 2N x 2N inverse has top-left block (I + B)^-1: its G(0,0) is not
    the bosonic (I - B)^-1, and every Wrap_tau replaces the propagated functions
    by unrelated ones (drifts of order the matrices themselves)."""
    p, opT, ch = _chain()
    G = ch.prop.Gr.copy()
    rec = {}
    ch.tau_sweep_R(fermion_sign=True,
                   on_slice=lambda nt, pg: rec.__setitem__(nt, pg.Gr00.copy()))
    assert np.max(np.abs(rec[p.Nwrap] - G)) > 0.1 * np.max(np.abs(G))
    assert max(ch.pg.Xmaxm) > 1e-2 * np.sum(np.abs(G))


def test_the_main_chain_is_untouched_and_u2_slot_matters():
    """The pass works on a copy: the chain's own state and RNG do not change.  The
    reference's U2-slot choice (dynamics.f90:52 passes the U1 field to the U2
    operator) gives different time-displaced functions whenever U2 is active."""
    p, opT, ch = _chain()
    before = (ch.seed, ch.prop.Gr.copy(), ch.prop.UUR.copy(), ch.phi.copy())
    out = {}
    for bug in (False, True):
        ch.tau_sweep_R(u2_slot_bug=bug)
        out[bug] = ch.pg.Grt0.copy()
    assert ch.seed == before[0]
    np.testing.assert_array_equal(ch.prop.Gr, before[1])
    np.testing.assert_array_equal(ch.prop.UUR, before[2])
    np.testing.assert_array_equal(ch.phi, before[3])
    assert np.max(np.abs(out[True] - out[False])) > 1e-3 * np.max(np.abs(out[False]))
    # with U2 = 0 the slot choice does not matter
    p, opT, ch = _chain(u2=0.0)
    ch.tau_sweep_R(u2_slot_bug=False)
    a = ch.pg.Grt0.copy()
    ch.tau_sweep_R(u2_slot_bug=True)
    np.testing.assert_array_equal(ch.pg.Grt0, a)


def test_a_sweep_with_the_pass_keeps_the_markov_chain():
    """Decisions, seeds and fields of a bin are the same with and without the pass."""
    runs = []
    for tau in (False, True):
        p = O.Params(U1=1.0, U2=-0.5, mu=-3.5, Nlx=3, Nly=3, Ltrot=20, Beta=1.0, NlxTherm=3, NlyTherm=3,
                     LtrotTherm=20, Nwrap=5, Nbin=1, Nsweep=1, shiftLoc=1.5, iniType=2, iniAmpl=1.0)
        _, _, (ch,) = O.init_chains(p, seeds=[99])
        ch.pre()
        ch.sweep_bin(tau=tau)
        runs.append((ch.seed, ch.phi.copy(), ch.prop.Gr.copy()))
    assert runs[0][0] == runs[1][0]
    np.testing.assert_array_equal(runs[0][1], runs[1][1])
    np.testing.assert_array_equal(runs[0][2], runs[1][2])


def test_pairing_pass_matches_dense_products():
    """The pairing solver's pass (src/pairing/src/dynamics.f90, multiply.f90:48-97)
    on the 4Ns matrices: the propagated functions equal the dense products of
    the slice matrices (B_nt = e^{-dtau H} D_nt, D_nt from opU_mmult_R on the
    identity; G(tau,0) = B G to 1e-10, the two with B^-1 to the dense inverse's
    own accuracy, 1e-14 cond(B)), the stabilised G(0,0) block reproduces G, and the functions keep
    the block structure of the Nambu matrices ({b, c^dagger} and {c, b^dagger}
    decoupled)."""
    p = O.Params(U1=1.0, U2=-0.5, mu=-5.0, Nlx=3, Nly=3, Ltrot=20, Beta=1.0, NlxTherm=3, NlyTherm=3,
                 LtrotTherm=20, Nwrap=5, Nbin=1, Nsweep=1, shiftLoc=1.5, iniType=2, iniAmpl=1.0, RDelta=0.3,
                 pairing=True)
    _, opT, (ch,) = O.init_chains(p, seeds=[5])
    ch.pre()
    ch.sweep_L()
    G = ch.prop.Gr.copy()
    n = G.shape[0]
    eye = np.eye(n)
    rec = {}
    ch.tau_sweep_R(on_slice=lambda nt, pg: rec.__setitem__(nt, (pg.Gr00.copy(), pg.Gr0t.copy(), pg.Grt0.copy(),
                                                                   pg.Grtt.copy())))
    B = np.eye(n, dtype=complex)
    ns = p.Lq
    blk = list(range(ns)) + list(range(3 * ns, 4 * ns))
    off = [i for i in range(n) if i not in blk]
    for nt in range(1, p.Ltrot + 1):
        D = np.eye(n, dtype=complex)
        for nf in (0, 1):
            if ch.op[nf].active:
                for ii in range(p.Nsite):
                    ch._mmult_R(D, nf, ii, ch.phi[nt - 1, ii, nf], 1)
        B = opT.expT_P @ D @ B
        g00, g0t, gt0, gtt = rec[nt]
        Binv = np.linalg.inv(B)
        # the dense inverse carries ~cond(B) eps (cond(B) reaches 8e6 at nt = 15, 1.5e9 at nt = 20)
        tol_inv = max(1e-10, 1e-14 * np.linalg.cond(B))
        for got, want, tol in ((gt0, B @ G, 1e-10), (g0t, -(eye - G) @ Binv, tol_inv),
                               (gtt, B @ G @ Binv, tol_inv)):
            scale = max(1.0, np.max(np.abs(want)))
            assert np.max(np.abs(got - want)) <= tol * scale, nt
            assert np.max(np.abs(got[np.ix_(blk, off)])) <= 1e-12 * scale
        if nt % p.Nwrap == 0:
            assert np.max(np.abs(g00 - G)) <= 1e-10 * max(1.0, np.max(np.abs(G)))
    assert max(ch.pg.Xmaxm) < 1e-10 * np.sum(np.abs(G))
