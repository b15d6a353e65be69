"""Mixed-precision slice products of the N <= 144 size class against the FP64
path.

The reference multiplies every slice in FP64 (multiply.f90:72-86, ZGEMM).
The mixed option runs those products on the tensor cores in 3xTF32-
compensated FP32 and keeps FP64 for the stabilisation, (I - B)^{-1}, the
ratios and the acceptance.  What it changes is therefore the Green's function
each decision reads: after G(beta) is built and after every mixed sweep, the
mixed chain's G is compared with G recomputed in FP64 (bafqmc_pre, itself
within 1e-10 of the oracle) from the same fields.  Bound: 1e-6 max-abs.
"""
import numpy as np
import pytest

from bafqmc_b200.params import SolverParams

pytestmark = pytest.mark.gpu

G_TOL = 1e-6


@pytest.fixture(scope="module")
def solver_mod():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from bafqmc_b200 import build, solver
    build.build()
    return solver


def point(lx, ly, L, beta, nwrap=10, mu=-5.0):
    return SolverParams(U1=1.0, U2=-0.5, mu=mu, Nlx=lx, Nly=ly, Ltrot=L, Beta=beta, NlxTherm=lx, NlyTherm=ly,
                        LtrotTherm=L, Nwrap=nwrap, Nbin=1, Nsweep=1, shiftLoc=1.5, iniType=2, iniAmpl=1.0)


def fp64_green(solver, p, seeds, phis):
    """G(beta) recomputed in FP64 from the given seeds and fields."""
    with solver.Ensemble([p], np.zeros(len(seeds), dtype=np.int32)) as ref:
        ref.set_state(seeds, phis)
        ref.pre()
        return [ref.green(c) for c in range(len(seeds))]


def max_green_error(solver, ens, p):
    seeds, phis = ens.get_state()
    ref = fp64_green(solver, p, seeds, phis)
    return max(float(np.max(np.abs(ens.green(c) - ref[c]))) for c in range(len(seeds)))


def test_12x12_beta10_green_error_every_sweep(solver_mod):
    """The 12x12, beta = 10 point (L = 200, Nwrap = 10): G after bafqmc_pre and
    after each of three mixed sweeps against FP64 from the same fields."""
    p = point(12, 12, 200, 10.0)
    seeds = [11, 12, 13, 14]
    with solver_mod.Ensemble([p], np.zeros(len(seeds), dtype=np.int32)) as ens:
        ens.set_precision("mixed")
        ens.fields_from_seeds(seeds)
        ens.pre()
        errs = [max_green_error(solver_mod, ens, p)]
        for _ in range(3):
            ens.sweep(1)
            errs.append(max_green_error(solver_mod, ens, p))
        cnt = ens.counters()
    print("max |G_mixed - G_fp64| after pre and each sweep:", ["%.2e" % e for e in errs])
    assert np.all(cnt[:, 6].astype(int) & 4 == 0), "a tensor-core product timed out"
    assert 0.7 < float(cnt[:, 0].mean()) / 3 < 0.95   # U1 acceptance per sweep, as in FP64 (0.85)
    assert max(errs) < G_TOL, errs


def test_ragged_sizes_and_other_classes_unchanged(solver_mod):
    """One handle with 9x9 and 10x11 chains (N <= 144 class, mixed) and 6x6
    chains (N <= 36 class, always FP64): the 6x6 chains are bit-identical to a
    run in FP64; the larger chains' G stays within the bound."""
    pts = [point(6, 6, 40, 2.0, nwrap=10), point(9, 9, 40, 2.0, nwrap=10), point(10, 11, 40, 2.0, nwrap=5)]
    chain_point = np.array([0, 1, 2, 0, 1, 2], dtype=np.int32)
    seeds = [101, 102, 103, 104, 105, 106]
    runs = {}
    for mode in ("fp64", "mixed"):
        with solver_mod.Ensemble(pts, chain_point) as ens:
            ens.set_precision(mode)
            ens.fields_from_seeds(seeds)
            ens.pre()
            ens.sweep(1)
            s, phi = ens.get_state()
            runs[mode] = (s, phi, ens.chain_obs_raw(), [ens.green(c) for c in range(len(seeds))])
    for c in np.nonzero(chain_point == 0)[0]:
        assert runs["mixed"][0][c] == runs["fp64"][0][c]
        np.testing.assert_array_equal(runs["mixed"][1][c], runs["fp64"][1][c])
        np.testing.assert_array_equal(runs["mixed"][2][c], runs["fp64"][2][c])
    for k in (1, 2):
        cs = [int(c) for c in np.nonzero(chain_point == k)[0]]
        ref = fp64_green(solver_mod, pts[k], [int(runs["mixed"][0][c]) for c in cs], [runs["mixed"][1][c] for c in cs])
        err = max(float(np.max(np.abs(runs["mixed"][3][c] - ref[i]))) for i, c in enumerate(cs))
        print(f"point {k}: max |G_mixed - G_fp64| = {err:.2e}")
        assert err < G_TOL


def test_9x9_near_band_edge_green_error_every_sweep(solver_mod):
    """9x9 (lowest free level -3) at mu = -3.02, beta = 8, U1 = 0.2, U2 = -0.05:
    G is far from the identity (largest singular values about 1.3-1.5, density
    0.01-0.02), so the propagation error of the mixed products is visible.  G
    after bafqmc_pre and after each of three mixed sweeps against FP64."""
    p = SolverParams(U1=0.2, U2=-0.05, mu=-3.02, Nlx=9, Nly=9, Ltrot=80, Beta=8.0, NlxTherm=9, NlyTherm=9,
                     LtrotTherm=80, Nwrap=10, Nbin=1, Nsweep=1, shiftLoc=1.5, iniType=2, iniAmpl=1.0)
    seeds = [5, 6, 7, 8]
    with solver_mod.Ensemble([p], np.zeros(len(seeds), dtype=np.int32)) as ens:
        ens.set_precision("mixed")
        ens.fields_from_seeds(seeds)
        ens.pre()
        errs = [max_green_error(solver_mod, ens, p)]
        for _ in range(3):
            ens.sweep(1)
            errs.append(max_green_error(solver_mod, ens, p))
        gmax = max(float(np.linalg.norm(ens.green(c) - np.eye(81), 2)) for c in range(len(seeds)))
        cnt = ens.counters()
    print("max |G_mixed - G_fp64| after pre and each sweep:", ["%.2e" % e for e in errs], "||G - I||_2 %.3f" % gmax)
    assert np.all(cnt[:, 6].astype(int) & 4 == 0), "a tensor-core product timed out"
    assert gmax > 0.2
    assert max(errs) < G_TOL, errs


def test_expired_product_wait_falls_back_to_fp64_exactly(solver_mod):
    """The give-up path of the products' bounded wait: in the wait-test mode
    the products issue no MMA and poll 1024 times, so each chain's first
    product times out, the chain records status bit 2 and continues in FP64.
    Nothing is left in flight (bit 3 stays clear), and seeds, fields and G
    are bit-identical to a plain FP64 run from the same start."""
    p = point(9, 9, 20, 1.0, nwrap=5)
    seeds0 = 515 + 17 * np.arange(4)
    out = {}
    for mode in ("fp64", "wait_test"):
        with solver_mod.Ensemble([p], np.zeros(len(seeds0), dtype=np.int32)) as ens:
            ens.set_precision(mode)
            ens.fields_from_seeds(seeds0)
            ens.pre()
            ens.sweep(1)
            s, phis = ens.get_state()
            out[mode] = (s, phis, [ens.green(c) for c in range(len(seeds0))], ens.counters())
    status = out["wait_test"][3][:, 6].astype(np.int64)
    assert np.all(status & 4), status
    assert not np.any(status & 8), status
    assert not np.any(out["fp64"][3][:, 6].astype(np.int64) & 12)
    np.testing.assert_array_equal(out["wait_test"][0], out["fp64"][0])
    for c in range(len(seeds0)):
        np.testing.assert_array_equal(out["wait_test"][1][c], out["fp64"][1][c])
        np.testing.assert_array_equal(out["wait_test"][2][c], out["fp64"][2][c])


def test_6x6_beta8_in_the_tensor_core_class(solver_mod):
    """The 6x6, beta = 8 point (L = 160) run in the N <= 144 class, the one with
    the tensor-core slice products, at mu = -3.1 (G departs from I by 8e-2):
    G after bafqmc_pre and after two mixed sweeps against FP64 from the same
    fields.  (The bench's mixed_at_6x6 line times the same configuration.)"""
    p = point(6, 6, 160, 8.0, mu=-3.1)
    seeds = [21, 22, 23, 24]
    with solver_mod.Ensemble([p], np.zeros(len(seeds), dtype=np.int32), classes=[6]) as ens:
        ens.set_precision("mixed")
        ens.fields_from_seeds(seeds)
        ens.pre()
        errs = [max_green_error(solver_mod, ens, p)]
        for _ in range(2):
            ens.sweep(1)
            errs.append(max_green_error(solver_mod, ens, p))
        status = ens.counters()[:, 6].astype(np.int64)
    print("6x6 mixed G error vs FP64:", errs)
    assert not np.any(status & 5), status
    assert max(errs) <= G_TOL
