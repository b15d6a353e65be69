"""A ragged batch in one launch per kernel class, compared point by point with
the same chains run alone.

The points are the ragged-batch grid of the benchmark configurations: Lx = Ly
in {3, 4, 6}, beta in {2, 4, 8} at dtau = 0.05, U1 = 1, U2 in {0, -0.5}, mu in
{-6, -5, -4}, for the number-conserving solver and the Nambu solver at Delta in
{0.25, 0.5, 1.0} (216 points; Nwrap = 10).  A deterministic subset of 24
points, two chains each, shares one handle; each point then runs in a handle
of its own from the same seeds.  Every chain's CTA does the same work whatever
else is in the launch, so fields, seeds and bin records agree bit for bit.
"""
import numpy as np
import pytest

from bafqmc_b200.workloads import ragged_grid

pytestmark = pytest.mark.gpu


def test_grid_has_216_points_in_three_size_classes():
    pts = ragged_grid()
    assert len(pts) == 216
    assert sorted({p.block_dim for p in pts}) == [9, 16, 18, 32, 36, 72]


@pytest.fixture(scope="module")
def solver_mod():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from bafqmc_b200 import build, solver
    build.build()
    return solver


def test_ragged_launch_equals_points_run_alone(solver_mod):
    grid = ragged_grid()
    rng = np.random.default_rng(2024)
    pick = sorted(rng.choice(len(grid), size=24, replace=False).tolist())
    # every size class and both sectors are in the sample
    pts = [grid[i] for i in pick]
    assert {p.sector for p in pts} == {0, 1}
    chain_point = np.repeat(np.arange(len(pts)), 2).astype(np.int32)
    seeds = (1000 + 17 * np.arange(chain_point.size)).astype(np.int32)
    with solver_mod.Ensemble(pts, chain_point) as ens:
        ens.fields_from_seeds(seeds)
        ens.pre()
        ens.sweep(1)
        obs = ens.chain_obs_raw()
        s_all, phi_all = ens.get_state()
    for k, p in enumerate(pts):
        cs = np.nonzero(chain_point == k)[0]
        with solver_mod.Ensemble([p], [0, 0]) as one:
            one.fields_from_seeds(seeds[cs])
            one.pre()
            one.sweep(1)
            o1 = one.chain_obs_raw()
            s1, phi1 = one.get_state()
        width = o1.shape[1]
        np.testing.assert_array_equal(s1, s_all[cs], err_msg=f"point {pick[k]} seeds")
        for a, c in enumerate(cs):
            np.testing.assert_array_equal(phi1[a], phi_all[c], err_msg=f"point {pick[k]} fields")
            np.testing.assert_array_equal(o1[a], obs[c, :width], err_msg=f"point {pick[k]} bins")
