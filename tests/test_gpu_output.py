"""Output side: on-device block statistics and the binary checkpoint.

The reference's analysis blocks the per-bin point averages
(benchmarks/paper/analysis.py:52-64): block means sum(block) / block_size,
mean sum(means) / n, standard error sqrt(sum((m - mean)^2) / (n - 1) / n),
each sum taken in order (Python 3.11, as its environment pins).  The device statistics must give the same numbers
from the same bins.  The binary checkpoint confout.npz holds exactly the
seeds and fields of confout.txt, and a run resumed from it equals a run
resumed from confout.txt bit for bit.
"""
import math
import shutil

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


def ordered_sum(values) -> float:
    """Python 3.11's built-in sum of floats: left to right from 0 (the reference's
    analysis environment pins python=3.11, benchmarks/paper/environment.yml;
    from 3.12 on, sum() is compensated and may differ in the last bit)."""
    s = 0.0
    for v in values:
        s = s + v
    return s


def analysis_block_stats(samples: list[float], block_size: int):
    """benchmarks/paper/analysis.py:52-64, restated with its sums in order."""
    usable = samples[: (len(samples) // block_size) * block_size]
    means = [ordered_sum(usable[i:i + block_size]) / block_size for i in range(0, len(usable), block_size)]
    mean = ordered_sum(means) / len(means)
    return mean, math.sqrt(ordered_sum((v - mean) ** 2 for v in means) / (len(means) - 1) / len(means)), len(means)


def test_device_block_statistics_equal_the_analysis_scripts(solver_mod):
    pts = [point(), SolverParams(U1=1.0, U2=0.0, mu=-5.0, Nlx=4, Nly=3, Ltrot=20, Beta=1.0, NlxTherm=4,
                                 NlyTherm=3, LtrotTherm=20, Nwrap=10, Nbin=1, Nsweep=1, shiftLoc=1.5,
                                 iniType=2, iniAmpl=1.0)]
    bins = []
    with solver_mod.Ensemble(pts, [0, 1, 0, 1]) as ens:
        ens.fields_from_seeds([3, 4, 5, 6])
        ens.pre()
        ens.stats_reset(block_size=5, max_blocks=16)
        for _ in range(23):   # 4 full blocks; the last 3 bins form no block
            ens.sweep(1)
            bins.append(ens.point_obs_raw().copy())
        mean, sem, nb = ens.stats_raw()
    assert nb == 4
    bins = np.array(bins)   # [bin][point][slot]
    for p in range(2):
        for k in range(bins.shape[2]):
            m, e, n = analysis_block_stats(bins[:, p, k].tolist(), 5)
            assert mean[p, k] == m and (sem[p, k] == e or (np.isnan(sem[p, k]) and np.isnan(e))), (p, k)


def test_binary_checkpoint_round_trip_and_resume(solver_mod, tmp_path):
    p = point(nbin=2)
    first = tmp_path / "first"
    first.mkdir()
    (first / "paramC_sets.txt").write_text(p.to_text())
    (first / "confin.txt").write_text("0\n")
    (first / "seeds.txt").write_text("31\n32\n")
    solver_mod.run_directory(first, nchains=2, log=lambda *a: None)
    z = np.load(first / "confout.npz")
    txt = solver_mod.read_confin(first / "confout.txt", p, 2)
    assert z["seeds"].tolist() == [s for s, _ in txt]
    for c in range(2):
        np.testing.assert_array_equal(z["phi"][c].ravel(), np.asarray(txt[c][1]).ravel())
    runs = {}
    for name, src, dst in (("txt", "confout.txt", "confin.txt"), ("npz", "confout.npz", "confin.npz")):
        d = tmp_path / name
        d.mkdir()
        (d / "paramC_sets.txt").write_text(point(nbin=1).to_text())
        (d / "seeds.txt").write_text("31\n32\n")
        (d / "confin.txt").write_text("0\n")
        shutil.copy(first / src, d / dst)
        solver_mod.run_directory(d, nchains=2, log=lambda *a: None)
        runs[name] = ((d / "density_total").read_text(), (d / "confout.txt").read_text())
    assert runs["txt"] == runs["npz"]


def test_time_displaced_run_directory(solver_mod, tmp_path):
    """is_tau = .true. with Nthermal = 1 over 3 bins (main.f90:49-50): the pass
    runs in bins 2 and 3 only, info.txt gets Dyn_control_print's six lines
    (dynamics.f90:74-79) after the acceptance lines, and the Markov chain (the
    checkpoint) is that of the same run without the pass, bit for bit."""
    import json
    import dataclasses
    out = {}
    for tau in (False, True):
        d = tmp_path / ("tau" if tau else "plain")
        d.mkdir()
        p = dataclasses.replace(point(nbin=3), is_tau=tau, Nthermal=1)
        (d / "paramC_sets.txt").write_text(p.to_text())
        (d / "confin.txt").write_text("0\n")
        (d / "seeds.txt").write_text("41\n42\n")
        solver_mod.run_directory(d, nchains=2, log=lambda *a: None)
        out[tau] = d
    assert (out[False] / "confout.txt").read_text() == (out[True] / "confout.txt").read_text()
    lines = (out[True] / "info.txt").read_text().splitlines()
    labels = [ln.split(":")[0].strip() for ln in lines]
    want = ["Max diff GRtt", "Mean diff GRtt", "Max diff GRt0", "Mean diff GRt0", "Max diff GR0t", "Mean diff GR0t"]
    i = labels.index("Max diff GRtt")
    assert labels[i:i + 6] == want
    assert labels[i - 1] == "Accept_U2_shift" and labels[i + 6] == "Max diff Matrix"
    vals = [float(lines[i + k].split(":")[1]) for k in range(6)]
    assert all(0 < v < 1e-8 for v in vals), vals
    assert "Max diff GRtt" not in (out[False] / "info.txt").read_text()
    rec = json.loads((out[True] / "run_record.json").read_text())
    assert rec["tau_passes"] == 2 * 2 and rec["tau_nonfinite"] == 0
