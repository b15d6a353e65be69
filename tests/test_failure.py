"""Failure detection on the host (no GPU): the reference stops on bad input
(calc_basic.f90:61-62,103) and has no recovery; here a corrupt confin.txt is
rejected with the chain and position named, and a rank that leaves a
multi-process run ends the others' next per-bin reduction with an error
instead of a hang."""
import os
from datetime import timedelta

import numpy as np
import pytest
import torch.multiprocessing as mp

from bafqmc_b200.params import SolverParams
from bafqmc_b200.solver import read_confin


def params():
    return SolverParams(U1=1.0, U2=-0.5, mu=-5.0, Nlx=3, Nly=3, Ltrot=4, Beta=0.4, NlxTherm=3, NlyTherm=3,
                        LtrotTherm=4, Nwrap=2, Nbin=1, Nsweep=1, shiftLoc=1.5, iniType=2, iniAmpl=1.0)


def confin_text(nchains, per, bad=None):
    rows = []
    for c in range(nchains):
        rows.append(f" {100 + c}")
        rows += [f" {0.01 * k:.17e}" for k in range(per)]
    if bad is not None:
        rows[bad[0]] = bad[1]
    return "\n".join(rows) + "\n"


def test_confin_zero_means_seeds(tmp_path):
    (tmp_path / "confin.txt").write_text("0\n")
    assert read_confin(tmp_path / "confin.txt", params(), 2) is None


def test_confin_round_trip(tmp_path):
    per = 4 * 9 * 2
    (tmp_path / "confin.txt").write_text(confin_text(2, per))
    out = read_confin(tmp_path / "confin.txt", params(), 2)
    assert [s for s, _ in out] == [100, 101]
    np.testing.assert_array_equal(out[1][1].ravel(), 0.01 * np.arange(per))


def test_truncated_confin_is_rejected(tmp_path):
    per = 4 * 9 * 2
    text = confin_text(2, per)
    (tmp_path / "confin.txt").write_text("\n".join(text.split("\n")[:-10]) + "\n")
    with pytest.raises(ValueError, match="needed for 2 chains"):
        read_confin(tmp_path / "confin.txt", params(), 2)


def test_corrupt_value_is_rejected_with_position(tmp_path):
    per = 4 * 9 * 2
    (tmp_path / "confin.txt").write_text(confin_text(2, per, bad=(5, " 1.0x-3")))
    with pytest.raises(ValueError, match=r"value 6 \('1.0x-3'\) is not a number"):
        read_confin(tmp_path / "confin.txt", params(), 2)


def test_non_finite_field_is_rejected(tmp_path):
    per = 4 * 9 * 2
    (tmp_path / "confin.txt").write_text(confin_text(2, per, bad=(per + 3, " NaN")))
    with pytest.raises(ValueError, match="non-finite field value in chain 1"):
        read_confin(tmp_path / "confin.txt", params(), 2)


def _rank(rank, world, port, out):
    import torch.distributed as dist
    from bafqmc_b200.multigpu import chain_average, torch_all_reduce
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=5))
    if rank == 1:   # this rank leaves between bins, before the reduction of the next bin
        out[rank] = "left"
        return
    try:
        chain_average(np.ones(8), 4, torch_all_reduce())
        out[rank] = "completed"
    except Exception as e:   # the survivor learns of it from the collective
        out[rank] = "error: " + type(e).__name__
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


@pytest.mark.timeout(120)
def test_rank_leaving_ends_the_next_bin_reduction_with_an_error():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = 31500 + os.getpid() % 1000
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert out[1] == "left"
    assert out[0].startswith("error"), out[0]


def test_time_displaced_request_outside_its_range_is_refused(tmp_path):
    """is_tau = .true. (calc_basic.f90:56) runs the time-displaced pass of
    dynamics.f90, built here for number-conserving chains with Ndim <= 72: a
    12x12 run (Ndim 144) is refused before any device work, instead of
    ignoring the flag."""
    import dataclasses
    from bafqmc_b200.params import ParamError
    from bafqmc_b200.solver import run_directory
    p = dataclasses.replace(params(), Nlx=12, Nly=12, NlxTherm=12, NlyTherm=12)
    text = p.to_text().splitlines()
    text[4] = ".true. 10"
    (tmp_path / "paramC_sets.txt").write_text("\n".join(text) + "\n")
    with pytest.raises(ParamError, match="is_tau"):
        run_directory(tmp_path, nchains=1)
    assert not (tmp_path / "info.txt").exists()


def test_drift_warnings_once_per_chain_and_kind():
    """The reference warns when a recomputed Green's function moved by 5.5e-5 or more
    (stabilization.f90:320, 358, 387-397); run directories report it once per
    chain and kind, from the drift maxima after each bin."""
    import numpy as np
    from bafqmc_b200.solver import drift_warnings
    seen, lines = set(), []
    drift = np.array([1e-12, 6e-5, 5.5e-5, 1e-3])
    ts = np.zeros((4, 8))
    ts[1, 1] = 1e-4   # G(tau,0) of chain 1
    new = drift_warnings(drift, ts, seen, 1, lines.append)
    assert new == lines and len(new) == 4
    assert [ln.split(":")[0] for ln in new] == [" WARNING", " WARNING", " WARNING", " WARNING"]
    assert "chain 1: drift" in new[0] and "chain 2: drift" in new[1] and "chain 3: drift" in new[2]
    assert "chain 1: GRT0 drift" in new[3]
    # already reported: nothing new; a new chain crossing the threshold is
    drift[0] = 1.0
    assert len(drift_warnings(drift, ts, seen, 2, lines.append)) == 1 and "by bin 2" in lines[-1]
    assert drift_warnings(drift, None, seen, 3, lines.append) == []
