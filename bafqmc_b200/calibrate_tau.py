"""Measure tau_int of rho, -E, Re S_SF(K), Re S_DW(K) for the plain sweep,
or for the learned sampler (one learned global move, then one local sweep,
per step).

    python -m bafqmc_b200.calibrate_tau --chains 1024 --warmup 200 --sweeps 300 \
        --out bafqmc_b200/data/tau_int_6x6_beta8.json
    python -m bafqmc_b200.calibrate_tau --chains 1024 --warmup 200 --sweeps 300 \
        --learned bafqmc_b200/data/proposer_6x6_beta8.npz \
        --out bafqmc_b200/data/tau_int_6x6_beta8_learned.json

Runs the batched number-conserving sweep at 6x6, beta=8 (U1=1, U2=-0.5,
mu=-5, dtau=0.05, Nwrap=10, shiftLoc=1.5), one bin per sweep, and records the
per-chain bin series after `warmup` full-weight sweeps.  tau_int is in units
of steps: one sweep (left + right traversal = one bin at Nsweep=1) for the
plain sampler, one learned move plus one sweep for the learned sampler.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from .ess import tau_blocking, tau_int
from .observables import COMPLEX_SLOTS, REAL_SLOTS
from .params import SolverParams

OBSERVABLES = ("density_total", "minus_energy", "sf_K", "dw_K")


def workload_6x6_beta8(**kw) -> SolverParams:
    base = dict(U1=1.0, U2=-0.5, mu=-5.0, Nlx=6, Nly=6, Ltrot=160, Beta=8.0, NlxTherm=6, NlyTherm=6,
                LtrotTherm=160, Nwrap=10, Nbin=1, Nsweep=1, shiftLoc=1.5, iniType=2, iniAmpl=1.0)
    base.update(kw)
    return SolverParams(**base)


def series_row(raw: np.ndarray, lq: int) -> np.ndarray:
    """[chains, 4] of rho, -E (= -Ns * energy_density), Re S_SF(K), Re S_DW(K)."""
    return np.stack([raw[:, REAL_SLOTS["density_total"]],
                     -lq * raw[:, REAL_SLOTS["energy_density"]],
                     raw[:, COMPLEX_SLOTS["sf_K"]],
                     raw[:, COMPLEX_SLOTS["dw_K"]]], axis=1)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--chains", type=int, default=1024)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--sweeps", type=int, default=300)
    ap.add_argument("--seed0", type=int, default=1000003)
    ap.add_argument("--learned", type=str, default="", help="proposer parameter file: the learned sampler")
    ap.add_argument("--out", type=str, default="")
    a = ap.parse_args(argv)
    from .solver import Ensemble
    p = workload_6x6_beta8()
    ens = Ensemble([p], np.zeros(a.chains, dtype=np.int32))
    ens.fields_from_seeds(a.seed0 + 7919 * np.arange(a.chains))
    ens.pre()
    net = None
    if a.learned:
        from .proposer import Proposer
        net = Proposer.load(a.learned)

    def step():
        if net is not None:
            ens.learned_move(net, want=False)
        ens.sweep(1)

    t0 = time.time()
    for _ in range(a.warmup):
        step()
    ens.synchronize()
    t1 = time.time()
    data = np.zeros((a.sweeps, a.chains, 4))
    for s in range(a.sweeps):
        step()
        data[s] = series_row(ens.chain_obs_raw(), p.Lq)
    t2 = time.time()
    x = data.transpose(2, 1, 0)   # [obs, chains, steps]
    kind = (f"learned sampler (one move of {Path(a.learned).name}, then one local sweep, per step)" if net
            else "plain FP64 local sweep")
    out = {"workload": f"6x6 beta=8 U1=1 U2=-0.5 mu=-5 dtau=0.05 Nwrap=10 shiftLoc=1.5, {kind}",
           "chains": a.chains, "warmup_sweeps": a.warmup, "sweeps": a.sweeps,
           "units": "steps (move + sweep)" if net else "sweeps",
           "seconds": {"warmup": t1 - t0, "measure": t2 - t1}, "tau_int": {}, "window": {}, "tau_blocking": {},
           "mean": {}, "sem_over_chains": {}}
    for k, name in enumerate(OBSERVABLES):
        tau, w = tau_int(x[k])
        out["tau_int"][name] = tau
        out["window"][name] = w
        out["tau_blocking"][name] = tau_blocking(x[k], max(1, a.sweeps // 10))
        out["mean"][name] = float(x[k].mean())
        out["sem_over_chains"][name] = float(x[k].mean(axis=1).std(ddof=1) / np.sqrt(a.chains))
    cnt = ens.counters()
    out["acceptance"] = (cnt[:, 0:2].mean(0) / (a.warmup + a.sweeps)).tolist()
    if net is not None:
        out["move_acceptance"] = float(cnt[:, 9].mean() / (a.warmup + a.sweeps))
    out["max_drift"] = float(cnt[:, 4].max())
    out["bad_chains"] = int(np.count_nonzero(cnt[:, 6]))
    js = json.dumps(out, indent=1)
    if a.out:
        Path(a.out).parent.mkdir(parents=True, exist_ok=True)
        Path(a.out).write_text(js + "\n")
    print(js)


if __name__ == "__main__":
    main()
