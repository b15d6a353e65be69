"""Train the learned proposer on configurations of the plain sampler.

    python -m bafqmc_b200.train_proposer --chains 1024 --sweeps 200 --lag 10 \
        --steps 3000 --batch 64 --out bafqmc_b200/data/proposer_6x6_beta8.npz

Workload: 6x6, beta = 8, dtau = 0.05 (L = 160), U1 = 1, U2 = -0.5, mu = -5,
Nwrap = 10, shiftLoc = 1.5.  `chains` chains of the plain FP64 sampler are
equilibrated for `equil` sweeps; the fields after each of the next `sweeps`
sweeps are collected on the device (chains x sweeps configurations, 2x10^5
at the defaults).  The network is then trained by Adam on pairs (phi, phi')
of one chain `lag` sweeps apart: it learns a Gaussian transition
phi -> mu(phi) + exp(lsig(phi)) xi that jumps as far as `lag` sweeps of the
plain sampler.  Every step of training (forward, loss, gradient, optimiser)
runs on the GPU in the library's own kernels.  The untrained network (zero
last layer) is the prior's independence sampler; after every chunk of
steps the network's moves are tried on the ensemble (`eval_moves` moves,
each followed by a local sweep) and the parameters with the highest exact
Metropolis-Hastings acceptance so far are kept (the untrained network
included), since the acceptance, not the training loss, sets what a move
is worth.
"""
from __future__ import annotations

import argparse
import json
import math
import time
from pathlib import Path

import numpy as np

from .calibrate_tau import workload_6x6_beta8
from .proposer import Proposer


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--chains", type=int, default=1024)
    ap.add_argument("--equil", type=int, default=100)
    ap.add_argument("--sweeps", type=int, default=200)
    ap.add_argument("--lag", type=int, default=10)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--width", type=int, default=64)
    ap.add_argument("--moves", type=int, default=20, help="trial moves after training")
    ap.add_argument("--eval-moves", type=int, default=3, help="moves per acceptance check")
    ap.add_argument("--seed0", type=int, default=7000001)
    ap.add_argument("--out", type=str, default="")
    a = ap.parse_args(argv)
    from .solver import Ensemble
    p = workload_6x6_beta8()
    rec = {"workload": "6x6 beta=8 U1=1 U2=-0.5 mu=-5 dtau=0.05 Nwrap=10 shiftLoc=1.5", "chains": a.chains,
           "equil_sweeps": a.equil, "collected_sweeps": a.sweeps, "configurations": a.chains * a.sweeps,
           "lag": a.lag, "steps": a.steps, "batch": a.batch, "lr": a.lr, "width": a.width, "seconds": {}}
    ens = Ensemble([p], np.zeros(a.chains, dtype=np.int32))
    ens.fields_from_seeds(a.seed0 + 7919 * np.arange(a.chains))
    ens.pre()
    t0 = time.time()
    ens.sweep(a.equil)
    net = Proposer(p.Nlx, p.Nly, p.Ltrot, a.width, seed=a.seed0 % 1000)
    net.reserve(a.chains, a.sweeps)
    for _ in range(a.sweeps):
        ens.sweep(1)
        net.collect(ens)
    ens.synchronize()
    t1 = time.time()
    rec["seconds"]["sampling"] = t1 - t0
    def acceptance(k):
        acc = []
        for _ in range(k):
            acc.append(ens.learned_move(net)[0].mean())
            ens.sweep(1)
        return float(np.mean(acc))

    # Adam with a cosine decay of the learning rate, in chunks; the parameters
    # with the best acceptance are kept
    best_acc, best_params, best_step = acceptance(a.eval_moves), net.get_params(), 0
    rec["acceptance_untrained"] = best_acc
    print(f"step 0: acceptance {best_acc:.4f}", flush=True)
    losses = []
    history = []
    chunk = 250
    done = 0
    while done < a.steps:
        n = min(chunk, a.steps - done)
        lr = a.lr * 0.5 * (1.0 + math.cos(math.pi * done / a.steps))
        losses.append(net.train(n, a.batch, a.lag, lr, seed=a.seed0 + done))
        done += n
        acc = acceptance(a.eval_moves)
        history.append((done, float(losses[-1][-50:].mean()), acc))
        print(f"step {done}: loss {losses[-1][-50:].mean():.5f} (lr {lr:.2e}) acceptance {acc:.4f}", flush=True)
        if acc >= best_acc:
            best_acc, best_params, best_step = acc, net.get_params(), done
    net.set_params(best_params)
    losses = np.concatenate(losses)
    t2 = time.time()
    rec["seconds"]["training"] = t2 - t1
    rec["loss_first_100"] = float(losses[:100].mean())
    rec["loss_last_100"] = float(losses[-100:].mean())
    rec["history"] = history
    rec["kept_step"] = best_step
    # the trained moves on the ensemble, each followed by a local sweep
    acc = []
    hst = []
    for _ in range(a.moves):
        ac, h = ens.learned_move(net)
        acc.append(ac.mean())
        hst.append(float(np.median(h)))
        ens.sweep(1)
    rec["move_acceptance"] = float(np.mean(acc))
    rec["median_hastings"] = float(np.median(hst))
    rec["seconds"]["moves"] = time.time() - t2
    print(json.dumps(rec, indent=1), flush=True)
    if a.out:
        Path(a.out).parent.mkdir(parents=True, exist_ok=True)
        net.save(a.out, **rec)
        Path(a.out).with_suffix(".json").write_text(json.dumps(rec, indent=1) + "\n")
    net.close()
    ens.close()


if __name__ == "__main__":
    main()
