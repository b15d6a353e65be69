#!/usr/bin/env python
"""Benchmark of the B200 BAFQMC sampler at 6x6, beta = 8.

Headline metric: effective samples per second per B200 of the learned
sampler against the plain FP64 sweep, at equal error bars on rho, -E,
Re S_SF(K) and Re S_DW(K).

* Plain arm: 4096 number-conserving chains, 6x6 triangular lattice (Ns = 36),
  t = 1, U1 = 1, U2 = -0.5, mu = -5, beta = 8, dtau = 0.05 (L = 160), Nwrap = 10,
  shiftLoc = 1.5, N(0,1) fields from per-chain seeds; a step is one sweep
  (left + right traversal, one measurement bin) of every chain, FP64.
* Learned arm (the line's value): the same point with 1024 chains; a step is
  one learned global move (the bf16 convolutional proposer of
  bafqmc_b200/data/proposer_6x6_beta8.npz, trained on the GPU on 2x10^5
  configurations of the plain sampler, accepted by the exact
  Metropolis-Hastings ratio) followed by one local sweep, FP64 sweeps.

ESS/s = (chain-steps/s) / (2 tau_int), tau_int the largest over the four
observables, calibrated per arm by bafqmc_b200.calibrate_tau (units: steps
of that arm).  At equal error bars the time each arm needs is inversely
proportional to its ESS/s, so ess_ratio = ESS/s(learned) / ESS/s(plain) is
the equal-error speed-up, reported against the 10x target.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--gpus N > 1 without a torchrun environment launches N ranks itself (one
process per GPU, chains sharded per rank, NCCL all-reduce of each bin
record in the end-to-end leg); under torchrun the ranks come from the
environment.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "effective samples/sec per B200 at 6x6 β=8: learned+mixed vs plain FP64, equal error"
UNIT = "effective samples/s"
TAU_FILE = ROOT / "bafqmc_b200" / "data" / "tau_int_6x6_beta8.json"
TAU_LEARNED_FILE = ROOT / "bafqmc_b200" / "data" / "tau_int_6x6_beta8_learned.json"
NET_FILE = ROOT / "bafqmc_b200" / "data" / "proposer_6x6_beta8.npz"
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
TARGET_RATIO = 10.0
# kernel launches of one learned step: the move (input pack + 4 layers, twice;
# proposal; Hastings term; pre of the proposal; two field norms; accept) and
# the sweep's bin graph (reset, sweep, finish)
LEARNED_STEP_LAUNCHES = 2 * 5 + 2 + 1 + 2 + 1 + 3
PLAIN_STEP_LAUNCHES = 3


def workload():
    from bafqmc_b200.calibrate_tau import workload_6x6_beta8
    return workload_6x6_beta8()


def tau_table(path: Path = TAU_FILE):
    if path.exists():
        d = json.loads(path.read_text())
        return d["tau_int"], f"{path.relative_to(ROOT)} ({d['chains']} chains x {d['sweeps']} steps)"
    return None, f"uncalibrated ({path.name} missing; tau_int = 0.5)"


def ess_rate(steps_per_s: float, path: Path = TAU_FILE):
    taus, src = tau_table(path)
    if not taus:
        return steps_per_s, {"tau_int": None, "tau_source": src}
    name = max(taus, key=lambda k: taus[k])
    return steps_per_s / (2.0 * taus[name]), {"tau_int_max": round(taus[name], 3), "tau_limiting": name,
                                              "tau_source": src}


def flops_per_chain_sweep(n: int, L: int, nwrap: int, naccept: float) -> float:
    """Algorithmic FP64 flops of one sweep of one chain: 2L slice steps of three
    N^3 products of a complex matrix with the real e^{-+dtau K} (4 N^3 each; the
    reference's ZGEMMs count 8 N^3 because they carry the zero imaginary part),
    8 N^2 per accepted rank-1 update, and 2L/Nwrap stabilisations at (15 + 45) N^3
    (pivoted QR + ZUNGQR + ZTRMM, and stab_green), by LAPACK's complex flop counts."""
    return 2 * L * 12.0 * n ** 3 + 8.0 * n ** 2 * naccept + (2.0 * L / nwrap) * 60.0 * n ** 3


def conv_flops(chains: int, L: int, ns: int, cin: int = 64, cout: int = 64) -> float:
    """Algorithmic flops of one periodic 3x3x3 convolution launch: 2 x 27 cin cout per point."""
    return 2.0 * 27 * cin * cout * chains * L * ns


# the profiling recipe's figures for this pool's B200s, used only when the
# measured file is absent (it is written per machine by the benchmark driver)
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}


def measured_peaks() -> tuple[dict, str]:
    try:
        return json.loads(PEAKS_FILE.read_text()), "of measured (MEASURED_PEAKS.json)"
    except (OSError, ValueError):
        return dict(FALLBACK_PEAKS), "of fallback (MEASURED_PEAKS.json absent on this machine)"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def fp64_gemm_peak(dev) -> float:
    """Measured cuBLAS FP64 GEMM throughput (TFLOP/s), the FP64 roofline."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = float("inf")
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


# ---------------------------------------------------------------------------
# CPU arm: the C++ restatement of the reference's sweep (oracle/csweep.cpp,
# checked against oracle.py) on the host cores, one chain per thread
def _cport():
    sys.path.insert(0, str(ROOT))
    from oracle import cport
    if not cport.LIB.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle")], check=True, capture_output=True)
    from oracle import oracle as O
    return cport, O


def cpu_sweep_rate(cores: int, sweeps_per_chain: int, seed0: int = 1000):
    """chain-sweeps/s of the C++ restatement, `cores` chains on `cores` threads
    (after each chain's pre); returns (rate, wall seconds)."""
    cport, O = _cport()
    p = workload()
    op = O.Params(U1=p.U1, U2=p.U2, mu=p.mu, Nlx=p.Nlx, Nly=p.Nly, Ltrot=p.Ltrot, Beta=p.Beta, NlxTherm=p.NlxTherm,
                  NlyTherm=p.NlyTherm, LtrotTherm=p.LtrotTherm, Nwrap=p.Nwrap, Nbin=1, Nsweep=1,
                  shiftLoc=p.shiftLoc, iniType=p.iniType, iniAmpl=p.iniAmpl)
    _, _, chains = O.init_chains(op, seeds=[seed0 + 17 * i for i in range(cores)])
    seeds = np.array([c.seed for c in chains], dtype=np.int32)
    phi = np.ascontiguousarray(np.stack([c.phi for c in chains]))
    t0 = time.perf_counter()
    out = cport.run(op, seeds, phi, sweeps_per_chain, nthreads=cores)
    wall = time.perf_counter() - t0
    return cores * sweeps_per_chain / out["sweep_seconds"], wall


def cpu_baseline(cores: int, sweeps_per_chain: int = 4):
    rate, wall = cpu_sweep_rate(cores, sweeps_per_chain)
    ess, _ = ess_rate(rate)
    return {"value": ess, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{cores} chains x {sweeps_per_chain} sweeps of the 6x6 beta=8 workload, one chain per thread "
                      f"(oracle/csweep.cpp, the C++ restatement of the reference's sweep checked against "
                      f"oracle.py), after pre; {rate:.2f} chain-sweeps/s"}


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    per = 2
    for k in range(args.warmup):
        cpu_sweep_rate(cores, 1, seed0=500 + k)
    rates, walls = [], []
    for k in range(args.steps):
        r, w = cpu_sweep_rate(cores, per, seed0=1000 + 100 * k)
        rates.append(r)
        walls.append(w)
    rate = float(np.mean(rates))
    ess, tau = ess_rate(rate)
    line = {"impl": "reference", "metric": METRIC, "value": ess, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(walls)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded N(0,1) HS fields)",
            "config": {"workload": "6x6 beta=8 (U1=1, U2=-0.5, mu=-5, dtau=0.05, L=160, Nwrap=10, shiftLoc=1.5): "
                                   "the reference's plain local sweep on the host cores (the reference has no "
                                   "learned sampler)", "sample_per_step":
                       f"{cores} chains x {per} sweeps on {cores} host threads", "chain_sweeps_per_s": rate, **tau},
            "cpu_baseline": {"value": ess, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{cores} chains x {per} sweeps per step, oracle/csweep.cpp (C++ "
                                       f"restatement of the reference's sweep), one chain per thread"},
            "e2e": {"value": ess, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def run_ragged(args):
    """The ragged batch: 216 parameter points (3x3, 4x4, 6x6; beta 2, 4, 8;
    number-conserving and Nambu) x 32 chains in one handle, kernel classes from
    the autotuner, one persistent launch per class and sweep; against the same
    points run one handle at a time (the sequential plain path)."""
    import torch
    from bafqmc_b200.solver import Ensemble, autotune
    from bafqmc_b200.workloads import ragged_grid
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    pts = ragged_grid()
    per = 32
    classes, _ = autotune(pts)
    chain_point = np.repeat(np.arange(len(pts)), per).astype(np.int32)
    seeds = 4242 + 7919 * np.arange(chain_point.size)
    ens = Ensemble(pts, chain_point, classes=classes)
    ens.fields_from_seeds(seeds)
    ens.pre()
    for _ in range(max(args.warmup, 3)):
        ens.sweep(1)
    ens.synchronize()
    stream = torch.cuda.ExternalStream(ens.stream, device=dev)
    clocks = ClockSampler(0)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        ens.sweep(1)
    e1.record(stream)
    e1.synchronize()
    clk = clocks.stop()
    ragged_s = e0.elapsed_time(e1) / 1e3 / args.steps
    ens.close()
    # the same chains, one point per handle, each timed alone
    seq_s = 0.0
    for k, p in enumerate(pts):
        with Ensemble([p], np.zeros(per, dtype=np.int32), classes=[int(classes[k])]) as one:
            one.fields_from_seeds(seeds[k * per:(k + 1) * per])
            one.pre()
            one.sweep(1)
            one.synchronize()
            st = torch.cuda.ExternalStream(one.stream, device=dev)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            one.sweep(1)
            b.record(st)
            b.synchronize()
            seq_s += a.elapsed_time(b) / 1e3
    n = int(chain_point.size)
    print(json.dumps({
        "metric": "chain-sweeps/s per B200, ragged batch (216 points x 32 chains, FP64)", "value": n / ragged_s,
        "unit": "chain-sweeps/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": 1e3 * ragged_s, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded N(0,1) HS fields)",
        "config": {"workload": "ragged grid: Lx=Ly in {3,4,6}, beta in {2,4,8}, U2 in {0,-0.5}, mu in {-6,-5,-4}, "
                               "number-conserving and Nambu Delta in {0.25,0.5,1}", "points": len(pts),
                   "chains_per_point": per, "chains": n,
                   "classes": {str(c): int(np.sum(classes == c)) for c in np.unique(classes)},
                   "sequential_ms_per_sweep": 1e3 * seq_s, "sequential_chain_sweeps_per_s": n / seq_s,
                   "speedup_vs_sequential": seq_s / ragged_s},
        "clocks": clk,
    }), flush=True)


def run_12x12(args):
    """12x12 (N = 144), U1 = 1, U2 = -0.5, mu = -5, beta = 10, dtau = 0.05 (L = 200),
    Nwrap = 10, 512 chains: the size class whose matrices live in HBM.  One
    line of chain-sweeps/s with the FP64 roofline, on one GPU."""
    import torch
    from bafqmc_b200.params import SolverParams
    from bafqmc_b200.solver import Ensemble
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    C = 512 if args.chains == 4096 else args.chains
    p = SolverParams(U1=1.0, U2=-0.5, mu=-5.0, Nlx=12, Nly=12, Ltrot=200, Beta=10.0, NlxTherm=12, NlyTherm=12,
                     LtrotTherm=200, Nwrap=10, Nbin=1, Nsweep=1, shiftLoc=1.5, iniType=2, iniAmpl=1.0)
    ens = Ensemble([p], np.zeros(C, dtype=np.int32))
    ens.set_precision(args.precision)
    ens.fields_from_seeds(20241203 + 7919 * np.arange(C))
    ens.pre()
    for _ in range(max(args.warmup, 3)):
        ens.sweep(1)
    ens.synchronize()
    stream = torch.cuda.ExternalStream(ens.stream, device=dev)
    cnt0 = ens.counters()
    clocks = ClockSampler(0)
    clocks.start()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        ens.sweep(1)
    e1.record(stream)
    e1.synchronize()
    clk = clocks.stop()
    dev_s = e0.elapsed_time(e1) / 1e3
    cnt1 = ens.counters()
    acc = (cnt1[:, 0:2] - cnt0[:, 0:2]).mean(0) / args.steps
    naccept = float(acc.sum()) * 2 * p.Ltrot * p.Ndim
    flops = flops_per_chain_sweep(p.Ndim, p.Ltrot, p.Nwrap, naccept) * C * args.steps
    achieved = flops / dev_s / 1e12
    peak = fp64_gemm_peak(dev)
    # G of a sample of chains against G recomputed in FP64 from the same fields
    sample = min(C, 16)
    seeds, phis = ens.get_state()
    with Ensemble([p], np.zeros(sample, dtype=np.int32)) as ref:
        ref.set_state(seeds[:sample], phis[:sample])
        ref.pre()
        g_err = max(float(np.max(np.abs(ens.green(c) - ref.green(c)))) for c in range(sample))
    print(json.dumps({
        "metric": f"chain-sweeps/s per B200 at 12x12 beta=10 ({args.precision})", "value": C * args.steps / dev_s,
        "unit": "chain-sweeps/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": 1e3 * dev_s / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "tf32x3+f64", "data": "synthetic (seeded N(0,1) HS fields)",
        "config": {"workload": f"12x12 beta=10 {args.precision} sweep (U1=1, U2=-0.5, mu=-5, dtau=0.05, L=200, "
                               "Nwrap=10, shiftLoc=1.5)", "chains_per_gpu": C, "acceptance": acc.tolist(),
                   "precision": "FP64" if args.precision == "fp64" else
                   "slice products 3xTF32 on the tensor cores (FP32 accumulate), the rest FP64",
                   "g_maxabs_err_vs_fp64": g_err, "g_err_sample_chains": sample,
                   "l2": "31 MB arena + 1.7 MB working region per chain x chains >> 126 MB L2 (no flush needed)"},
        "roofline": {"bound": "tensor", "pipe": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None,
                     "peak_source": "cuBLAS FP64 GEMM 8192^3 measured in this run",
                     "note": "achieved counts the algorithm's FP64-equivalent flops"},
        "clocks": clk, "gpu_launches": 3 * args.steps,
    }), flush=True)
    ens.close()


# ---------------------------------------------------------------------------
# the two GPU arms of the headline
def _timed_steps(ens, stream, step, steps, world, dev, sweep_events=False):
    """Device time of `steps` calls of step() on the ensemble's stream (max over
    ranks), bracketed by a barrier and synchronize on both sides; with
    sweep_events, also the summed device time of the sweeps inside the steps."""
    import torch
    import torch.distributed as dist
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sw = []
    e0.record(stream)
    for _ in range(steps):
        step(sw if sweep_events else None)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    dev_s = e0.elapsed_time(e1) / 1e3
    sweep_s = sum(a.elapsed_time(b) for a, b in sw) / 1e3 if sw else None
    if world > 1:
        t = torch.tensor([dev_s, sweep_s or 0.0], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_s, sweep_s = float(t[0]), (float(t[1]) if sweep_s is not None else None)
    return dev_s, sweep_s


def plain_arm(args, rank, world, dev):
    """4096 chains per GPU of the plain FP64 sweep: device-timed chain-sweeps/s."""
    import torch
    from bafqmc_b200.solver import Ensemble
    p = workload()
    C = args.chains
    ens = Ensemble([p], np.zeros(C, dtype=np.int32), device=dev.index)
    ens.fields_from_seeds(20240601 + 7919 * (rank * C + np.arange(C)))
    ens.pre()
    for _ in range(max(args.warmup, 3)):
        ens.sweep(1)
    ens.synchronize()
    stream = torch.cuda.ExternalStream(ens.stream, device=dev)
    cnt0 = ens.counters()

    def step(_):
        ens.sweep(1)

    dev_s, _ = _timed_steps(ens, stream, step, args.steps, world, dev)
    cnt1 = ens.counters()
    acc = (cnt1[:, 0:2] - cnt0[:, 0:2]).mean(0) / args.steps
    ens.close()
    rate = world * C * args.steps / dev_s
    ess, tau = ess_rate(rate, TAU_FILE)
    naccept = float(acc.sum()) * 2 * p.Ltrot * p.Ndim
    return {"chains_per_gpu": C, "ms_per_step": 1e3 * dev_s / args.steps, "chain_sweeps_per_s": rate,
            "ess_per_s": ess, "acceptance": acc.tolist(), **tau,
            "sweep_flops_per_chain": flops_per_chain_sweep(p.Ndim, p.Ltrot, p.Nwrap, naccept)}


def learned_arm(args, rank, world, dev):
    """1024 chains per GPU of the learned sampler (one learned move, then one
    local sweep, per step): device-timed chain-steps/s, the sweeps' share, the
    move acceptance, the network layers' times and the end-to-end leg."""
    import torch
    from bafqmc_b200.proposer import Proposer
    from bafqmc_b200.solver import Ensemble
    p = workload()
    C = args.learned_chains
    net = Proposer.load(NET_FILE, device=dev.index)
    ens = Ensemble([p], np.zeros(C, dtype=np.int32), device=dev.index)
    ens.fields_from_seeds(31000007 + 7919 * (rank * C + np.arange(C)))
    ens.pre()
    ens.sweep(10)
    for _ in range(max(args.warmup, 3)):
        ens.learned_move(net, want=False)
        ens.sweep(1)
    ens.synchronize()
    stream = torch.cuda.ExternalStream(ens.stream, device=dev)
    cnt0 = ens.counters()

    def step(sw):
        ens.learned_move(net, want=False)
        if sw is None:
            ens.sweep(1)
            return
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ens.sweep(1)
        b.record(stream)
        sw.append((a, b))

    clocks = ClockSampler(dev.index)
    clocks.start()
    dev_s, sweep_s = _timed_steps(ens, stream, step, args.steps, world, dev, sweep_events=True)
    clk = clocks.stop()
    cnt1 = ens.counters()
    acc = (cnt1[:, 0:2] - cnt0[:, 0:2]).mean(0) / args.steps
    move_acc = float((cnt1[:, 9] - cnt0[:, 9]).mean() / args.steps)
    naccept = float(acc.sum()) * 2 * p.Ltrot * p.Ndim
    rate = world * C * args.steps / dev_s
    ess, tau = ess_rate(rate, TAU_LEARNED_FILE)
    out = {"chains_per_gpu": C, "ms_per_step": 1e3 * dev_s / args.steps, "chain_steps_per_s": rate,
           "ess_per_s": ess, "acceptance": acc.tolist(), "move_acceptance": move_acc, **tau,
           "sweep_ms_per_step": 1e3 * sweep_s / args.steps,
           "sweep_flops_per_chain": flops_per_chain_sweep(p.Ndim, p.Ltrot, p.Nwrap, naccept), "clocks": clk,
           "net_file": str(NET_FILE.relative_to(ROOT)),
           "net_sha256_16": hashlib.sha256(NET_FILE.read_bytes()).hexdigest()[:16]}
    # the network's layers, device-timed at the arm's chain count
    ms = net.time_layers(C, reps=5)
    out["layer_ms"] = ms.tolist()

    # ---- end to end through the C ABI with host buffers: every step is one
    # checkpointed step, as a reference run from confin.txt to confout.txt: the
    # chains' seeds and fields go host -> device from pinned memory
    # (bafqmc_set_state), bafqmc_pre rebuilds the UDV slots, one learned move and
    # one sweep, and the bin records, seeds and fields come back device -> host.
    from bafqmc_b200.multigpu import chain_average, torch_all_reduce
    import torch.distributed as dist
    reduce = torch_all_reduce(device=dev) if world > 1 else (lambda b: b)
    nphi = int(ens.phi_offsets[-1])
    h_seeds = torch.empty(C, dtype=torch.int32, pin_memory=True).numpy()
    h_phi = torch.empty(nphi, dtype=torch.float64, pin_memory=True).numpy()
    ens.get_state_flat(h_seeds, h_phi)
    h2d = h_seeds.nbytes + h_phi.nbytes
    d2h = 0
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ens.set_state_flat(h_seeds, h_phi)
        ens.pre()
        ens.learned_move(net, want=False)
        ens.sweep(1)
        pt = ens.point_obs_raw()
        ch = ens.chain_obs_raw()
        ens.get_state_flat(h_seeds, h_phi)
        d2h = pt.nbytes + ch.nbytes + h_seeds.nbytes + h_phi.nbytes
        chain_average(pt[0] * C, C, reduce)   # job-wide average (m_process_obs_equal's MPI_REDUCE)
    torch.cuda.synchronize(dev)
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value, _ = ess_rate(world * C * args.steps / e2e_s, TAU_LEARNED_FILE)
    out["e2e"] = {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                  "step": "checkpointed step: set_state (pinned h2d) + pre + learned move + 1 sweep + bins and "
                          "state d2h"}
    ens.close()
    net.close()
    return out


def mixed_at_6x6(dev, steps: int = 2):
    """The mixed-precision slice products at the metric's shape.  Only the
    N <= 144 kernel class has the tensor-core product path; the 6x6 point runs
    in it as well, so the same 148 chains (one CTA per SM) are timed in that
    class in FP64 and in mixed precision, and G of the mixed chains is compared
    with G recomputed in FP64 from the same fields."""
    import torch
    from bafqmc_b200.solver import Ensemble
    p = workload()
    C = 148
    out = {"chains": C, "kernel_class": 6}
    for mode in ("fp64", "mixed"):
        ens = Ensemble([p], np.zeros(C, dtype=np.int32), device=dev.index, classes=[6])
        ens.set_precision(mode)
        ens.fields_from_seeds(5151 + 7919 * np.arange(C))
        ens.pre()
        ens.sweep(1)
        ens.synchronize()
        stream = torch.cuda.ExternalStream(ens.stream, device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ens.sweep(steps)
        e1.record(stream)
        e1.synchronize()
        out[f"ms_per_chain_sweep_{mode}"] = e0.elapsed_time(e1) / (steps * C)
        if mode == "mixed":
            seeds, phis = ens.get_state()
            n = 16
            with Ensemble([p], np.zeros(n, dtype=np.int32), device=dev.index) as ref:
                ref.set_state(seeds[:n], phis[:n])
                ref.pre()
                out["g_maxabs_err_vs_fp64"] = max(float(np.max(np.abs(ens.green(c) - ref.green(c))))
                                                  for c in range(n))
        ens.close()
    return out


def run_headline(args, rank, world, local):
    # the CPU baseline runs before any CUDA call
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.cpu_cores or (os.cpu_count() or 1))
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    plain = plain_arm(args, rank, world, dev)
    learned = learned_arm(args, rank, world, dev)
    mixed = mixed_at_6x6(dev) if rank == 0 else None
    peaks, peaks_src = measured_peaks()
    if rank == 0:
        fp64_peak = fp64_gemm_peak(dev)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    p = workload()
    C = learned["chains_per_gpu"]
    # dominant kernel: the FP64 sweep (timed inside the learned steps)
    sweep_tflops = learned["sweep_flops_per_chain"] * C / (learned["sweep_ms_per_step"] / 1e3) / 1e12
    traffic = None
    tfile = ROOT / "profiles" / "sweep_kernel_6x6_beta8.md"
    if tfile.exists():
        import re
        m = re.search(r"dram_bytes_per_launch_4096_chains:\s*(\d+)", tfile.read_text())
        if m:   # per launch, scaled to this run's chain count
            traffic = int(m.group(1)) * C // 4096
    bf16_peak = peaks.get("bf16_tflops")
    conv_ms = float(np.mean(learned["layer_ms"][1:3]))
    conv_tflops = conv_flops(C, p.Ltrot, p.Lq) / (conv_ms / 1e3) / 1e12
    ratio = learned["ess_per_s"] / plain["ess_per_s"]
    line = {
        "metric": METRIC, "value": learned["ess_per_s"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": learned["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 sweeps + bf16 network (f32 accumulate)",
        "data": "synthetic (seeded N(0,1) HS fields)",
        "config": {
            "workload": "6x6 beta=8 learned sampler (U1=1, U2=-0.5, mu=-5, dtau=0.05, L=160, Nwrap=10, "
                        "shiftLoc=1.5): one learned global move + one local sweep per step, 1024 chains per GPU",
            "parallelism": f"chains x {world} GPU",
            "precision": "sweeps, stabilisation, (I-B)^-1, ratios and acceptance FP64: the 3xTF32 slice products "
                         "exist in the N<=144 kernel class only, and at 6x6 that class is slower in either precision "
                         "than the FP64 N<=36 class the arms use (mixed_at_6x6); proposer network bf16 with f32 "
                         "accumulation on tcgen05",
            "g_maxabs_err_vs_fp64": 0.0,
            "mixed_at_6x6": dict(
                mixed, ms_per_chain_sweep_fp64_class_used=plain["ms_per_step"] / plain["chains_per_gpu"],
                # the plain sampler's ESS/s on one GPU with the mixed products (148 chains fill the class's one
                # CTA per SM), at the plain chain's tau_int
                ess_per_s_plain_sampler_mixed=(1e3 / mixed["ms_per_chain_sweep_mixed"]) / (2.0 * plain["tau_int_max"])),
            "l2": "working set 1.5 MB/chain x chains >> 126 MB L2 (no flush needed)",
            "learned": {k: v for k, v in learned.items() if k not in ("e2e", "clocks")},
            "plain": plain,
            "ess_ratio_learned_vs_plain": ratio, "target_ratio": TARGET_RATIO,
            "meets_target": bool(ratio >= TARGET_RATIO),
            "equal_error": "time to a given SEM on all four observables is 2 tau_int / (chain-steps/s) per "
                           "effective sample, so the ESS/s ratio is the equal-error speed-up",
        },
        "roofline": {"bound": "tensor", "pipe": "fp64",
                     "limiter": "FP64 dependency latency and barriers (the sweep issues DFMA, no tensor instruction)",
                     "kernel": "sweep_kernel<36,0>", "achieved": sweep_tflops, "peak": fp64_peak,
                     "unit": "TFLOP/s", "frac": sweep_tflops / fp64_peak, "traffic": traffic,
                     "traffic_source": "dram bytes of one launch from the ncu capture in "
                                       "profiles/sweep_kernel_6x6_beta8.md, scaled to this chain count "
                                       "(not measured in this run)",
                     "peak_source": "cuBLAS FP64 GEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no "
                                    "FP64 figure)"},
        "roofline_network": {"bound": "tensor", "pipe": "bf16 tcgen05", "kernel": "conv_tc_kernel (64->64 layers)",
                             "achieved": conv_tflops, "peak": bf16_peak, "unit": "TFLOP/s",
                             "frac": conv_tflops / bf16_peak if bf16_peak else None,
                             "peak_source": f"bf16_tflops (burst) {peaks_src}"},
        "clocks": learned["clocks"],
        "e2e": learned["e2e"],
        "gpu_launches": LEARNED_STEP_LAUNCHES * args.steps,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def _bench_rank(rank, world, args):
    import os
    os.environ.setdefault("NCCL_DEBUG", "INFO")   # NCCL's init log shows the ranks and transports
    run_headline(args, rank, world, rank)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--chains", type=int, default=4096, help="chains per GPU of the plain arm")
    ap.add_argument("--learned-chains", type=int, default=1024, help="chains per GPU of the learned arm")
    ap.add_argument("--cpu-cores", type=int, default=0, help="cores for the CPU baseline (0 = all)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64",
                    help="12x12 workload: FP64 slice products, or 3xTF32 on the tensor cores")
    ap.add_argument("--workload", choices=["6x6", "12x12", "ragged"], default="6x6",
                    help="6x6: the headline line; 12x12: the beta=10 point (512 chains, device time only); "
                         "ragged: 216 points x 32 chains in one launch per kernel class")
    args = ap.parse_args()
    if args.workload == "12x12":
        run_12x12(args)
        return
    if args.workload == "ragged":
        run_ragged(args)
        return
    env_world = os.environ.get("WORLD_SIZE")
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, rank, int(env_world or 1))
        return
    if env_world is None and args.gpus > 1:
        # no launcher: one process per GPU, spawned here (chains sharded by rank)
        from bafqmc_b200.multigpu import launch_ranks
        launch_ranks(_bench_rank, args.gpus, args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(env_world or 1)
    local = int(os.environ.get("LOCAL_RANK", "0"))
    run_headline(args, rank, world, local)


if __name__ == "__main__":
    main()
