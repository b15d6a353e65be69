"""Drop-in for `mpirun -np N build/bosonDQMC.out` in a run directory (or,
with --pairing, for the Nambu pairing program of src/pairing).

    python -m bafqmc_b200 --np N [--device D] [--no-pole] [--pairing] [RUN_DIR]

Reads paramC_sets.txt, confin.txt and seeds.txt from RUN_DIR (default: the
current directory) and writes the per-bin files, info.txt and confout.txt
there, running the N chains (the reference's N MPI ranks) on one GPU.
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m bafqmc_b200")
    ap.add_argument("run_dir", nargs="?", default=".")
    ap.add_argument("--np", type=int, default=1, help="number of chains (MPI ranks of the reference)")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--no-pole", action="store_true", help="skip the per-bin pole diagnostics files")
    ap.add_argument("--pairing", action="store_true",
                    help="the Nambu pairing program: RDelta on line 1 of paramC_sets.txt, pairing file set")
    a = ap.parse_args(argv)
    from .params import ParamError
    from .solver import run_directory
    try:
        run_directory(Path(a.run_dir), nchains=a.np, device=a.device, pole=not a.no_pole, pairing=a.pairing)
    except ParamError as e:   # the reference `stop`s with a message
        print(str(e))
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
