"""Generate the golden vectors under tests/golden/ from the reference's own tests.

Run once in a checkout that has the reference tree available:

    python tests/golden/make_golden.py /path/to/BAFQMC

It imports the pure-NumPy halves of the reference's physics tests and records
their outputs, so the committed fixtures are exactly what those tests compare
the Fortran solver against:

* ``tests/physics/test_fixed_field_solver.py``: ``prescribed_fields`` and
  ``direct_fixed_field_reference`` (dense G = (I - B_tau...B_1 B_L...B_tau+1)^-1
  for 3x3, L=6, beta=0.6, mu=-5, U1=0.7, U2=-0.1) -> ``fixed_field.json``
* ``tests/physics/test_gaussian_solvers.py``: ``gaussian_observables`` (closed
  Bogoliubov forms at U1=U2=0, 3x3, beta=1, mu=-5) -> ``gaussian.json``
* ``benchmarks/paper/data/number_conserving/ed/*.json`` and
  ``benchmarks/paper/data/pairing/ed/triangle_pairing_delta_3x3_D0_mum5_b4.json``:
  stored ED chain averages for 3x3 points -> ``ed_3x3.json`` (observables only)
* ``benchmarks/paper/data/index.json`` and ``benchmarks/paper/data/*/inputs/*/
  paramC_sets.txt``: for each paper case (number-conserving and pairing 3x3
  points), the run parameters and, per observable (density_total,
  energy_density, S_SF_K, S_DW_K), the ED value and the reference solver's
  own DQMC mean and standard error -> ``paper_3x3.json``
"""

from __future__ import annotations

import importlib.util
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _load(path: Path, name: str):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _jsonable(v):
    if isinstance(v, np.ndarray):
        return v.tolist()
    if isinstance(v, (np.floating, float)):
        return float(v)
    return v


def main(ref_root: str) -> None:
    root = Path(ref_root)
    ff = _load(root / "tests/physics/test_fixed_field_solver.py", "ref_fixed_field")
    fields = ff.prescribed_fields()
    ref = ff.direct_fixed_field_reference(fields)
    fixed = {
        "source": "tests/physics/test_fixed_field_solver.py:40-119",
        "params": {"Lx": ff.LX, "Ly": ff.LY, "Ltrot": ff.NSLICE, "beta": ff.BETA, "mu": ff.MU,
                   "U1": ff.U1, "U2": ff.U2, "Nbin": ff.NBIN, "tolerance": ff.TOLERANCE,
                   "nwrap": [1, 2, ff.NSLICE]},
        "fields_t_site_aux": fields.tolist(),
        "expected": {k: _jsonable(v) for k, v in ref.items()},
    }
    (HERE / "fixed_field.json").write_text(json.dumps(fixed, indent=1) + "\n")

    gs = _load(root / "tests/physics/test_gaussian_solvers.py", "ref_gaussian")
    gauss = {
        "source": "tests/physics/test_gaussian_solvers.py:44-77",
        "params": {"Lx": 3, "Ly": 3, "beta": gs.BETA, "mu": gs.MU, "abs_tol": gs.ABS_TOL,
                   "rel_tol": gs.REL_TOL, "Nbin": gs.NBIN, "nwrap": [10, 2], "Ltrot": 100},
        "expected": {"0.0": gs.gaussian_observables(0.0), "0.2": gs.gaussian_observables(0.2)},
    }
    (HERE / "gaussian.json").write_text(json.dumps(gauss, indent=1) + "\n")

    ed = {}
    for path in sorted((root / "benchmarks/paper/data/number_conserving/ed").glob("*.json")):
        d = json.loads(path.read_text())
        ed[path.stem] = {"parameters": d["parameters"], "observables": d["observables"]}
    p = root / "benchmarks/paper/data/pairing/ed/triangle_pairing_delta_3x3_D0_mum5_b4.json"
    d = json.loads(p.read_text())
    ed[p.stem] = {k: d[k] for k in ("parameters", "observables") if k in d}
    (HERE / "ed_3x3.json").write_text(json.dumps(ed, indent=1) + "\n")

    data = root / "benchmarks/paper/data"
    index = json.loads((data / "index.json").read_text())
    cases = {}
    for c in index["cases"]:
        lines = (data / c["model"] / "inputs" / c["id"] / "paramC_sets.txt").read_text().splitlines()
        cases[c["id"]] = {
            "model": c["model"],
            "paramC_sets": [ln.split() for ln in lines[:7]],
            "samples": c["samples"],
            "observables": {k: {f: v[f] for f in ("ed", "dqmc", "stderr")} for k, v in c["observables"].items()},
        }
    (HERE / "paper_3x3.json").write_text(json.dumps({"source": "benchmarks/paper/data/index.json", "cases": cases},
                                                    indent=1) + "\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
