"""oracle/ed.py (exact diagonalisation, up to 4 bosons in all) against the
reference's stored ED results (tests/golden/ed_3x3.json, which keep up to 8-10
bosons): agreement to 1e-4 relative, the truncation of the smaller space, 100x
below the statistical errors of the QMC comparisons it serves."""
import json

import pytest

from oracle import ed


@pytest.mark.parametrize("key", ["triangle_3x3_U2_-0.5_mu-7_b1", "triangle_3x3_U1_0.5_mu-3.5_b4"])
def test_own_ed_matches_stored_ed(root, key):
    g = json.loads((root / "tests/golden/ed_3x3.json").read_text())[key]
    pr, obs = g["parameters"], g["observables"]
    r = ed.observables(3, 3, pr["U1"], pr["U2"], pr["mu"], pr["beta"], n_max_total=4)
    for k, v in r.items():
        ref = obs[k]["value"] if isinstance(obs[k], dict) else obs[k]
        assert abs(v / ref - 1.0) < 1e-4, (k, v, ref)
