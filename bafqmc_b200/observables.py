"""Observable slots of a chain's bin record and the reference's per-bin files.

Slot order is the accumulator layout of the device estimators; names are the
files that m_write_obs_equal appends to (fourier_trans.f90:250-348).
"""
from __future__ import annotations

import numpy as np

OBS_SCALARS = 26
REAL_SLOTS = {
    "density_up": 0, "density_do": 1, "density_total": 2, "kinetic": 3, "doubleOcc": 4,
    "squareOcc": 5, "num_up": 6, "num_do": 7, "numsquare_up": 8, "numsquare_do": 9,
    "onsite_n2_up": 10, "onsite_n2_do": 11, "interaction_energy_density": 12, "energy_density": 13,
}
COMPLEX_SLOTS = {"sf_K": 14, "psf_Gamma": 16, "dw_K": 18}
# sum over r of den_corr(r)/Lq; the k=0 Fourier component divides once more by Lq
DEN_SLOTS = {"den_upup_sub11": 20, "den_dodo_sub11": 22, "den_updo": 24}
SITE_SLOT = 26

# file order of m_write_obs_equal
FILE_ORDER = ("density_up", "density_do", "density_total", "density_site_total", "kinetic", "doubleOcc",
              "squareOcc", "num_up", "num_do", "numsquare_up", "numsquare_do", "onsite_n2_up", "onsite_n2_do",
              "interaction_energy_density", "energy_density", "sf_K", "psf_Gamma", "dw_K",
              "den_upup_sub11", "den_dodo_sub11", "den_updo")


def decode(row: np.ndarray, lq: int) -> dict:
    """One chain's (or one point's chain-averaged) bin record -> named values."""
    out = {k: float(row[i]) for k, i in REAL_SLOTS.items()}
    for k, i in COMPLEX_SLOTS.items():
        out[k] = complex(row[i], row[i + 1])
    for k, i in DEN_SLOTS.items():
        out[k] = complex(row[i], row[i + 1]) / float(lq)
    out["density_site_total"] = np.array(row[SITE_SLOT:SITE_SLOT + lq], dtype=np.float64)
    return out
