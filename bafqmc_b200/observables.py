"""Observable slots of a chain's bin record and the reference's per-bin files.

Slot order is the accumulator layout of the device estimators; names are the
files that m_write_obs_equal appends to (fourier_trans.f90:250-348 for the
number-conserving program, src/pairing/src/fourier_trans.f90:276-405 for the
pairing program).
"""
from __future__ import annotations

import numpy as np

OBS_SCALARS = 32
REAL_SLOTS = {
    "density_up": 0, "density_do": 1, "density_total": 2, "kinetic": 3, "doubleOcc": 4,
    "squareOcc": 5, "num_up": 6, "num_do": 7, "numsquare_up": 8, "numsquare_do": 9,
    "onsite_n2_up": 10, "onsite_n2_do": 11, "interaction_energy_density": 12, "energy_density": 13,
}
COMPLEX_SLOTS = {"sf_K": 14, "psf_Gamma": 16, "dw_K": 18}
# sum over r of den_corr(r)/Lq; the k=0 Fourier component divides once more by Lq
DEN_SLOTS = {"den_upup_sub11": 20, "den_dodo_sub11": 22, "den_updo": 24}
# written by the pairing program only (src/pairing/src/obser_equal.f90:10-15)
PAIR_SLOTS = {"density": 26, "local_numsquare": 27, "pair_equal": 28, "pairing_energy_density": 29,
              "chemical_energy_density": 30, "grand_energy_density": 31}
SITE_SLOT = 32

# file order of m_write_obs_equal
FILE_ORDER = ("density_up", "density_do", "density_total", "density_site_total", "kinetic", "doubleOcc",
              "squareOcc", "num_up", "num_do", "numsquare_up", "numsquare_do", "onsite_n2_up", "onsite_n2_do",
              "interaction_energy_density", "energy_density", "sf_K", "psf_Gamma", "dw_K",
              "den_upup_sub11", "den_dodo_sub11", "den_updo")
FILE_ORDER_PAIRING = ("density_up", "density_do", "density", "density_total", "density_site_total", "num_up",
                      "num_do", "kinetic", "doubleOcc", "squareOcc", "local_numsquare", "numsquare_up",
                      "numsquare_do", "onsite_n2_up", "onsite_n2_do", "pair_equal", "interaction_energy_density",
                      "pairing_energy_density", "chemical_energy_density", "grand_energy_density",
                      "energy_density", "sf_K", "dw_K", "psf_Gamma", "den_upup_sub11", "den_dodo_sub11",
                      "den_updo")


def decode(row: np.ndarray, lq: int, pairing: bool = False) -> dict:
    """One chain's (or one point's chain-averaged) bin record -> named values."""
    out = {k: float(row[i]) for k, i in REAL_SLOTS.items()}
    if pairing:
        out.update({k: float(row[i]) for k, i in PAIR_SLOTS.items()})
    for k, i in COMPLEX_SLOTS.items():
        out[k] = complex(row[i], row[i + 1])
    for k, i in DEN_SLOTS.items():
        out[k] = complex(row[i], row[i + 1]) / float(lq)
    out["density_site_total"] = np.array(row[SITE_SLOT:SITE_SLOT + lq], dtype=np.float64)
    return out
