"""Exact diagonalisation of the two-species boson Hubbard model on small
triangular clusters, for cross-checks of the sweep's chain averages at points
the reference's stored ED results do not cover.  Test infrastructure, like
oracle.py.

Model (the reference's ED convention, src/number_conserving/benchmarks/ed/
EDtriangle_symm_NEblock.py:136-172 and EDtriangle_quspin_3x3.py:460-505):
  H = t sum_{<i,j> directed} (b_i^+ b_j + c_i^+ c_j)
      + (U1 + U2) sum_i (n_b,i^2 + n_c,i^2) + 2 (U2 - U1) sum_i n_b,i n_c,i
in the grand-canonical ensemble exp(-beta (H - mu N)), with the six directed
neighbours (+-1, 0), (0, +-1), (-1, +1), (+1, -1) under periodic boundaries.
Observables (per site or per site squared as the per-bin files hold them):
density_total = <N>/Lq; energy_density = (<K> + <V>)/Lq;
S_SF(K) = (1/Lq^2) sum_ij e^{i K (r_i - r_j)} <b_i^+ b_j + c_i^+ c_j>;
S_DW(K) = (1/Lq^2) sum_ij e^{i K (r_i - r_j)} <n_i n_j>, n = n_b + n_c;
with the phase 2 pi (kx dx / Lx + ky dy / Ly), (kx, ky) = (2 Lx / 3, Ly / 3).

The Fock space is truncated at n_max_total bosons of both species together;
each (N_b, N_c) block is diagonalised densely.
"""
from __future__ import annotations

import itertools
import math

import numpy as np

DIRECTIONS = ((1, 0), (0, 1), (-1, 1), (-1, 0), (0, -1), (1, -1))


def _configs(nsite: int, n: int) -> list[tuple[int, ...]]:
    """Occupations of nsite sites with n bosons in total."""
    out = []
    for cut in itertools.combinations(range(n + nsite - 1), nsite - 1):
        prev, occ = -1, []
        for c in cut:
            occ.append(c - prev - 1)
            prev = c
        occ.append(n + nsite - 1 - prev - 1)
        out.append(tuple(occ))
    return out


def _one_body(configs, index, pairs_coeff) -> np.ndarray:
    """sum coeff * a_i^+ a_j in the fixed-number space of one species."""
    dim = len(configs)
    m = np.zeros((dim, dim), dtype=complex)
    for col, occ in enumerate(configs):
        for (i, j), coeff in pairs_coeff:
            if occ[j] == 0:
                continue
            if i == j:
                m[col, col] += coeff * occ[j]
                continue
            new = list(occ)
            f = math.sqrt((new[i] + 1) * new[j])
            new[i] += 1
            new[j] -= 1
            m[index[tuple(new)], col] += coeff * f
    return m


def observables(lx: int, ly: int, U1: float, U2: float, mu: float, beta: float, t: float = 1.0,
                n_max_total: int = 4) -> dict[str, float]:
    lq = lx * ly

    def site(x, y):
        return (y % ly) * lx + (x % lx)

    hop = [((site(x, y), site(x + dx, y + dy)), t) for y in range(ly) for x in range(lx) for dx, dy in DIRECTIONS]
    hasK = lx % 3 == 0 and ly % 3 == 0
    phase = np.zeros((lq, lq), dtype=complex)
    if hasK:
        for i in range(lq):
            for j in range(lq):
                dx, dy = (i % lx - j % lx) % lx, (i // lx - j // lx) % ly
                a = 2.0 * math.pi * ((2 * lx // 3) * dx / lx + (ly // 3) * dy / ly)
                phase[i, j] = complex(math.cos(a), math.sin(a))
    sf_pairs = [((i, j), phase[i, j] / lq ** 2) for i in range(lq) for j in range(lq)]
    spaces = {}
    for n in range(n_max_total + 1):
        cfg = _configs(lq, n)
        idx = {c: k for k, c in enumerate(cfg)}
        occ = np.array(cfg, dtype=float).reshape(len(cfg), lq)
        spaces[n] = (occ, _one_body(cfg, idx, hop), _one_body(cfg, idx, sf_pairs))
    Z = 0.0
    acc = {"N": 0.0, "K": 0.0, "V": 0.0, "SF": 0.0, "DW": 0.0}
    logs = []
    blocks = []
    for nb in range(n_max_total + 1):
        for nc in range(n_max_total + 1 - nb):
            ob, Tb, Sb = spaces[nb]
            oc, Tc, Sc = spaces[nc]
            db, dc = len(ob), len(oc)
            Ib, Ic = np.eye(db), np.eye(dc)
            K = (np.kron(Tb, Ic) + np.kron(Ib, Tc)).real
            nbv = np.repeat(ob, dc, axis=0)         # [state][site] occupations of b
            ncv = np.tile(oc, (db, 1))
            vdiag = (U1 + U2) * np.sum(nbv ** 2 + ncv ** 2, axis=1) + 2.0 * (U2 - U1) * np.sum(nbv * ncv, axis=1)
            H = K + np.diag(vdiag)
            E, V = np.linalg.eigh(H)
            blocks.append((nb + nc, E, V, K, vdiag, np.kron(Sb, Ic) + np.kron(Ib, Sc), nbv + ncv))
            logs.append(np.max(-beta * (E - mu * (nb + nc))))
    shift = max(logs)
    for ntot, E, V, K, vdiag, S, ntv in blocks:
        w = np.exp(-beta * (E - mu * ntot) - shift)
        Z += float(np.sum(w))
        def expect(M):   # sum_n w_n <n|M|n>
            return float(np.real(np.sum(w * np.sum(V.conj() * (M @ V), axis=0))))
        p = np.abs(V) ** 2
        acc["N"] += float(np.sum(w)) * ntot
        acc["K"] += expect(K)
        acc["V"] += float(np.sum(w * (p.T @ vdiag)))
        acc["SF"] += expect(S)
        dw = np.real(np.sum((ntv @ phase) * ntv, axis=1)) / lq ** 2
        acc["DW"] += float(np.sum(w * (p.T @ dw)))
    return {"density_total": acc["N"] / Z / lq, "energy_density": (acc["K"] + acc["V"]) / Z / lq,
            "S_SF_K": acc["SF"] / Z, "S_DW_K": acc["DW"] / Z}
