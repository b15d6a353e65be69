"""Parameter sets of the measured workloads.

ragged_grid: the ragged batch across both solvers -- Lx = Ly in {3, 4, 6},
beta in {2, 4, 8} at dtau = 0.05, U1 = 1, U2 in {0, -0.5}, mu in {-6, -5, -4},
number-conserving (shiftLoc 1.5) and Nambu at Delta in {0.25, 0.5, 1.0}
(shiftLoc 1.0); Nwrap = 10, N(0,1) initial fields.  3 x 3 x 2 x 3 = 54
(L, beta, U2, mu) combinations times 4 solver settings = 216 points.
"""
from __future__ import annotations

import itertools

from .params import SolverParams


def ragged_grid() -> list[SolverParams]:
    pts = []
    for lx, beta, u2, mu, delta in itertools.product((3, 4, 6), (2.0, 4.0, 8.0), (0.0, -0.5), (-6.0, -5.0, -4.0),
                                                     (None, 0.25, 0.5, 1.0)):
        L = int(round(beta / 0.05))
        kw = dict(U1=1.0, U2=u2, mu=mu, Nlx=lx, Nly=lx, Ltrot=L, Beta=beta, NlxTherm=lx, NlyTherm=lx, LtrotTherm=L,
                  Nwrap=10, Nbin=1, Nsweep=1, iniType=2, iniAmpl=1.0)
        if delta is None:
            pts.append(SolverParams(**kw, shiftLoc=1.5))
        else:
            pts.append(SolverParams(**kw, shiftLoc=1.0, delta=delta, sector=1))
    return pts
