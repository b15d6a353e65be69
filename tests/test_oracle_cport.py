"""The C++ restatement of the number-conserving sweep (oracle/csweep.cpp, the
timed CPU baseline) against oracle.py: from the same seeds and fields, seeds
and fields after every sweep bit-exact (same decisions, same draws), G and the
estimators within 1e-10 relative."""
import numpy as np
import pytest

from oracle import cport
from oracle import oracle as O

pytestmark = pytest.mark.skipif(not cport.LIB.exists(), reason="oracle/libcsweep.so not built (make -C oracle)")


def params(**kw):
    base = dict(U1=1.0, U2=-0.5, mu=-5.0, Nlx=3, Nly=3, Ltrot=20, Beta=1.0, NlxTherm=3, NlyTherm=3, LtrotTherm=20,
                Nwrap=5, Nbin=1, Nsweep=1, shiftLoc=1.5, iniType=2, iniAmpl=1.0)
    base.update(kw)
    for a, b in (("Nlx", "NlxTherm"), ("Nly", "NlyTherm"), ("Ltrot", "LtrotTherm")):
        if a in kw:
            base[b] = kw[a]
    return O.Params(**base)


@pytest.mark.parametrize("kw", [dict(), dict(Nlx=4, Nly=3), dict(U2=0.0, Ltrot=40, Beta=4.0, Nwrap=10)])
def test_cport_matches_oracle(kw):
    p = params(**kw)
    seeds0 = [101, 202]
    _, _, chains = O.init_chains(p, seeds=seeds0)
    seeds = np.array([c.seed for c in chains], dtype=np.int32)
    phi = np.ascontiguousarray(np.stack([c.phi for c in chains]))
    for c in chains:
        c.pre()
    for sweep in range(2):
        out = cport.run(p, seeds, phi, 1, nthreads=2, want_green=True)   # pre from the updated state, one sweep
        for c in chains:
            c.sweep_bin()
        for k, c in enumerate(chains):
            assert int(seeds[k]) == c.seed, f"sweep {sweep} chain {k} seed"
            np.testing.assert_array_equal(phi[k], c.phi, err_msg=f"sweep {sweep} chain {k} fields")
            g = c.prop.Gr
            assert np.max(np.abs(out["G"][k] - g)) <= 1e-10 * np.max(np.abs(g))
            d = c.obs.as_dict(c.latt)
            ref = [d["density_total"], d["energy_density"], d["kinetic"], d["doubleOcc"], d["numsquare_up"],
                   d["sf_K"].real, d["sf_K"].imag, d["dw_K"].real, d["dw_K"].imag, d["psf_Gamma"].real,
                   d["psf_Gamma"].imag]
            np.testing.assert_allclose(out["obs"][k, :11], ref, rtol=1e-10, atol=1e-13)
