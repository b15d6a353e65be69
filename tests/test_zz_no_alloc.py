"""GPU test of bafqmc_sweep_noalloc, the entry point that allocates no device memory.

It serves callers that cannot call cudaMalloc while they run (another
runtime's caching allocator owns the device, or all device memory is sized
before a campaign): they pass their own device buffers, and the library keeps
its scratch in a fixed device array.  The test calls it through the C ABI twice
in a row -- the second call continuing from the first call's fields and seeds,
so the array holds the first call's contents when the second starts -- and
checks each call against the handle-based entry points (bafqmc_set_state +
bafqmc_pre + bafqmc_sweep) on the same inputs: bins within the 1e-10 tolerance
of the other parity tests, fields and seeds bit-exact.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-10
ATOL = 1e-12


def _setup():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from bafqmc_b200 import _lib, build
    lib = _lib.load(build.build())
    return torch, lib


def _point(**kw):
    from bafqmc_b200.params import SolverParams
    base = dict(U1=1.0, U2=-0.5, mu=-5.0, Nlx=3, Nly=3, Ltrot=20, Beta=2.0, NlxTherm=3, NlyTherm=3, LtrotTherm=20,
                Nwrap=5, Nbin=1, Nsweep=2, shiftLoc=1.5, iniType=2, iniAmpl=1.0)
    base.update(kw)
    return SolverParams(**base)


def _handle_path(p, seeds, phis, nsweep):
    from bafqmc_b200.solver import Ensemble
    with Ensemble([p], np.zeros(len(seeds), dtype=np.int32)) as ens:
        ens.set_state(seeds, phis)
        ens.pre()
        ens.sweep(nsweep)
        obs = ens.chain_obs_raw()
        s, ph = ens.get_state()
    from bafqmc_b200 import _lib
    return obs[:, : _lib.OBS_SCALARS + p.Lq], s, ph


def test_noalloc_matches_handle_path_on_two_calls():
    torch, lib = _setup()
    from bafqmc_b200 import _lib
    from bafqmc_b200.solver import Ensemble, point_struct
    p = _point()
    nchains, nsweep, stride = 6, 2, _lib.OBS_SCALARS + p.Lq
    with Ensemble([p], np.zeros(nchains, dtype=np.int32)) as ens:
        ens.fields_from_seeds(4099 + 31 * np.arange(nchains))
        seeds, phis = ens.get_state()
    pt = point_struct(p)
    dev_seeds = torch.tensor(seeds, dtype=torch.int32, device="cuda")
    dev_phi = torch.tensor(np.concatenate([f.ravel() for f in phis]), dtype=torch.float64, device="cuda")
    dev_obs = torch.zeros(nchains * stride, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        in_seeds = dev_seeds.cpu().numpy().copy()
        in_phis = dev_phi.cpu().numpy().reshape(nchains, p.Ltrot, p.Lq, 2).copy()
        dev_obs.fill_(float("nan"))
        rc = lib.bafqmc_sweep_noalloc(C.byref(pt), nchains, dev_seeds.data_ptr(), dev_phi.data_ptr(), nsweep,
                                      dev_obs.data_ptr(), stream)
        if rc != 0:
            raise AssertionError(lib.bafqmc_last_error().decode())
        torch.cuda.synchronize()
        got_obs = dev_obs.cpu().numpy().reshape(nchains, stride)
        ref_obs, ref_seeds, ref_phis = _handle_path(p, in_seeds, list(in_phis), nsweep)
        np.testing.assert_allclose(got_obs, ref_obs, rtol=RTOL, atol=ATOL, err_msg=f"call {call} bins")
        np.testing.assert_array_equal(dev_seeds.cpu().numpy(), ref_seeds, err_msg=f"call {call} seeds")
        np.testing.assert_array_equal(dev_phi.cpu().numpy().reshape(nchains, p.Ltrot, p.Lq, 2),
                                      np.stack(ref_phis), err_msg=f"call {call} fields")
        assert not np.array_equal(in_seeds, ref_seeds)


def test_noalloc_rejects_sizes_beyond_the_array():
    torch, lib = _setup()
    from bafqmc_b200.solver import point_struct
    p = _point(Nlx=6, Nly=6, Ltrot=160, Beta=8.0, LtrotTherm=160, NlxTherm=6, NlyTherm=6, Nwrap=10)
    n = 4096
    seeds = torch.zeros(n, dtype=torch.int32, device="cuda")
    phi = torch.zeros(1, dtype=torch.float64, device="cuda")
    obs = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = lib.bafqmc_sweep_noalloc(C.byref(point_struct(p)), n, seeds.data_ptr(), phi.data_ptr(), 1, obs.data_ptr(),
                                  torch.cuda.current_stream().cuda_stream)
    assert rc == -1
    assert b"scratch" in lib.bafqmc_last_error()


def test_noalloc_rejects_non_finite_fields():
    """A NaN field is refused as bafqmc_set_state refuses it, naming the chain."""
    torch, lib = _setup()
    from bafqmc_b200 import _lib
    from bafqmc_b200.solver import point_struct
    p = _point()
    nchains, stride = 3, _lib.OBS_SCALARS + p.Lq
    seeds = torch.tensor([11, 12, 13], dtype=torch.int32, device="cuda")
    phi = torch.zeros(nchains * p.Ltrot * p.Lq * 2, dtype=torch.float64, device="cuda")
    phi[p.Ltrot * p.Lq * 2 + 5] = float("nan")   # chain 1
    obs = torch.zeros(nchains * stride, dtype=torch.float64, device="cuda")
    rc = lib.bafqmc_sweep_noalloc(C.byref(point_struct(p)), nchains, seeds.data_ptr(), phi.data_ptr(), 1,
                                  obs.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == -1
    assert b"chain 1" in lib.bafqmc_last_error()
