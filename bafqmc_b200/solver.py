"""Host side of the B200 sweep: a batch of chains behind the C ABI, and the
reference's run-directory contract on top of it.

`Ensemble` holds one handle of libbafqmc_b200.so (chains of one or several
parameter points, number-conserving and Nambu mixed).  `run_directory`
reproduces `mpirun -np N bosonDQMC.out` (src/number_conserving/src/main.f90:22-85,
or the pairing program src/pairing/src/main.f90:19-83 with pairing=True) for
N chains on one GPU: it reads paramC_sets.txt / confin.txt / seeds.txt and
appends the same per-bin files, info.txt and confout.txt.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import time
from pathlib import Path

import numpy as np

from . import _lib
from .observables import FILE_ORDER, FILE_ORDER_PAIRING, OBS_SCALARS, decode
from .params import NAUX, ParamError, SolverParams, conf_transfer


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def point_struct(p: SolverParams) -> _lib.Point:
    return _lib.Point(
        sector=p.sector, Lx=p.Nlx, Ly=p.Nly, Ltrot=p.Ltrot, beta=p.Beta, U1=p.U1, U2=p.U2, mu=p.mu,
        delta=p.delta, Nwrap=p.Nwrap, shiftLoc=p.shiftLoc, iniType=p.iniType, iniAmpl=p.iniAmpl,
        iniBias1=p.iniBias[0], iniBias2=p.iniBias[1], LxTherm=p.NlxTherm, LyTherm=p.NlyTherm,
        LtrotTherm=p.LtrotTherm)


class Ensemble:
    """Independent Markov chains (the reference's MPI ranks) on one GPU."""

    def __init__(self, points: list[SolverParams], chain_point, device: int = 0, classes=None):
        """classes: optional kernel class per point (from autotune), -1 for the default."""
        self.lib = _lib.load()
        self.points = list(points)
        self.chain_point = np.ascontiguousarray(chain_point, dtype=np.int32)
        self.nchains = int(self.chain_point.size)
        arr = (_lib.Point * len(points))(*[point_struct(p) for p in points])
        h = C.c_void_p()
        if classes is None:
            _lib.check(self.lib.bafqmc_create(arr, len(points), _iptr(self.chain_point), self.nchains, device,
                                              C.byref(h)))
        else:
            cls = np.ascontiguousarray(classes, dtype=np.int32)
            _lib.check(self.lib.bafqmc_create_tuned(arr, len(points), _iptr(self.chain_point), self.nchains, device,
                                                    _iptr(cls), C.byref(h)))
        self.h = h
        self.stride = self.lib.bafqmc_obs_stride(h)
        self.dims = []
        for i in range(len(points)):
            nd, lq, lt, nst = C.c_int(), C.c_int(), C.c_int(), C.c_int()
            _lib.check(self.lib.bafqmc_point_dim(h, i, C.byref(nd), C.byref(lq), C.byref(lt), C.byref(nst)))
            self.dims.append((nd.value, lq.value, lt.value, nst.value))
        # fields: [Ltrot][Lx*Ly][2] per chain in both sectors
        self.phi_sizes = [self.dims[p][2] * self.dims[p][1] * NAUX for p in self.chain_point]
        self.phi_offsets = np.concatenate([[0], np.cumsum(self.phi_sizes)]).astype(np.int64)

    def close(self):
        if getattr(self, "h", None):
            self.lib.bafqmc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- state
    def fields_from_seeds(self, seeds):
        s = np.ascontiguousarray(seeds, dtype=np.int32)
        assert s.size == self.nchains
        _lib.check(self.lib.bafqmc_fields_from_seeds(self.h, _iptr(s)))

    def set_state(self, seeds, phis):
        s = np.ascontiguousarray(seeds, dtype=np.int32)
        flat = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.float64).ravel() for p in phis]))
        assert flat.size == self.phi_offsets[-1]
        _lib.check(self.lib.bafqmc_set_state(self.h, _iptr(s), _dptr(flat)))

    def set_state_flat(self, seeds: np.ndarray, phi_flat: np.ndarray):
        """set_state from caller-owned contiguous buffers (int32 seeds, float64
        fields of all chains back to back), e.g. views of pinned host memory."""
        assert seeds.dtype == np.int32 and seeds.flags.c_contiguous and seeds.size == self.nchains
        assert phi_flat.dtype == np.float64 and phi_flat.flags.c_contiguous and phi_flat.size == self.phi_offsets[-1]
        _lib.check(self.lib.bafqmc_set_state(self.h, _iptr(seeds), _dptr(phi_flat)))

    def get_state_flat(self, seeds: np.ndarray, phi_flat: np.ndarray):
        """get_state into caller-owned contiguous buffers (see set_state_flat)."""
        assert seeds.dtype == np.int32 and seeds.flags.c_contiguous and seeds.size == self.nchains
        assert phi_flat.dtype == np.float64 and phi_flat.flags.c_contiguous and phi_flat.size == self.phi_offsets[-1]
        _lib.check(self.lib.bafqmc_get_state(self.h, _iptr(seeds), _dptr(phi_flat)))

    def get_state(self):
        s = np.zeros(self.nchains, dtype=np.int32)
        flat = np.zeros(int(self.phi_offsets[-1]), dtype=np.float64)
        _lib.check(self.lib.bafqmc_get_state(self.h, _iptr(s), _dptr(flat)))
        phis = []
        for c in range(self.nchains):
            _, lq, lt, _ = self.dims[self.chain_point[c]]
            phis.append(flat[self.phi_offsets[c]:self.phi_offsets[c + 1]].reshape(lt, lq, NAUX))
        return s, phis

    # ---- the sweep path
    def warmup_prior(self, nwarm: int):
        _lib.check(self.lib.bafqmc_warmup_prior(self.h, int(nwarm)))

    def pre(self):
        _lib.check(self.lib.bafqmc_pre(self.h))

    def sweep(self, nsweep: int = 1):
        _lib.check(self.lib.bafqmc_sweep(self.h, int(nsweep)))

    def synchronize(self):
        _lib.check(self.lib.bafqmc_synchronize(self.h))

    @property
    def stream(self) -> int:
        return int(self.lib.bafqmc_stream(self.h) or 0)

    # ---- results
    def chain_obs_raw(self) -> np.ndarray:
        out = np.zeros((self.nchains, self.stride))
        _lib.check(self.lib.bafqmc_bin_chain_obs(self.h, _dptr(out)))
        return out

    def point_obs_raw(self) -> np.ndarray:
        out = np.zeros((len(self.points), self.stride))
        _lib.check(self.lib.bafqmc_bin_point_obs(self.h, _dptr(out)))
        return out

    def chain_obs(self) -> list[dict]:
        raw = self.chain_obs_raw()
        out = []
        for c in range(self.nchains):
            pt = self.chain_point[c]
            out.append(decode(raw[c], self.dims[pt][1], self.points[pt].sector == 1))
        return out

    def point_obs(self) -> list[dict]:
        raw = self.point_obs_raw()
        return [decode(raw[p], self.dims[p][1], self.points[p].sector == 1) for p in range(len(self.points))]

    def green(self, chain: int) -> np.ndarray:
        """The stored Green's function: Prop%Gr, or the {b, c^dagger} block of a Nambu chain."""
        nd = self.dims[self.chain_point[chain]][0]
        out = np.zeros(2 * nd * nd)
        _lib.check(self.lib.bafqmc_get_green(self.h, int(chain), _dptr(out)))
        return out.view(np.complex128).reshape(nd, nd)

    def log_weight(self) -> np.ndarray:
        out = np.zeros(self.nchains)
        _lib.check(self.lib.bafqmc_log_weight(self.h, _dptr(out)))
        return out

    def set_precision(self, mode: str):
        """"fp64" (default) or "mixed": slice products of chains with 72 < Ndim <= 144
        on the tensor cores in 3xTF32-compensated FP32 (bafqmc_set_precision);
        "wait_test" is the test hook of the products' bounded wait."""
        _lib.check(self.lib.bafqmc_set_precision(self.h, _lib.PRECISION[mode]))

    def set_time_displaced(self, enable: bool = True, probe_nt: int = 0):
        """Run the time-displaced pass (Dyn_sweep_R, dynamics.f90:44-57) in every
        following sweep, between the left and right traversals; probe_nt in
        1..Ltrot keeps the four functions of that slice (bafqmc_set_time_displaced)."""
        _lib.check(self.lib.bafqmc_set_time_displaced(self.h, 1 if enable else 0, int(probe_nt)))

    def time_displaced_stats(self, reset: bool = False) -> np.ndarray:
        """[nchains, 8]: drift max of G(0,tau), G(tau,0), G(tau,tau), their sums,
        passes run, non-finite recomputations (bafqmc_time_displaced_stats)."""
        out = np.zeros((self.nchains, 8), dtype=np.float64)
        _lib.check(self.lib.bafqmc_time_displaced_stats(self.h, _dptr(out), 1 if reset else 0))
        return out

    def time_displaced_probe(self, chain: int):
        """(G(0,0), G(0,tau), G(tau,0), G(tau,tau)) of the chain at the probe slice."""
        n = self.dims[self.chain_point[chain]][0]
        out = np.zeros((4, n, n, 2), dtype=np.float64)
        _lib.check(self.lib.bafqmc_time_displaced_probe(self.h, int(chain), _dptr(out)))
        z = out[..., 0] + 1j * out[..., 1]
        return z[0], z[1], z[2], z[3]

    def global_shift(self, shift) -> np.ndarray:
        """One global shift move per chain (bafqmc_global_shift): every field of
        channel ns shifted by (u - 1/2)|shift[ns]|, accepted by the exact weight
        ratio; returns 0/1 per chain."""
        sh = np.ascontiguousarray(shift, dtype=np.float64)
        assert sh.size == 2
        acc = np.zeros(self.nchains, dtype=np.int32)
        _lib.check(self.lib.bafqmc_global_shift(self.h, _dptr(sh), _iptr(acc)))
        return acc

    def learned_move(self, net, want: bool = True):
        """One learned global move per chain (bafqmc_learned_move) with the
        network `net` (a bafqmc_b200.proposer.Proposer).  Returns (accepted,
        hastings) per chain, or None without synchronising if want is False."""
        if not want:
            _lib.check(self.lib.bafqmc_learned_move(self.h, net.h, None, None))
            return None
        acc = np.zeros(self.nchains, dtype=np.int32)
        hst = np.zeros(self.nchains, dtype=np.float64)
        _lib.check(self.lib.bafqmc_learned_move(self.h, net.h, _iptr(acc), _dptr(hst)))
        return acc, hst

    def stats_reset(self, block_size: int, max_blocks: int = 1024):
        """Start on-device block statistics of the per-bin point averages (bafqmc_stats_reset)."""
        _lib.check(self.lib.bafqmc_stats_reset(self.h, int(block_size), int(max_blocks)))

    def stats_raw(self):
        """(mean, sem) as [npts, stride] arrays over the completed blocks, and the block count."""
        mean = np.zeros((len(self.points), self.stride))
        sem = np.zeros_like(mean)
        nb = np.zeros(1, dtype=np.int32)
        _lib.check(self.lib.bafqmc_stats(self.h, _dptr(mean), _dptr(sem), _iptr(nb)))
        return mean, sem, int(nb[0])

    def stats(self) -> list[dict]:
        """Per point: {observable: (mean, sem)}; complex observables give complex mean and
        complex sem (the SEM of the real and of the imaginary part)."""
        mean, sem, _ = self.stats_raw()
        out = []
        for p in range(len(self.points)):
            pair = self.points[p].sector == 1
            m, e = decode(mean[p], self.dims[p][1], pair), decode(sem[p], self.dims[p][1], pair)
            out.append({k: (m[k], e[k]) for k in m})
        return out

    def quarantined(self) -> list[int]:
        """Chains whose Green's function became non-finite (status bit 0): later
        sweeps skip them and the point averages leave them out."""
        st = self.counters()[:, 6].astype(np.int64)
        return [int(c) for c in np.nonzero(st & 1)[0]]

    POLE_NAMES = ("pole_distance", "pole_x", "green_spectral_radius", "green_smax", "log_weight")

    def pole_diagnostics(self) -> list[dict | None]:
        """PoleDiagnostics (pole_diagnostics.f90:91-123) of every chain's current G,
        computed on the device: the poles z = 1/lambda (the chain's pole_z row)
        and the five scalar files.  None for a Nambu chain."""
        zs = max([self.dims[self.chain_point[c]][0] for c in range(self.nchains)] + [1])
        z = np.zeros((self.nchains, zs, 2))
        sc = np.zeros((self.nchains, _lib.POLE_SCALARS))
        _lib.check(self.lib.bafqmc_pole_diagnostics(self.h, _dptr(z), zs, _dptr(sc)))
        out = []
        for c in range(self.nchains):
            p = self.chain_point[c]
            if self.points[p].sector == 1:
                out.append(None)
                continue
            nd = self.dims[p][0]
            d = {k: float(sc[c, i]) for i, k in enumerate(self.POLE_NAMES)}
            d["pole_z"] = z[c, :nd, 0] + 1j * z[c, :nd, 1]
            out.append(d)
        return out

    def phase_timers(self, enable: bool = True) -> np.ndarray:
        """Enable per-phase cycle counting; returns the [nchains, 4] cycles so far."""
        out = np.zeros((self.nchains, 4))
        _lib.check(self.lib.bafqmc_phase_timers(self.h, 1 if enable else 0, _dptr(out)))
        return out

    def counters(self) -> np.ndarray:
        out = np.zeros((self.nchains, _lib.COUNTERS))
        _lib.check(self.lib.bafqmc_counters(self.h, _dptr(out)))
        return out


def autotune(points: list[SolverParams], trial_chains: int = 0, device: int = 0):
    """bafqmc_autotune: the fastest kernel class per point, and the measured
    milliseconds per chain-sweep of every candidate class ([npts, 7], NaN where
    a class cannot hold the point)."""
    lib = _lib.load()
    arr = (_lib.Point * len(points))(*[point_struct(p) for p in points])
    classes = np.full(len(points), -1, dtype=np.int32)
    table = np.full((len(points), _lib.NUM_CLASSES), np.nan)
    _lib.check(lib.bafqmc_autotune(arr, len(points), device, int(trial_chains), _iptr(classes), _dptr(table)))
    return classes, table


def nambu_green(block: np.ndarray) -> np.ndarray:
    """The pairing program's 4Ns Prop%Gr from the {b, c^dagger} block.

    Sector order b, c, b^dagger, c^dagger (src/pairing/src/lattice.f90:26-35):
    the block sits on {b, c^dagger}, its complex conjugate on {c, b^dagger},
    zeros elsewhere."""
    n2 = block.shape[0]
    ns = n2 // 2
    g = np.zeros((4 * ns, 4 * ns), dtype=np.complex128)
    one = list(range(ns)) + list(range(3 * ns, 4 * ns))
    two = list(range(ns, 2 * ns)) + list(range(2 * ns, 3 * ns))
    g[np.ix_(one, one)] = block
    g[np.ix_(two, two)] = np.conj(block)
    return g


# ---------------------------------------------------------------------------
# output formats of the reference writer
def _scalar(v):
    """A numpy scalar as the Python int/float it holds (numpy 2 reprs carry the type name)."""
    return v.item() if isinstance(v, np.generic) else v


def _lst(*vals) -> str:
    """Fortran list-directed record: blank-separated values, lossless."""
    return " " + "  ".join(repr(float(v)) for v in vals) + "\n"


def _es(v: float, width: int = 24, digits: int = 16, expdigits: int = 2) -> str:
    """Fortran ESw.dEe; a non-finite value is written as gfortran does (NaN, Infinity)."""
    if not math.isfinite(v):
        return ("NaN" if v != v else ("-Infinity" if v < 0 else "Infinity")).rjust(width)
    m, e = f"{v:.{digits}E}".split("E")
    ei = int(e)
    s = f"{m}E{'-' if ei < 0 else '+'}{abs(ei):0{expdigits}d}"
    return s.rjust(width)


def _e(v: float, width: int = 24, digits: int = 16) -> str:
    """Fortran Ew.d: 0.ddd...E+xx (mantissa in [0.1, 1))."""
    if v == 0.0 or not math.isfinite(v):
        s = f"0.{'0' * digits}E+00" if v == 0.0 else str(v)
        return s.rjust(width)
    m, e = f"{abs(v):.{digits - 1}E}".split("E")
    ei = int(e) + 1
    s = f"{'-' if v < 0 else ''}0.{m.replace('.', '')}E{'-' if ei < 0 else '+'}{abs(ei):02d}"
    return s.rjust(width)


def append_bin(run_dir: Path, obs: dict, pairing: bool = False) -> None:
    """m_write_obs_equal (fourier_trans.f90:250-348; src/pairing/src/fourier_trans.f90:276-405)."""
    for name in (FILE_ORDER_PAIRING if pairing else FILE_ORDER):
        v = obs[name]
        with open(run_dir / name, "a") as f:
            if name == "density_site_total" and pairing:   # '(1X,E24.16)' per site
                f.write("".join(" " + _e(x) for x in v) + "\n")
            elif name == "density_site_total":
                f.write("".join(_es(x) + " " for x in v) + "\n")
            elif isinstance(v, complex):
                f.write(_lst(v.real, v.imag))
            else:
                f.write(_lst(v))


def append_pole(run_dir: Path, diags: list[dict]) -> None:
    """PoleDiagnostics_write (pole_diagnostics.f90:126-187): one row per chain."""
    with open(run_dir / "pole_z", "a") as f:
        for d in diags:
            f.write("".join(" " + _es(z.real, expdigits=3) + " " + _es(z.imag, expdigits=3) for z in d["pole_z"]))
            f.write("\n")
    for name in ("pole_distance", "pole_x", "green_spectral_radius", "green_smax", "log_weight"):
        with open(run_dir / name, "a") as f:
            for d in diags:
                f.write(_es(d[name], expdigits=3) + "\n")


def _fortran_float(tok: str, path, pos: int) -> float:
    try:
        return float(tok.replace("D", "E").replace("d", "e"))
    except ValueError:
        raise ValueError(f"{path}: value {pos + 1} ({tok!r}) is not a number") from None


def read_confin(path: Path, p: SolverParams, nchains: int):
    """conf_therm_in's confin.txt (fields.f90:64-103): 0, or per chain a seed and
    LtrotTherm*NlxTherm*NlyTherm*2 field values.  A truncated or corrupt file
    raises ValueError naming the chain and position (the reference would read
    past the end or stop)."""
    toks = Path(path).read_text().split()
    if not toks:
        raise ValueError(f"{path}: empty")
    if int(_fortran_float(toks[0], path, 0)) == 0:
        return None
    per = p.LtrotTherm * p.NlxTherm * p.NlyTherm * NAUX
    need = nchains * (per + 1)
    if len(toks) < need:
        raise ValueError(f"{path}: {len(toks)} values, {need} needed for {nchains} chains of {per} fields")
    out, pos = [], 0
    for c in range(nchains):
        seed = _fortran_float(toks[pos], path, pos)
        if seed != int(seed):
            raise ValueError(f"{path}: seed of chain {c} ({toks[pos]!r}) is not an integer")
        pos += 1
        vals = np.array([_fortran_float(t, path, pos + i) for i, t in enumerate(toks[pos:pos + per])])
        if not np.all(np.isfinite(vals)):
            raise ValueError(f"{path}: non-finite field value in chain {c}")
        pos += per
        out.append((int(seed), conf_transfer(p, vals)))
    return out


def read_confin_npz(path: Path, p: SolverParams, nchains: int):
    """The binary checkpoint confout.npz written by run_directory (seeds
    [nchains] int32, phi [nchains][Ltrot][Lq][2] float64), read back as
    read_confin's (seed, fields) list."""
    with np.load(path) as z:
        seeds, phi = z["seeds"], z["phi"]
    if seeds.shape != (nchains,) or phi.shape != (nchains, p.Ltrot, p.Lq, NAUX):
        raise ValueError(f"{path}: seeds {seeds.shape} and fields {phi.shape} do not match {nchains} chains of "
                         f"({p.Ltrot}, {p.Lq}, {NAUX})")
    if not np.all(np.isfinite(phi)):
        raise ValueError(f"{path}: non-finite field value")
    return [(int(seeds[c]), phi[c]) for c in range(nchains)]


UNSTABLE_DRIFT = 5.5e-5   # the reference's warning threshold (stabilization.f90:320, 358)


def drift_warnings(drift, tau_stats, seen: set, nbin: int, log=print) -> list[str]:
    """The reference's stability warnings (stabilization.f90:320, 358, 387-397): a
    drift of 5.5e-5 or more between the propagated and the recomputed functions.
    The reference prints one line per wrap; here one line per chain and kind, from
    the drift maxima after bin nbin (drift: per chain, of G; tau_stats: the
    time-displaced statistics, or None).  seen holds what was reported already.
    Returns the new lines."""
    out = []
    kinds = [("G", np.asarray(drift))]
    if tau_stats is not None:
        kinds += [(name, np.asarray(tau_stats)[:, k]) for k, name in enumerate(("GR0T", "GRT0", "GRTT"))]
    for name, d in kinds:
        for c in np.nonzero(d >= UNSTABLE_DRIFT)[0]:
            if (name, int(c)) in seen:
                continue
            seen.add((name, int(c)))
            what = "drift" if name == "G" else f"{name} drift"
            out.append(f" WARNING: chain {int(c)}: {what} {d[c]:.3e} >= {UNSTABLE_DRIFT} by bin {nbin} (ortho unstable)")
    for line in out:
        log(line)
    return out


def run_directory(run_dir, nchains: int = 1, device: int = 0, pole: bool = True, log=print,
                  pairing: bool = False) -> dict:
    """The reference program for `mpirun -np nchains` in run_dir, on one GPU.

    pairing=True runs the Nambu program (src/pairing/src/main.f90): RDelta is
    read from line 1 of paramC_sets.txt, the pairing file set is written, and
    there are no pole diagnostics."""
    run_dir = Path(run_dir)
    t0 = time.time()
    p = SolverParams.from_file(run_dir / "paramC_sets.txt", pairing=pairing)
    if p.is_tau and p.block_dim > 72:
        # the time-displaced pass (dynamics.f90) is built for stored dimensions up to 72
        raise ParamError("is_tau = .true. (line 5 of paramC_sets.txt) is supported up to a stored dimension of 72 "
                         f"(this run: {p.block_dim}); set is_tau = .false.")
    info = open(run_dir / "info.txt", "w")
    w = lambda label, v: info.write(f" {label:<47}:{_scalar(v)!r:>26}\n")
    if pairing:   # write_info (src/pairing/src/calc_basic.f90:140-180)
        info.write(" =========================\n DQMC for pairing Bose Hubbard on triangular lattice\n")
        w("Linear lengh Lx", p.Nlx); w("Linear lengh Ly", p.Nly); w("Hopping t", 1.0)
        w("Relative-density U1 (>=0)", p.U1); w("Total-density U2 (<=0)", p.U2); w("pairing Delta", p.delta)
    else:         # write_info (calc_basic.f90:137-175)
        info.write(" =========================\n DQMC for boson Hubbard on triangular lattice\n")
        w("Linear lengh Lx", p.Nlx); w("Linear lengh Ly", p.Nly); w("Hopping t", 1.0)
        w("Hubbard U1 (relative-density, repulsive)", p.U1); w("Hubbard U2 (total-density, attractive)", p.U2)
    w("chemical potential", p.mu); w("Local update auxiliary field magnitude Shift", p.shiftLoc)
    if p.is_warm:
        w("# Warm", p.Nwarm)
        if pairing:
            w("Thermalize auxiliary field magnitude for U1", p.shiftWarm[0])
            w("Thermalize auxiliary field magnitude for U2", p.shiftWarm[1])
        else:
            w("Thermalize U1 relative-field magnitude", p.shiftWarm[0])
            w("Thermalize U2 total-field magnitude", p.shiftWarm[1])
    w("Choosing initial distribution type", p.iniType); w("Magnitude of Gaussian distribution", p.iniAmpl)
    w("Beta", p.Beta); w("Trotter number", p.Ltrot); w("=>Dtau", p.Dtau); w("N_Ortho", p.Nwrap)
    w("# Bins", p.Nbin); w("# Nsweep in one bin", p.Nsweep); w("# Cores", nchains)
    ens = Ensemble([p], np.zeros(nchains, dtype=np.int32), device=device)
    if (run_dir / "confin.npz").exists():   # binary checkpoint, read in place of confin.txt
        confin = read_confin_npz(run_dir / "confin.npz", p, nchains)
    else:
        confin = read_confin(run_dir / "confin.txt", p, nchains)
    if confin is None:
        seeds = [int(r.split()[0]) for r in (run_dir / "seeds.txt").read_text().split("\n") if r.strip()][:nchains]
        if len(seeds) < nchains:
            raise ValueError("seeds.txt has fewer rows than chains")
        ens.fields_from_seeds(seeds)
    else:
        ens.set_state([s for s, _ in confin], [phi for _, phi in confin])
    if p.is_warm:
        ens.warmup_prior(p.Nwarm)
        cnt = ens.counters()
        for ch, name in ((0, "Thermalize U1 Accept Ratio"), (1, "Thermalize U2 Accept Ratio")):
            if abs((p.U1, p.U2)[ch]) > 1e-10:
                w(name, float(cnt[:, 2 + ch].sum() / (nchains * p.Nwarm)))
    else:
        info.write(" Skipping Bosonic warm-up\n")
    ens.pre()
    seen = set()
    istau = False
    tau_record = {}
    for nbc in range(p.Nbin):
        if nbc + 1 > p.Nthermal and p.is_tau and not istau:   # main.f90:49-50
            istau = True
            ens.set_time_displaced(True)
        ens.sweep(p.Nsweep)
        for c in ens.quarantined():
            if c not in seen:   # the reference has no counterpart: it would carry the NaN on
                seen.add(c)
                log(f" WARNING: chain {c} quarantined after bin {nbc + 1}: non-finite Green's function")
        ts = (ens.time_displaced_stats() * (2.0 if pairing else 1.0)) if istau else None
        drift_warnings(ens.counters()[:, 4], ts, seen, nbc + 1, log)
        append_bin(run_dir, ens.point_obs()[0], pairing=pairing)
        if pole and not pairing:
            append_pole(run_dir, ens.pole_diagnostics())
    cnt = ens.counters()
    for ch, name in ((0, "U1"), (1, "U2")):
        if abs((p.U1, p.U2)[ch]) > 1e-10:
            w(f"Accept_{name}_shift", float(cnt[:, ch].sum() / (nchains * p.Nbin)))
            if pairing:   # Local_control_print (src/pairing/src/local_sweep.f90:163-213)
                nprop, nacc = float(cnt[:, 10 + ch].sum()), float(cnt[:, 12 + ch].sum())
                if nprop > 0:
                    w(f"Phase_{name}_mean_abs_arg_proposed", 0.0)
                if nacc > 0:
                    w(f"Phase_{name}_mean_abs_arg_accepted", 0.0)
                if nprop > 0:
                    w(f"Phase_{name}_branch_pi_fraction", 0.0)
                w(f"Phase_{name}_local_proposals", nprop)
    if istau:
        # Dyn_control_print (dynamics.f90:59-82): the sums are divided by chains * Nbin * Nst * Nsweep
        # whatever Nthermal is, and the labels are those the reference prints: its
        # Xmaxm(1..3) hold the drifts of G(0,tau), G(tau,0), G(tau,tau) in that order
        # (stabilization.f90:384-398) while the lines name them GRtt, GRt0, GR0t.
        ts = ens.time_displaced_stats()
        if pairing:   # the reference's 4Ns matrices hold the block and its complex conjugate
            ts[:, :6] *= 2.0
        tau_record = {"tau_passes": int(ts[:, 6].sum()), "tau_drift_max": [float(ts[:, k].max()) for k in range(3)],
                      "tau_nonfinite": int(ts[:, 7].sum())}
        norm = nchains * p.Nbin * p.Nst * p.Nsweep
        for k, label in enumerate(("GRtt", "GRt0", "GR0t")):
            w(f"Max diff {label}", float(ts[:, k].max()))
            w(f"Mean diff {label}", float(ts[:, 3 + k].sum() / norm))
    quarantined = ens.quarantined()
    if quarantined:
        info.write(" non-finite Green's function, chains quarantined: "
                   + " ".join(str(i) for i in quarantined) + "\n")
    w("Max diff Matrix", float(cnt[:, 4].max()))
    w("Mean diff Matrix", float(cnt[:, 5].sum() / (2 * nchains * p.Nbin * p.Nst * p.Nsweep)))
    elapsed = time.time() - t0
    w("Tot CPU time", elapsed)
    info.close()
    record = {   # machine-readable summary of the run (no counterpart in the reference)
        "program": "pairing" if pairing else "number_conserving", "chains": nchains, "bins": p.Nbin,
        "sweeps_per_bin": p.Nsweep, "Ndim": p.Ndim, "Ltrot": p.Ltrot, "wall_s": elapsed,
        "chain_sweeps_per_s": nchains * p.Nbin * p.Nsweep / elapsed,
        "acceptance": [float(cnt[:, ch].sum() / (nchains * p.Nbin)) for ch in (0, 1)],
        "drift_max": float(cnt[:, 4].max()), "quarantined_chains": quarantined,
        "status": [int(v) for v in cnt[:, 6]], **tau_record,
    }
    (run_dir / "run_record.json").write_text(json.dumps(record, indent=1) + "\n")
    seeds, phis = ens.get_state()
    # binary checkpoint beside confout.txt: the same seeds and fields, exact and compact
    np.savez(run_dir / "confout.npz", seeds=np.asarray(seeds, dtype=np.int32),
             phi=np.stack([np.asarray(x, dtype=np.float64).reshape(p.Ltrot, p.Lq, NAUX) for x in phis]))
    with open(run_dir / "confout.txt", "w") as f:   # conf_out (fields.f90:236-278)
        for c in range(nchains):
            f.write(f" {int(seeds[c])}\n")
            f.write("".join(f" {float(v)!r}\n" for v in phis[c].ravel()))
    ens.close()
    return {"params": p, "counters": cnt}
