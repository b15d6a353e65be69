// C ABI of the B200 BAFQMC sweep (include/bafqmc_b200.h): host-side model set
// up (lattice tables, kinetic propagators, HS factors, initial fields) and the
// device state of a batch of chains of the number-conserving and Nambu
// pairing solvers.
#include <algorithm>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/bafqmc_b200.h"
#include "kernels.h"
#include "net.h"
#include "sweep.cuh"

using bq::ChainDev;
using bq::ChainScalars;
using bq::PointDev;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}
// NVTX range over one C-ABI call, so that a profiler timeline shows the
// host-side phases (set-up, pre, bins, diagnostics) around the kernels.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

int cuda_fail(cudaError_t e, const char* where) {
    return fail(BAFQMC_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
#define CK(call)                                                 \
    do {                                                         \
        cudaError_t _e = (call);                                 \
        if (_e != cudaSuccess) return cuda_fail(_e, #call);      \
    } while (0)

typedef std::vector<double> dvec;
struct zmat {   // row-major complex n x n
    int n;
    std::vector<double> a;   // interleaved
    explicit zmat(int n_ = 0) : n(n_), a(2 * (size_t)n_ * n_, 0.0) {}
    double& re(int i, int j) { return a[2 * ((size_t)i * n + j)]; }
};

zmat zmul(const zmat& A, const zmat& B) {
    const int n = A.n;
    zmat C(n);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k) {
            const double ar = A.a[2 * ((size_t)i * n + k)], ai = A.a[2 * ((size_t)i * n + k) + 1];
            if (ar == 0.0 && ai == 0.0) continue;
            for (int j = 0; j < n; ++j) {
                const double br = B.a[2 * ((size_t)k * n + j)], bi = B.a[2 * ((size_t)k * n + j) + 1];
                C.a[2 * ((size_t)i * n + j)] += ar * br - ai * bi;
                C.a[2 * ((size_t)i * n + j) + 1] += ar * bi + ai * br;
            }
        }
    return C;
}

// exp(s * H) by scaling and squaring of the Taylor series (degree 24 after
// scaling to norm <= 1/2; truncation error < 1e-30 relative before squaring).
// Stands in for the ZHEEV-based opT_set (non_interact.f90:74-109) and, for the
// non-Hermitian Nambu block, the ZGEEV-based exp_general_matrix
// (src/pairing/src/non_interact.f90:131-178); it needs no eigenvectors.
zmat expm_scaled(const zmat& H, double s) {
    const int n = H.n;
    zmat A(n);
    double norm1 = 0.0;
    for (int j = 0; j < n; ++j) {
        double col = 0.0;
        for (int i = 0; i < n; ++i) col += std::hypot(H.a[2 * ((size_t)i * n + j)], H.a[2 * ((size_t)i * n + j) + 1]);
        norm1 = std::max(norm1, col);
    }
    norm1 *= std::fabs(s);
    int sq = 0;
    while (norm1 > 0.5) {
        norm1 *= 0.5;
        ++sq;
    }
    const double scale = s * std::ldexp(1.0, -sq);
    for (size_t k = 0; k < A.a.size(); ++k) A.a[k] = H.a[k] * scale;
    zmat E(n), term(n);
    for (int i = 0; i < n; ++i) {
        E.re(i, i) = 1.0;
        term.re(i, i) = 1.0;
    }
    for (int k = 1; k <= 24; ++k) {
        term = zmul(term, A);
        const double inv = 1.0 / k;
        for (size_t q = 0; q < term.a.size(); ++q) term.a[q] *= inv;
        for (size_t q = 0; q < E.a.size(); ++q) E.a[q] += term.a[q];
    }
    for (int k = 0; k < sq; ++k) E = zmul(E, E);
    return E;
}

const double kPI = std::acos(-1.0);

struct HostLattice {   // lattice.f90:21-125 (Norb = 1)
    int nlx, nly, lq;
    std::vector<int> cellx, celly, inv_cell, bonds, imj;
    std::vector<double> aimj, xk;
    bool hasK;
    int indexK;
    int cell(int nx, int ny) const { return inv_cell[(size_t)(ny - 1) * nlx + (nx - 1)]; }

    HostLattice(int lx, int ly) : nlx(lx), nly(ly), lq(lx * ly) {
        inv_cell.assign((size_t)lq, 0);
        cellx.resize(lq);
        celly.resize(lq);
        int nc = 0;
        for (int ny = 1; ny <= nly; ++ny)
            for (int nx = 1; nx <= nlx; ++nx) {
                cellx[nc] = nx;
                celly[nc] = ny;
                inv_cell[(size_t)(ny - 1) * nlx + (nx - 1)] = nc;
                ++nc;
            }
        auto npbc = [](int nr, int L) { return nr > L ? nr - L : (nr < 1 ? nr + L : nr); };
        imj.resize((size_t)lq * lq);
        for (int jj = 0; jj < lq; ++jj)
            for (int ii = 0; ii < lq; ++ii) {
                const int dx = ((cellx[ii] - cellx[jj]) % nlx + nlx) % nlx + 1;
                const int dy = ((celly[ii] - celly[jj]) % nly + nly) % nly + 1;
                imj[(size_t)ii * lq + jj] = cell(dx, dy);
            }
        const double a1[2] = {1.0, 0.0}, a2[2] = {0.5, std::sqrt(3.0) / 2.0};
        const double b1[2] = {2.0 * kPI, -2.0 * kPI / std::sqrt(3.0)}, b2[2] = {0.0, 4.0 * kPI / std::sqrt(3.0)};
        aimj.resize(2 * (size_t)lq);
        xk.resize(2 * (size_t)lq);
        for (int ii = 0; ii < lq; ++ii) {
            const int ix = cellx[ii], iy = celly[ii];
            aimj[2 * ii] = (ix - 1) * a1[0] + (iy - 1) * a2[0];
            aimj[2 * ii + 1] = (ix - 1) * a1[1] + (iy - 1) * a2[1];
            xk[2 * ii] = (ix - 1) * b1[0] / nlx + (iy - 1) * b2[0] / nly;
            xk[2 * ii + 1] = (ix - 1) * b1[1] / nlx + (iy - 1) * b2[1] / nly;
        }
        bonds.resize(3 * (size_t)lq);
        for (int iy = 1; iy <= nly; ++iy)
            for (int ix = 1; ix <= nlx; ++ix) {
                const int i = cell(ix, iy);
                bonds[3 * i + 0] = cell(npbc(ix + 1, nlx), npbc(iy, nly));
                bonds[3 * i + 1] = cell(npbc(ix, nlx), npbc(iy + 1, nly));
                bonds[3 * i + 2] = cell(npbc(ix - 1, nlx), npbc(iy + 1, nly));
            }
        hasK = (nlx % 3 == 0) && (nly % 3 == 0);
        indexK = hasK ? cell(2 * nlx / 3 + 1, nly / 3 + 1) : 0;
    }
    double k_dot_r(int k, int r) const { return xk[2 * k] * aimj[2 * r] + xk[2 * k + 1] * aimj[2 * r + 1]; }
};

struct PointHost {
    bafqmc_point p;
    int N, Lq, Nst;
    int pairing;   // Nambu chain: N = 2 Lq, the {b, c^dagger} block
    double dtau;
    zmat expP, expM;
    std::vector<double> phaseR;   // interleaved complex, Lq entries
    double alpha_re[2], alpha_im[2];
    int active[2];
    int flip[2];
    int cls = -1;   // kernel class of the point's chains (default: the smallest that holds N)
};

double ranf(int32_t& seed) {   // src/common/random.f90:1-11
    const long long v = (48828125LL * (long long)seed) % 2147483648LL;
    seed = (int32_t)(v < 0 ? v + 2147483648LL : v);
    return (double)seed / 2147483648.0;
}
double rng_gaussian(int32_t& seed) {   // fields.f90:280-288
    const double x1 = ranf(seed);
    const double x2 = ranf(seed);
    return std::sqrt(-2.0 * std::log(x1)) * std::cos(2.0 * kPI * x2);
}

}  // namespace

int bq::net_fail(int code, const std::string& msg) { return fail(code, msg); }

struct bafqmc_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    int npts = 0, nchains = 0, obs_stride = 0;
    std::vector<PointHost> pts;
    std::vector<int> chain_point;
    std::vector<long long> arena_off, phi_off;
    long long arena_total = 0, phi_total = 0;
    std::vector<int> cls_list[bq::kNumClasses];
    int* d_cls[bq::kNumClasses] = {};
    int* d_pstart = nullptr;
    int* d_plist = nullptr;
    double* d_pout = nullptr;
    double* d_tmp = nullptr;
    double* d_pole = nullptr;   // pole diagnostics: [nchains][kPoleScalars] then [nchains][pole_n][2]
    double2* d_pole_mat = nullptr;   // per-chain matrices of the pole kernel above its shared-memory size
    int pole_n = 0;
    PointDev* d_pts = nullptr;
    ChainDev* d_chains = nullptr;
    double2* d_mats = nullptr;
    double2* d_arena = nullptr;
    double* d_phi = nullptr;
    double* d_obs = nullptr;
    ChainScalars* d_sc = nullptr;
    bool have_fields = false, pre_done = false, bin_done = false;
    int timers = 0;
    int mixed = 0;   // bafqmc_set_precision
    // the launches of one bin (reset, nsweep sweeps of every class, finish),
    // captured once per (nsweep, timers) and replayed as one graph launch
    // proposal state of the global moves (bafqmc_global_shift): arena, fields,
    // chain scalars and field norms, allocated on first use
    double2* d_arena2 = nullptr;
    double* d_phi2 = nullptr;
    ChainScalars* d_sc2 = nullptr;
    double* d_fn2 = nullptr;
    int* d_acc = nullptr;
    // on-device block statistics of the per-bin point averages (bafqmc_stats_reset)
    int stats_block = 0, stats_max = 0, stats_in_block = 0, stats_blocks = 0;
    double* d_stats = nullptr;   // [npts*stride] x (current block sum, mean, sem, then stats_max block means)
    cudaGraphExec_t bin_graph = nullptr;
    int graph_nsweep = 0, graph_timers = 0, graph_mixed = 0, graph_tau = 0, graph_probe = 0;
    // time-displaced pass (bafqmc_set_time_displaced): the chains it runs, one
    // matrix region per CTA, per-chain drift statistics, the optional probe
    int tau_on = 0, tau_probe_nt = 0, tau_grid = 0;
    int* d_tau_idx = nullptr;
    double2* d_tau_ws = nullptr;
    double* d_tau_stats = nullptr;
    double2* d_tau_probe = nullptr;

    bq::KernelArgs args() const {
        bq::KernelArgs ka;
        ka.pts = d_pts;
        ka.chains = d_chains;
        ka.nchains = nchains;
        ka.obs_stride = obs_stride;
        ka.arena = d_arena;
        ka.phi = d_phi;
        ka.obs = d_obs;
        ka.sc = d_sc;
        ka.timers = timers;
        ka.mixed = mixed;
        if (tau_on) {
            ka.tau_ws = d_tau_ws;
            ka.tau_stats = d_tau_stats;
            ka.tau_probe = tau_probe_nt > 0 ? d_tau_probe : nullptr;
            ka.tau_probe_nt = tau_probe_nt;
        }
        return ka;
    }
    bq::KernelArgs args2() const {   // the proposal state of the global moves
        bq::KernelArgs ka = args();
        ka.arena = d_arena2;
        ka.phi = d_phi2;
        ka.sc = d_sc2;
        ka.timers = 0;
        return ka;
    }
};

namespace {

int setup_point(const bafqmc_point& p, PointHost& out) {
    if (p.sector != 0 && p.sector != 1) return fail(BAFQMC_EARG, "sector must be 0 (number-conserving) or 1 (Nambu)");
    if (p.sector == 0 && p.delta != 0.0) return fail(BAFQMC_EARG, "delta must be 0 for the number-conserving sector");
    if (p.Lx < 1 || p.Ly < 1 || p.Ltrot < 1 || p.Nwrap < 1) return fail(BAFQMC_EARG, "non-positive lattice size");
    if (p.Ltrot % p.Nwrap != 0) return fail(BAFQMC_EARG, "Ltrot is not a multiple of Nwrap");
    if (p.U1 < -bq::kZero) return fail(BAFQMC_EARG, "U1 must be non-negative (relative-density channel)");
    if (p.U2 > bq::kZero) return fail(BAFQMC_EARG, "U2 must be non-positive (total-density channel)");
    if (p.LxTherm < 1 || p.LyTherm < 1 || p.LtrotTherm < 1 || p.LxTherm > p.Lx || p.LyTherm > p.Ly ||
        p.LtrotTherm > p.Ltrot)
        return fail(BAFQMC_EARG, "therm field size must not exceed the lattice");
    if (p.iniType < 1 || p.iniType > 3) return fail(BAFQMC_EARG, "incorrect initype input");
    out.p = p;
    out.pairing = p.sector == 1 ? 1 : 0;
    out.Lq = p.Lx * p.Ly;
    out.N = out.pairing ? 2 * out.Lq : out.Lq;
    out.Nst = p.Ltrot / p.Nwrap;
    out.dtau = p.beta / (double)p.Ltrot;
    if (bq::class_of(out.N, out.pairing) < 0)
        return fail(BAFQMC_EUNSUPPORTED, "Ndim above the largest size class of this build (144 number-conserving, 72 Nambu)");
    HostLattice lat(p.Lx, p.Ly);
    const int ns = out.Lq, n = out.N;
    zmat H(n);   // def_hamT (non_interact.f90:33-72), t = 1
    for (int ii = 0; ii < ns; ++ii)
        for (int nb = 0; nb < 3; ++nb) {
            const int jj = lat.bonds[3 * ii + nb];
            H.re(ii, jj) += 1.0;
            H.re(jj, ii) += 1.0;
            if (out.pairing) {   // c^dagger block: -t on the transposed bond (src/pairing/src/non_interact.f90:61-66)
                H.re(ns + jj, ns + ii) -= 1.0;
                H.re(ns + ii, ns + jj) -= 1.0;
            }
        }
    for (int ii = 0; ii < ns; ++ii) {
        H.re(ii, ii) -= p.mu;
        if (out.pairing) {   // pairing (:70-81) and chemical potential (:83-94) of the {b, c^dagger} block
            H.re(ii, ns + ii) += p.delta;
            H.re(ns + ii, ii) -= p.delta;
            H.re(ns + ii, ns + ii) += p.mu;
        }
    }
    out.expP = expm_scaled(H, -out.dtau);
    out.expM = expm_scaled(H, out.dtau);
    out.phaseR.assign(2 * (size_t)out.Lq, 0.0);
    if (lat.hasK) {   // phaseK = exp(i k_dot_r(indexK, imj)) (obser_equal.f90:157)
        for (int r = 0; r < out.Lq; ++r) {
            const double kr = lat.k_dot_r(lat.indexK, r);
            out.phaseR[2 * r] = std::cos(kr);
            out.phaseR[2 * r + 1] = std::sin(kr);
        }
    }
    const double U[2] = {p.U1, p.U2};
    for (int ch = 0; ch < 2; ++ch) {   // opU_set (operator_Hubbard.f90:36-43)
        out.alpha_re[ch] = 0.0;
        out.alpha_im[ch] = 0.0;
        if (U[ch] < -bq::kZero) out.alpha_re[ch] = std::sqrt(-2.0 * U[ch] * out.dtau);
        if (U[ch] > bq::kZero) out.alpha_im[ch] = std::sqrt(2.0 * U[ch] * out.dtau);
        out.active[ch] = std::fabs(U[ch]) > bq::kZero ? 1 : 0;
    }
    // Nambu sector factors on c^dagger: e^{+alpha phi} for U1, e^{-alpha phi} for U2
    // (src/pairing/src/operator_Hubbard.f90:155-166)
    out.flip[0] = 0;
    out.flip[1] = out.pairing;
    return BAFQMC_OK;
}

int point_class(const PointHost& ph) { return ph.cls >= 0 ? ph.cls : bq::class_of(ph.N, ph.pairing); }

// Whether kernel class cls can run a point of dimension n and the given sector.
bool class_holds(int cls, int n, int pairing) {
    if (cls < 0 || cls >= bq::kNumClasses || n > bq::class_nmax(cls)) return false;
    const int cls_pair = (cls >= 3 && cls < 6) ? 1 : 0;
    return cls_pair == pairing;
}

// Device descriptor of a point whose expP | expM | phase table start at mats.
PointDev point_dev(const PointHost& ph, const double2* mats) {
    PointDev d;
    std::memset(&d, 0, sizeof d);
    const size_t nn = (size_t)ph.N * ph.N;
    d.N = ph.N;
    d.L = ph.p.Ltrot;
    d.Nwrap = ph.p.Nwrap;
    d.Nst = ph.Nst;
    d.Lq = ph.Lq;
    d.hasK = (ph.p.Lx % 3 == 0 && ph.p.Ly % 3 == 0) ? 1 : 0;
    d.Lx = ph.p.Lx;
    d.Ly = ph.p.Ly;
    d.Ns = ph.Lq;
    d.pairing = ph.pairing;
    for (int ch = 0; ch < 2; ++ch) {
        d.active[ch] = ph.active[ch];
        d.flip[ch] = ph.flip[ch];
        d.alpha_re[ch] = ph.alpha_re[ch];
        d.alpha_im[ch] = ph.alpha_im[ch];
    }
    d.shiftLoc = ph.p.shiftLoc;
    d.U1 = ph.p.U1;
    d.U2 = ph.p.U2;
    d.RT = 1.0;
    d.mu = ph.p.mu;
    d.Delta = ph.pairing ? ph.p.delta : 0.0;
    d.expP = mats;
    d.expM = mats + nn;
    d.phaseR = mats + 2 * nn;
    return d;
}

void free_handle(bafqmc_handle* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    void* ptrs[] = {h->d_pts, h->d_chains, h->d_mats, h->d_arena, h->d_phi, h->d_obs, h->d_sc,
                    h->d_pstart, h->d_plist, h->d_pout, h->d_tmp, h->d_pole, h->d_pole_mat, h->d_stats,
                    h->d_arena2, h->d_phi2, h->d_sc2, h->d_fn2, h->d_acc, h->d_tau_idx, h->d_tau_ws,
                    h->d_tau_stats, h->d_tau_probe};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (int c = 0; c < bq::kNumClasses; ++c)
        if (h->d_cls[c]) cudaFree(h->d_cls[c]);
    if (h->bin_graph) cudaGraphExecDestroy(h->bin_graph);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

}  // namespace

namespace {
// the proposal state of the global moves, allocated on first use
int ensure_proposal_state(bafqmc_handle* h) {
    if (h->d_arena2) return BAFQMC_OK;
    CK(cudaMalloc(&h->d_arena2, sizeof(double2) * h->arena_total));
    CK(cudaMalloc(&h->d_phi2, sizeof(double) * h->phi_total));
    CK(cudaMalloc(&h->d_sc2, sizeof(ChainScalars) * h->nchains));
    CK(cudaMemset(h->d_sc2, 0, sizeof(ChainScalars) * h->nchains));
    CK(cudaMalloc(&h->d_fn2, sizeof(double) * h->nchains));
    CK(cudaMalloc(&h->d_acc, sizeof(int) * h->nchains));
    return BAFQMC_OK;
}
// every chain of the handle is a number-conserving chain of the network's lattice
int check_net_chains(const bafqmc_handle* h, const bafqmc_net* n) {
    for (int c = 0; c < h->nchains; ++c) {
        const PointHost& p = h->pts[h->chain_point[c]];
        if (p.pairing)
            return fail(BAFQMC_EUNSUPPORTED, "the learned proposer runs number-conserving chains only (chain " +
                                                 std::to_string(c) + " is a Nambu chain)");
        if (p.p.Lx != n->shape.Lx || p.p.Ly != n->shape.Ly || p.p.Ltrot != n->shape.L)
            return fail(BAFQMC_EARG, "chain " + std::to_string(c) + " is not on the network's lattice (" +
                                         std::to_string(n->shape.Lx) + "x" + std::to_string(n->shape.Ly) + ", Ltrot " +
                                         std::to_string(n->shape.L) + ")");
    }
    return BAFQMC_OK;
}
}  // namespace

extern "C" {

const char* bafqmc_last_error(void) { return g_err.c_str(); }

int bafqmc_create(const bafqmc_point* pts, int npts, const int32_t* chain_point, int nchains, int device,
                  bafqmc_handle** out) {
    return bafqmc_create_tuned(pts, npts, chain_point, nchains, device, nullptr, out);
}

int bafqmc_create_tuned(const bafqmc_point* pts, int npts, const int32_t* chain_point, int nchains, int device,
                        const int* classes, bafqmc_handle** out) {
    NvtxRange nvtx_("bafqmc_create");
    if (!out || !pts || npts < 1 || nchains < 1 || !chain_point) return fail(BAFQMC_EARG, "bad create arguments");
    *out = nullptr;
    bafqmc_handle* h = new bafqmc_handle();
    h->device = device;
    h->npts = npts;
    h->nchains = nchains;
    h->pts.resize(npts);
    int maxlq = 0;
    for (int i = 0; i < npts; ++i) {
        int rc = setup_point(pts[i], h->pts[i]);
        if (rc != BAFQMC_OK) {
            delete h;
            return rc;
        }
        if (classes && classes[i] >= 0) {
            if (!class_holds(classes[i], h->pts[i].N, h->pts[i].pairing)) {
                delete h;
                return fail(BAFQMC_EARG, "kernel class " + std::to_string(classes[i]) + " cannot run point " +
                                             std::to_string(i));
            }
            h->pts[i].cls = classes[i];
        }
        maxlq = std::max(maxlq, h->pts[i].Lq);
    }
    h->obs_stride = bq::kObsScalars + maxlq;
    h->chain_point.assign(chain_point, chain_point + nchains);
    h->arena_off.resize(nchains);
    h->phi_off.resize(nchains);
    std::vector<std::vector<int>> per_point(npts);
    for (int c = 0; c < nchains; ++c) {
        const int p = chain_point[c];
        if (p < 0 || p >= npts) {
            delete h;
            return fail(BAFQMC_EARG, "chain_point out of range");
        }
        const PointHost& ph = h->pts[p];
        h->arena_off[c] = h->arena_total;
        h->arena_total += bq::arena_size(ph.N, ph.Nst, bq::class_work_elems(point_class(ph)));
        h->phi_off[c] = h->phi_total;
        h->phi_total += (long long)ph.p.Ltrot * ph.Lq * 2;
        h->cls_list[point_class(ph)].push_back(c);
        per_point[p].push_back(c);
    }
    // Within a class launch, CTAs start in list order: longest chains first
    // (cost ~ Ltrot * N^3 * active channels), so that a ragged batch does not end
    // on a tail of long chains started last.  Results do not depend on the order.
    for (int k = 0; k < bq::kNumClasses; ++k) {
        auto cost = [&](int c) {
            const PointHost& q = h->pts[h->chain_point[c]];
            return (double)q.p.Ltrot * q.N * q.N * q.N * (q.active[0] + q.active[1]);
        };
        std::stable_sort(h->cls_list[k].begin(), h->cls_list[k].end(),
                         [&](int a, int b) { return cost(a) > cost(b); });
    }
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        delete h;
        return cuda_fail(e, "cudaSetDevice");
    }
    auto bail = [&](cudaError_t err, const char* where) {
        int rc = cuda_fail(err, where);
        free_handle(h);
        return rc;
    };
    if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(e, "cudaStreamCreate");
    // a^k mod 2^31 table for the in-kernel skip-ahead of the LCG
    std::vector<uint32_t> apow(bq::kMaxPow);
    unsigned long long v = 1;
    for (int k = 0; k < bq::kMaxPow; ++k) {
        apow[k] = (uint32_t)v;
        v = (v * 48828125ull) & 0x7fffffffull;
    }
    if ((e = bq::upload_pow_table(apow.data(), bq::kMaxPow)) != cudaSuccess) return bail(e, "upload_pow_table");
    // point matrices: expP, expM (N*N each) and the K phase table (Lq) per point
    size_t mat_total = 0;
    std::vector<size_t> mat_off(npts);
    for (int i = 0; i < npts; ++i) {
        mat_off[i] = mat_total;
        mat_total += 2 * (size_t)h->pts[i].N * h->pts[i].N + h->pts[i].Lq;
    }
    std::vector<double> mats(2 * mat_total);
    for (int i = 0; i < npts; ++i) {
        const PointHost& ph = h->pts[i];
        const size_t nn = (size_t)ph.N * ph.N;
        std::memcpy(&mats[2 * mat_off[i]], ph.expP.a.data(), sizeof(double) * 2 * nn);
        std::memcpy(&mats[2 * (mat_off[i] + nn)], ph.expM.a.data(), sizeof(double) * 2 * nn);
        std::memcpy(&mats[2 * (mat_off[i] + 2 * nn)], ph.phaseR.data(), sizeof(double) * 2 * ph.Lq);
    }
    if ((e = cudaMalloc(&h->d_mats, sizeof(double2) * mat_total)) != cudaSuccess) return bail(e, "cudaMalloc mats");
    if ((e = cudaMemcpy(h->d_mats, mats.data(), sizeof(double2) * mat_total, cudaMemcpyHostToDevice)) != cudaSuccess)
        return bail(e, "upload mats");
    std::vector<PointDev> pd(npts);
    for (int i = 0; i < npts; ++i) pd[i] = point_dev(h->pts[i], h->d_mats + mat_off[i]);
    std::vector<ChainDev> cd(nchains);
    for (int c = 0; c < nchains; ++c) {
        cd[c].point = chain_point[c];
        cd[c].pad = 0;
        cd[c].arena_off = h->arena_off[c];
        cd[c].phi_off = h->phi_off[c];
    }
    std::vector<int> pstart(npts + 1, 0), plist;
    for (int p = 0; p < npts; ++p) {
        pstart[p + 1] = pstart[p] + (int)per_point[p].size();
        plist.insert(plist.end(), per_point[p].begin(), per_point[p].end());
    }
    if ((e = cudaMalloc(&h->d_pts, sizeof(PointDev) * npts)) != cudaSuccess) return bail(e, "cudaMalloc pts");
    if ((e = cudaMalloc(&h->d_chains, sizeof(ChainDev) * nchains)) != cudaSuccess) return bail(e, "cudaMalloc chains");
    if ((e = cudaMalloc(&h->d_arena, sizeof(double2) * h->arena_total)) != cudaSuccess) return bail(e, "cudaMalloc arena");
    if ((e = cudaMalloc(&h->d_phi, sizeof(double) * h->phi_total)) != cudaSuccess) return bail(e, "cudaMalloc phi");
    if ((e = cudaMalloc(&h->d_obs, sizeof(double) * (size_t)nchains * h->obs_stride)) != cudaSuccess)
        return bail(e, "cudaMalloc obs");
    if ((e = cudaMalloc(&h->d_sc, sizeof(ChainScalars) * nchains)) != cudaSuccess) return bail(e, "cudaMalloc sc");
    if ((e = cudaMalloc(&h->d_pstart, sizeof(int) * (npts + 1))) != cudaSuccess) return bail(e, "cudaMalloc pstart");
    if ((e = cudaMalloc(&h->d_plist, sizeof(int) * nchains)) != cudaSuccess) return bail(e, "cudaMalloc plist");
    if ((e = cudaMalloc(&h->d_pout, sizeof(double) * (size_t)npts * h->obs_stride)) != cudaSuccess)
        return bail(e, "cudaMalloc pout");
    if ((e = cudaMalloc(&h->d_tmp, sizeof(double) * nchains)) != cudaSuccess) return bail(e, "cudaMalloc tmp");
    for (int c = 0; c < bq::kNumClasses; ++c) {
        if (h->cls_list[c].empty()) continue;
        if ((e = cudaMalloc(&h->d_cls[c], sizeof(int) * h->cls_list[c].size())) != cudaSuccess)
            return bail(e, "cudaMalloc cls");
        if ((e = cudaMemcpy(h->d_cls[c], h->cls_list[c].data(), sizeof(int) * h->cls_list[c].size(),
                            cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail(e, "upload cls");
    }
    if ((e = cudaMemcpy(h->d_pts, pd.data(), sizeof(PointDev) * npts, cudaMemcpyHostToDevice)) != cudaSuccess)
        return bail(e, "upload pts");
    if ((e = cudaMemcpy(h->d_chains, cd.data(), sizeof(ChainDev) * nchains, cudaMemcpyHostToDevice)) != cudaSuccess)
        return bail(e, "upload chains");
    if ((e = cudaMemcpy(h->d_pstart, pstart.data(), sizeof(int) * (npts + 1), cudaMemcpyHostToDevice)) != cudaSuccess)
        return bail(e, "upload pstart");
    if ((e = cudaMemcpy(h->d_plist, plist.data(), sizeof(int) * nchains, cudaMemcpyHostToDevice)) != cudaSuccess)
        return bail(e, "upload plist");
    if ((e = cudaMemset(h->d_arena, 0, sizeof(double2) * h->arena_total)) != cudaSuccess) return bail(e, "memset arena");
    if ((e = cudaMemset(h->d_obs, 0, sizeof(double) * (size_t)nchains * h->obs_stride)) != cudaSuccess)
        return bail(e, "memset obs");
    if ((e = cudaMemset(h->d_sc, 0, sizeof(ChainScalars) * nchains)) != cudaSuccess) return bail(e, "memset sc");
    if ((e = cudaMemset(h->d_phi, 0, sizeof(double) * h->phi_total)) != cudaSuccess) return bail(e, "memset phi");
    *out = h;
    return BAFQMC_OK;
}

void bafqmc_destroy(bafqmc_handle* h) { free_handle(h); }

int bafqmc_point_dim(const bafqmc_handle* h, int point, int* ndim, int* lq, int* ltrot, int* nst) {
    if (!h || point < 0 || point >= h->npts) return fail(BAFQMC_EARG, "bad point");
    const PointHost& p = h->pts[point];
    if (ndim) *ndim = p.N;
    if (lq) *lq = p.Lq;
    if (ltrot) *ltrot = p.p.Ltrot;
    if (nst) *nst = p.Nst;
    return BAFQMC_OK;
}
int bafqmc_obs_stride(const bafqmc_handle* h) { return h ? h->obs_stride : fail(BAFQMC_EARG, "null handle"); }
int bafqmc_num_chains(const bafqmc_handle* h) { return h ? h->nchains : fail(BAFQMC_EARG, "null handle"); }

static int upload_state(bafqmc_handle* h, const int32_t* seeds, const double* phi) {
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(h->d_phi, phi, sizeof(double) * h->phi_total, cudaMemcpyHostToDevice, h->stream));
    std::vector<ChainScalars> sc(h->nchains);
    std::memset(sc.data(), 0, sizeof(ChainScalars) * h->nchains);
    for (int c = 0; c < h->nchains; ++c) sc[c].seed = (uint32_t)seeds[c];
    CK(cudaMemcpyAsync(h->d_sc, sc.data(), sizeof(ChainScalars) * h->nchains, cudaMemcpyHostToDevice, h->stream));
    // fields must be finite (the reference would carry a NaN into every weight)
    int* d_bad = reinterpret_cast<int*>(h->d_tmp);
    CK(bq::launch_field_check(h->args(), d_bad, h->stream));
    std::vector<int> bad(h->nchains);
    CK(cudaMemcpyAsync(bad.data(), d_bad, sizeof(int) * h->nchains, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->pre_done = false;
    h->bin_done = false;
    for (int c = 0; c < h->nchains; ++c)
        if (bad[c]) {
            h->have_fields = false;
            return fail(BAFQMC_EARG, "non-finite field value (NaN or Inf) in chain " + std::to_string(c));
        }
    h->have_fields = true;
    return BAFQMC_OK;
}

int bafqmc_fields_from_seeds(bafqmc_handle* h, const int32_t* seeds) {
    NvtxRange nvtx_("bafqmc_fields_from_seeds");
    if (!h || !seeds) return fail(BAFQMC_EARG, "null argument");
    std::vector<double> phi(h->phi_total);
    std::vector<int32_t> adv(h->nchains);
    for (int c = 0; c < h->nchains; ++c) {
        const PointHost& ph = h->pts[h->chain_point[c]];
        const bafqmc_point& p = ph.p;
        int32_t s = seeds[c];
        const int ndT = p.LxTherm * p.LyTherm;
        std::vector<double> therm((size_t)p.LtrotTherm * ndT * 2);
        const double bias[2] = {p.iniBias1, p.iniBias2};
        for (int nt = 0; nt < p.LtrotTherm; ++nt)   // conf_set (fields.f90:115-154)
            for (int ii = 0; ii < ndT; ++ii)
                for (int ns = 0; ns < 2; ++ns) {
                    double x;
                    if (p.iniType == 1) {
                        x = ranf(s);
                        x = bias[ns] + p.iniAmpl * (x - 0.5);
                    } else if (p.iniType == 2) {
                        x = bias[ns] + p.iniAmpl * rng_gaussian(s);
                    } else {
                        x = bias[ns] + p.iniAmpl * std::fabs(rng_gaussian(s));
                    }
                    therm[((size_t)nt * ndT + ii) * 2 + ns] = x;
                }
        adv[c] = s;
        double* out = phi.data() + h->phi_off[c];   // conf_transfer (fields.f90:156-234)
        const int n = ph.Lq;
        for (int nt = 0; nt < p.LtrotTherm; ++nt)
            for (int ny = 1; ny <= p.Ly; ++ny)
                for (int nx = 1; nx <= p.Lx; ++nx) {
                    const int tx = nx > p.LxTherm ? nx - p.LxTherm : nx;
                    const int ty = ny > p.LyTherm ? ny - p.LyTherm : ny;
                    const int iit = (ty - 1) * p.LxTherm + (tx - 1);
                    const int ii = (ny - 1) * p.Lx + (nx - 1);
                    for (int ns = 0; ns < 2; ++ns)
                        out[((size_t)nt * n + ii) * 2 + ns] = therm[((size_t)nt * ndT + iit) * 2 + ns];
                }
        for (int nt = p.LtrotTherm; nt < p.Ltrot; ++nt)
            for (int k = 0; k < 2 * n; ++k) out[(size_t)nt * n * 2 + k] = out[(size_t)(nt - p.LtrotTherm) * n * 2 + k];
    }
    return upload_state(h, adv.data(), phi.data());
}

int bafqmc_set_state(bafqmc_handle* h, const int32_t* seeds, const double* phi) {
    NvtxRange nvtx_("bafqmc_set_state");
    if (!h || !seeds || !phi) return fail(BAFQMC_EARG, "null argument");
    return upload_state(h, seeds, phi);
}

int bafqmc_get_state(bafqmc_handle* h, int32_t* seeds, double* phi) {
    NvtxRange nvtx_("bafqmc_get_state");
    if (!h) return fail(BAFQMC_EARG, "null handle");
    CK(cudaSetDevice(h->device));
    if (phi) CK(cudaMemcpyAsync(phi, h->d_phi, sizeof(double) * h->phi_total, cudaMemcpyDeviceToHost, h->stream));
    std::vector<ChainScalars> sc(h->nchains);
    CK(cudaMemcpyAsync(sc.data(), h->d_sc, sizeof(ChainScalars) * h->nchains, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (seeds)
        for (int c = 0; c < h->nchains; ++c) seeds[c] = (int32_t)sc[c].seed;
    return BAFQMC_OK;
}

int bafqmc_warmup_prior(bafqmc_handle* h, int nwarm) {
    NvtxRange nvtx_("bafqmc_warmup_prior");
    if (!h || nwarm < 0) return fail(BAFQMC_EARG, "bad warm-up arguments");
    if (!h->have_fields) return fail(BAFQMC_ESTATE, "fields not initialised");
    if (nwarm == 0) return BAFQMC_OK;
    CK(cudaSetDevice(h->device));
    CK(bq::launch_warmup(h->args(), nwarm, h->stream));
    h->pre_done = false;
    return BAFQMC_OK;
}

int bafqmc_pre(bafqmc_handle* h) {
    NvtxRange nvtx_("bafqmc_pre");
    if (!h) return fail(BAFQMC_EARG, "null handle");
    if (!h->have_fields) return fail(BAFQMC_ESTATE, "fields not initialised");
    CK(cudaSetDevice(h->device));
    for (int c = 0; c < bq::kNumClasses; ++c)
        CK(bq::launch_pre(c, h->args(), h->d_cls[c], (int)h->cls_list[c].size(), h->stream));
    h->pre_done = true;
    return BAFQMC_OK;
}

namespace {
// The launches of one bin: accumulator reset, nsweep persistent sweep launches
// per kernel class, bin averages.  With the time-displaced pass on, each sweep
// is a left-traversal launch, the pass, and a right-traversal launch
// (Local_sweep_R's toggle, local_sweep.f90:119-123).
cudaError_t record_bin(bafqmc_handle* h, int nsweep) {
    const bq::KernelArgs ka = h->args();
    bq::KernelArgs kl = ka, kr = ka;
    kl.traverse = 1;
    kr.traverse = 2;
    cudaError_t e = bq::launch_bin_reset(ka, h->stream);
    for (int s = 0; s < nsweep && e == cudaSuccess; ++s) {
        if (h->tau_on) {
            for (int c = 0; c < bq::kNumClasses && e == cudaSuccess; ++c)
                e = bq::launch_sweep(c, kl, h->d_cls[c], (int)h->cls_list[c].size(), h->stream);
            if (e == cudaSuccess) e = bq::launch_tau(ka, h->d_tau_idx, h->nchains, h->tau_grid, h->stream);
            for (int c = 0; c < bq::kNumClasses && e == cudaSuccess; ++c)
                e = bq::launch_sweep(c, kr, h->d_cls[c], (int)h->cls_list[c].size(), h->stream);
        } else {
            for (int c = 0; c < bq::kNumClasses && e == cudaSuccess; ++c)
                e = bq::launch_sweep(c, ka, h->d_cls[c], (int)h->cls_list[c].size(), h->stream);
        }
    }
    if (e == cudaSuccess) e = bq::launch_bin_finish(ka, h->stream);
    return e;
}
}  // namespace

int bafqmc_sweep(bafqmc_handle* h, int nsweep) {
    NvtxRange nvtx_("bafqmc_sweep");
    if (!h || nsweep < 1) return fail(BAFQMC_EARG, "bad sweep arguments");
    if (!h->pre_done) return fail(BAFQMC_ESTATE, "bafqmc_pre has not run");
    CK(cudaSetDevice(h->device));
    if (!h->bin_graph || h->graph_nsweep != nsweep || h->graph_timers != h->timers || h->graph_mixed != h->mixed ||
        h->graph_tau != h->tau_on || h->graph_probe != h->tau_probe_nt) {
        if (h->bin_graph) {
            CK(cudaGraphExecDestroy(h->bin_graph));
            h->bin_graph = nullptr;
        }
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeRelaxed));
        const cudaError_t e = record_bin(h, nsweep);
        const cudaError_t e2 = cudaStreamEndCapture(h->stream, &g);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return cuda_fail(e != cudaSuccess ? e : e2, "capture of the bin launches");
        }
        const cudaError_t e3 = cudaGraphInstantiate(&h->bin_graph, g, 0);
        cudaGraphDestroy(g);
        if (e3 != cudaSuccess) {
            h->bin_graph = nullptr;
            return cuda_fail(e3, "cudaGraphInstantiate");
        }
        h->graph_nsweep = nsweep;
        h->graph_timers = h->timers;
        h->graph_mixed = h->mixed;
        h->graph_tau = h->tau_on;
        h->graph_probe = h->tau_probe_nt;
    }
    CK(cudaGraphLaunch(h->bin_graph, h->stream));
    h->bin_done = true;
    if (h->stats_block > 0 && h->stats_blocks < h->stats_max) {
        const int n = h->npts * h->obs_stride;
        const bool finish = h->stats_in_block + 1 == h->stats_block;
        CK(bq::launch_point_average(h->args(), h->npts, h->d_pstart, h->d_plist, h->d_pout, h->stream));
        CK(bq::launch_stats_add(h->d_pout, h->d_stats, h->d_stats + (size_t)(3 + h->stats_blocks) * n, n,
                                finish ? 1 : 0, h->stats_block, h->stream));
        h->stats_in_block = finish ? 0 : h->stats_in_block + 1;
        if (finish) ++h->stats_blocks;
    }
    return BAFQMC_OK;
}

int bafqmc_global_shift(bafqmc_handle* h, const double* shift, int* accepted) {
    NvtxRange nvtx_("bafqmc_global_shift");
    if (!h || !shift) return fail(BAFQMC_EARG, "null argument");
    if (!h->pre_done) return fail(BAFQMC_ESTATE, "bafqmc_pre has not run");
    CK(cudaSetDevice(h->device));
    int rc = ensure_proposal_state(h);
    if (rc != BAFQMC_OK) return rc;
    const bq::KernelArgs ka = h->args(), kp = h->args2();
    CK(bq::launch_global_propose(ka, kp, shift, h->stream));
    for (int c = 0; c < bq::kNumClasses; ++c)
        CK(bq::launch_pre(c, kp, h->d_cls[c], (int)h->cls_list[c].size(), h->stream));
    CK(bq::launch_field_norm(ka, h->d_tmp, h->stream));
    CK(bq::launch_field_norm(kp, h->d_fn2, h->stream));
    CK(bq::launch_global_accept(ka, kp, h->d_tmp, h->d_fn2, nullptr, h->d_acc, h->stream));
    if (accepted) {
        CK(cudaMemcpyAsync(accepted, h->d_acc, sizeof(int) * h->nchains, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    return BAFQMC_OK;
}


int bafqmc_net_collect(bafqmc_net* n, bafqmc_handle* h) {
    NvtxRange nvtx_("bafqmc_net_collect");
    if (!n || !h) return fail(BAFQMC_EARG, "null argument");
    if (!h->have_fields) return fail(BAFQMC_ESTATE, "fields not initialised");
    int rc = check_net_chains(h, n);
    if (rc != BAFQMC_OK) return rc;
    if (!n->d_data || n->data_chains != h->nchains)
        return fail(BAFQMC_ESTATE, "bafqmc_net_reserve_data has not reserved a set of this handle's chain count");
    if (n->data_used >= n->data_slots) return fail(BAFQMC_ESTATE, "the training set is full");
    CK(cudaSetDevice(h->device));
    cudaStream_t own = n->stream;
    n->stream = h->stream;
    const cudaError_t e = bq::launch_collect(n, h->args(), n->data_used);
    n->stream = own;
    CK(e);
    n->data_used += 1;
    return BAFQMC_OK;
}

int bafqmc_learned_move(bafqmc_handle* h, bafqmc_net* n, int* accepted, double* hastings) {
    NvtxRange nvtx_("bafqmc_learned_move");
    if (!h || !n) return fail(BAFQMC_EARG, "null argument");
    if (!h->pre_done) return fail(BAFQMC_ESTATE, "bafqmc_pre has not run");
    int rc = check_net_chains(h, n);
    if (rc != BAFQMC_OK) return rc;
    CK(cudaSetDevice(h->device));
    if ((rc = ensure_proposal_state(h)) != BAFQMC_OK) return rc;
    if ((rc = bq::net_ensure_cap(n, h->nchains)) != BAFQMC_OK) return rc;
    if (n->move_cap < h->nchains) {
        if (n->d_lqf) CK(cudaFree(n->d_lqf));
        if (n->d_hastings) CK(cudaFree(n->d_hastings));
        n->d_lqf = n->d_hastings = nullptr;
        CK(cudaMalloc(&n->d_lqf, sizeof(double) * h->nchains));
        CK(cudaMalloc(&n->d_hastings, sizeof(double) * h->nchains));
        n->move_cap = h->nchains;
    }
    // the network's kernels run on the handle's stream for the move
    cudaStream_t own = n->stream;
    n->stream = h->stream;
    const bq::KernelArgs ka = h->args(), kp = h->args2();
    cudaError_t e = bq::launch_pack_chains(n, ka);
    if (e == cudaSuccess) e = bq::net_forward(n, h->nchains);
    if (e == cudaSuccess) e = bq::launch_learned_propose(n, ka, kp, n->d_lqf);
    if (e == cudaSuccess) e = bq::launch_pack_chains(n, kp);
    if (e == cudaSuccess) e = bq::net_forward(n, h->nchains);
    if (e == cudaSuccess) e = bq::launch_learned_reverse(n, ka, kp, n->d_lqf, n->d_hastings);
    n->stream = own;
    CK(e);
    for (int c = 0; c < bq::kNumClasses; ++c)
        CK(bq::launch_pre(c, kp, h->d_cls[c], (int)h->cls_list[c].size(), h->stream));
    CK(bq::launch_field_norm(ka, h->d_tmp, h->stream));
    CK(bq::launch_field_norm(kp, h->d_fn2, h->stream));
    CK(bq::launch_global_accept(ka, kp, h->d_tmp, h->d_fn2, n->d_hastings, h->d_acc, h->stream));
    if (accepted) CK(cudaMemcpyAsync(accepted, h->d_acc, sizeof(int) * h->nchains, cudaMemcpyDeviceToHost, h->stream));
    if (hastings)
        CK(cudaMemcpyAsync(hastings, n->d_hastings, sizeof(double) * h->nchains, cudaMemcpyDeviceToHost, h->stream));
    if (accepted || hastings) {
        int st = 0;
        CK(cudaMemcpyAsync(&st, n->d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (st) return fail(BAFQMC_ETIMEOUT, "a bounded wait of the tensor-core convolution expired (status " +
                                                 std::to_string(st) + ")");
    }
    return BAFQMC_OK;
}

int bafqmc_stats_reset(bafqmc_handle* h, int block_size, int max_blocks) {
    if (!h || block_size < 1 || max_blocks < 2) return fail(BAFQMC_EARG, "block_size >= 1 and max_blocks >= 2");
    CK(cudaSetDevice(h->device));
    const size_t n = (size_t)h->npts * h->obs_stride;
    if (h->d_stats && max_blocks > h->stats_max) {
        CK(cudaFree(h->d_stats));
        h->d_stats = nullptr;
    }
    if (!h->d_stats) {
        CK(cudaMalloc(&h->d_stats, sizeof(double) * n * (3 + (size_t)max_blocks)));
        h->stats_max = max_blocks;
    }
    CK(cudaMemsetAsync(h->d_stats, 0, sizeof(double) * n, h->stream));
    h->stats_block = block_size;
    h->stats_in_block = 0;
    h->stats_blocks = 0;
    return BAFQMC_OK;
}

int bafqmc_stats(bafqmc_handle* h, double* mean, double* sem, int* nblocks) {
    if (!h || !mean || !sem) return fail(BAFQMC_EARG, "null argument");
    if (h->stats_block < 1) return fail(BAFQMC_ESTATE, "bafqmc_stats_reset has not run");
    if (nblocks) *nblocks = h->stats_blocks;
    CK(cudaSetDevice(h->device));
    const size_t n = (size_t)h->npts * h->obs_stride;
    double* d_mean = h->d_stats + n;
    double* d_sem = h->d_stats + 2 * n;
    CK(bq::launch_stats_final(h->d_stats + 3 * n, h->stats_blocks, (int)n, d_mean, d_sem, h->stream));
    CK(cudaMemcpyAsync(mean, d_mean, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(sem, d_sem, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return BAFQMC_OK;
}

int bafqmc_bin_chain_obs(bafqmc_handle* h, double* chain_obs) {
    NvtxRange nvtx_("bafqmc_bin_chain_obs");
    if (!h || !chain_obs) return fail(BAFQMC_EARG, "null argument");
    if (!h->bin_done) return fail(BAFQMC_ESTATE, "no bin has been measured");
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(chain_obs, h->d_obs, sizeof(double) * (size_t)h->nchains * h->obs_stride,
                       cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return BAFQMC_OK;
}

int bafqmc_bin_point_obs(bafqmc_handle* h, double* point_obs) {
    NvtxRange nvtx_("bafqmc_bin_point_obs");
    if (!h || !point_obs) return fail(BAFQMC_EARG, "null argument");
    if (!h->bin_done) return fail(BAFQMC_ESTATE, "no bin has been measured");
    CK(cudaSetDevice(h->device));
    CK(bq::launch_point_average(h->args(), h->npts, h->d_pstart, h->d_plist, h->d_pout, h->stream));
    CK(cudaMemcpyAsync(point_obs, h->d_pout, sizeof(double) * (size_t)h->npts * h->obs_stride,
                       cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return BAFQMC_OK;
}

int bafqmc_get_green(bafqmc_handle* h, int chain, double* G) {
    if (!h || !G || chain < 0 || chain >= h->nchains) return fail(BAFQMC_EARG, "bad chain");
    CK(cudaSetDevice(h->device));
    const int n = h->pts[h->chain_point[chain]].N;
    CK(cudaMemcpyAsync(G, h->d_arena + h->arena_off[chain], sizeof(double2) * n * n, cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return BAFQMC_OK;
}

int bafqmc_log_weight(bafqmc_handle* h, double* out) {
    if (!h || !out) return fail(BAFQMC_EARG, "null argument");
    CK(cudaSetDevice(h->device));
    CK(bq::launch_field_norm(h->args(), h->d_tmp, h->stream));
    std::vector<double> fn(h->nchains);
    std::vector<ChainScalars> sc(h->nchains);
    CK(cudaMemcpyAsync(fn.data(), h->d_tmp, sizeof(double) * h->nchains, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(sc.data(), h->d_sc, sizeof(ChainScalars) * h->nchains, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int c = 0; c < h->nchains; ++c)
        out[c] = h->pts[h->chain_point[c]].pairing ? std::nan("") : fn[c] - 2.0 * sc[c].logdetM;
    return BAFQMC_OK;
}

int bafqmc_pole_diagnostics(bafqmc_handle* h, double* z, int zstride, double* scalars) {
    NvtxRange nvtx_("bafqmc_pole_diagnostics");
    if (!h || !scalars) return fail(BAFQMC_EARG, "null argument");
    if (!h->pre_done) return fail(BAFQMC_ESTATE, "bafqmc_pre has not run");
    int nmax = 0;
    for (int c = 0; c < h->nchains; ++c) {
        const PointHost& p = h->pts[h->chain_point[c]];
        if (!p.pairing) nmax = std::max(nmax, p.N);
    }
    if (z && zstride < nmax) return fail(BAFQMC_EARG, "zstride is below the largest Ndim of a number-conserving chain");
    const double nan = std::nan("");
    for (size_t k = 0; k < (size_t)h->nchains * BAFQMC_POLE_SCALARS; ++k) scalars[k] = nan;
    if (z)
        for (size_t k = 0; k < (size_t)h->nchains * zstride * 2; ++k) z[k] = nan;
    if (nmax == 0) return BAFQMC_OK;
    CK(cudaSetDevice(h->device));
    const size_t per = bq::kPoleScalars + 2 * (size_t)nmax;
    if (!h->d_pole) {
        CK(cudaMalloc(&h->d_pole, sizeof(double) * per * h->nchains));
        h->pole_n = nmax;
        const long long hm = bq::pole_hbm_elems(nmax);
        if (hm > 0) CK(cudaMalloc(&h->d_pole_mat, sizeof(double2) * (size_t)hm * h->nchains));
    }
    double* d_s = h->d_pole;
    double* d_z = h->d_pole + (size_t)bq::kPoleScalars * h->nchains;
    CK(bq::launch_pole(h->args(), nmax, h->pole_n, d_z, d_s, h->d_pole_mat, h->stream));
    CK(bq::launch_field_norm(h->args(), h->d_tmp, h->stream));
    std::vector<double> hs((size_t)bq::kPoleScalars * h->nchains), hz(2 * (size_t)h->pole_n * h->nchains),
        fn(h->nchains);
    std::vector<ChainScalars> sc(h->nchains);
    CK(cudaMemcpyAsync(hs.data(), d_s, sizeof(double) * hs.size(), cudaMemcpyDeviceToHost, h->stream));
    if (z) CK(cudaMemcpyAsync(hz.data(), d_z, sizeof(double) * hz.size(), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(fn.data(), h->d_tmp, sizeof(double) * h->nchains, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(sc.data(), h->d_sc, sizeof(ChainScalars) * h->nchains, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    int bad = -1;
    for (int c = 0; c < h->nchains; ++c) {
        const PointHost& p = h->pts[h->chain_point[c]];
        if (p.pairing || (sc[c].status & 1)) continue;   // NaN rows for quarantined chains
        const double* s = hs.data() + (size_t)c * bq::kPoleScalars;
        double* o = scalars + (size_t)c * BAFQMC_POLE_SCALARS;
        for (int k = 0; k < 4; ++k) o[k] = s[k];
        o[4] = fn[c] - 2.0 * sc[c].logdetM;
        if (s[4] != 0.0 && bad < 0) bad = c;
        if (z)
            for (int i = 0; i < 2 * p.N; ++i) z[(size_t)c * zstride * 2 + i] = hz[(size_t)c * h->pole_n * 2 + i];
    }
    if (bad >= 0)
        return fail(BAFQMC_ENUMERIC, "eigenvalue iteration of the pole diagnostics did not converge for chain " +
                                         std::to_string(bad));
    return BAFQMC_OK;
}

int bafqmc_counters(bafqmc_handle* h, double* out) {
    if (!h || !out) return fail(BAFQMC_EARG, "null argument");
    CK(cudaSetDevice(h->device));
    std::vector<ChainScalars> sc(h->nchains);
    CK(cudaMemcpyAsync(sc.data(), h->d_sc, sizeof(ChainScalars) * h->nchains, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int c = 0; c < h->nchains; ++c) {
        double* o = out + (size_t)c * BAFQMC_COUNTERS;
        o[0] = sc[c].acc_sum[0];
        o[1] = sc[c].acc_sum[1];
        o[2] = sc[c].therm_acc_sum[0];
        o[3] = sc[c].therm_acc_sum[1];
        o[4] = sc[c].xmax;
        o[5] = sc[c].xmean;
        o[6] = (double)sc[c].status;
        o[7] = (double)sc[c].seed;
        o[8] = (double)sc[c].nobs;
        o[9] = sc[c].glb_acc;
        o[10] = sc[c].prop_tot[0];
        o[11] = sc[c].prop_tot[1];
        o[12] = sc[c].acc_tot[0];
        o[13] = sc[c].acc_tot[1];
    }
    return BAFQMC_OK;
}

int bafqmc_autotune(const bafqmc_point* pts, int npts, int device, int trial_chains, int* classes,
                    double* ms_per_chain_sweep) {
    NvtxRange nvtx_("bafqmc_autotune");
    if (!pts || npts < 1 || !classes) return fail(BAFQMC_EARG, "bad autotune arguments");
    std::vector<PointHost> ph(npts);
    for (int i = 0; i < npts; ++i) {
        int rc = setup_point(pts[i], ph[i]);
        if (rc != BAFQMC_OK) return rc;
    }
    CK(cudaSetDevice(device));
    if (trial_chains <= 0) {
        int sms = 0;
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        trial_chains = 4 * sms;   // whole waves at one, two and four CTAs per SM
    }
    if (ms_per_chain_sweep)
        for (int k = 0; k < npts * bq::kNumClasses; ++k) ms_per_chain_sweep[k] = std::nan("");
    // one trial per distinct (Ndim, sector), on the first point that has it
    std::vector<int> done(npts, 0);
    for (int i = 0; i < npts; ++i) {
        if (done[i]) continue;
        int best = -1;
        double best_t = 0.0;
        std::vector<int32_t> cp(trial_chains, 0), seeds(trial_chains);
        for (int c = 0; c < trial_chains; ++c) seeds[c] = 1000003 + 7919 * c;
        for (int cls = 0; cls < bq::kNumClasses; ++cls) {
            if (!class_holds(cls, ph[i].N, ph[i].pairing)) continue;
            bafqmc_handle* t = nullptr;
            int rc = bafqmc_create_tuned(&pts[i], 1, cp.data(), trial_chains, device, &cls, &t);
            if (rc == BAFQMC_OK) rc = bafqmc_fields_from_seeds(t, seeds.data());
            if (rc == BAFQMC_OK) rc = bafqmc_pre(t);
            if (rc == BAFQMC_OK) rc = bafqmc_sweep(t, 1);   // warm-up (captures the bin graph)
            float ms = 0.0f;
            if (rc == BAFQMC_OK) {
                cudaEvent_t e0, e1;
                cudaEventCreate(&e0);
                cudaEventCreate(&e1);
                cudaEventRecord(e0, t->stream);
                rc = bafqmc_sweep(t, 1);
                cudaEventRecord(e1, t->stream);
                cudaEventSynchronize(e1);
                cudaEventElapsedTime(&ms, e0, e1);
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
            }
            if (t) bafqmc_destroy(t);
            if (rc != BAFQMC_OK) return rc;
            const double per = (double)ms / trial_chains;
            for (int j = i; j < npts; ++j)
                if (ph[j].N == ph[i].N && ph[j].pairing == ph[i].pairing && ms_per_chain_sweep)
                    ms_per_chain_sweep[(size_t)j * bq::kNumClasses + cls] = per;
            if (best < 0 || per < best_t) {
                best = cls;
                best_t = per;
            }
        }
        for (int j = i; j < npts; ++j)
            if (ph[j].N == ph[i].N && ph[j].pairing == ph[i].pairing) {
                classes[j] = best;
                done[j] = 1;
            }
    }
    return BAFQMC_OK;
}

int bafqmc_set_precision(bafqmc_handle* h, int mode) {
    if (!h) return fail(BAFQMC_EARG, "null handle");
    if (mode != BAFQMC_PRECISION_FP64 && mode != BAFQMC_PRECISION_MIXED && mode != BAFQMC_PRECISION_WAIT_TEST)
        return fail(BAFQMC_EARG,
                    "precision must be BAFQMC_PRECISION_FP64, BAFQMC_PRECISION_MIXED or BAFQMC_PRECISION_WAIT_TEST");
    h->mixed = mode;
    return BAFQMC_OK;
}

int bafqmc_set_time_displaced(bafqmc_handle* h, int enable, int probe_nt) {
    if (!h) return fail(BAFQMC_EARG, "null handle");
    if (!enable) {
        h->tau_on = 0;
        h->tau_probe_nt = 0;
        return BAFQMC_OK;
    }
    for (int c = 0; c < h->nchains; ++c) {
        const PointHost& p = h->pts[h->chain_point[c]];
        if (p.N > bq::kTauMaxN)
            return fail(BAFQMC_EUNSUPPORTED, "the time-displaced pass needs N <= " + std::to_string(bq::kTauMaxN) +
                                                 " (chain " + std::to_string(c) + " has N = " + std::to_string(p.N) + ")");
        if (probe_nt < 0 || probe_nt > p.p.Ltrot)
            return fail(BAFQMC_EARG, "probe slice outside 0..Ltrot");
    }
    CK(cudaSetDevice(h->device));
    // each buffer on its own, so that a failed allocation is retried by the next call
    if (!h->tau_grid) {
        int sms = 0;
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
        h->tau_grid = std::max(1, std::min(sms, h->nchains));
    }
    if (!h->d_tau_idx) {
        std::vector<int> idx(h->nchains);
        for (int c = 0; c < h->nchains; ++c) idx[c] = c;
        int* p = nullptr;
        CK(cudaMalloc(&p, sizeof(int) * h->nchains));
        const cudaError_t e = cudaMemcpy(p, idx.data(), sizeof(int) * h->nchains, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(p);
            return cuda_fail(e, "chain list of the time-displaced pass");
        }
        h->d_tau_idx = p;
    }
    if (!h->d_tau_ws) CK(cudaMalloc(&h->d_tau_ws, sizeof(double2) * bq::tau_region_elems() * h->tau_grid));
    if (!h->d_tau_stats) {
        double* p = nullptr;
        CK(cudaMalloc(&p, sizeof(double) * bq::kTauStats * h->nchains));
        const cudaError_t e = cudaMemset(p, 0, sizeof(double) * bq::kTauStats * h->nchains);
        if (e != cudaSuccess) {
            cudaFree(p);
            return cuda_fail(e, "drift statistics of the time-displaced pass");
        }
        h->d_tau_stats = p;
    }
    if (probe_nt > 0 && !h->d_tau_probe) {
        double2* p = nullptr;
        CK(cudaMalloc(&p, sizeof(double2) * bq::kTauProbeElems * h->nchains));
        const cudaError_t e = cudaMemset(p, 0, sizeof(double2) * bq::kTauProbeElems * h->nchains);
        if (e != cudaSuccess) {
            cudaFree(p);
            return cuda_fail(e, "probe of the time-displaced pass");
        }
        h->d_tau_probe = p;
    }
    h->tau_on = 1;
    h->tau_probe_nt = probe_nt;
    return BAFQMC_OK;
}

int bafqmc_time_displaced_stats(bafqmc_handle* h, double* out, int reset) {
    if (!h) return fail(BAFQMC_EARG, "null handle");
    if (!h->d_tau_stats) return fail(BAFQMC_ESTATE, "the time-displaced pass has not been enabled");
    CK(cudaSetDevice(h->device));
    if (out)
        CK(cudaMemcpyAsync(out, h->d_tau_stats, sizeof(double) * bq::kTauStats * h->nchains, cudaMemcpyDeviceToHost,
                           h->stream));
    if (reset) CK(cudaMemsetAsync(h->d_tau_stats, 0, sizeof(double) * bq::kTauStats * h->nchains, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return BAFQMC_OK;
}

int bafqmc_time_displaced_probe(bafqmc_handle* h, int chain, double* out) {
    if (!h || !out || chain < 0 || chain >= h->nchains) return fail(BAFQMC_EARG, "bad probe arguments");
    if (!h->d_tau_probe) return fail(BAFQMC_ESTATE, "no probe slice has been set");
    const int n = h->pts[h->chain_point[chain]].N;
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(out, h->d_tau_probe + (size_t)chain * bq::kTauProbeElems, sizeof(double2) * 4 * n * n,
                       cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return BAFQMC_OK;
}

int bafqmc_phase_timers(bafqmc_handle* h, int enable, double* out) {
    if (!h) return fail(BAFQMC_EARG, "null handle");
    h->timers = enable ? 1 : 0;
    if (!out) return BAFQMC_OK;
    CK(cudaSetDevice(h->device));
    std::vector<ChainScalars> sc(h->nchains);
    CK(cudaMemcpyAsync(sc.data(), h->d_sc, sizeof(ChainScalars) * h->nchains, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int c = 0; c < h->nchains; ++c)
        for (int k = 0; k < 4; ++k) out[(size_t)c * 4 + k] = (double)sc[c].cyc[k];
    return BAFQMC_OK;
}

int bafqmc_synchronize(bafqmc_handle* h) {
    if (!h) return fail(BAFQMC_EARG, "null handle");
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaGetLastError());
    return BAFQMC_OK;
}

void* bafqmc_stream(bafqmc_handle* h) { return h ? (void*)h->stream : nullptr; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc once they are running: a host program
// whose device memory is fully claimed by another runtime's caching allocator,
// or a production driver that sizes all device memory before a long campaign
// and forbids allocation afterwards.  bafqmc_sweep_noalloc runs the same
// kernels as bafqmc_pre + bafqmc_sweep, but keeps every piece of scratch state
// (chain descriptors, e^{-+dtau K}, UDV slots, Green's functions, accumulators)
// in one file-scope device array of fixed size.  The caller passes its own
// device buffers for the inputs and outputs.
namespace {

constexpr size_t kNoAllocBytes = (size_t)BAFQMC_NOALLOC_MAX_BYTES;
// Host code must never use this name as a device address: it is a host-side
// stand-in.  The device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
unsigned char* g_noalloc_base[kNoAllocMaxDevices] = {};
std::once_flag g_noalloc_once[kNoAllocMaxDevices];
cudaError_t g_noalloc_setup_err[kNoAllocMaxDevices] = {};

// a^k mod 2^31 for the kernels' LCG skip-ahead, filled once (thread-safe static)
const uint32_t* lcg_pow_table() {
    static const std::vector<uint32_t> tab = [] {
        std::vector<uint32_t> t(bq::kMaxPow);
        unsigned long long v = 1;
        for (int k = 0; k < bq::kMaxPow; ++k) {
            t[k] = (uint32_t)v;
            v = (v * 48828125ull) & 0x7fffffffull;
        }
        return t;
    }();
    return tab.data();
}

// Set-up of a device, once, with that device current: the scratch array's
// device address and the LCG power table in constant memory.
void noalloc_setup(int dev) {
    void* base = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&base, g_noalloc_scratch);
    if (e == cudaSuccess) e = bq::upload_pow_table(lcg_pow_table(), bq::kMaxPow);
    g_noalloc_setup_err[dev] = e;
    if (e == cudaSuccess) g_noalloc_base[dev] = static_cast<unsigned char*>(base);
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

__global__ void noalloc_seeds_in(ChainScalars* sc, const int32_t* seeds, int nchains) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nchains) {
        ChainScalars z;
        memset(&z, 0, sizeof(z));
        z.seed = (uint32_t)seeds[c];
        sc[c] = z;
    }
}

__global__ void noalloc_seeds_out(const ChainScalars* sc, int32_t* seeds, int nchains) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nchains) seeds[c] = (int32_t)sc[c].seed;
}

}  // namespace

extern "C" int bafqmc_sweep_noalloc(const bafqmc_point* pt, int nchains, int32_t* seeds, double* phi, int nsweep,
                                    double* chain_obs, void* stream) {
    if (!pt || nchains < 1 || !seeds || !phi || nsweep < 1 || !chain_obs)
        return fail(BAFQMC_EARG, "bafqmc_sweep_noalloc: bad arguments");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(BAFQMC_EARG, "bafqmc_sweep_noalloc: device index too large");
    std::call_once(g_noalloc_once[dev], noalloc_setup, dev);
    if (g_noalloc_setup_err[dev] != cudaSuccess)
        return cuda_fail(g_noalloc_setup_err[dev], "bafqmc_sweep_noalloc set-up (cudaGetSymbolAddress, LCG table)");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cap));
    if (cap != cudaStreamCaptureStatusNone)
        return fail(BAFQMC_ESTATE, "bafqmc_sweep_noalloc copies host-side set-up data and reads results back on "
                                   "every call; it cannot run inside a stream capture");
    PointHost ph;
    int rc = setup_point(*pt, ph);
    if (rc != BAFQMC_OK) return rc;
    const int n = ph.N, cls = point_class(ph);
    const int stride = bq::kObsScalars + ph.Lq;
    const long long asz = bq::arena_size(n, ph.Nst, bq::class_work_elems(cls));
    // scratch layout: point | chains | scalars | index list | matrices | observables | arenas
    const size_t o_pt = 0;
    const size_t o_ch = align256(o_pt + sizeof(PointDev));
    const size_t o_sc = align256(o_ch + sizeof(ChainDev) * nchains);
    const size_t o_ix = align256(o_sc + sizeof(ChainScalars) * nchains);
    const size_t o_bad = align256(o_ix + sizeof(int) * nchains);
    const size_t o_mt = align256(o_bad + sizeof(int) * nchains);
    const size_t nn = (size_t)n * n;
    const size_t o_ob = align256(o_mt + sizeof(double2) * (2 * nn + ph.Lq));
    const size_t o_ar = align256(o_ob + sizeof(double) * (size_t)nchains * stride);
    const size_t total = o_ar + sizeof(double2) * (size_t)asz * nchains;
    if (total > kNoAllocBytes) {
        char msg[256];
        snprintf(msg, sizeof msg,
                 "bafqmc_sweep_noalloc: %d chains of Ndim=%d, Ltrot=%d need %zu bytes of scratch; the fixed "
                 "array holds %zu bytes (BAFQMC_NOALLOC_MAX_BYTES)",
                 nchains, n, pt->Ltrot, total, kNoAllocBytes);
        return fail(BAFQMC_EARG, msg);
    }
    unsigned char* base = g_noalloc_base[dev];
    // descriptors staged on the host, copied into the array in one transfer
    std::vector<unsigned char> stage(o_ob, 0);
    const PointDev d = point_dev(ph, reinterpret_cast<const double2*>(base + o_mt));
    std::memcpy(stage.data() + o_pt, &d, sizeof d);
    ChainDev* cd = reinterpret_cast<ChainDev*>(stage.data() + o_ch);
    int* ix = reinterpret_cast<int*>(stage.data() + o_ix);
    for (int c = 0; c < nchains; ++c) {
        cd[c].point = 0;
        cd[c].pad = 0;
        cd[c].arena_off = (long long)c * asz;
        cd[c].phi_off = (long long)c * ph.p.Ltrot * ph.Lq * 2;
        ix[c] = c;
    }
    std::memcpy(stage.data() + o_mt, ph.expP.a.data(), sizeof(double2) * nn);
    std::memcpy(stage.data() + o_mt + sizeof(double2) * nn, ph.expM.a.data(), sizeof(double2) * nn);
    std::memcpy(stage.data() + o_mt + 2 * sizeof(double2) * nn, ph.phaseR.data(), sizeof(double2) * ph.Lq);
    CK(cudaMemcpyAsync(base, stage.data(), o_ob, cudaMemcpyHostToDevice, st));
    // the array keeps the previous call's contents: reset what is accumulated
    CK(cudaMemsetAsync(base + o_ob, 0, o_ar - o_ob, st));
    ChainScalars* sc = reinterpret_cast<ChainScalars*>(base + o_sc);
    noalloc_seeds_in<<<(nchains + 127) / 128, 128, 0, st>>>(sc, seeds, nchains);
    CK(cudaGetLastError());
    bq::KernelArgs ka;
    ka.pts = reinterpret_cast<const PointDev*>(base + o_pt);
    ka.chains = reinterpret_cast<const ChainDev*>(base + o_ch);
    ka.nchains = nchains;
    ka.obs_stride = stride;
    ka.arena = reinterpret_cast<double2*>(base + o_ar);
    ka.phi = phi;
    ka.obs = reinterpret_cast<double*>(base + o_ob);
    ka.sc = sc;
    ka.timers = 0;
    ka.mixed = 0;
    const int* d_ix = reinterpret_cast<const int*>(base + o_ix);
    // fields must be finite, as bafqmc_set_state requires
    int* d_bad = reinterpret_cast<int*>(base + o_bad);
    CK(bq::launch_field_check(ka, d_bad, st));
    std::vector<int> bad(nchains);
    CK(cudaMemcpyAsync(bad.data(), d_bad, sizeof(int) * nchains, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int c = 0; c < nchains; ++c)
        if (bad[c])
            return fail(BAFQMC_EARG, "bafqmc_sweep_noalloc: non-finite field value (NaN or Inf) in chain " +
                                         std::to_string(c));
    CK(bq::launch_pre(cls, ka, d_ix, nchains, st));
    CK(bq::launch_bin_reset(ka, st));
    for (int s = 0; s < nsweep; ++s) CK(bq::launch_sweep(cls, ka, d_ix, nchains, st));
    CK(bq::launch_bin_finish(ka, st));
    CK(cudaMemcpyAsync(chain_obs, ka.obs, sizeof(double) * (size_t)nchains * stride, cudaMemcpyDeviceToDevice, st));
    noalloc_seeds_out<<<(nchains + 127) / 128, 128, 0, st>>>(sc, seeds, nchains);
    CK(cudaGetLastError());
    // quarantined chains (status bit 0: a non-finite Green's function)
    std::vector<ChainScalars> scs(nchains);
    CK(cudaMemcpyAsync(scs.data(), sc, sizeof(ChainScalars) * nchains, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    int quarantined = 0;
    for (int c = 0; c < nchains; ++c) quarantined += (scs[c].status & 1) ? 1 : 0;
    return quarantined;
}
