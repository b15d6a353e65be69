// Device-side data layout and per-chain sweep routines for the BAFQMC
// number-conserving solver (src/number_conserving/src/*.f90) and the Nambu
// pairing solver (src/pairing/src/*.f90).
//
// One CTA owns one Markov chain for a whole sweep.  Shared memory holds four
// N x N complex matrices: G, the current U factor of the propagated side, and
// two workspaces that hold e^{-dtau K} / e^{+dtau K} while slices are
// propagated and serve the QR stabilisation at wrap slices.  The stored UDV
// slots, the V/D factors and the fields stay in HBM.
//
// Nambu chains.  The reference's 4Ns matrices (sectors b, c, b^dagger,
// c^dagger) are block diagonal: the kinetic matrix couples only b with
// c^dagger and c with b^dagger (src/pairing/src/non_interact.f90:44-93), the
// HS factors are diagonal, and for real t, Delta and the reference's HS
// constants the {c, b^dagger} block is the complex conjugate of the
// {b, c^dagger} block.  A Nambu chain therefore propagates only the
// {b, c^dagger} block, N = 2Ns, index i = b_i and Ns+i = c^dagger_i.
#pragma once
#include "linalg.cuh"

namespace bq {

constexpr double kZero = 1.0e-10;          // calc_basic.f90:5
constexpr uint32_t kLcgA = 48828125u;       // random.f90:9
constexpr int kMaxPow = 2 * 160 + 2;        // a^k mod 2^31 table for k <= 2*NMAX_ALL + 1

// Observable accumulator layout per chain (obser_equal.f90:6-18 and the bin
// writer fourier_trans.f90:250-348).  Complex values take two slots.
enum ObsIndex {
    O_DENSITY_UP = 0, O_DENSITY_DO, O_DENSITY_TOTAL, O_KINETIC, O_DOUBLEOCC, O_SQUAREOCC,
    O_NUM_UP, O_NUM_DO, O_NUMSQUARE_UP, O_NUMSQUARE_DO, O_ONSITE_N2_UP, O_ONSITE_N2_DO,
    O_INTERACTION, O_ENERGY,
    O_SF_K = 14,        // re, im
    O_PSF_GAMMA = 16,   // re, im
    O_DW_K = 18,        // re, im
    O_DEN_UPUP = 20,    // re, im  (sum over r of den_corr_up(r)/Lq == FFT at k=0)
    O_DEN_DODO = 22,    // re, im
    O_DEN_UPDO = 24,    // re, im
    // written by the Nambu solver only (src/pairing/src/obser_equal.f90:10-15)
    O_DENSITY = 26, O_LOCAL_NUMSQUARE, O_PAIR_EQUAL, O_PAIRING_ENERGY, O_CHEMICAL_ENERGY, O_GRAND_ENERGY,
    O_SITE = 32,        // Lq values of density_site_total
};
constexpr int kObsScalars = 32;

struct PointDev {
    int N, L, Nwrap, Nst, Lq, hasK, Lx, Ly;
    int Ns;         // lattice sites (fields per slice and channel); N = Ns, or 2Ns for a Nambu chain
    int pairing;    // 1: Nambu chain propagating the {b, c^dagger} block
    int active[2];
    int flip[2];    // Nambu: the c^dagger factor of channel ch is e^{-alpha phi} (U2) rather than e^{+alpha phi} (U1)
    double alpha_re[2], alpha_im[2];
    double shiftLoc, U1, U2, RT, mu, Delta;
    const cplx* expP;      // e^{-dtau K}, N*N row-major
    const cplx* expM;      // e^{+dtau K}
    const cplx* phaseR;    // exp(i K.r) for the Lq lattice displacements r (only if hasK)
};

struct ChainScalars {
    uint32_t seed;
    int status;
    long long nc[2], nacc[2];   // current bin, per channel (AccCounter)
    long long nobs;             // measurements in the current bin
    double acc_sum[2];          // sum over bins of nacc/nc (AccCounter%acc)
    double therm_acc_sum[2];    // sum over warm-up sweeps of nacc/nc
    double xmax, xmean;         // stabilisation drift (Prop%Xmaxm, Prop%Xmeanm)
    double logdetM;             // sum log D of the last (I-B) factorisation at tau = beta
    double pad;
    long long cyc[4];           // SM cycles per phase: local updates, slice products, measurement, wraps
    double prop_tot[2];         // proposals over all bins (PhaseCounter%count_proposed)
    double acc_tot[2];          // accepted over all bins (PhaseCounter%count_accepted)
    double glb_prop, glb_acc;   // global moves proposed and accepted (bafqmc_global_shift)
};

struct ChainDev {
    int point;
    int pad;
    long long arena_off;   // in cplx units
    long long phi_off;     // in doubles
};

// Per-chain arena layout (cplx units).
struct Arena {
    cplx *G, *URc, *VRc, *ULc, *VLc, *DRc, *DLc, *slots;
    int N;
    DEVI cplx* URs(int s) const { return slots + (long)s * (4 * N * N + 2 * N); }
    DEVI cplx* VRs(int s) const { return URs(s) + N * N; }
    DEVI cplx* ULs(int s) const { return URs(s) + 2 * N * N; }
    DEVI cplx* VLs(int s) const { return URs(s) + 3 * N * N; }
    DEVI cplx* DRs(int s) const { return URs(s) + 4 * N * N; }
    DEVI cplx* DLs(int s) const { return URs(s) + 4 * N * N + N; }
};

__host__ __device__ inline long long arena_base(int N, int Nst) {
    return 5LL * N * N + 2LL * N + (long long)(Nst + 1) * (4LL * N * N + 2LL * N);
}
// Kernel classes that keep the two workspaces (e^{-+dtau K} during slice
// products, QR workspace at wraps) in HBM append them after the arena:
// work = 2 * NMAX * LD complex values of the class, 0 otherwise.
__host__ __device__ inline long long arena_size(int N, int Nst, long long work) {
    return arena_base(N, Nst) + work;
}

DEVI Arena make_arena(cplx* base, int N) {
    Arena a;
    a.N = N;
    a.G = base;
    a.URc = base + N * N;
    a.VRc = base + 2 * N * N;
    a.ULc = base + 3 * N * N;
    a.VLc = base + 4 * N * N;
    a.DRc = base + 5 * N * N;
    a.DLc = base + 5 * N * N + N;
    a.slots = base + 5 * N * N + 2 * N;
    return a;
}

DEVI uint32_t lcg_mul(uint32_t apow, uint32_t s) {
    return (uint32_t)(((unsigned long long)apow * (unsigned long long)s) & 0x7fffffffull);
}
DEVI double lcg_u(uint32_t s) { return (double)s * (1.0 / 2147483648.0); }

// a^k mod 2^31 by square-and-multiply (any k >= 0).
DEVI uint32_t lcg_pow(unsigned long long k) {
    unsigned long long r = 1, b = kLcgA;
    while (k) {
        if (k & 1ull) r = (r * b) & 0x7fffffffull;
        b = (b * b) & 0x7fffffffull;
        k >>= 1;
    }
    return (uint32_t)r;
}

}  // namespace bq
