// Sweep kernels for the BAFQMC number-conserving and Nambu pairing solvers on
// sm_100a.
//
// One CTA = one Markov chain.  sweep_kernel runs one full sweep (left then
// right traversal of imaginary time, local_sweep.f90:96-134 with is_beta
// = .true.) including every local update, slice propagation, stabilisation
// and equal-time measurement of that chain.  pre_kernel builds the right UDV
// slots and G(beta) (local_sweep.f90:80-94); warmup_kernel is the prior-only
// warm-up (local_sweep.f90:64-78).  Both sweep kernels are instantiated per
// shared-memory size class and per sector (PAIR: Nambu chains).
#include "sweep.cuh"
#include "kernels.h"
#include "linalg_big.cuh"
#include "tc.cuh"

namespace bq {

__constant__ uint32_t c_apow[kMaxPow];   // a^k mod 2^31 for k = 0 .. kMaxPow-1

template <int NMAX> struct Cfg;
// R8 rows per lane and CPS columns per 8-lane segment for the register-resident
// factorisation routines: R8 >= NMAX/8, CPS >= NMAX/(THREADS/8).
// LD: leading dimension of the shared-memory matrices, odd so that a column
// walk over 16-byte elements touches all eight bank groups.  MINB: CTAs per SM for the register
// budget.  GW: the two workspaces live in HBM (after the chain's arena) and
// only G and U in shared memory.
template <> struct Cfg<16> {
    static constexpr bool TCORE = false;
    static constexpr int THREADS = 128, TR = 1, TC = 2, MAXE = 2, KB = 4, R8 = 2, CPS = 1, LD = 17, MINB = 2;
    static constexpr bool GW = false, GG = false;
    static constexpr int RW = 1, CPW = 1;
};
static_assert(16 % 1 == 0 && 16 % 2 == 0, "tile must divide NMAX");
// N <= 36: two CTAs per SM, all four matrices in shared memory.  (Three CTAs
// per SM at 192 threads with the workspaces in HBM measured 42% slower: the
// slice products and wraps slow down more than the third chain adds.)
template <> struct Cfg<36> {
    static constexpr bool TCORE = false;
    static constexpr int THREADS = 256, TR = 2, TC = 3, MAXE = 6, KB = 4, R8 = 5, CPS = 2, LD = 37, MINB = 2;
    static constexpr bool GW = false, GG = false;
    static constexpr int RW = 2, CPW = 1;
};
// N <= 72: G and U in shared memory, the workspaces in HBM (one CTA per SM)
template <> struct Cfg<72> {
    static constexpr bool TCORE = false;
    static constexpr int THREADS = 512, TR = 3, TC = 4, MAXE = 11, KB = 4, R8 = 9, CPS = 2, LD = 73, MINB = 1;
    static constexpr bool GW = true, GG = false;
    static constexpr int RW = 3, CPW = 1;
};
// N <= 144 (up to the 12x12 lattice, number-conserving): G, U, both
// workspaces and a product scratch in HBM after the chain's arena (L2-resident
// while the chain runs), one CTA of 512 threads per SM.  Neither shared memory
// nor the register file holds these n x n matrices, so products loop over
// TR x TC tiles out of place and the factorisations use linalg_big.cuh (one
// warp per column, RW rows per lane, CPW columns at a time).
static_assert(kTcPer * 512 >= 144 * kTcKC, "tensor-core staging: elements per thread must cover a chunk");
template <> struct Cfg<144> {
    static constexpr bool TCORE = true;   // slice products may run on the tensor cores (tc.cuh)
    static constexpr int THREADS = 512, TR = 2, TC = 3, MAXE = 41, KB = 4, R8 = 18, CPS = 3, LD = 145,
                         MINB = 1;
    static constexpr bool GW = true, GG = true;
    static constexpr int RW = 5, CPW = 2;
};
template <int NMAX>
constexpr bool cfg_ok() {
    using C = Cfg<NMAX>;
    return NMAX % C::TR == 0 && NMAX % C::TC == 0 && (C::GG || (NMAX / C::TR) * (NMAX / C::TC) <= C::THREADS) &&
           (!C::GG || (C::RW * 32 >= NMAX && C::THREADS >= NMAX && C::GW)) &&
           C::MAXE * C::THREADS >= NMAX * NMAX && C::R8 * 8 >= NMAX && C::CPS * (C::THREADS / 8) >= NMAX &&
           (C::LD & 1) == 1 && C::LD >= NMAX;
}
static_assert(cfg_ok<16>() && cfg_ok<36>() && cfg_ok<72>() && cfg_ok<144>(),
              "class tiles and register layouts must cover NMAX");
static_assert(36 % 2 == 0 && 36 % 3 == 0, "tile must divide NMAX");
static_assert(Cfg<16>::R8 * 8 >= 16 && Cfg<16>::CPS * (Cfg<16>::THREADS / 8) >= 16, "register layout must cover NMAX");
static_assert(Cfg<36>::R8 * 8 >= 36 && Cfg<36>::CPS * (Cfg<36>::THREADS / 8) >= 36, "register layout must cover NMAX");

// Dynamic shared memory of the sweep kernels.  Every buffer sits at a
// compile-time offset, so device code addresses it without holding pointers.
extern __shared__ __align__(16) unsigned char bq_smem[];

template <int NMAX>
struct Smem {
    static constexpr int kRed = 32 * (Cfg<NMAX>::THREADS / 32);
    static constexpr size_t MM = sizeof(cplx) * NMAX * Cfg<NMAX>::LD, VC = sizeof(cplx) * NMAX, VD = sizeof(double) * NMAX;
    static constexpr bool GW = Cfg<NMAX>::GW;   // workspaces in HBM
    static constexpr bool GG = Cfg<NMAX>::GG;   // G and U in HBM as well
    static constexpr size_t oG = 0, oU = MM, oW1 = 2 * MM, oW2 = 3 * MM;
    static constexpr int KB = Cfg<NMAX>::KB;
    static constexpr size_t oTau = (GG ? 0 : (GW ? 2 : 4)) * MM, oCol = oTau + VC, oRow = oCol + KB * VC, oDelta = oRow + KB * VC;
    static constexpr size_t oDelta2 = oDelta + VC;
    static constexpr size_t oEao = oDelta2 + VC, oEan = oEao + VC, oEbo = oEan + VC, oEbn = oEbo + VC;
    static constexpr size_t oPh = oEbn + VC, oCoef = oPh + VC, oCbc = oCoef + KB * sizeof(cplx);
    static constexpr size_t oP = oCbc + 4 * sizeof(cplx);
    static constexpr size_t oRg = oP + ((sizeof(PointDev) + 15) / 16) * 16;
    static constexpr size_t oU2 = oRg + VD, oPhin = oU2 + VD, oVn1 = oPhin + VD, oVn2 = oVn1 + VD, oD = oVn2 + VD;
    static constexpr size_t oRed = oD + VD, oObs = oRed + sizeof(double) * kRed;
    static constexpr size_t oPiv = oObs + sizeof(double) * (kObsScalars + NMAX);
    static constexpr size_t oIpiv = oPiv + sizeof(int) * NMAX, oAccf = oIpiv + sizeof(int) * NMAX;
    static constexpr size_t oIbc = oAccf + sizeof(int) * NMAX, oSeed = oIbc + 4 * sizeof(int);
    static constexpr size_t oSxy = oSeed + 16;   // site coordinates x | y << 16
    static constexpr size_t oCnt = oSxy + ((sizeof(int) * NMAX + 15) / 16) * 16;   // nacc[2], nc[2], nobs of the sweep
    // tensor-core staging (classes with Cfg::TCORE): A hi | A lo | B hi | B lo, then
    // the MMA barrier, the tensor-memory base, the barrier parity and the on flag
    static constexpr bool TCORE = Cfg<NMAX>::TCORE;
    static constexpr size_t oTc = ((oCnt + 48 + 127) / 128) * 128;
    static constexpr size_t oTcBar = oTc + 2 * kTcABytes + 2 * kTcBBytes;
    static constexpr size_t bytes() { return TCORE ? oTcBar + 32 : oCnt + 48; }

    template <class T>
    static DEVI T* at(size_t off) { return reinterpret_cast<T*>(bq_smem + off); }
    DEVI cplx* G() const { return at<cplx>(oG); }
    DEVI cplx* U() const { return at<cplx>(oU); }
    DEVI cplx* W1() const { return at<cplx>(oW1); }   // shared-memory workspaces (N <= 36 classes)
    DEVI cplx* W2() const { return at<cplx>(oW2); }
    DEVI cplx* tau() const { return at<cplx>(oTau); }
    DEVI cplx* col(int m) const { return at<cplx>(oCol) + m * NMAX; }   // column of the m-th site of a block
    DEVI cplx* row(int m) const { return at<cplx>(oRow) + m * NMAX; }   // row of the m-th site of a block
    DEVI cplx* delta() const { return at<cplx>(oDelta); }
    DEVI cplx* delta2() const { return at<cplx>(oDelta2); }   // Nambu: Delta of the c^dagger index
    DEVI cplx* eao() const { return at<cplx>(oEao); }
    DEVI cplx* ean() const { return at<cplx>(oEan); }
    DEVI cplx* ebo() const { return at<cplx>(oEbo); }
    DEVI cplx* ebn() const { return at<cplx>(oEbn); }
    DEVI cplx* ph() const { return at<cplx>(oPh); }
    DEVI cplx* coef() const { return at<cplx>(oCoef); }
    DEVI cplx* cbc() const { return at<cplx>(oCbc); }
    DEVI PointDev* P() const { return at<PointDev>(oP); }
    DEVI double* rg() const { return at<double>(oRg); }
    DEVI double* u2() const { return at<double>(oU2); }
    DEVI double* phin() const { return at<double>(oPhin); }
    DEVI double* vn1() const { return at<double>(oVn1); }
    DEVI double* vn2() const { return at<double>(oVn2); }
    DEVI double* d() const { return at<double>(oD); }
    DEVI double* red() const { return at<double>(oRed); }
    DEVI double* obs() const { return at<double>(oObs); }
    DEVI int* piv() const { return at<int>(oPiv); }
    DEVI int* ipiv() const { return at<int>(oIpiv); }
    DEVI int* accf() const { return at<int>(oAccf); }
    DEVI int* ibc() const { return at<int>(oIbc); }
    DEVI uint32_t* seed() const { return at<uint32_t>(oSeed); }
    DEVI int* sxy() const { return at<int>(oSxy); }
    DEVI long long* cnt() const { return at<long long>(oCnt); }
    DEVI int* strip_warp() const { return at<int>(oCnt + 40); }
    DEVI uint64_t* tc_mbar() const { return at<uint64_t>(oTcBar); }
    DEVI uint32_t* tc_slot() const { return at<uint32_t>(oTcBar + 8); }
    DEVI uint32_t* tc_phase() const { return at<uint32_t>(oTcBar + 12); }
    DEVI int* tc_on() const { return at<int>(oTcBar + 16); }
    DEVI uint32_t* tc_pending() const { return at<uint32_t>(oTcBar + 20); }   // 2 + parity of a group left in flight
    DEVI int* tc_test() const { return at<int>(oTcBar + 24); }                // the wait-test mode of the products
    DEVI TcBufs tcb() const {
        return TcBufs{at<uint32_t>(oTc), at<uint32_t>(oTc + kTcABytes), at<uint32_t>(oTc + 2 * kTcABytes),
                      at<uint32_t>(oTc + 2 * kTcABytes + kTcBBytes), tc_mbar(), *tc_slot()};
    }
    DEVI QRScratch qr() const { return QRScratch{tau(), piv(), ipiv(), vn1(), vn2(), d(), cbc(), ibc()}; }
};

// green_from_M keeps n complex reciprocals in vn1 | vn2
static_assert(Smem<16>::oVn1 % 16 == 0 && Smem<36>::oVn1 % 16 == 0 && Smem<72>::oVn1 % 16 == 0 &&
                  Smem<144>::oVn1 % 16 == 0 &&
                  Smem<16>::oVn2 == Smem<16>::oVn1 + 8 * 16 && Smem<36>::oVn2 == Smem<36>::oVn1 + 8 * 36 &&
                  Smem<72>::oVn2 == Smem<72>::oVn1 + 8 * 72 && Smem<144>::oVn2 == Smem<144>::oVn1 + 8 * 144,
              "vn1 | vn2 must hold NMAX aligned complex values");
template <int NMAX>
constexpr bool smem_fits() { return Cfg<NMAX>::MINB * (Smem<NMAX>::bytes() + 1024) <= 228 * 1024; }
static_assert(smem_fits<16>() && smem_fits<36>() && smem_fits<72>() && smem_fits<144>(),
              "shared memory per SM for MINB CTAs");

// Per-chain view: the chain's arena base and fields in registers, the point
// parameters in shared memory.
template <int NMAX>
struct Ctx {
    Smem<NMAX> s;
    cplx* abase;
    double* phi;
    ChainScalars* sc;
    cplx* wg;   // HBM region after the arena: W1, W2 (N > 36), then G, U and a product scratch (N > 72)
    int n;
    int sw0;    // the local update's deciding warp
    DEVI const PointDev& P() const { return *s.P(); }
    DEVI Arena A() const { return make_arena(abase, n); }
    DEVI cplx* W1() const {
        if constexpr (Smem<NMAX>::GW) return wg;
        else return s.W1();
    }
    DEVI cplx* W2() const {
        if constexpr (Smem<NMAX>::GW) return wg + NMAX * Cfg<NMAX>::LD;
        else return s.W2();
    }
    DEVI cplx* G() const {
        if constexpr (Smem<NMAX>::GG) return wg + 2 * NMAX * Cfg<NMAX>::LD;
        else return s.G();
    }
    DEVI cplx* U() const {
        if constexpr (Smem<NMAX>::GG) return wg + 3 * NMAX * Cfg<NMAX>::LD;
        else return s.U();
    }
    DEVI cplx* S() const { return wg + 4 * NMAX * Cfg<NMAX>::LD; }   // product scratch (HBM-resident classes)
};

// ---------------------------------------------------------------------------
// Linear algebra per size class: the register-resident 8-lane-segment
// routines of linalg.cuh for the shared-memory classes, the warp-per-column
// routines of linalg_big.cuh (out of place through x.S()) for the HBM class.
template <int NMAX>
DEVI void gemm_any(Ctx<NMAX>& x, cplx* C, MatOp A, MatOp B, int tri = TRI_NONE) {
    using C_ = Cfg<NMAX>;
    if constexpr (C_::GG) {
        gemm_big<C_::TR, C_::TC>(x.n, C_::LD, x.S(), A, B, tri);
        copy_mat(x.n, C_::LD, C, x.S());
    } else {
        gemm_rs<C_::TR, C_::TC>(x.n, C_::LD, C, A, B, tri);
    }
}
template <int NMAX, bool RIGHT_REAL>
DEVI void gemm_real_any(Ctx<NMAX>& x, cplx* C, const void* A, const void* B) {
    using C_ = Cfg<NMAX>;
    if constexpr (C_::GG) {
        gemm_big_real<C_::TR, C_::TC, RIGHT_REAL>(x.n, C_::LD, x.S(), A, B);
        copy_mat(x.n, C_::LD, C, x.S());
    } else {
        gemm_smem_real<C_::TR, C_::TC, RIGHT_REAL>(x.n, C_::LD, C, A, B);
    }
}
template <int NMAX>
DEVI void qrp_any(Ctx<NMAX>& x, cplx* A) {
    using C_ = Cfg<NMAX>;
    if constexpr (C_::GG) {
        // factorised in a column-major copy in S, so each warp's column walk is
        // contiguous; the operations and their order are those of the row-major call
        const int n = x.n;
        cplx* S = x.S();
        for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
            const int r = e / n, c = e - r * n;
            S[c * C_::LD + r] = A[r * C_::LD + c];
        }
        __syncthreads();
        qrp_big<C_::RW, true>(n, C_::LD, S, x.s.qr());
        for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
            const int r = e / n, c = e - r * n;
            A[r * C_::LD + c] = S[c * C_::LD + r];
        }
        __syncthreads();
    } else {
        qrp_inplace<C_::R8, C_::CPS>(x.n, C_::LD, A, x.s.qr());
    }
}
template <int NMAX>
DEVI void form_q_any(Ctx<NMAX>& x, const cplx* F, cplx* Q, bool conjT) {
    using C_ = Cfg<NMAX>;
    if constexpr (C_::GG) {
        copy_col_major(x.n, C_::LD, x.S(), F);
        form_q_big<C_::RW, C_::CPW, true>(x.n, C_::LD, x.S(), x.s.tau(), Q, conjT);
    } else form_q<C_::R8, C_::CPS>(x.n, C_::LD, F, x.s.tau(), Q, conjT);
}
template <int NMAX>
DEVI void apply_qh_left_any(Ctx<NMAX>& x, const cplx* F, cplx* C) {
    using C_ = Cfg<NMAX>;
    if constexpr (C_::GG) {
        copy_col_major(x.n, C_::LD, x.S(), F);
        apply_qh_left_big<C_::RW, C_::CPW, true>(x.n, C_::LD, x.S(), x.s.tau(), C);
    } else apply_qh_left<C_::R8, C_::CPS>(x.n, C_::LD, F, x.s.tau(), C);
}
template <int NMAX>
DEVI void apply_q_right_any(Ctx<NMAX>& x, const cplx* F, cplx* C) {
    using C_ = Cfg<NMAX>;
    if constexpr (C_::GG) {
        copy_col_major(x.n, C_::LD, x.S(), F);
        apply_q_right_big<C_::RW, C_::CPW, true>(x.n, C_::LD, x.S(), x.s.tau(), C);
    } else apply_q_right<C_::R8, C_::CPS>(x.n, C_::LD, F, x.s.tau(), C);
}
template <int NMAX>
DEVI void trsm_left_any(Ctx<NMAX>& x, const cplx* F, const cplx* rinv, const double* rs, cplx* C) {
    using C_ = Cfg<NMAX>;
    if constexpr (C_::GG) {
        copy_col_major(x.n, C_::LD, x.S(), F);
        trsm_left_upper_big<C_::RW, C_::CPW, true>(x.n, C_::LD, x.S(), rinv, rs, C);
    } else trsm_left_upper<C_::R8, C_::CPS>(x.n, C_::LD, F, rinv, rs, C);
}
template <int NMAX>
DEVI void trsm_right_any(Ctx<NMAX>& x, const cplx* F, const cplx* rinv, const double* cs, cplx* C) {
    using C_ = Cfg<NMAX>;
    if constexpr (C_::GG) {
        copy_col_major(x.n, C_::LD, x.S(), F);
        trsm_right_upperH_big<C_::RW, C_::CPW, true>(x.n, C_::LD, x.S(), rinv, cs, C);
    } else trsm_right_upperH<C_::R8, C_::CPS>(x.n, C_::LD, F, rinv, cs, C);
}
template <int NMAX>
DEVI void permute_rows_any(Ctx<NMAX>& x, cplx* C, bool forward) {
    using C_ = Cfg<NMAX>;
    if constexpr (C_::GG) permute_rows_big(x.n, C_::LD, C, x.s.piv(), x.s.ipiv(), forward, x.S());
    else permute_rows<C_::MAXE>(x.n, C_::LD, C, x.s.piv(), x.s.ipiv(), forward);
}
template <int NMAX>
DEVI void permute_cols_any(Ctx<NMAX>& x, cplx* C, bool forward) {
    using C_ = Cfg<NMAX>;
    if constexpr (C_::GG) permute_cols_big(x.n, C_::LD, C, x.s.piv(), x.s.ipiv(), forward, x.S());
    else permute_cols<C_::MAXE>(x.n, C_::LD, C, x.s.piv(), x.s.ipiv(), forward);
}
template <int NMAX>
DEVI void conj_transpose_any(Ctx<NMAX>& x, cplx* A) {
    using C_ = Cfg<NMAX>;
    if constexpr (C_::GG) conj_transpose_big(x.n, C_::LD, A, x.S());
    else conj_transpose_inplace<C_::MAXE>(x.n, C_::LD, A);
}

// One slice product in place: X <- X R (RIGHT) or X <- R X, R = e^{-+dtau K}
// real.  With the mixed-precision option on, classes with tensor-core staging
// run it as tc_product; a product that did not complete within its wait bound
// leaves X unchanged, flags the chain (status bit 2) and the kernel continues
// in FP64 (the tensor cores stay off for the rest of the launch, so the MMA
// barrier's parity bookkeeping is not used again).
template <int NMAX, bool RIGHT>
DEVI void slice_mult(Ctx<NMAX>& x, cplx* X, const double* R) {
    if constexpr (Cfg<NMAX>::TCORE) {
        if (*x.s.tc_on()) {
            if (tc_product(x.n, Cfg<NMAX>::LD, X, R, RIGHT, x.s.tcb(), x.s.tc_phase(), *x.s.tc_test() != 0,
                           x.s.tc_pending()))
                return;
            if (threadIdx.x == 0) {
                *x.s.tc_on() = 0;
                x.sc->status |= 4;
            }
            __syncthreads();
        }
    }
    if constexpr (RIGHT) gemm_real_any<NMAX, true>(x, X, X, R);
    else gemm_real_any<NMAX, false>(x, X, R, X);
}

// Tensor memory and the MMA barrier of a CTA that runs mixed-precision products
// (one CTA per SM in the classes with Cfg::TCORE): allocated after set-up, freed at exit.
template <int NMAX>
DEVI void tc_begin(Ctx<NMAX>& x, const KernelArgs& ka) {
    if constexpr (Cfg<NMAX>::TCORE) {
        if (threadIdx.x == 0) {
            *x.s.tc_on() = ka.mixed ? 1 : 0;
            *x.s.tc_phase() = 0;
            *x.s.tc_pending() = 0;
            *x.s.tc_test() = ka.mixed == 2 ? 1 : 0;
        }
        if (ka.mixed) {
            if (threadIdx.x < 32) tmem_alloc(smem_u32(x.s.tc_slot()), kTcCols);
            if (threadIdx.x == 0) mbar_init(smem_u32(x.s.tc_mbar()), 1);
            tc_fence_before();
        }
        __syncthreads();
        if (ka.mixed) tc_fence_after();
    }
}
// The tensor memory is released only after every MMA group the CTA issued has
// completed: a group that a product gave up on gets one more bounded wait here;
// if it still has not arrived the chain's status gets bit 3.
template <int NMAX>
DEVI void tc_end(Ctx<NMAX>& x, const KernelArgs& ka) {
    if constexpr (Cfg<NMAX>::TCORE) {
        if (ka.mixed) {
            tc_fence_before();
            __syncthreads();
            const uint32_t pend = *x.s.tc_pending();
            if (pend) {
                const bool done = mbar_wait(smem_u32(x.s.tc_mbar()), pend - 2u);
                if (threadIdx.x == 0 && !done) x.sc->status |= 8;
                __syncthreads();
            }
            tc_fence_after();
            if (threadIdx.x < 32) tmem_dealloc(*x.s.tc_slot(), kTcCols);
        }
    }
}

// ---------------------------------------------------------------------------
// small CTA helpers
DEVI void gcopy(cplx* dst, const cplx* src, int count) {
    for (int e = threadIdx.x; e < count; e += blockDim.x) dst[e] = src[e];
}
// identity in an n x n matrix with leading dimension ld
DEVI void set_identity(int n, int ld, cplx* A) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - (e / n) * n;
        A[r * ld + c] = cmk(r == c ? 1.0 : 0.0, 0.0);
    }
}
// dense n x n (global) <-> shared n x n with leading dimension ld
DEVI void sload(int n, int ld, cplx* dst, const cplx* src) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - (e / n) * n;
        dst[r * ld + c] = src[e];
    }
}
DEVI void sstore(int n, int ld, cplx* dst, const cplx* src) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - (e / n) * n;
        dst[e] = src[r * ld + c];
    }
}
DEVI void scopy(int n, int ld, cplx* dst, const cplx* src) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - (e / n) * n;
        dst[r * ld + c] = src[r * ld + c];
    }
}

// e^{-dtau K} (real) into W1 and e^{+dtau K} into W2 as doubles with the
// matrices' leading dimension.
DEVI void sload_real(int n, int ld, double* dst, const cplx* src) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - (e / n) * n;
        dst[r * ld + c] = src[e].x;
    }
}
template <int NMAX>
DEVI void load_expT(Ctx<NMAX>& x) {
    sload_real(x.n, Cfg<NMAX>::LD, reinterpret_cast<double*>(x.W1()), x.P().expP);
    sload_real(x.n, Cfg<NMAX>::LD, reinterpret_cast<double*>(x.W2()), x.P().expM);
    __syncthreads();
}

// ---------------------------------------------------------------------------
// local update of one channel over all sites of one slice, fused with the
// V-wrap of G (LocalU_prop_L / LocalU_prop_R, localU.f90:79-113, and
// LocalU_metro, localU.f90:31-77).
//
// Sites are strictly sequential.  They are taken in blocks of KB consecutive
// sites.  Within a block one warp runs the sites one after another, with
// warp-level synchronisation only: for each site it wraps and records the
// site's column and row, makes the Metropolis decision (every lane computes
// the same one), and applies the rank-1 update to the rows and columns of the
// block's sites -- the only elements the block's later sites read.  After the
// block, the whole CTA adds the block's KB rank-1 terms to the remaining
// elements, which the wraps of the block's sites do not touch.  The terms are
// the reference's ZGERU updates; only the order of the additions changes.

// e^{+alpha phi} and e^{-alpha phi} for the HS coupling alpha = ar + i ai of one
// channel, which the reference makes purely real (U2) or purely imaginary (U1)
// (operator_Hubbard.f90:36-43): a real alpha needs only exp, an imaginary one
// one sincos with e^{-i theta} = conj(e^{i theta}).
DEVI void hs_factors(double ar, double ai, double p, cplx& ep, cplx& em) {
    if (ai == 0.0) {
        ep = cmk(exp(ar * p), 0.0);
        em = cmk(exp(-(ar * p)), 0.0);
    } else if (ar == 0.0) {
        double sn, cs;
        sincos(ai * p, &sn, &cs);
        ep = cmk(cs, sn);
        em = cmk(cs, -sn);
    } else {
        ep = cexpz(cmk(ar * p, ai * p));
        em = cexpz(cmk(-(ar * p), -(ai * p)));
    }
}
// e_new / e_old for those factors: a real quotient, or e_new conj(e_old) on the unit circle.
DEVI cplx ratio_unit(double ar, double ai, cplx en, cplx eo) {
    if (ai == 0.0) return cmk(en.x / eo.x, 0.0);
    if (ar == 0.0) return cmulcj(en, eo);
    return cdiv(en, eo);
}

// Metropolis ratio for the (wrapped) diagonal element gjj: ratio_det = 1/w,
// w = 1 + Delta (1 - G_jj); accept if r_gauss |ratio_det|^2 > u; on accept the
// rank-1 coefficient is -ratio_det * Delta (localU.f90:56-71).
DEVI bool metro_ratio(cplx d, double rg, double u, cplx gjj, cplx& coef) {
    const cplx w = cmk(1.0 + (d.x * (1.0 - gjj.x) + d.y * gjj.y), d.y * (1.0 - gjj.x) - d.x * gjj.y);
    const double inv = 1.0 / (w.x * w.x + w.y * w.y);
    const bool accept = rg * inv > u;
    const cplx t = cmulcj(d, w);   // Delta * conj(w)
    coef = accept ? cmk(-t.x * inv, -t.y * inv) : cmk(0.0, 0.0);
    return accept;
}

// prop_channel visits the sites of a channel in blocks of KB.  Per block:
//  1. lead_block: one warp makes the block's Metropolis decisions in visiting
//     order on the block's kb x kb submatrix of G, held in registers, applying
//     each accepted rank-1 term to the submatrix (no barrier per site);
//  2. block_vectors: the full update vectors of the block from the recorded
//     coefficients and block values;
//  3. rank_tile / rank_rows: G += sum_m X_m Y_m^T on every element.
// The rank-1 term of a site i (localU.f90:56-71, ZGERU) is
// G <- G + coef G(:,i) (e_i - G(i,:))^T.  For any diagonal E it satisfies
// F_i(E G E^-1) = E F_i(G) E^-1, and coef depends only on G(i,i), which E
// leaves unchanged, so the wraps of the sites (row i by e^{a phi_i}, column i
// by e^{-a phi_i} before the decision in the right traversal, with the old
// field; row i by e^{-a phi_i} and column i by e^{a phi_i} after it in the left
// traversal, with the final field) commute with the updates and are applied
// once, as one diagonal similarity, in the last block's rank pass.

static_assert(Cfg<16>::KB * Cfg<16>::KB <= 16 && Cfg<36>::KB * Cfg<36>::KB <= 16 && Cfg<72>::KB * Cfg<72>::KB <= 16 &&
                  Cfg<144>::KB * Cfg<144>::KB <= 16,
              "the block records (tau, delta2, the vn1 | vn2 snapshot) hold KB x KB values in NMAX >= 16 entries, "
              "and the lead warp one element per lane");

// the channel's deferred wrap: factor of row r and of column c
template <int NMAX, bool LEFT>
DEVI cplx wrap_row(const Smem<NMAX>& s, int r) {
    if constexpr (LEFT) return s.accf()[r] ? s.ebn()[r] : s.ebo()[r];
    else return s.eao()[r];
}
template <int NMAX, bool LEFT>
DEVI cplx wrap_col(const Smem<NMAX>& s, int c) {
    if constexpr (LEFT) return s.accf()[c] ? s.ean()[c] : s.eao()[c];
    else return s.ebo()[c];
}

// Step 1, by the lead warp (warp sw0 of the CTA).  Lane l < KB*KB holds
// the element (l / KB, l % KB) of the block's kb x kb submatrix of the current
// G; the decisions run in visiting order, every lane computing the same
// Metropolis ratio from the diagonal element it receives by shuffle.  Records
// per visited slot m: coef (coef()), X_m on the later block sites (xb = tau(),
// [m][a], a > m) and Y_m on them (yb = delta2(), [m][b], b > m), where
// X_m = coef G_{m-1}(:, i_m) and Y_m = e_{i_m} - G_{m-1}(i_m, :)^T.  Only the
// trailing submatrix (sites after m) is updated: nothing later reads the
// rest.  A rejected site has coef = 0, so its update adds exact zeros.

// the submatrix at block start k0 into the QR norm vectors (vn1 | vn2, free
// during local updates); the lead warp reads it back after the barrier, when
// the rank pass may already be writing G
template <int NMAX, bool LEFT>
DEVI void block_snapshot(const Smem<NMAX>& s, const cplx* G, int n, int k0, int kb) {
    constexpr int KB = Cfg<NMAX>::KB, LD = Cfg<NMAX>::LD;
    const int lane = threadIdx.x & 31;
    if (lane < KB * KB) {
        const int a = lane / KB, b = lane % KB;
        const int sa = LEFT ? n - 1 - (k0 + min(a, kb - 1)) : k0 + min(a, kb - 1);
        const int sb = LEFT ? n - 1 - (k0 + min(b, kb - 1)) : k0 + min(b, kb - 1);
        reinterpret_cast<cplx*>(s.vn1())[lane] = (a < kb && b < kb) ? G[sa * LD + sb] : cmk(0.0, 0.0);
    }
}

DEVI cplx shfl_c(cplx v, int src) {
    return cmk(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// The snapshot, the previous block's kbp rank terms (in the order and with the
// operations of the rank pass, so the lanes hold exactly the G the pass
// writes there), then the decisions.  Returns the accepted count.
template <int NMAX, bool LEFT>
COLD long long lead_block(Ctx<NMAX> x, int n, int k0, int kb, int kbp) {
    constexpr int KB = Cfg<NMAX>::KB;
    const auto& s = x.s;
    const int lane = threadIdx.x & 31;
    const bool own = lane < KB * KB;
    const int a = own ? lane / KB : KB - 1, b = lane % KB;
    cplx* xb = s.tau();
    cplx* yb = s.delta2();
    cplx g = reinterpret_cast<const cplx*>(s.vn1())[a * KB + b];
    if (kbp > 0 && a < kb && b < kb) {
        const int sa = LEFT ? n - 1 - (k0 + a) : k0 + a, sb = LEFT ? n - 1 - (k0 + b) : k0 + b;
#pragma unroll
        for (int m = 0; m < KB; ++m) {
            if (m >= kbp) break;
            g = cfma(s.col(m)[sa], s.row(m)[sb], g);
        }
    }
    long long nacc = 0;
#pragma unroll
    for (int m = 0; m < KB; ++m) {
        if (m >= kb) break;
        const int i = LEFT ? n - 1 - (k0 + m) : k0 + m;
        const cplx gmm = shfl_c(g, m * KB + m);
        const cplx gam = shfl_c(g, a * KB + m);
        const cplx gmb = shfl_c(g, m * KB + b);
        cplx coef;
        const bool accept = metro_ratio(s.delta()[i], s.rg()[i], s.u2()[i], gmm, coef);
        const cplx xv = cmul(coef, gam);
        const cplx yv = cmk(-gmb.x, -gmb.y);
        if (a > m && b > m) g = cfma(xv, yv, g);
        if (own && b == m && a > m) xb[m * KB + a] = xv;
        if (own && a == m && b > m) yb[m * KB + b] = yv;
        if (lane == 0) {
            s.accf()[i] = accept ? 1 : 0;
            s.coef()[m] = coef;
        }
        nacc += accept ? 1 : 0;
    }
    return nacc;
}

// Step 2.  X_k(r) = coef_k (G(r, i_k) + sum_{j<k} X_j(r) Y_j(i_k)) into col(k),
// Y_k(c) = delta(c, i_k) - (G(i_k, c) + sum_{j<k} X_j(i_k) Y_j(c)) into row(k);
// threads 0..n-1 build the X rows, n..2n-1 the Y columns.
template <int NMAX, bool LEFT>
DEVI void block_vectors(const Ctx<NMAX>& x, const cplx* G, int n, int k0, int kb) {
    constexpr int KB = Cfg<NMAX>::KB, LD = Cfg<NMAX>::LD;
    const auto& s = x.s;
    const cplx* xb = s.tau();
    const cplx* yb = s.delta2();
    for (int t = threadIdx.x; t < 2 * n; t += blockDim.x) {
        const bool isx = t < n;
        const int v = isx ? t : t - n;
        cplx acc[KB];
#pragma unroll
        for (int k = 0; k < KB; ++k) {
            if (k >= kb) break;
            const int ik = LEFT ? n - 1 - (k0 + k) : k0 + k;
            cplx a = isx ? G[v * LD + ik] : G[ik * LD + v];
#pragma unroll
            for (int j = 0; j < k; ++j) a = isx ? cfma(acc[j], yb[j * KB + k], a) : cfma(xb[j * KB + k], acc[j], a);
            if (isx) {
                acc[k] = cmul(s.coef()[k], a);
                s.col(k)[v] = acc[k];
            } else {
                acc[k] = cmk((v == ik ? 1.0 : 0.0) - a.x, -a.y);
                s.row(k)[v] = acc[k];
            }
        }
    }
}

// Step 3 on one TR x TC tile at (r0, c0): G(r,c) += sum_m X_m(r) Y_m(c), then
// (WRAP, the channel's last block) the deferred wrap.  Rejected slots have
// X_m = 0 and add exact zeros; coef() is not read (the lead thread is already
// writing the next block's coefficients).
template <int NMAX, bool LEFT, bool WRAP>
DEVI void rank_tile(const Ctx<NMAX>& x, cplx* G, int n, int kb, int r0, int c0) {
    constexpr int TR = Cfg<NMAX>::TR, TC = Cfg<NMAX>::TC, KB = Cfg<NMAX>::KB, LD = Cfg<NMAX>::LD;
    const auto& s = x.s;
    cplx g[TR][TC];
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) g[a][b] = G[min(r0 + a, n - 1) * LD + min(c0 + b, n - 1)];
#pragma unroll
    for (int m = 0; m < KB; ++m) {
        if (m >= kb) break;
        cplx cr[TR], y[TC];
#pragma unroll
        for (int a = 0; a < TR; ++a) cr[a] = s.col(m)[min(r0 + a, n - 1)];
#pragma unroll
        for (int b = 0; b < TC; ++b) y[b] = s.row(m)[min(c0 + b, n - 1)];
#pragma unroll
        for (int a = 0; a < TR; ++a)
#pragma unroll
            for (int b = 0; b < TC; ++b) g[a][b] = cfma(cr[a], y[b], g[a][b]);
    }
    if constexpr (WRAP) {
        cplx fb[TC];
#pragma unroll
        for (int b = 0; b < TC; ++b) fb[b] = wrap_col<NMAX, LEFT>(s, min(c0 + b, n - 1));
#pragma unroll
        for (int a = 0; a < TR; ++a) {
            const cplx fa = wrap_row<NMAX, LEFT>(s, min(r0 + a, n - 1));
#pragma unroll
            for (int b = 0; b < TC; ++b) g[a][b] = cmul(cmul(g[a][b], fa), fb[b]);
        }
    }
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b)
            if (r0 + a < n && c0 + b < n) G[(r0 + a) * LD + c0 + b] = g[a][b];
}

// Step 3 for the classes whose G lives in HBM/L2.  Items are (32-column chunk,
// PR-row block): a warp's load or store of one row of an item is a coalesced
// 512-byte segment.  Warp w (of nw, the lead's warp excluded) takes items
// w, w + nw, ...
template <int NMAX, bool LEFT, bool WRAP>
DEVI void rank_rows(const Ctx<NMAX>& x, cplx* G, int n, int kb, int w, int nw) {
    constexpr int KB = Cfg<NMAX>::KB, LD = Cfg<NMAX>::LD, PR = 9;
    const auto& s = x.s;
    const int lane = threadIdx.x & 31;
    const int nch = (n + 31) >> 5, items = nch * ((n + PR - 1) / PR);
    for (int it = w; it < items; it += nw) {
        const int c = (it % nch) * 32 + lane, rb = (it / nch) * PR;
        if (c >= n) continue;
        cplx g[PR];
#pragma unroll
        for (int a = 0; a < PR; ++a) g[a] = G[min(rb + a, n - 1) * LD + c];
#pragma unroll
        for (int m = 0; m < KB; ++m) {
            if (m >= kb) break;
            const cplx y = s.row(m)[c];
            const cplx* cr = s.col(m);
#pragma unroll
            for (int a = 0; a < PR; ++a) g[a] = cfma(cr[min(rb + a, n - 1)], y, g[a]);
        }
        if constexpr (WRAP) {
            const cplx fb = wrap_col<NMAX, LEFT>(s, c);
#pragma unroll
            for (int a = 0; a < PR; ++a) g[a] = cmul(cmul(g[a], wrap_row<NMAX, LEFT>(s, min(rb + a, n - 1))), fb);
        }
#pragma unroll
        for (int a = 0; a < PR; ++a)
            if (rb + a < n) G[(rb + a) * LD + c] = g[a];
    }
}

template <int NMAX, bool LEFT>
COLD void prop_channel(Ctx<NMAX> x, int ch, int slice) {
    constexpr int TR = Cfg<NMAX>::TR, TC = Cfg<NMAX>::TC, KB = Cfg<NMAX>::KB, LD = Cfg<NMAX>::LD;
    auto& s = x.s;
    const int n = x.n, tid = threadIdx.x;
    const double ar = x.P().alpha_re[ch], ai = x.P().alpha_im[ch];
    const double shift = fabs(x.P().shiftLoc);
    const uint32_t s0 = *s.seed();
    double* phis = x.phi + (long)slice * n * 2;
    cplx* G = x.G();

    // per-site proposals; draw order follows the visiting order of the sites
    for (int i = tid; i < n; i += blockDim.x) {
        const int m = LEFT ? (n - 1 - i) : i;
        const double xflip = lcg_u(lcg_mul(c_apow[2 * m + 1], s0));
        const double rnd = lcg_u(lcg_mul(c_apow[2 * m + 2], s0));
        const double po = phis[i * 2 + ch];
        const double xdif = (xflip - 0.5) * shift;
        const double pn = po + xdif;
        const double go = exp(-0.5 * po * po), gn = exp(-0.5 * pn * pn);
        cplx eo, en, ebo, ebn;
        hs_factors(ar, ai, po, eo, ebo);
        hs_factors(ar, ai, pn, en, ebn);
        s.eao()[i] = eo;
        s.ean()[i] = en;
        s.ebo()[i] = ebo;
        s.ebn()[i] = ebn;
        s.delta()[i] = csub(ratio_unit(ar, ai, en, eo), cmk(1.0, 0.0));
        s.rg()[i] = gn / go;
        s.u2()[i] = rnd;
        s.phin()[i] = pn;
        s.accf()[i] = 0;
    }
    __syncthreads();

    // Blocks of KB sites in visiting order.  The lead warp (warp sw0) decides
    // block b + 1 while the other warps run block b's rank pass: it
    // copies block b + 1's submatrix during block b's vector step (G is not
    // written then) and adds block b's terms itself, exactly as the pass does.  The last block's pass applies the channel's deferred wrap.
    constexpr int NT = Cfg<NMAX>::THREADS;
    const bool lead = tid == 32 * x.sw0;
    const int warp = tid >> 5;
    const bool lwarp = warp == x.sw0;
    const int rt = tid - (warp > x.sw0 ? 32 : 0);   // rank-pass thread index (lead warp excluded)
    const int ncg = (n + TC - 1) / TC, ntiles = ncg * ((n + TR - 1) / TR);
    long long nacc = 0;   // accepted proposals, counted by the lead
    if (lwarp) {
        block_snapshot<NMAX, LEFT>(s, G, n, 0, min(KB, n));
        __syncwarp();
        const long long c = lead_block<NMAX, LEFT>(x, n, 0, min(KB, n), 0);
        if (lead) nacc += c;
    }
    __syncthreads();
    for (int k0 = 0; k0 < n; k0 += KB) {
        const int kb = min(KB, n - k0), k1 = k0 + KB, kb1 = min(KB, n - k1);
        const bool more = k1 < n;
        block_vectors<NMAX, LEFT>(x, G, n, k0, kb);
        if (lwarp && more) block_snapshot<NMAX, LEFT>(s, G, n, k1, kb1);
        __syncthreads();
        if (lwarp) {
            if (more) {
                const long long c = lead_block<NMAX, LEFT>(x, n, k1, kb1, kb);
                if (lead) nacc += c;
            }
        } else if constexpr (Cfg<NMAX>::GG) {
            const int w = warp - (warp > x.sw0 ? 1 : 0), nw = NT / 32 - 1;
            if (more) rank_rows<NMAX, LEFT, false>(x, G, n, kb, w, nw);
            else rank_rows<NMAX, LEFT, true>(x, G, n, kb, w, nw);
        } else {
            for (int tt = rt; tt < ntiles; tt += NT - 32) {
                const int r0 = (tt / ncg) * TR, c0 = (tt % ncg) * TC;
                if (more) rank_tile<NMAX, LEFT, false>(x, G, n, kb, r0, c0);
                else rank_tile<NMAX, LEFT, true>(x, G, n, kb, r0, c0);
            }
        }
        __syncthreads();
    }
    // accepted fields, counters, seed, and the U factor wrap with the final fields
    for (int i = tid; i < n; i += blockDim.x)
        if (s.accf()[i]) phis[i * 2 + ch] = s.phin()[i];
    if (tid == 32 * x.sw0) {   // the lead thread: AccCounter%count, kept in shared memory
        s.cnt()[ch] += nacc;
        s.cnt()[2 + ch] += n;
        *s.seed() = lcg_mul(c_apow[2 * n], s0);
    }
    {
        constexpr int MAXE = Cfg<NMAX>::MAXE, T = Cfg<NMAX>::THREADS;
        int r = tid / n, c = tid - (tid / n) * n;
        const int dr = T / n, dc = T - (T / n) * n;
#pragma unroll
        for (int k = 0; k < MAXE; ++k) {
            const int e = tid + k * T;
            if (e < n * n) {
                const int site = LEFT ? c : r;
                const cplx f = s.accf()[site] ? s.ean()[site] : s.eao()[site];
                x.U()[r * LD + c] = cmul(x.U()[r * LD + c], f);
            }
            c += dc;
            r += dr;
            if (c >= n) {
                c -= n;
                ++r;
            }
        }
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Nambu local update of one channel over all sites of one slice, fused with
// the V-wrap of G (LocalU_prop_L / LocalU_prop_R and LocalU_metro,
// src/pairing/src/localU.f90:33-149), on the {b, c^dagger} block.
//
// For site i the reference forms the 4x4 P = I + Delta (I - G[isec,isec]) over
// the sectors b, c, b^dagger, c^dagger of the site, takes
// ratio_det = det(P)^(-1/2), and on acceptance applies the rank-4 update
// G -= G[:,isec] P^{-1} Delta (I[isec,:] - G[isec,:]).  With the block
// structure P splits into the 2x2 block P1 on {b_i, c^dagger_i} and its
// complex conjugate on {c_i, b^dagger_i}, so det(P) = |det P1|^2 (real and
// positive: ratio_det = 1/|det P1|, and the ratio's phase that PhaseCounter
// records is zero), and the update of the block is the rank-2 term
// G1 -= G1[:,s] P1^{-1} D1 (I[s,:] - G1[s,:]), s = (i, Ns+i).
//
// Sites are sequential.  Every thread keeps the same MAXE elements of G in
// registers for the whole slice; per site the owners of rows and columns i
// and Ns+i stage them in shared memory (double-buffered by site parity), one
// barrier, then every thread makes the same decision from the staged 2x2 and
// updates its own elements.
template <int NMAX, bool LEFT>
COLD void prop_channel_pair(Ctx<NMAX> x, int ch, int slice) {
    constexpr int MAXE = Cfg<NMAX>::MAXE, LD = Cfg<NMAX>::LD;
    auto& s = x.s;
    const int n = x.n, ns = x.P().Ns, tid = threadIdx.x;
    const double ar = x.P().alpha_re[ch], ai = x.P().alpha_im[ch];
    const double shift = fabs(x.P().shiftLoc);
    const bool flip = x.P().flip[ch] != 0;
    const bool total = (ch == 1);
    const uint32_t s0 = *s.seed();
    double* phis = x.phi + (long)slice * ns * 2;
    cplx* G = x.G();

    // per-site proposals (opU_get_delta, src/pairing/src/operator_Hubbard.f90:100-137)
    for (int i = tid; i < ns; i += blockDim.x) {
        const int m = LEFT ? (ns - 1 - i) : i;
        const double xflip = lcg_u(lcg_mul(c_apow[2 * m + 1], s0));
        const double rnd = lcg_u(lcg_mul(c_apow[2 * m + 2], s0));
        const double po = phis[i * 2 + ch];
        const double pn = po + (xflip - 0.5) * shift;
        const double go = exp(-0.5 * po * po), gn = exp(-0.5 * pn * pn);
        const cplx eo = cexpz(cmk(ar * po, ai * po)), en = cexpz(cmk(ar * pn, ai * pn));
        const double dphi = pn - po;
        const cplx dp = csub(cexpz(cmk(ar * dphi, ai * dphi)), cmk(1.0, 0.0));
        const cplx dm = csub(cexpz(cmk(-(ar * dphi), -(ai * dphi))), cmk(1.0, 0.0));
        s.eao()[i] = eo;
        s.ean()[i] = en;
        s.ebo()[i] = cexpz(cmk(-(ar * po), -(ai * po)));
        s.ebn()[i] = cexpz(cmk(-(ar * pn), -(ai * pn)));
        s.delta()[i] = dp;                  // b_i: e^{+alpha dphi} - 1 in both channels
        s.delta2()[i] = flip ? dm : dp;     // c^dagger_i
        // |ratio_gaussian * ratio_constant|; ratio_constant = e^{alpha(phi_old - phi_new)} for U2
        const double rc = total ? cabsv(cdiv(eo, en)) : 1.0;
        s.rg()[i] = (gn / go) * rc;
        s.u2()[i] = rnd;
        s.phin()[i] = pn;
        s.accf()[i] = 0;
    }
    __syncthreads();

    cplx g[MAXE];
    int er[MAXE], ec[MAXE];
    long long nacc = 0;   // accepted proposals, counted by thread 0
#pragma unroll
    for (int k = 0; k < MAXE; ++k) {
        const int e = tid + k * blockDim.x;
        er[k] = (e < n * n) ? e / n : -1;
        ec[k] = (e < n * n) ? e - (e / n) * n : -1;
        g[k] = (e < n * n) ? G[er[k] * LD + ec[k]] : cmk(0.0, 0.0);
    }
    for (int q = 0; q < ns; ++q) {
        const int i = LEFT ? ns - 1 - q : q;
        const int a = i, b = ns + i;
        const int buf = (q & 1) * 2;
        cplx* xa = s.col(buf);
        cplx* xb = s.col(buf + 1);
        cplx* ya = s.row(buf);
        cplx* yb = s.row(buf + 1);
        if (!LEFT) {   // opU_mmult_R(+1) then opU_mmult_L(-1) with the current field
            const cplx ep = s.eao()[i], em = s.ebo()[i];
#pragma unroll
            for (int k = 0; k < MAXE; ++k) {
                if (er[k] == a) g[k] = cmul(ep, g[k]);
                else if (er[k] == b) g[k] = cmul(flip ? em : ep, g[k]);
                if (ec[k] == a) g[k] = cmul(g[k], em);
                else if (ec[k] == b) g[k] = cmul(g[k], flip ? ep : em);
            }
        }
#pragma unroll
        for (int k = 0; k < MAXE; ++k) {
            if (ec[k] == a) xa[er[k]] = g[k];
            if (ec[k] == b) xb[er[k]] = g[k];
            if (er[k] == a) ya[ec[k]] = g[k];
            if (er[k] == b) yb[ec[k]] = g[k];
        }
        __syncthreads();
        // P1 = I + D1 (I - G1[s,s]);  accept if |rg rc| / |det P1| > u
        const cplx d0 = s.delta()[i], d1 = s.delta2()[i];
        const cplx gaa = ya[a], gab = ya[b], gba = yb[a], gbb = yb[b];
        const cplx p00 = cadd(cmk(1.0, 0.0), cmul(d0, cmk(1.0 - gaa.x, -gaa.y)));
        const cplx p01 = cmul(d0, cmk(-gab.x, -gab.y));
        const cplx p10 = cmul(d1, cmk(-gba.x, -gba.y));
        const cplx p11 = cadd(cmk(1.0, 0.0), cmul(d1, cmk(1.0 - gbb.x, -gbb.y)));
        const cplx det = csub(cmul(p00, p11), cmul(p01, p10));
        const double det2 = det.x * det.x + det.y * det.y;
        const bool accept = s.rg()[i] / sqrt(det2) > s.u2()[i];
        if (tid == 0) {
            s.accf()[i] = accept ? 1 : 0;
            nacc += accept ? 1 : 0;
        }
        if (accept) {
            // M = P1^{-1} D1, P1^{-1} = adj(P1) conj(det) / |det|^2
            const cplx id = cmk(det.x / det2, -det.y / det2);
            const cplx m00 = cmul(cmul(p11, id), d0);
            const cplx m01 = cmul(cmul(cmk(-p01.x, -p01.y), id), d1);
            const cplx m10 = cmul(cmul(cmk(-p10.x, -p10.y), id), d0);
            const cplx m11 = cmul(cmul(p00, id), d1);
#pragma unroll
            for (int k = 0; k < MAXE; ++k) {
                if (er[k] < 0) continue;
                const int r = er[k], c = ec[k];
                const cplx ca = xa[r], cb = xb[r];
                const cplx x0 = cadd(cmul(ca, m00), cmul(cb, m10));
                const cplx x1 = cadd(cmul(ca, m01), cmul(cb, m11));
                const cplx y0 = cmk(((c == a) ? 1.0 : 0.0) - ya[c].x, -ya[c].y);
                const cplx y1 = cmk(((c == b) ? 1.0 : 0.0) - yb[c].x, -yb[c].y);
                g[k] = csub(g[k], cadd(cmul(x0, y0), cmul(x1, y1)));
            }
        }
        if (LEFT) {   // opU_mmult_L(+1) then opU_mmult_R(-1) with the final field
            const cplx ep = accept ? s.ean()[i] : s.eao()[i];
            const cplx em = accept ? s.ebn()[i] : s.ebo()[i];
#pragma unroll
            for (int k = 0; k < MAXE; ++k) {
                if (ec[k] == a) g[k] = cmul(g[k], ep);
                else if (ec[k] == b) g[k] = cmul(g[k], flip ? em : ep);
                if (er[k] == a) g[k] = cmul(em, g[k]);
                else if (er[k] == b) g[k] = cmul(flip ? ep : em, g[k]);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < MAXE; ++k)
        if (er[k] >= 0) G[er[k] * LD + ec[k]] = g[k];
    __syncthreads();
    for (int i = tid; i < ns; i += blockDim.x)
        if (s.accf()[i]) phis[i * 2 + ch] = s.phin()[i];
    if (tid == 0) {
        s.cnt()[ch] += nacc;
        s.cnt()[2 + ch] += ns;
        *s.seed() = lcg_mul(c_apow[2 * ns], s0);
    }
    // U_L columns (left) or U_R rows (right) of both indices of every site, final fields
#pragma unroll
    for (int k = 0; k < MAXE; ++k) {
        const int e = tid + k * blockDim.x;
        if (e < n * n) {
            const int idx = LEFT ? ec[k] : er[k];
            const int site = idx < ns ? idx : idx - ns;
            const bool acc = s.accf()[site] != 0;
            const cplx ep = acc ? s.ean()[site] : s.eao()[site];
            const cplx em = acc ? s.ebn()[site] : s.ebo()[site];
            const cplx f = (idx >= ns && flip) ? em : ep;
            cplx* u = x.U() + er[k] * LD + ec[k];
            *u = LEFT ? cmul(*u, f) : cmul(f, *u);
        }
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// propT_L / propT_R (multiply.f90:72-86): G <- e^{+dK} G e^{-dK}, U_L <- U_L e^{-dK}
// for the left traversal; G <- e^{-dK} G e^{+dK}, U_R <- e^{-dK} U_R for the
// right.  e^{-dtau K} is in W1, e^{+dtau K} in W2.
template <int NMAX, bool LEFT>
COLD void slice_products(Ctx<NMAX> x) {
    auto& s = x.s;
    const int n = x.n;
    const double* P = reinterpret_cast<const double*>(x.W1());   // e^{-dtau K}, real
    const double* M = reinterpret_cast<const double*>(x.W2());   // e^{+dtau K}, real
    if (LEFT) {
        slice_mult<NMAX, true>(x, x.G(), P);
        slice_mult<NMAX, false>(x, x.G(), M);
        slice_mult<NMAX, true>(x, x.U(), P);
    } else {
        slice_mult<NMAX, false>(x, x.G(), P);
        slice_mult<NMAX, true>(x, x.G(), M);
        slice_mult<NMAX, false>(x, x.U(), P);
    }
}

// ---------------------------------------------------------------------------
// equal-time estimators (Obs_equal_calc, obser_equal.f90:95-198).  The c
// flavour's Green's function is the complex conjugate of the b flavour's
// (obser_equal.f90:112-113), so every c-flavour sum is the conjugate of the
// b-flavour sum and is not recomputed.  The K-point phase depends only on the
// displacement r = i - j, so it comes from an Lq-entry table in shared memory.
template <int NMAX>
COLD void measure(Ctx<NMAX> x) {
    constexpr int LD = Cfg<NMAX>::LD;
    auto& s = x.s;
    const PointDev& P = x.P();
    const int n = x.n, tid = threadIdx.x, lx = P.Lx, ly = P.Ly;
    const double lq = (double)P.Lq, lq2 = lq * lq;
    const cplx* G = x.G();
    const cplx* ph = s.ph();
    const bool hasK = P.hasK;
    // v: 0 sum Re(t_up), 1 sum |Gc|^2, 2-3 sf_K, 4-5 dw_K, 6-7 sum t_up, 8-9 sum du_i conj(du_j),
    //    10 kinetic, 11 sum Re du, 12 sum |du|^2, 13 sum Re du^2
    double v[14];
#pragma unroll
    for (int k = 0; k < 14; ++k) v[k] = 0.0;
    const int* sxy = s.sxy();
    const int T = blockDim.x, di = T / n, dj = T - (T / n) * n;
    int i = tid / n, j = tid - (tid / n) * n;
    for (int e = tid; e < n * n; e += T) {
        const cplx a = G[i * LD + j];                 // Grup(i,j)
        cplx gc = G[j * LD + i];                      // Grupc(i,j) = G(j,i) - delta_ij
        if (i == j) gc.x -= 1.0;
        const cplx dui = cmk(G[i * LD + i].x - 1.0, G[i * LD + i].y);
        const cplx duj = cmk(G[j * LD + j].x - 1.0, G[j * LD + j].y);
        const cplx tup = cadd(cmul(dui, duj), cmul(gc, a));   // b-flavour density correlator
        const cplx tud = cmulcj(dui, duj);                     // du_i * dd_j
        v[0] += tup.x;
        v[1] += gc.x * gc.x + gc.y * gc.y;
        v[6] += tup.x;
        v[7] += tup.y;
        v[8] += tud.x;
        v[9] += tud.y;
        if (hasK) {
            const int pi = sxy[i], pj = sxy[j];
            int dx = (pi & 0xffff) - (pj & 0xffff), dy = (pi >> 16) - (pj >> 16);
            dx += (dx < 0) ? lx : 0;
            dy += (dy < 0) ? ly : 0;
            const cplx p = ph[dy * lx + dx];
            const double sfr = 2.0 * gc.x;                     // Grupc + Grdoc
            const double dwr = 2.0 * tup.x + 2.0 * tud.x;      // t_up + t_do + du_i dd_j + dd_i du_j
            v[2] += p.x * sfr;
            v[3] += p.y * sfr;
            v[4] += p.x * dwr;
            v[5] += p.y * dwr;
        }
        j += dj;
        i += di;
        if (j >= n) {
            j -= n;
            ++i;
        }
    }
    for (int e = tid; e < 3 * n; e += blockDim.x) {   // bonds (x+1,y), (x,y+1), (x-1,y+1) (lattice.f90:98-111)
        const int i = e / 3, nb = e - (e / 3) * 3;
        const int ix = sxy[i] & 0xffff, iy = sxy[i] >> 16;
        const int jx = (nb == 0) ? (ix + 1) % lx : (nb == 1 ? ix : (ix + lx - 1) % lx);
        const int jy = (nb == 0) ? iy : (iy + 1) % ly;
        const int jj = jy * lx + jx;
        cplx gij = G[jj * LD + i], gji = G[i * LD + jj];   // Grupc(i,jj), Grupc(jj,i)
        if (i == jj) { gij.x -= 1.0; gji.x -= 1.0; }
        v[10] += 2.0 * (gij.x + gji.x);
    }
    for (int i = tid; i < n; i += blockDim.x) {
        const cplx du = cmk(G[i * LD + i].x - 1.0, G[i * LD + i].y);
        v[11] += du.x;
        v[12] += du.x * du.x + du.y * du.y;
        v[13] += du.x * du.x - du.y * du.y;
        s.obs()[O_SITE + i] += 2.0 * du.x;
    }
    block_sum<14>(v, s.red());
    if (tid == 0) {
        double* o = s.obs();
        const double onsite = 2.0 * v[13] + v[11];          // sum Re(2 du^2 + du)
        const double dbl = v[12] / lq;                       // doubleOcc sample
        const double kin = P.RT * v[10] / lq;
        const double inter = (P.U1 + P.U2) * (2.0 * onsite) / lq + 2.0 * (P.U2 - P.U1) * dbl;
        o[O_DENSITY_UP] += v[11] / lq;
        o[O_DENSITY_DO] += v[11] / lq;
        o[O_DENSITY_TOTAL] += 2.0 * v[11] / lq;
        o[O_KINETIC] += kin;
        o[O_DOUBLEOCC] += dbl;
        o[O_SQUAREOCC] += 2.0 * v[13] / lq;
        o[O_NUM_UP] += v[11];
        o[O_NUM_DO] += v[11];
        o[O_NUMSQUARE_UP] += v[0];
        o[O_NUMSQUARE_DO] += v[0];
        o[O_ONSITE_N2_UP] += onsite;
        o[O_ONSITE_N2_DO] += onsite;
        o[O_INTERACTION] += inter;
        o[O_ENERGY] += kin + inter;
        o[O_PSF_GAMMA] += v[1] / lq2;
        o[O_SF_K] += v[2] / lq2;
        o[O_SF_K + 1] += v[3] / lq2;
        o[O_DW_K] += v[4] / lq2;
        o[O_DW_K + 1] += v[5] / lq2;
        o[O_DEN_UPUP] += v[6] / lq;
        o[O_DEN_UPUP + 1] += v[7] / lq;
        o[O_DEN_DODO] += v[6] / lq;
        o[O_DEN_DODO + 1] -= v[7] / lq;
        o[O_DEN_UPDO] += v[8] / lq;
        o[O_DEN_UPDO + 1] += v[9] / lq;
        s.cnt()[4] += 1;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Nambu equal-time estimators (Obs_equal_calc, src/pairing/src/obser_equal.f90:112-271)
// from the {b, c^dagger} block.  With A = G1[b,b], B = G1[b,c^dagger],
// C = G1[c^dagger,b], D = G1[c^dagger,c^dagger], the reference's sixteen
// sub-blocks are A, -B, conj(A), -conj(B), conj(C), -conj(D), C, -D and zeros:
// n_b(i) = -conj(D_ii), n_c(i) = -D_ii, and every c-flavour sum is the complex
// conjugate of the b-flavour sum.  Pair terms:
//   Dbb(i,j) = n_b(i) n_b(j) - conj(D_ij) A_ij,  Dbc(i,j) = n_b(i) n_c(j) - conj(C_ij) B_ij,
//   Dcc = conj(Dbb), Dcb = conj(Dbc).
template <int NMAX>
COLD void measure_pair(Ctx<NMAX> x) {
    constexpr int LD = Cfg<NMAX>::LD;
    auto& s = x.s;
    const PointDev& P = x.P();
    const int n = x.n, ns = P.Ns, tid = threadIdx.x, lx = P.Lx, ly = P.Ly;
    const double lq = (double)P.Lq, lq2 = lq * lq, dns = (double)ns;
    const cplx* G = x.G();
    const cplx* ph = s.ph();
    const bool hasK = P.hasK;
    // v: 0-1 sum Dbb, 2-3 sum Dbc, 4 sum |D_ij|^2, 5-6 sf_K, 7-8 dw_K, 9 kinetic bonds,
    //    10 sum Re n_b, 11 sum Re Dbc(i,i), 12 sum Re n_b^2, 13 sum Re Dbb(i,i),
    //    14 sum Re(C_ii - B_ii), 15-16 tr B, 17-18 tr C
    double v[19];
#pragma unroll
    for (int k = 0; k < 19; ++k) v[k] = 0.0;
    const int* sxy = s.sxy();
    const int T = blockDim.x, stepi = T / ns, stepj = T - (T / ns) * ns;
    int i = tid / ns, j = tid - (tid / ns) * ns;
    for (int e = tid; e < ns * ns; e += T) {
        const cplx A = G[i * LD + j], B = G[i * LD + ns + j], C = G[(ns + i) * LD + j], D = G[(ns + i) * LD + ns + j];
        const cplx di = G[(ns + i) * LD + ns + i], dj = G[(ns + j) * LD + ns + j];
        const cplx nbi = cmk(-di.x, di.y), nbj = cmk(-dj.x, dj.y), ncj = cmk(-dj.x, -dj.y);
        const cplx dbb = csub(cmul(nbi, nbj), cmul(cconj(D), A));
        const cplx dbc = csub(cmul(nbi, ncj), cmul(cconj(C), B));
        v[0] += dbb.x;
        v[1] += dbb.y;
        v[2] += dbc.x;
        v[3] += dbc.y;
        v[4] += D.x * D.x + D.y * D.y;
        if (hasK) {
            const int pi = sxy[i], pj = sxy[j];
            int dx = (pi & 0xffff) - (pj & 0xffff), dy = (pi >> 16) - (pj >> 16);
            dx += (dx < 0) ? lx : 0;
            dy += (dy < 0) ? ly : 0;
            const cplx p = ph[dy * lx + dx];
            const double sfr = -2.0 * D.x;                 // G_bdag_b + G_cdag_c
            const double dwr = 2.0 * (dbb.x + dbc.x);      // Dbb + Dcc + Dbc + Dcb
            v[5] += p.x * sfr;
            v[6] += p.y * sfr;
            v[7] += p.x * dwr;
            v[8] += p.y * dwr;
        }
        j += stepj;
        i += stepi;
        if (j >= ns) {
            j -= ns;
            ++i;
        }
    }
    for (int e = tid; e < 3 * ns; e += blockDim.x) {   // bonds (x+1,y), (x,y+1), (x-1,y+1)
        const int i = e / 3, nb = e - (e / 3) * 3;
        const int ix = sxy[i] & 0xffff, iy = sxy[i] >> 16;
        const int jx = (nb == 0) ? (ix + 1) % lx : (nb == 1 ? ix : (ix + lx - 1) % lx);
        const int jy = (nb == 0) ? iy : (iy + 1) % ly;
        const int jj = jy * lx + jx;
        v[9] += -2.0 * (G[(ns + i) * LD + ns + jj].x + G[(ns + jj) * LD + ns + i].x);
    }
    for (int i = tid; i < ns; i += blockDim.x) {
        const cplx A = G[i * LD + i], B = G[i * LD + ns + i], C = G[(ns + i) * LD + i], D = G[(ns + i) * LD + ns + i];
        const cplx nb = cmk(-D.x, D.y);
        const double nbnc = D.x * D.x + D.y * D.y;          // n_b n_c = |D_ii|^2
        const cplx cb = cmul(cconj(C), B);
        const cplx dbb = cadd(cmul(nb, nb), cmul(nb, A));
        v[10] += nb.x;
        v[11] += nbnc - cb.x;
        v[12] += nb.x * nb.x - nb.y * nb.y;
        v[13] += dbb.x;
        v[14] += C.x - B.x;
        v[15] += B.x;
        v[16] += B.y;
        v[17] += C.x;
        v[18] += C.y;
        s.obs()[O_SITE + i] += 2.0 * nb.x;
    }
    block_sum<19>(v, s.red());
    if (tid == 0) {
        double* o = s.obs();
        const double dens = 2.0 * v[10] / dns;
        const double dbl = v[11] / dns;
        const double pair = v[14] / dns;
        const double kin = P.RT * v[9] / dns;
        const double inter = (P.U1 + P.U2) * (2.0 * v[13]) / dns + 2.0 * (P.U2 - P.U1) * dbl;
        const double epair = P.Delta * pair;
        const double chem = -P.mu * dens;
        const double energy = kin + inter + epair;
        // tr C tr B; psf_Gamma = (-conj(trC trB) + sum |D_ij|^2) / Lq^2
        const double tcb_re = v[17] * v[15] - v[18] * v[16], tcb_im = v[17] * v[16] + v[18] * v[15];
        o[O_DENSITY_UP] += v[10] / dns;
        o[O_DENSITY_DO] += v[10] / dns;
        o[O_DENSITY] += dens;
        o[O_DENSITY_TOTAL] += dens;
        o[O_NUM_UP] += v[10];
        o[O_NUM_DO] += v[10];
        o[O_DOUBLEOCC] += dbl;
        o[O_SQUAREOCC] += 2.0 * v[12] / dns;
        o[O_LOCAL_NUMSQUARE] += 2.0 * v[13] / dns;
        o[O_PAIR_EQUAL] += pair;
        o[O_NUMSQUARE_UP] += v[0];
        o[O_NUMSQUARE_DO] += v[0];
        o[O_ONSITE_N2_UP] += v[13];
        o[O_ONSITE_N2_DO] += v[13];
        o[O_KINETIC] += kin;
        o[O_INTERACTION] += inter;
        o[O_PAIRING_ENERGY] += epair;
        o[O_CHEMICAL_ENERGY] += chem;
        o[O_ENERGY] += energy;
        o[O_GRAND_ENERGY] += energy + chem;
        o[O_SF_K] += v[5] / lq2;
        o[O_SF_K + 1] += v[6] / lq2;
        o[O_DW_K] += v[7] / lq2;
        o[O_DW_K + 1] += v[8] / lq2;
        o[O_PSF_GAMMA] += (v[4] - tcb_re) / lq2;
        o[O_PSF_GAMMA + 1] += tcb_im / lq2;
        o[O_DEN_UPUP] += v[0] / lq;
        o[O_DEN_UPUP + 1] += v[1] / lq;
        o[O_DEN_DODO] += v[0] / lq;
        o[O_DEN_DODO + 1] -= v[1] / lq;
        o[O_DEN_UPDO] += v[2] / lq;
        o[O_DEN_UPDO + 1] += v[3] / lq;
        s.cnt()[4] += 1;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// stabilisation (stabilization.f90:69-190)

// stab_UR: (U_R D_R) P = Q R;  D_R <- |diag R|;  V_R <- R P^T V_R;  U_R <- Q.
// U_R is x.U(); on exit the new V_R is in x.W2() and in A.VRc, D_R in A.DRc.
template <int NMAX>
COLD void stab_UR(Ctx<NMAX> x) {
    constexpr int LD = Cfg<NMAX>::LD;
    auto& s = x.s;
    const int n = x.n;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - (e / n) * n;
        x.W1()[r * LD + c] = cmul(x.U()[r * LD + c], x.A().DRc[c]);
    }
    __syncthreads();
    qrp_any(x, x.W1());
    for (int i = threadIdx.x; i < n; i += blockDim.x) x.A().DRc[i] = cmk(s.d()[i], 0.0);
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - (e / n) * n;
        x.W2()[r * LD + c] = x.A().VRc[s.piv()[r] * n + c];
    }
    __syncthreads();
    gemm_any(x, x.W2(), op_n(x.W1(), LD), op_n(x.W2(), LD), TRI_A_UPPER);
    form_q_any(x, x.W1(), x.U(), false);
    sstore(n, LD, x.A().VRc, x.W2());
    __syncthreads();
}

// stab_UL: (U_L^H D_L) P = Q R;  D_L <- |diag R|;  V_L <- V_L P R^H;  U_L <- Q^H.
template <int NMAX>
COLD void stab_UL(Ctx<NMAX> x) {
    constexpr int LD = Cfg<NMAX>::LD;
    auto& s = x.s;
    const int n = x.n;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - (e / n) * n;
        x.W1()[r * LD + c] = cmul(cconj(x.U()[c * LD + r]), x.A().DLc[c]);
    }
    __syncthreads();
    qrp_any(x, x.W1());
    for (int i = threadIdx.x; i < n; i += blockDim.x) x.A().DLc[i] = cmk(s.d()[i], 0.0);
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - (e / n) * n;
        x.W2()[r * LD + c] = x.A().VLc[r * n + s.piv()[c]];
    }
    __syncthreads();
    gemm_any(x, x.W2(), op_n(x.W2(), LD), op_c(x.W1(), LD), TRI_B_LOWER_FROM_C);
    form_q_any(x, x.W1(), x.U(), true);
    sstore(n, LD, x.A().VLc, x.W2());
    __syncthreads();
}

// M = U_R^H U_L^H - D_R V_R V_L D_L is in W2 (W1 free); finish stab_green:
// factor M (or M^H for nt > L/2) and write G = (I - B)^{-1} into W2.  The
// D^{-1} scaling before ZTRSM is applied as the solve loads its operand; the
// reciprocals of R's diagonal and of D live in the QR norm vectors (free once
// the factorisation is done) and in u2.
//
// right_local: the right side (U_R) is in shared memory and U_L in HBM
// (stab_green_right_local); otherwise the left side is local and U_R in HBM.
// The HBM factor of the final product is staged into W2 (free after the
// triangular solve) so that every product runs on shared memory.
template <int NMAX>
COLD void green_from_M(Ctx<NMAX> x, int nt, bool right_local, bool want_logdet) {
    constexpr int LD = Cfg<NMAX>::LD;
    auto& s = x.s;
    const int n = x.n, L = x.P().L;
    cplx* rinv = reinterpret_cast<cplx*>(s.vn1());   // vn1 | vn2, n complex
    double* dinv = s.u2();
    const MatOp Uloc = op_c(x.U(), LD);
    const MatOp URh = right_local ? Uloc : op_c(x.A().URc, n);
    const MatOp ULh = right_local ? op_c(x.A().ULc, n) : Uloc;
    if (nt > L / 2) conj_transpose_any(x, x.W2());
    qrp_any(x, x.W2());
    if (nt < L / 2 + 1) {
        copy_op(n, LD, x.W1(), URh);
        apply_qh_left_any(x, x.W2(), x.W1());
        diag_inverse(n, LD, x.W2(), s.d(), rinv, dinv);
        trsm_left_any(x, x.W2(), rinv, dinv, x.W1());
        permute_rows_any(x, x.W1(), false);
        if (right_local) {   // U_L^H from HBM, staged
            sload(n, LD, x.W2(), x.A().ULc);
            __syncthreads();
            gemm_any(x, x.W2(), op_c(x.W2(), LD), op_n(x.W1(), LD));
        } else {
            gemm_any(x, x.W2(), Uloc, op_n(x.W1(), LD));
        }
    } else {
        copy_op(n, LD, x.W1(), ULh);
        apply_q_right_any(x, x.W2(), x.W1());
        diag_inverse(n, LD, x.W2(), s.d(), rinv, dinv);
        trsm_right_any(x, x.W2(), rinv, dinv, x.W1());
        permute_cols_any(x, x.W1(), false);
        if (right_local) {
            gemm_any(x, x.W2(), op_n(x.W1(), LD), Uloc);
        } else {             // U_R^H from HBM, staged
            sload(n, LD, x.W2(), x.A().URc);
            __syncthreads();
            gemm_any(x, x.W2(), op_n(x.W1(), LD), op_c(x.W2(), LD));
        }
    }
    if (want_logdet) {
        double v[1] = {0.0};
        for (int i = threadIdx.x; i < n; i += blockDim.x) v[0] += log(s.d()[i]);
        block_sum<1>(v, s.red());
        if (threadIdx.x == 0) x.sc->logdetM = v[0];
    }
}

// M = invULUR - D_R (V_R V_L) D_L with V_R V_L already in W1 and invULUR in W2.
template <int NMAX>
DEVI void form_M(Ctx<NMAX>& x) {
    constexpr int LD = Cfg<NMAX>::LD;
    auto& s = x.s;
    const int n = x.n;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - (e / n) * n;
        const cplx t = cmul(x.A().DLc[c], x.W1()[r * LD + c]);
        x.W2()[r * LD + c] = csub(x.W2()[r * LD + c], cmul(x.A().DRc[r], t));
    }
    __syncthreads();
}

// compare_mat + G <- G_new (stabilization.f90:256-266, 339-344)
template <int NMAX>
DEVI void drift_and_replace(Ctx<NMAX>& x) {
    auto& s = x.s;
    const int n = x.n;
    double v[1] = {0.0};
    constexpr int LD = Cfg<NMAX>::LD;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - (e / n) * n;
        v[0] += cabsv(csub(x.W2()[r * LD + c], x.G()[r * LD + c]));
    }
    block_sum<1>(v, s.red());
    if (threadIdx.x == 0) {
        const double dif = v[0];
        if (dif > x.sc->xmax) x.sc->xmax = dif;
        x.sc->xmean += dif;
        if (!(dif == dif) || dif > 1.0e300) x.sc->status |= 1;
    }
    scopy(n, LD, x.G(), x.W2());
    __syncthreads();
}

// stab_green with the right side factored in shared memory (U = U_R, W2 = V_R)
// and the left side in HBM (A.ULc, A.VLc, A.DLc).
template <int NMAX>
COLD void stab_green_right_local(Ctx<NMAX> x, int nt, bool want_logdet) {
    constexpr int LD = Cfg<NMAX>::LD;
    auto& s = x.s;
    const int n = x.n;
    // HBM operands are staged into the workspace the product overwrites (the
    // products stage their results in registers, so C may alias an operand);
    // V_R in W2 is no longer needed after the first product (VRc holds it).
    sload(n, LD, x.W1(), x.A().VLc);
    __syncthreads();
    gemm_any(x, x.W1(), op_n(x.W2(), LD), op_n(x.W1(), LD));   // V_R V_L
    sload(n, LD, x.W2(), x.A().ULc);
    __syncthreads();
    gemm_any(x, x.W2(), op_c(x.U(), LD), op_c(x.W2(), LD));    // U_R^H U_L^H
    form_M(x);
    green_from_M(x, nt, true, want_logdet);
}

// stab_green with the left side in shared memory (U = U_L, W2 = V_L) and the
// right side in HBM.
template <int NMAX>
COLD void stab_green_left_local(Ctx<NMAX> x, int nt) {
    constexpr int LD = Cfg<NMAX>::LD;
    auto& s = x.s;
    const int n = x.n;
    sload(n, LD, x.W1(), x.A().VRc);
    __syncthreads();
    gemm_any(x, x.W1(), op_n(x.W1(), LD), op_n(x.W2(), LD));   // V_R V_L
    sload(n, LD, x.W2(), x.A().URc);
    __syncthreads();
    gemm_any(x, x.W2(), op_c(x.W2(), LD), op_c(x.U(), LD));    // U_R^H U_L^H
    form_M(x);
    green_from_M(x, nt, false, false);
}

// Wrap_L (stabilization.f90:301-331)
template <int NMAX>
COLD void wrap_L(Ctx<NMAX> x, int nt) {
    auto& s = x.s;
    const int n = x.n, st = nt / x.P().Nwrap;
    gcopy(x.A().URc, x.A().URs(st), n * n);
    gcopy(x.A().VRc, x.A().VRs(st), n * n);
    gcopy(x.A().DRc, x.A().DRs(st), n);
    __syncthreads();
    if (nt != x.P().L) {
        stab_UL(x);
        stab_green_left_local(x, nt);
        drift_and_replace(x);
    }
    sstore(n, Cfg<NMAX>::LD, x.A().ULs(st), x.U());
    gcopy(x.A().VLs(st), x.A().VLc, n * n);
    gcopy(x.A().DLs(st), x.A().DLc, n);
    __syncthreads();
    load_expT(x);
}

// Wrap_R (stabilization.f90:333-366)
template <int NMAX>
COLD void wrap_R(Ctx<NMAX> x, int nt) {
    auto& s = x.s;
    const int n = x.n, st = nt / x.P().Nwrap;
    gcopy(x.A().ULc, x.A().ULs(st), n * n);
    gcopy(x.A().VLc, x.A().VLs(st), n * n);
    gcopy(x.A().DLc, x.A().DLs(st), n);
    __syncthreads();
    if (nt != 0) {
        stab_UR(x);
        stab_green_right_local(x, nt, nt == x.P().L);
        drift_and_replace(x);
    }
    sstore(n, Cfg<NMAX>::LD, x.A().URs(st), x.U());
    gcopy(x.A().VRs(st), x.A().VRc, n * n);
    gcopy(x.A().DRs(st), x.A().DRc, n);
    __syncthreads();
    load_expT(x);
}

// ---------------------------------------------------------------------------
template <int NMAX>
DEVI bool setup_ctx(Ctx<NMAX>& x, const KernelArgs& ka, int chain) {
    const ChainDev cd = ka.chains[chain];
    if (threadIdx.x == 0) {
        *x.s.P() = ka.pts[cd.point];
        // The SM's schedulers take warps by slot modulo 4, so the deciding warps
        // of two CTAs on one SM would share a scheduler if both used warp 0.  A
        // CTA whose warp slots start at an odd multiple of 8 decides on warp 2.
        // Thread 0 decides for the whole CTA.
        unsigned slot;
        asm volatile("mov.u32 %0, %%warpid;" : "=r"(slot));
        *x.s.strip_warp() = (Cfg<NMAX>::THREADS >= 192 && ((slot >> 3) & 1)) ? 2 : 0;
    }
    __syncthreads();
    x.n = x.P().N;
    if (x.P().hasK)
        for (int r = threadIdx.x; r < x.P().Lq && r < NMAX; r += blockDim.x) x.s.ph()[r] = x.P().phaseR[r];
    for (int i = threadIdx.x; i < x.P().Lq && i < NMAX; i += blockDim.x) {
        const int lx = x.P().Lx;
        x.s.sxy()[i] = (i % lx) | ((i / lx) << 16);
    }
    x.abase = ka.arena + cd.arena_off;
    x.wg = x.abase + arena_base(x.n, x.P().Nst);
    x.sw0 = *x.s.strip_warp();
    x.phi = ka.phi + cd.phi_off;
    x.sc = ka.sc + chain;
    return x.n <= NMAX;
}

template <int NMAX>
DEVI void load_obs(Ctx<NMAX>& x) {
    for (int k = threadIdx.x; k < kObsScalars + NMAX; k += blockDim.x) x.s.obs()[k] = 0.0;
}
template <int NMAX>
DEVI void flush_obs(Ctx<NMAX>& x, double* gobs) {
    for (int k = threadIdx.x; k < kObsScalars + x.P().Lq; k += blockDim.x) gobs[k] += x.s.obs()[k];
}

template <int NMAX, bool PAIR, bool LEFT>
DEVI void prop_any(Ctx<NMAX>& x, int ch, int slice) {
    if constexpr (PAIR) prop_channel_pair<NMAX, LEFT>(x, ch, slice);
    else prop_channel<NMAX, LEFT>(x, ch, slice);
}
template <int NMAX, bool PAIR>
DEVI void measure_any(Ctx<NMAX>& x) {
    if constexpr (PAIR) measure_pair<NMAX>(x);
    else measure<NMAX>(x);
}

// one sweep: Local_sweep_L then Local_sweep_R (local_sweep.f90:96-134)
template <int NMAX, bool PAIR>
__global__ void __launch_bounds__(Cfg<NMAX>::THREADS, Cfg<NMAX>::MINB) sweep_kernel(KernelArgs ka, const int* idx, int count) {
    if ((int)blockIdx.x >= count) return;
    const int chain = idx[blockIdx.x];
    Ctx<NMAX> x;
    if (!setup_ctx(x, ka, chain)) return;
    if (x.sc->status & 1) return;   // quarantined: non-finite G, skipped until its state is set again
    tc_begin(x, ka);
    auto& s = x.s;
    const int n = x.n, L = x.P().L;
    const bool tm = ka.timers && threadIdx.x == 0;
    long long tk = tm ? clock64() : 0;
#define lap(ph)                                      \
    do {                                             \
        if (tm) {                                    \
            const long long t_ = clock64();          \
            x.sc->cyc[ph] += t_ - tk;                \
            tk = t_;                                 \
        }                                            \
    } while (0)
    if (threadIdx.x == 0) {
        *s.seed() = x.sc->seed;
        for (int k = 0; k < 5; ++k) s.cnt()[k] = 0;
    }
    load_obs(x);
    sload(n, Cfg<NMAX>::LD, x.G(), x.A().G);
    sload(n, Cfg<NMAX>::LD, x.U(), x.A().ULc);
    __syncthreads();
    load_expT(x);
    lap(3);
    // ---- left traversal (skipped by a right-only launch, which continues from
    // the G, U_L and counters a left-only launch left in the arena)
    if (ka.traverse != 2) {
        for (int nt = L; nt >= 1; --nt) {
            if (nt % x.P().Nwrap == 0) {
                wrap_L(x, nt);
                lap(3);
            }
            measure_any<NMAX, PAIR>(x);
            lap(2);
            slice_products<NMAX, true>(x);
            lap(1);
            if (x.P().active[1]) prop_any<NMAX, PAIR, true>(x, 1, nt - 1);
            if (x.P().active[0]) prop_any<NMAX, PAIR, true>(x, 0, nt - 1);
            lap(0);
        }
        wrap_L(x, 0);
        sstore(n, Cfg<NMAX>::LD, x.A().ULc, x.U());
        __syncthreads();
    }
    // ---- right traversal
    if (ka.traverse != 1) {
    sload(n, Cfg<NMAX>::LD, x.U(), x.A().URc);
    __syncthreads();
    wrap_R(x, 0);
    lap(3);
    for (int nt = 1; nt <= L; ++nt) {
        if (x.P().active[0]) prop_any<NMAX, PAIR, false>(x, 0, nt - 1);
        if (x.P().active[1]) prop_any<NMAX, PAIR, false>(x, 1, nt - 1);
        lap(0);
        slice_products<NMAX, false>(x);
        lap(1);
        if (nt % x.P().Nwrap == 0) {
            wrap_R(x, nt);
            lap(3);
        }
        measure_any<NMAX, PAIR>(x);
        lap(2);
    }
    sstore(n, Cfg<NMAX>::LD, x.A().URc, x.U());
    }
    sstore(n, Cfg<NMAX>::LD, x.A().G, x.G());
    flush_obs(x, ka.obs + (long)chain * ka.obs_stride);
    if (threadIdx.x == 0) {
        x.sc->seed = *s.seed();
        x.sc->nacc[0] += s.cnt()[0];
        x.sc->nacc[1] += s.cnt()[1];
        x.sc->nc[0] += s.cnt()[2];
        x.sc->nc[1] += s.cnt()[3];
        x.sc->nobs += s.cnt()[4];
    }
    lap(3);
#undef lap
    tc_end(x, ka);
}

// Local_sweep_pre (local_sweep.f90:80-94) with Prop_make's identities
// (process_matrix.f90:37-47).  propU_pre scales the rows of U_R by the HS
// factors (multiply.f90:7-16); for a Nambu chain row Ns+i (c^dagger_i) takes
// e^{-alpha phi} in the U2 channel (src/pairing/src/operator_Hubbard.f90:155-166).
template <int NMAX, bool PAIR>
__global__ void __launch_bounds__(Cfg<NMAX>::THREADS, Cfg<NMAX>::MINB) pre_kernel(KernelArgs ka, const int* idx, int count) {
    constexpr int LD = Cfg<NMAX>::LD;
    if ((int)blockIdx.x >= count) return;
    const int chain = idx[blockIdx.x];
    Ctx<NMAX> x;
    if (!setup_ctx(x, ka, chain)) return;
    tc_begin(x, ka);
    auto& s = x.s;
    const int n = x.n, L = x.P().L;
    set_identity(n, LD, x.U());
    set_identity(n, LD, x.G());
    set_identity(n, n, x.A().VRc);
    set_identity(n, n, x.A().ULc);
    set_identity(n, n, x.A().VLc);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        x.A().DRc[i] = cmk(1.0, 0.0);
        x.A().DLc[i] = cmk(1.0, 0.0);
    }
    __syncthreads();
    sstore(n, LD, x.A().URs(0), x.U());
    gcopy(x.A().VRs(0), x.A().VRc, n * n);
    gcopy(x.A().DRs(0), x.A().DRc, n);
    sload_real(n, LD, reinterpret_cast<double*>(x.W1()), x.P().expP);
    __syncthreads();
    const int ns = x.P().Ns;
    for (int nt = 1; nt <= L; ++nt) {
        const double* ph = x.phi + (long)(nt - 1) * ns * 2;
        for (int ch = 0; ch < 2; ++ch) {
            if (!x.P().active[ch]) continue;
            const double ar = x.P().alpha_re[ch], ai = x.P().alpha_im[ch];
            const bool flip = x.P().flip[ch] != 0;
            for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
                const int r = e / n, c = e - (e / n) * n;
                const int site = (PAIR && r >= ns) ? r - ns : r;
                const double p = ph[site * 2 + ch];
                const bool neg = PAIR && r >= ns && flip;
                const cplx f = neg ? cexpz(cmk(-(ar * p), -(ai * p))) : cexpz(cmk(ar * p, ai * p));
                x.U()[r * LD + c] = cmul(f, x.U()[r * LD + c]);
            }
            __syncthreads();
        }
        slice_mult<NMAX, false>(x, x.U(), reinterpret_cast<const double*>(x.W1()));
        if (nt % x.P().Nwrap == 0) {
            const int st = nt / x.P().Nwrap;
            stab_UR(x);
            sstore(n, LD, x.A().URs(st), x.U());
            gcopy(x.A().VRs(st), x.A().VRc, n * n);
            gcopy(x.A().DRs(st), x.A().DRc, n);
            __syncthreads();
            if (nt == L) {
                stab_green_right_local(x, nt, true);
                scopy(n, LD, x.G(), x.W2());
                __syncthreads();
            }
            sload_real(n, LD, reinterpret_cast<double*>(x.W1()), x.P().expP);
            __syncthreads();
        }
    }
    sstore(n, LD, x.A().URc, x.U());
    sstore(n, LD, x.A().G, x.G());
    // a chain whose G(beta) is not finite (overflowing fields) is quarantined
    {
        double v[1] = {0.0};
        for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
            const cplx g = x.A().G[e];
            if (!isfinite(g.x) || !isfinite(g.y)) v[0] += 1.0;
        }
        block_sum<1>(v, x.s.red());
        if (threadIdx.x == 0 && v[0] > 0.0) x.sc->status |= 1;
    }
    tc_end(x, ka);
}

// LocalU_prop_therm / LocalU_metro_therm over the whole field, nwarm sweeps
// (localU.f90:115-156, local_sweep.f90:64-78).  Each field value sees only its
// own proposals, so fields are updated in parallel; the draw index of a
// proposal is its position in the reference's sequential order.
__global__ void warmup_kernel(KernelArgs ka, int nwarm) {
    const int chain = blockIdx.x;
    if (chain >= ka.nchains) return;
    const ChainDev cd = ka.chains[chain];
    const PointDev P = ka.pts[cd.point];
    ChainScalars* sc = ka.sc + chain;
    double* phi = ka.phi + cd.phi_off;
    __shared__ double red[2 * 32];
    __shared__ int chs[2];
    __shared__ int nact;
    if (threadIdx.x == 0) {
        int a = 0;
        for (int ch = 0; ch < 2; ++ch)
            if (P.active[ch]) chs[a++] = ch;
        nact = a;
    }
    __syncthreads();
    const int A = nact, n = P.Ns, L = P.L;
    const uint32_t s0 = sc->seed;
    const unsigned long long per_sweep = (unsigned long long)L * A * n;
    const uint32_t step = lcg_pow(2ull * per_sweep);
    const double shift = fabs(P.shiftLoc);
    double cnt[2] = {0.0, 0.0};
    for (long long m = threadIdx.x; m < (long long)per_sweep; m += blockDim.x) {
        const int i = (int)(m % n);
        const int chpos = (int)((m / n) % A);
        const int nt = (int)(m / ((long long)n * A));
        const int ch = chs[chpos];
        double p = phi[((long)nt * n + i) * 2 + ch];
        uint32_t d1 = lcg_mul(lcg_pow(2ull * m + 1ull), s0);
        for (int w = 0; w < nwarm; ++w) {
            const uint32_t d2 = lcg_mul(kLcgA, d1);
            const double xflip = lcg_u(d1), rnd = lcg_u(d2);
            const double pn = p + (xflip - 0.5) * shift;
            const double ratio = exp(-0.5 * pn * pn) / exp(-0.5 * p * p);
            if (ratio > rnd) {
                p = pn;
                cnt[chpos] += 1.0;
            }
            d1 = lcg_mul(step, d1);
        }
        phi[((long)nt * n + i) * 2 + ch] = p;
    }
    double v[2] = {cnt[0], cnt[1]};
    block_sum<2>(v, red);
    if (threadIdx.x == 0) {
        for (int k = 0; k < A; ++k) sc->therm_acc_sum[chs[k]] += v[k] / ((double)L * n);
        sc->seed = lcg_mul(lcg_pow(2ull * per_sweep * (unsigned long long)nwarm), s0);
    }
}

// Start of a bin: Local_sweep_reset (local_sweep.f90:54-62).
__global__ void bin_reset_kernel(KernelArgs ka) {
    const int chain = blockIdx.x;
    if (chain >= ka.nchains) return;
    double* o = ka.obs + (long)chain * ka.obs_stride;
    for (int k = threadIdx.x; k < ka.obs_stride; k += blockDim.x) o[k] = 0.0;
    if (threadIdx.x == 0) {
        ChainScalars* sc = ka.sc + chain;
        sc->nc[0] = sc->nc[1] = 0;
        sc->nacc[0] = sc->nacc[1] = 0;
        sc->nobs = 0;
    }
}

// End of a bin: Obs_equal_ave and AccCounter%ratio (obser_equal.f90:66-93,
// operator_Hubbard.f90:124-129).
__global__ void bin_finish_kernel(KernelArgs ka) {
    const int chain = blockIdx.x;
    if (chain >= ka.nchains) return;
    ChainScalars* sc = ka.sc + chain;
    const int lq = ka.pts[ka.chains[chain].point].Lq;
    const double z = 1.0 / (double)sc->nobs;
    double* o = ka.obs + (long)chain * ka.obs_stride;
    for (int k = threadIdx.x; k < kObsScalars + lq; k += blockDim.x) o[k] *= z;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int ch = 0; ch < 2; ++ch) {
            if (sc->nc[ch] > 0) sc->acc_sum[ch] += (double)sc->nacc[ch] / (double)sc->nc[ch];
            sc->prop_tot[ch] += (double)sc->nc[ch];
            sc->acc_tot[ch] += (double)sc->nacc[ch];
        }
    }
}

// Chain average per point (m_process_obs_equal, fourier_trans.f90:350-457):
// out[p][k] = sum over the chains of point p of obs[chain][k] / (chains of p),
// over the chains that are not quarantined (NaN if none is left).
__global__ void point_average_kernel(KernelArgs ka, const int* point_chain_start, const int* point_chain_list,
                                     double* out) {
    const int p = blockIdx.x;
    const int b = point_chain_start[p], e = point_chain_start[p + 1];
    for (int k = threadIdx.x; k < ka.obs_stride; k += blockDim.x) {
        double s = 0.0;
        int m = 0;
        for (int c = b; c < e; ++c) {
            const int ch = point_chain_list[c];
            if (ka.sc[ch].status & 1) continue;   // quarantined chains leave the average
            s += ka.obs[(long)ch * ka.obs_stride + k];
            ++m;
        }
        out[(long)p * ka.obs_stride + k] = m > 0 ? s / (double)m : __longlong_as_double(0x7ff8000000000000LL);
    }
}

// Block statistics of the per-bin point averages: cur += pout (bins summed in
// order); when a block completes, blk = cur / block_size and cur restarts.
__global__ void stats_add_kernel(const double* pout, double* cur, double* blk, int n, int finish, int block_size) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const double v = cur[k] + pout[k];
        if (finish) {
            blk[k] = v / (double)block_size;
            cur[k] = 0.0;
        } else {
            cur[k] = v;
        }
    }
}
// mean and standard error over nb block means, each element summed over the
// blocks in order: mean = sum / nb, sem = sqrt(sum (m - mean)^2 / (nb - 1) / nb)
__global__ void stats_final_kernel(const double* blk, int nb, int n, double* mean, double* sem) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nb; ++b) s += blk[(long)b * n + k];
        const double m = s / (double)nb;
        double v = 0.0;
        for (int b = 0; b < nb; ++b) {   // square rounded, then added (no fused multiply-add)
            const double d = blk[(long)b * n + k] - m;
            v = __dadd_rn(v, __dmul_rn(d, d));
        }
        mean[k] = m;
        sem[k] = nb > 1 ? sqrt(v / (double)(nb - 1) / (double)nb) : __longlong_as_double(0x7ff8000000000000LL);
    }
}

// Global shift move: the shift part of Global_flip (global_update.f90:193-208),
// under this model's weight.  Per chain, two draws of the chain's LCG give a
// uniform shift X_ns = (u - 1/2) |shift_ns| of every field of auxiliary channel
// ns; the shifted field goes to the proposal state kp (same layout).
__global__ void global_propose_kernel(KernelArgs ka, KernelArgs kp, double shift0, double shift1) {
    const int chain = blockIdx.x;
    if (chain >= ka.nchains) return;
    const ChainDev cd = ka.chains[chain];
    const PointDev& P = ka.pts[cd.point];
    ChainScalars* sc = ka.sc + chain;
    if (sc->status & 1) return;   // quarantined
    __shared__ double X[2];
    if (threadIdx.x == 0) {
        uint32_t seed = sc->seed;
        const double amp[2] = {fabs(shift0), fabs(shift1)};
        for (int ns = 0; ns < 2; ++ns) {
            seed = lcg_mul(kLcgA, seed);
            X[ns] = (lcg_u(seed) - 0.5) * amp[ns];
        }
        sc->seed = seed;
        kp.sc[chain].status = 0;
    }
    __syncthreads();
    const long long tot = (long long)P.L * P.Ns * 2;
    const double* phi = ka.phi + cd.phi_off;
    double* phi2 = kp.phi + cd.phi_off;
    for (long long k = threadIdx.x; k < tot; k += blockDim.x) phi2[k] = phi[k] + X[k & 1];
}

// Exact Metropolis-Hastings decision of a global move (global_update.f90:237-249:
// accept if w'/w >= u, u the chain's next draw), with log w = -sum phi^2 / 2
// - f log|det(I - B(beta,0))| from the two states' last factorisations at
// tau = beta: f = 2 for a number-conserving chain (flavours b and c = conj(b)),
// f = 1 for a Nambu chain (the 4Ns determinant to the power -1/2 is the
// squared modulus of its {b, c^dagger} block's, to the power -1/2).
// hastings (optional) adds log q(phi|phi') - log q(phi'|phi) of a
// non-symmetric proposal; a non-finite exponent rejects.  An accepted chain
// takes the proposal's fields and UDV arena.
__global__ void global_accept_kernel(KernelArgs ka, KernelArgs kp, const double* fn, const double* fn2,
                                     const double* hastings, int* accepted) {
    const int chain = blockIdx.x;
    if (chain >= ka.nchains) return;
    const ChainDev cd = ka.chains[chain];
    const PointDev& P = ka.pts[cd.point];
    ChainScalars* sc = ka.sc + chain;
    __shared__ int acc;
    if (threadIdx.x == 0) {
        acc = 0;
        if (!(sc->status & 1)) {
            const double f = P.pairing ? 1.0 : 2.0;
            const double lw = fn[chain] - f * sc->logdetM;
            const double lw2 = fn2[chain] - f * kp.sc[chain].logdetM;
            const double x = lw2 - lw + (hastings ? hastings[chain] : 0.0);
            const uint32_t seed = lcg_mul(kLcgA, sc->seed);
            sc->seed = seed;
            acc = !(kp.sc[chain].status & 1) && !isnan(x) && x < INFINITY && exp(x) >= lcg_u(seed);
            sc->glb_prop += 1.0;
            if (acc) {
                sc->glb_acc += 1.0;
                sc->logdetM = kp.sc[chain].logdetM;
            }
        }
        if (accepted) accepted[chain] = acc;
    }
    __syncthreads();
    if (!acc) return;
    const long long na = arena_base(P.N, P.Nst), nphi = (long long)P.L * P.Ns * 2;
    const double2* a2 = kp.arena + cd.arena_off;
    double2* a = ka.arena + cd.arena_off;
    for (long long k = threadIdx.x; k < na; k += blockDim.x) a[k] = a2[k];
    const double* p2 = kp.phi + cd.phi_off;
    double* p = ka.phi + cd.phi_off;
    for (long long k = threadIdx.x; k < nphi; k += blockDim.x) p[k] = p2[k];
}

// bad[chain] = 1 if any field value of the chain is NaN or infinite
__global__ void field_check_kernel(KernelArgs ka, int* bad) {
    const int chain = blockIdx.x;
    if (chain >= ka.nchains) return;
    const ChainDev cd = ka.chains[chain];
    const PointDev& P = ka.pts[cd.point];
    const double* phi = ka.phi + cd.phi_off;
    const long long tot = (long long)P.L * P.Ns * 2;
    int any = 0;
    for (long long k = threadIdx.x; k < tot; k += blockDim.x) any |= !isfinite(phi[k]);
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) bad[chain] = any;
}

// -0.5 * sum(phi^2) per chain (AuxConf_log_weight, fields.f90:29-33)
__global__ void field_norm_kernel(KernelArgs ka, double* out) {
    const int chain = blockIdx.x;
    if (chain >= ka.nchains) return;
    const ChainDev cd = ka.chains[chain];
    const PointDev P = ka.pts[cd.point];
    __shared__ double red[32];
    const double* phi = ka.phi + cd.phi_off;
    double v[1] = {0.0};
    const long long tot = (long long)P.L * P.Ns * 2;
    for (long long k = threadIdx.x; k < tot; k += blockDim.x) v[0] += phi[k] * phi[k];
    block_sum<1>(v, red);
    if (threadIdx.x == 0) out[chain] = -0.5 * v[0];
}

// ---------------------------------------------------------------------------
// Time-displaced Green's functions (Dyn_reset + Dyn_sweep_R, dynamics.f90:38-58;
// propgrU_R / propgrT_R, multiply.f90:48-97; Wrap_tau and stab_green_big,
// stabilization.f90:192-254, 368-404) of a number-conserving chain with
// N <= 72, run between its left and right traversals (Local_sweep_R's toggle,
// local_sweep.f90:119-123).  From G(0,0) and the left factors the left
// traversal stored, G(tau,0) = B(tau,0) G, G(0,tau) = -(I - G) B(tau,0)^-1 and
// G(tau,tau) = B(tau,0) G B(tau,0)^-1 are propagated slice by slice, and every
// Nwrap slices recomputed from the stabilised factors as blocks of
//   diag(V_R^-1, U_L^H) [[(V_R V_L)^-1, -D_L], [-D_R, (U_L U_R)^H]]^-1 diag(V_L^-1, U_R^H),
// the inverse of [[I, -B(beta,tau)], [-B(tau,0), I]]; the L1 distance between
// the propagated and the recomputed matrices is the drift Wrap_tau records.
// Two departures from the reference, both deliberate: the U2 operator uses the
// U2 field (dynamics.f90:52 passes the U1 field), and the 2N x 2N matrix has
// the bosonic -D_L (stabilization.f90:206-209 has +D_L, whose inverse is the
// fermionic (I + B)^-1 in its G(0,0) block).  The chain's own state is not
// touched: the pass works on copies in its own region of global memory, with
// the routines of the N <= 144 class (2N <= 144 rows).
namespace taud {
// The pass of an N <= 36 chain runs in the N <= 72 class's context (2N <= 72;
// G and U in shared memory, register-resident factorisations), that of a
// 36 < N <= 72 chain in the N <= 144 class's.  Matrices of the region have the
// class's leading dimension.
template <int NMAX> constexpr int LD = Cfg<NMAX>::LD;
template <int NMAX> constexpr long long MAT = (long long)NMAX * Cfg<NMAX>::LD;   // complex values per slot
// slots of a CTA's region; 0..4 are the class context's W1, W2 (and, N <= 144, G, U, S)
// (G holds G(0,0) of the pass, U the propagated right factor U_R)
enum { GT0 = 5, G0T = 6, GTT = 7, VR = 8, BIG = 9, X = 10, VRI = 11, VLI = 12, UL = 13, VEC = 14, EP = 15, EM = 16, SLOTS = 17 };
constexpr long long REGION = SLOTS * MAT<144>;   // the larger class's region serves both
template <int NMAX> DEVI cplx* slot(const Ctx<NMAX>& x, int k) { return x.wg + k * MAT<NMAX>; }
}  // namespace taud

long long tau_region_elems() { return taud::REGION; }

// C <- A^-1 C for the x.n x x.n matrix A, which is destroyed: pivoted QR,
// Q^H C, R^-1 D^-1, the row permutation back.
template <int NMAX>
COLD void tau_solve(Ctx<NMAX>& x, cplx* A, cplx* C) {
    qrp_any(x, A);
    apply_qh_left_any(x, A, C);
    cplx* rinv = reinterpret_cast<cplx*>(x.s.vn1());
    double* dinv = x.s.u2();
    diag_inverse(x.n, taud::LD<NMAX>, A, x.s.d(), rinv, dinv);
    trsm_left_any(x, A, rinv, dinv, C);
    permute_rows_any(x, C, false);
}

template <int NMAX>
DEVI void tau_copy(int n, cplx* dst, const cplx* src) {   // both with the class's leading dimension
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - r * n;
        dst[r * taud::LD<NMAX> + c] = src[r * taud::LD<NMAX> + c];
    }
    __syncthreads();
}

// L1 distance of two n x n matrices (compare_mat, stabilization.f90:256-266),
// valid in thread 0
template <int NMAX>
DEVI double tau_l1(Ctx<NMAX>& x, int n, const cplx* a, const cplx* b) {
    double v[1] = {0.0};
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - r * n;
        const cplx d = csub(a[r * taud::LD<NMAX> + c], b[r * taud::LD<NMAX> + c]);
        v[0] += sqrt(d.x * d.x + d.y * d.y);
    }
    block_sum<1>(v, x.s.red());
    return v[0];
}

// slice nt (1-based, propgrU_R then propgrT_R, multiply.f90:48-97 of both
// solvers): the HS factors of both channels, then e^{-dtau K} from the left and
// e^{+dtau K} from the right (real, in the EP and EM slots)
template <int NMAX>
COLD void tau_slice(Ctx<NMAX>& x, int nt) {
    constexpr int LD = taud::LD<NMAX>;
    const int n = x.n;
    const PointDev& P = x.P();
    cplx *T0 = taud::slot(x, taud::GT0), *T1 = taud::slot(x, taud::G0T), *T2 = taud::slot(x, taud::GTT);
    cplx* U = x.U();
    cplx *ep = x.s.ean(), *em = x.s.ebn();
    for (int ch = 0; ch < 2; ++ch) {
        if (!P.active[ch]) continue;
        // row i's factor e^{+-alpha phi}; on a Nambu chain's {b, c^dagger} block
        // row Ns + i (c^dagger_i) takes site i's field, with the inverse factor in
        // a flipped channel (src/pairing/src/operator_Hubbard.f90:139-199)
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const bool cd = i >= P.Ns;
            const int site = cd ? i - P.Ns : i;
            cplx a, b;
            hs_factors(P.alpha_re[ch], P.alpha_im[ch], x.phi[((long)(nt - 1) * P.Ns + site) * 2 + ch], a, b);
            const bool inv = cd && P.flip[ch];
            ep[i] = inv ? b : a;
            em[i] = inv ? a : b;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
            const int r = e / n, c = e - r * n;
            T0[r * LD + c] = cmul(ep[r], T0[r * LD + c]);
            T1[r * LD + c] = cmul(T1[r * LD + c], em[c]);
            T2[r * LD + c] = cmul(cmul(ep[r], T2[r * LD + c]), em[c]);
            U[r * LD + c] = cmul(ep[r], U[r * LD + c]);
        }
        __syncthreads();
    }
    const double *kp = reinterpret_cast<const double*>(taud::slot(x, taud::EP)),
                 *km = reinterpret_cast<const double*>(taud::slot(x, taud::EM));
    gemm_real_any<NMAX, false>(x, T0, kp, T0);
    gemm_real_any<NMAX, true>(x, T1, T1, km);
    gemm_real_any<NMAX, false>(x, T2, kp, T2);
    gemm_real_any<NMAX, true>(x, T2, T2, km);
    gemm_real_any<NMAX, false>(x, U, kp, U);
}

// Wrap_tau at slice nt (stabilization.f90:368-404): stab_UR of the propagated
// right factors, the 2N x 2N inverse, the drifts of G(0,tau), G(tau,0),
// G(tau,tau) against the propagated ones (thread 0 accumulates them in dr:
// max[3], sum[3], non-finite count), then the replacement.
template <int NMAX>
COLD void tau_wrap(Ctx<NMAX>& x, const Arena& A, int nt, double* dr) {
    using namespace taud;
    constexpr int LD = taud::LD<NMAX>;
    const int n = x.n, st = nt / x.P().Nwrap;
    cplx *W1 = x.W1(), *W2 = x.W2(), *U = x.U();
    cplx *M = slot(x, BIG), *Xi = slot(x, X), *VRi = slot(x, VRI), *VLi = slot(x, VLI), *ULs = slot(x, UL);
    stab_UR(x);                      // U = U_R, A.DRc = D_R, A.VRc and W2 = V_R
    tau_copy<NMAX>(n, M, W2);
    set_identity(n, LD, VRi);
    __syncthreads();
    tau_solve(x, M, VRi);            // V_R^-1
    sload(n, LD, M, A.VLs(st));
    set_identity(n, LD, VLi);
    __syncthreads();
    tau_solve(x, M, VLi);            // V_L^-1
    sload(n, LD, ULs, A.ULs(st));
    for (int e = threadIdx.x; e < 4 * n * n; e += blockDim.x) {
        const int r = e / (2 * n), c = e - r * (2 * n);
        M[r * LD + c] = cmk(0.0, 0.0);
    }
    __syncthreads();
    gemm_any(x, M, op_n(VLi, LD), op_n(VRi, LD));               // (V_R V_L)^-1
    gemm_any(x, M + n * LD + n, op_c(U, LD), op_c(ULs, LD));    // (U_L U_R)^H
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const cplx dl = A.DLs(st)[i], drv = A.DRc[i];
        M[i * LD + n + i] = cmk(-dl.x, -dl.y);
        M[(n + i) * LD + i] = cmk(-drv.x, -drv.y);
    }
    x.n = 2 * n;
    set_identity(2 * n, LD, Xi);
    __syncthreads();
    tau_solve(x, M, Xi);
    x.n = n;
    // G(0,0) = V_R^-1 X00 V_L^-1
    gemm_any(x, W1, op_n(VRi, LD), op_n(Xi, LD));
    gemm_any(x, x.G(), op_n(W1, LD), op_n(VLi, LD));
    // index 0: G(0,tau) = V_R^-1 X01 U_R^H; 1: G(tau,0) = U_L^H X10 V_L^-1; 2: G(tau,tau) = U_L^H X11 U_R^H
    cplx* dst[3] = {slot(x, G0T), slot(x, GT0), slot(x, GTT)};
    const MatOp left[3] = {op_n(VRi, LD), op_c(ULs, LD), op_c(ULs, LD)};
    const cplx* blk[3] = {Xi + n, Xi + n * LD, Xi + n * LD + n};
    const MatOp right[3] = {op_c(U, LD), op_n(VLi, LD), op_c(U, LD)};
    for (int k = 0; k < 3; ++k) {
        gemm_any(x, W1, left[k], op_n(blk[k], LD));
        gemm_any(x, W2, op_n(W1, LD), right[k]);
        const double dif = tau_l1(x, n, W2, dst[k]);
        if (threadIdx.x == 0) {
            if (dif == dif && dif <= 1.0e300) {
                if (dif > dr[k]) dr[k] = dif;
                dr[3 + k] += dif;
            } else {
                dr[6] += 1.0;
            }
        }
        tau_copy<NMAX>(n, dst[k], W2);
    }
}

// Dyn_reset + Dyn_sweep_R of one chain (dynamics.f90:37-57): copies of G and of
// the right factors, L slices, a wrap every Nwrap slices; the arena's D_R and
// V_R (which stab_UR updates) are put back at the end.
template <int NMAX>
COLD void tau_pass(Ctx<NMAX>& x, const KernelArgs& ka, int chain) {
    using namespace taud;
    constexpr int LD = taud::LD<NMAX>;
    const int n = x.n, L = x.P().L;
    const Arena A = x.A();
    cplx *G = x.G(), *T0 = slot(x, GT0), *T1 = slot(x, G0T), *T2 = slot(x, GTT);
    cplx *sv = slot(x, VEC), *svr = slot(x, VR);
    gcopy(sv, A.DRc, n);
    gcopy(svr, A.VRc, n * n);
    sload_real(n, LD, reinterpret_cast<double*>(slot(x, EP)), x.P().expP);
    sload_real(n, LD, reinterpret_cast<double*>(slot(x, EM)), x.P().expM);
    sload(n, LD, G, A.G);
    sload(n, LD, x.U(), A.URc);
    __syncthreads();
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - r * n;
        const cplx g = G[r * LD + c];
        T0[r * LD + c] = g;
        T2[r * LD + c] = g;
        T1[r * LD + c] = cmk(g.x - (r == c ? 1.0 : 0.0), g.y);   // -(I - G)
    }
    __syncthreads();
    double dr[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int nt = 1; nt <= L; ++nt) {
        tau_slice(x, nt);
        if (nt % x.P().Nwrap == 0) tau_wrap(x, A, nt, dr);
        if (nt == ka.tau_probe_nt && ka.tau_probe) {
            cplx* pr = ka.tau_probe + (long long)chain * kTauProbeElems;
            const cplx* src[4] = {G, T1, T0, T2};   // G(0,0), G(0,tau), G(tau,0), G(tau,tau)
            for (int k = 0; k < 4; ++k) sstore(n, LD, pr + (long long)k * n * n, src[k]);
        }
    }
    gcopy(A.DRc, sv, n);
    gcopy(A.VRc, svr, n * n);
    if (threadIdx.x == 0) {
        double* o = ka.tau_stats + (long long)chain * kTauStats;
        for (int k = 0; k < 3; ++k) {
            o[k] = fmax(o[k], dr[k]);
            o[3 + k] += dr[3 + k];
        }
        o[6] += 1.0;
        o[7] += dr[6];
    }
    __syncthreads();
}

// One CTA per SM walks its share of the listed chains; its matrix region of
// tau_region_elems() complex values is indexed by blockIdx.x.  The N <= 72
// class's kernel takes the chains with N <= 36, the N <= 144 class's those
// with 36 < N <= kTauMaxN.
template <int NMAX>
__global__ void __launch_bounds__(Cfg<NMAX>::THREADS, 1) tau_kernel(KernelArgs ka, const int* idx, int count) {
    for (int k = blockIdx.x; k < count; k += gridDim.x) {
        const int chain = idx[k];
        Ctx<NMAX> x;
        const bool ok = setup_ctx(x, ka, chain) && 2 * x.n <= NMAX && (NMAX == 72 || 2 * x.n > 72) &&
                        x.n <= kTauMaxN && !(x.sc->status & 1);
        if (ok) {
            x.wg = ka.tau_ws + (long long)blockIdx.x * taud::REGION;
            tau_pass(x, ka, chain);
        }
        __syncthreads();
    }
}

template <int NMAX>
static cudaError_t launch_tau_cls(const KernelArgs& ka, const int* idx, int count, int grid, cudaStream_t st) {
    const size_t sm = Smem<NMAX>::bytes();
    const cudaError_t e = cudaFuncSetAttribute(tau_kernel<NMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    tau_kernel<NMAX><<<grid < count ? grid : count, Cfg<NMAX>::THREADS, sm, st>>>(ka, idx, count);
    return cudaGetLastError();
}
cudaError_t launch_tau(const KernelArgs& ka, const int* idx, int count, int grid, cudaStream_t st) {
    if (count <= 0) return cudaSuccess;
    const cudaError_t e = launch_tau_cls<72>(ka, idx, count, grid, st);
    return e != cudaSuccess ? e : launch_tau_cls<144>(ka, idx, count, grid, st);
}

// ---------------------------------------------------------------------------
template <int NMAX, bool PAIR>
static cudaError_t launch_cls(int which, const KernelArgs& ka, const int* idx, int count, cudaStream_t st) {
    if (count <= 0) return cudaSuccess;
    const size_t sm = Smem<NMAX>::bytes();
    cudaError_t e;
    if (which == 0) {
        e = cudaFuncSetAttribute(sweep_kernel<NMAX, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        sweep_kernel<NMAX, PAIR><<<count, Cfg<NMAX>::THREADS, sm, st>>>(ka, idx, count);
    } else {
        e = cudaFuncSetAttribute(pre_kernel<NMAX, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        pre_kernel<NMAX, PAIR><<<count, Cfg<NMAX>::THREADS, sm, st>>>(ka, idx, count);
    }
    return cudaGetLastError();
}

// class index: size class (NMAX 16 / 36 / 72) + 3 * Nambu sector; 6 = NMAX 144, number-conserving
static cudaError_t launch_any(int which, int cls, const KernelArgs& ka, const int* idx, int count, cudaStream_t st) {
    switch (cls) {
        case 0: return launch_cls<16, false>(which, ka, idx, count, st);
        case 1: return launch_cls<36, false>(which, ka, idx, count, st);
        case 2: return launch_cls<72, false>(which, ka, idx, count, st);
        case 3: return launch_cls<16, true>(which, ka, idx, count, st);
        case 4: return launch_cls<36, true>(which, ka, idx, count, st);
        case 5: return launch_cls<72, true>(which, ka, idx, count, st);
        case 6: return launch_cls<144, false>(which, ka, idx, count, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t upload_pow_table(const uint32_t* tab, int count) {
    if (count > kMaxPow) return cudaErrorInvalidValue;
    return cudaMemcpyToSymbol(c_apow, tab, sizeof(uint32_t) * count);
}

cudaError_t launch_sweep(int cls, const KernelArgs& ka, const int* idx, int count, cudaStream_t st) {
    return launch_any(0, cls, ka, idx, count, st);
}
cudaError_t launch_pre(int cls, const KernelArgs& ka, const int* idx, int count, cudaStream_t st) {
    return launch_any(1, cls, ka, idx, count, st);
}
cudaError_t launch_warmup(const KernelArgs& ka, int nwarm, cudaStream_t st) {
    warmup_kernel<<<ka.nchains, 256, 0, st>>>(ka, nwarm);
    return cudaGetLastError();
}
cudaError_t launch_bin_reset(const KernelArgs& ka, cudaStream_t st) {
    bin_reset_kernel<<<ka.nchains, 64, 0, st>>>(ka);
    return cudaGetLastError();
}
cudaError_t launch_bin_finish(const KernelArgs& ka, cudaStream_t st) {
    bin_finish_kernel<<<ka.nchains, 64, 0, st>>>(ka);
    return cudaGetLastError();
}
cudaError_t launch_point_average(const KernelArgs& ka, int npts, const int* start, const int* list, double* out,
                                 cudaStream_t st) {
    point_average_kernel<<<npts, 64, 0, st>>>(ka, start, list, out);
    return cudaGetLastError();
}
cudaError_t launch_stats_add(const double* pout, double* cur, double* blk, int n, int finish, int block_size,
                             cudaStream_t st) {
    stats_add_kernel<<<(n + 255) / 256, 256, 0, st>>>(pout, cur, blk, n, finish, block_size);
    return cudaGetLastError();
}
cudaError_t launch_stats_final(const double* blk, int nb, int n, double* mean, double* sem, cudaStream_t st) {
    stats_final_kernel<<<(n + 255) / 256, 256, 0, st>>>(blk, nb, n, mean, sem);
    return cudaGetLastError();
}
cudaError_t launch_global_propose(const KernelArgs& ka, const KernelArgs& kp, const double* shift, cudaStream_t st) {
    global_propose_kernel<<<ka.nchains, 256, 0, st>>>(ka, kp, shift[0], shift[1]);
    return cudaGetLastError();
}
cudaError_t launch_global_accept(const KernelArgs& ka, const KernelArgs& kp, const double* fn, const double* fn2,
                                 const double* hastings, int* accepted, cudaStream_t st) {
    global_accept_kernel<<<ka.nchains, 256, 0, st>>>(ka, kp, fn, fn2, hastings, accepted);
    return cudaGetLastError();
}
cudaError_t launch_field_check(const KernelArgs& ka, int* bad, cudaStream_t st) {
    field_check_kernel<<<ka.nchains, 256, 0, st>>>(ka, bad);
    return cudaGetLastError();
}
cudaError_t launch_field_norm(const KernelArgs& ka, double* out, cudaStream_t st) {
    field_norm_kernel<<<ka.nchains, 256, 0, st>>>(ka, out);
    return cudaGetLastError();
}
long long class_work_elems(int cls) {
    if (cls == 6) return 5LL * 144 * Cfg<144>::LD;   // W1, W2, G, U, product scratch
    const int sz = cls % 3;
    auto w = [](int nmax, int ld, bool gw) { return gw ? 2LL * nmax * ld : 0LL; };
    return sz == 0 ? w(16, Cfg<16>::LD, Cfg<16>::GW)
                   : (sz == 1 ? w(36, Cfg<36>::LD, Cfg<36>::GW) : w(72, Cfg<72>::LD, Cfg<72>::GW));
}
size_t smem_bytes(int cls) {
    if (cls == 6) return Smem<144>::bytes();
    const int sz = cls % 3;
    return sz == 0 ? Smem<16>::bytes() : (sz == 1 ? Smem<36>::bytes() : Smem<72>::bytes());
}
int class_nmax(int cls) {
    if (cls == 6) return 144;
    const int sz = cls % 3;
    return sz == 0 ? 16 : (sz == 1 ? 36 : 72);
}
int class_of(int n, int pairing) {
    for (int c = 0; c < 3; ++c)
        if (n <= class_nmax(c)) return c + (pairing ? 3 : 0);
    if (!pairing && n <= 144) return 6;
    return -1;
}

}  // namespace bq
