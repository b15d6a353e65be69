// CTA-level dense complex FP64 linear algebra on matrices resident in shared
// memory (row-major n x n with leading dimension ld; the sweep kernels use an
// odd ld so that a column walk touches every shared-memory bank group).  Every routine is called by all
// threads of the block and returns with the block synchronised.
//
// These restate the LAPACK/BLAS operations the reference sweep calls
// (src/number_conserving/src/stabilization.f90:41-190 and
// src/common/mymats.f90:20-29): ZGEMM, ZTRMM, ZGEQP3 (unblocked ZLAQP2 path,
// which LAPACK takes for the matrix sizes here), ZUNGQR, ZUNMQR, ZTRSM,
// ZLAPMR/ZLAPMT.  They are written for the sweep's sizes (n <= 64): one CTA
// owns one matrix.  The reflector and triangular-solve sequences run on 8-lane
// segments that each keep their columns (or rows) of the operand in registers
// for the whole sequence and reduce with shuffles, so no step needs a block
// barrier; divisions are replaced by precomputed reciprocals.
#pragma once
#include "cplx.cuh"

// Factorisation routines are kept out of line: they run once per wrap, and
// inlining them into the sweep kernel costs registers on the per-slice path.
#define COLD static __device__ __noinline__

// Strided operand view: element (r, c) = p[r*sr + c*sc], optionally conjugated.
// A transposed view swaps the strides.  p may point to shared or global memory.
struct MatOp {
    const cplx* p;
    int sr, sc;
    int cj;
    DEVI cplx at(int r, int c) const {
        cplx v = p[(long)r * sr + (long)c * sc];
        return cj ? cconj(v) : v;
    }
};
DEVI MatOp op_n(const cplx* p, int ld) { return MatOp{p, ld, 1, 0}; }
DEVI MatOp op_c(const cplx* p, int ld) { return MatOp{p, 1, ld, 1}; }   // conjugate transpose

enum { TRI_NONE = 0, TRI_A_UPPER = 1, TRI_B_LOWER_FROM_C = 2 };

// C = A * B for n x n operands, each thread computing a TR x TC micro-tile.
// C may alias A or B: results are staged in registers across a barrier.
// tri = TRI_A_UPPER zeroes A(r,k) for k < r (ZTRMM 'L','U','N');
// tri = TRI_B_LOWER_FROM_C zeroes B(k,c) for k < c (ZTRMM 'R','U','C').
template <int TR, int TC>
COLD void gemm_rs(int n, int ld, cplx* C, MatOp A, MatOp B, int tri = TRI_NONE) {
    const int ncg = (n + TC - 1) / TC, nrg = (n + TR - 1) / TR;
    const int g = threadIdx.x;
    const bool active = g < ncg * nrg;
    const int r0 = active ? (g / ncg) * TR : 0, c0 = active ? (g % ncg) * TC : 0;
    cplx acc[TR][TC];
#pragma unroll
    for (int i = 0; i < TR; ++i)
#pragma unroll
        for (int j = 0; j < TC; ++j) acc[i][j] = cmk(0.0, 0.0);
    if (active) {
        for (int k = 0; k < n; ++k) {
            cplx a[TR], b[TC];
#pragma unroll
            for (int i = 0; i < TR; ++i) {
                int r = r0 + i;
                a[i] = (r < n) ? A.at(r, k) : cmk(0.0, 0.0);
                if (tri == TRI_A_UPPER && k < r) a[i] = cmk(0.0, 0.0);
            }
#pragma unroll
            for (int j = 0; j < TC; ++j) {
                int c = c0 + j;
                b[j] = (c < n) ? B.at(k, c) : cmk(0.0, 0.0);
                if (tri == TRI_B_LOWER_FROM_C && k < c) b[j] = cmk(0.0, 0.0);
            }
#pragma unroll
            for (int i = 0; i < TR; ++i)
#pragma unroll
                for (int j = 0; j < TC; ++j) acc[i][j] = cfma(a[i], b[j], acc[i][j]);
        }
    }
    __syncthreads();
    if (active) {
#pragma unroll
        for (int i = 0; i < TR; ++i)
#pragma unroll
            for (int j = 0; j < TC; ++j) {
                int r = r0 + i, c = c0 + j;
                if (r < n && c < n) C[r * ld + c] = acc[i][j];
            }
    }
    __syncthreads();
}

// C = A * B with A, B, C n x n row-major in shared memory (C may alias A or
// B); the per-slice propagation products.
template <int TR, int TC>
DEVI void gemm_smem(int n, int ld, cplx* C, const cplx* A, const cplx* B) {
    const int ncg = (n + TC - 1) / TC, nrg = (n + TR - 1) / TR;
    const int g = threadIdx.x;
    const bool active = g < ncg * nrg;
    const int r0 = active ? (g / ncg) * TR : 0, c0 = active ? (g % ncg) * TC : 0;
    cplx acc[TR][TC];
#pragma unroll
    for (int i = 0; i < TR; ++i)
#pragma unroll
        for (int j = 0; j < TC; ++j) acc[i][j] = cmk(0.0, 0.0);
    if (active) {
        int ra[TR], cb[TC];
#pragma unroll
        for (int i = 0; i < TR; ++i) ra[i] = min(r0 + i, n - 1) * ld;
#pragma unroll
        for (int j = 0; j < TC; ++j) cb[j] = min(c0 + j, n - 1);
        for (int k = 0; k < n; ++k) {
            cplx a[TR], b[TC];
#pragma unroll
            for (int i = 0; i < TR; ++i) a[i] = A[ra[i] + k];
#pragma unroll
            for (int j = 0; j < TC; ++j) b[j] = B[k * ld + cb[j]];
#pragma unroll
            for (int i = 0; i < TR; ++i)
#pragma unroll
                for (int j = 0; j < TC; ++j) acc[i][j] = cfma(a[i], b[j], acc[i][j]);
        }
    }
    __syncthreads();
    if (active) {
#pragma unroll
        for (int i = 0; i < TR; ++i)
#pragma unroll
            for (int j = 0; j < TC; ++j) {
                const int r = r0 + i, c = c0 + j;
                if (r < n && c < n) C[r * ld + c] = acc[i][j];
            }
    }
    __syncthreads();
}

// The slice propagators e^{-+dtau K} are real (real hopping, chemical
// potential and pairing amplitude), so the per-slice products are complex x
// real.  Real operands are stored as doubles with the same leading dimension.
// acc += a * b with real b is (fma(a.x, b, acc.x), fma(a.y, b, acc.y)): the same
// values as the complex product with a zero imaginary part, in half the FLOPs.
template <int TR, int TC, bool RIGHT_REAL>
DEVI void gemm_smem_real(int n, int ld, cplx* C, const void* Ap, const void* Bp) {
    const int ncg = (n + TC - 1) / TC, nrg = (n + TR - 1) / TR;
    const int g = threadIdx.x;
    const bool active = g < ncg * nrg;
    const int r0 = active ? (g / ncg) * TR : 0, c0 = active ? (g % ncg) * TC : 0;
    cplx acc[TR][TC];
#pragma unroll
    for (int i = 0; i < TR; ++i)
#pragma unroll
        for (int j = 0; j < TC; ++j) acc[i][j] = cmk(0.0, 0.0);
    if (active) {
        int ra[TR], cb[TC];
#pragma unroll
        for (int i = 0; i < TR; ++i) ra[i] = min(r0 + i, n - 1) * ld;
#pragma unroll
        for (int j = 0; j < TC; ++j) cb[j] = min(c0 + j, n - 1);
        for (int k = 0; k < n; ++k) {
            if (RIGHT_REAL) {   // C = A (complex) * B (real)
                const cplx* A = static_cast<const cplx*>(Ap);
                const double* B = static_cast<const double*>(Bp);
                cplx a[TR];
                double b[TC];
#pragma unroll
                for (int i = 0; i < TR; ++i) a[i] = A[ra[i] + k];
#pragma unroll
                for (int j = 0; j < TC; ++j) b[j] = B[k * ld + cb[j]];
#pragma unroll
                for (int i = 0; i < TR; ++i)
#pragma unroll
                    for (int j = 0; j < TC; ++j)
                        acc[i][j] = cmk(fma(a[i].x, b[j], acc[i][j].x), fma(a[i].y, b[j], acc[i][j].y));
            } else {            // C = A (real) * B (complex)
                const double* A = static_cast<const double*>(Ap);
                const cplx* B = static_cast<const cplx*>(Bp);
                double a[TR];
                cplx b[TC];
#pragma unroll
                for (int i = 0; i < TR; ++i) a[i] = A[ra[i] + k];
#pragma unroll
                for (int j = 0; j < TC; ++j) b[j] = B[k * ld + cb[j]];
#pragma unroll
                for (int i = 0; i < TR; ++i)
#pragma unroll
                    for (int j = 0; j < TC; ++j)
                        acc[i][j] = cmk(fma(a[i], b[j].x, acc[i][j].x), fma(a[i], b[j].y, acc[i][j].y));
            }
        }
    }
    __syncthreads();
    if (active) {
#pragma unroll
        for (int i = 0; i < TR; ++i)
#pragma unroll
            for (int j = 0; j < TC; ++j) {
                const int r = r0 + i, c = c0 + j;
                if (r < n && c < n) C[r * ld + c] = acc[i][j];
            }
    }
    __syncthreads();
}

// dst = op(src) elementwise copy for an n x n matrix (dst must not alias src
// unless op is the identity view).
COLD void copy_op(int n, int ld, cplx* dst, MatOp src) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - (e / n) * n;
        dst[r * ld + c] = src.at(r, c);
    }
    __syncthreads();
}

// In-place conjugate transpose via register staging; MAXE >= ceil(n*n/blockDim).
template <int MAXE>
COLD void conj_transpose_inplace(int n, int ld, cplx* A) {
    cplx v[MAXE];
#pragma unroll
    for (int k = 0; k < MAXE; ++k) {
        const int e = threadIdx.x + k * blockDim.x;
        if (e < n * n) {
            const int r = e / n, c = e - (e / n) * n;
            v[k] = cconj(A[c * ld + r]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < MAXE; ++k) {
        const int e = threadIdx.x + k * blockDim.x;
        if (e < n * n) {
            const int r = e / n, c = e - (e / n) * n;
            A[r * ld + c] = v[k];
        }
    }
    __syncthreads();
}

// Segmented (8-lane) reductions used by the column-parallel reflector passes.
// The mask covers only the calling thread's aligned 8-lane segment, so the
// segments of one warp may run different trip counts.
DEVI unsigned seg8_mask() { return 0xffu << (threadIdx.x & 24); }
DEVI double seg8_sum(double v) {
    const unsigned m = seg8_mask();
    v += __shfl_xor_sync(m, v, 4);
    v += __shfl_xor_sync(m, v, 2);
    v += __shfl_xor_sync(m, v, 1);
    return v;
}
DEVI double seg8_max(double v) {
    const unsigned m = seg8_mask();
    v = fmax(v, __shfl_xor_sync(m, v, 4));
    v = fmax(v, __shfl_xor_sync(m, v, 2));
    v = fmax(v, __shfl_xor_sync(m, v, 1));
    return v;
}

// Overflow-safe 2-norm of column j, rows [r0, n), computed by one 8-lane segment.
DEVI double seg8_colnorm(int n, int ld, const cplx* A, int j, int r0, int lane8) {
    double m = 0.0;
    for (int r = r0 + lane8; r < n; r += 8) m = fmax(m, fmax(fabs(A[r * ld + j].x), fabs(A[r * ld + j].y)));
    m = seg8_max(m);
    if (m == 0.0) return 0.0;
    double s = 0.0;
    for (int r = r0 + lane8; r < n; r += 8) {
        double a = A[r * ld + j].x / m, b = A[r * ld + j].y / m;
        s += a * a + b * b;
    }
    s = seg8_sum(s);
    return m * sqrt(s);
}

// Sum of squares of column j, rows r0..n-1, by one 8-lane segment.
DEVI double seg8_sumsq_col(int n, int ld, const cplx* A, int j, int r0, int lane8) {
    double ss = 0.0;
    for (int r = r0 + lane8; r < n; r += 8) {
        const cplx a = A[r * ld + j];
        ss = fma(a.x, a.x, fma(a.y, a.y, ss));
    }
    return seg8_sum(ss);
}

DEVI bool sumsq_unsafe(double ss) { return !(ss <= 1.0e300) || (ss != 0.0 && ss < 1.0e-290); }

// 2-norm of column j rows r0..n-1 (one segment); scaled only when the plain sum
// of squares would over- or underflow.
DEVI double seg8_norm(int n, int ld, const cplx* A, int j, int r0, int lane8) {
    const double ss = seg8_sumsq_col(n, ld, A, j, r0, lane8);
    if (!sumsq_unsafe(ss)) return sqrt(ss);
    return seg8_colnorm(n, ld, A, j, r0, lane8);
}

// Shared scratch for the factorisations (lives in shared memory, size ~ 6n).
struct QRScratch {
    cplx* tau;      // n
    int* piv;       // n   (0-based: (A P)[:, j] = A[:, piv[j]])
    int* ipiv;      // n   inverse permutation
    double* vn1;    // n
    double* vn2;    // n
    double* d;      // n   |R_ii|
    cplx* bcast;    // 4   broadcast slots
    int* ibcast;    // 4
};

// ZGEQP3 (unblocked ZLAQP2 recurrence) on A (n x n) followed by the reference's
// QDRP_decompose post-step (stabilization.f90:41-67): d[i] = |R_ii| and row i of
// the upper triangle divided by d[i].  On exit A holds the scaled R in its upper
// triangle and the Householder vectors (unit leading entry implicit) below it.
//
// Two barriers per column.  Every warp finds the pivot (IDAMAX of the partial
// norms) and every 8-lane segment forms the reflector (ZLARFG) itself from the
// pivot column, so neither needs a barrier of its own; each segment keeps its
// target columns in registers from the read phase to the write phase.  The
// norm downdate is ZLAQP2's, with its quotients multiplied out (no division).
// R8 >= ceil(n/8) rows per lane, CPS >= ceil(n/segments) columns per segment.
template <int R8, int CPS>
COLD void qrp_inplace(int n, int ld, cplx* A, QRScratch s) {
    const int tid = threadIdx.x, lane = tid & 31, lane8 = tid & 7, seg = tid >> 3, nseg = blockDim.x >> 3;
    const double tol3z = 1.0536712127723509e-08;   // sqrt(2^-53), LAPACK's sqrt(dlamch('E'))
    for (int j = seg; j < n; j += nseg) {
        const double v = seg8_norm(n, ld, A, j, 0, lane8);
        if (lane8 == 0) { s.vn1[j] = v; s.vn2[j] = v; s.piv[j] = j; }
    }
    __syncthreads();
    for (int i = 0; i < n; ++i) {
        // pivot: first index of max vn1[i..n) (IDAMAX), every warp
        double best = -1.0;
        int bi = n;
        for (int j = i + lane; j < n; j += 32) {
            const double v = s.vn1[j];
            if (v > best) { best = v; bi = j; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
        }
        const int pvt = (bi < n) ? bi : i;   // all-NaN norms: keep column i
        // reflector of the pivot column (ZLARFG), every segment
        cplx v[R8];
        double ss = 0.0;
#pragma unroll
        for (int k = 0; k < R8; ++k) {
            const int r = lane8 + 8 * k;
            v[k] = (r < n && r > i) ? A[r * ld + pvt] : cmk(0.0, 0.0);
            ss = fma(v[k].x, v[k].x, fma(v[k].y, v[k].y, ss));
        }
        ss = seg8_sum(ss);
        const cplx alpha = A[i * ld + pvt];
        double xn = sqrt(ss);
        if (sumsq_unsafe(ss)) xn = seg8_colnorm(n, ld, A, pvt, i + 1, lane8);
        cplx tau = cmk(0.0, 0.0), beta = alpha, scl = cmk(0.0, 0.0);
        if (!(xn == 0.0 && alpha.y == 0.0)) {
            const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn * xn);
            const double b = (alpha.x >= 0.0) ? -nrm : nrm;
            const double ib = 1.0 / b;
            tau = cmk((b - alpha.x) * ib, -alpha.y * ib);
            const cplx d = cmk(alpha.x - b, alpha.y);           // scl = 1 / d
            const double id2 = 1.0 / (d.x * d.x + d.y * d.y);
            scl = cmk(d.x * id2, -d.y * id2);
            beta = cmk(b, 0.0);
        }
#pragma unroll
        for (int k = 0; k < R8; ++k) {
            const int r = lane8 + 8 * k;
            v[k] = (r == i) ? cmk(1.0, 0.0) : cmul(scl, v[k]);
        }
        // target columns j = i+1+seg+q*nseg; logical column pvt holds the old column i
        cplx a[CPS][R8];
        double t1[CPS], t2[CPS];
#pragma unroll
        for (int q = 0; q < CPS; ++q) {
            const int j = i + 1 + seg + q * nseg;
            const int src = (j == pvt) ? i : j;
            const bool ok = j < n;
#pragma unroll
            for (int k = 0; k < R8; ++k) {
                const int r = lane8 + 8 * k;
                a[q][k] = (ok && r < n && r >= i) ? A[r * ld + src] : cmk(0.0, 0.0);
            }
            t1[q] = ok ? s.vn1[src] : 0.0;
            t2[q] = ok ? s.vn2[src] : 0.0;
        }
        cplx ui = cmk(0.0, 0.0), up = cmk(0.0, 0.0);   // rows < i of columns i and pvt
        if (tid < i) {
            ui = A[tid * ld + i];
            up = A[tid * ld + pvt];
        }
        __syncthreads();
        if (pvt != i && tid < i) {
            A[tid * ld + i] = up;
            A[tid * ld + pvt] = ui;
        }
        if (seg == 0) {
#pragma unroll
            for (int k = 0; k < R8; ++k) {
                const int r = lane8 + 8 * k;
                if (r < n && r > i) A[r * ld + i] = v[k];
            }
            if (lane8 == 0) {
                A[i * ld + i] = beta;
                s.tau[i] = tau;
            }
        }
        if (tid == 0 && pvt != i) {
            const int t = s.piv[pvt];
            s.piv[pvt] = s.piv[i];
            s.piv[i] = t;
        }
        const cplx ctau = cconj(tau);
#pragma unroll
        for (int q = 0; q < CPS; ++q) {
            const int j = i + 1 + seg + q * nseg;
            if (j >= n) continue;   // uniform within the segment
            cplx w = cmk(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < R8; ++k) w = cfmacj(v[k], a[q][k], w);
            w.x = seg8_sum(w.x);
            w.y = seg8_sum(w.y);
            const cplx f = cmul(ctau, w);
            double ai2 = 0.0, rest = 0.0;
#pragma unroll
            for (int k = 0; k < R8; ++k) {
                const int r = lane8 + 8 * k;
                a[q][k] = csub(a[q][k], cmul(v[k], f));
                const double m2 = a[q][k].x * a[q][k].x + a[q][k].y * a[q][k].y;
                if (r == i) ai2 = m2;
                if (r > i && r < n) rest += m2;
                if (r < n && r >= i) A[r * ld + j] = a[q][k];
            }
            ai2 = seg8_sum(ai2);
            rest = seg8_sum(rest);
            // ZLAQP2 norm downdate: temp = max(1 - (|a_ij|/vn1)^2, 0),
            // recompute if temp (vn1/vn2)^2 <= tol3z, else vn1 *= sqrt(temp);
            // written as max(vn1^2 - |a_ij|^2, 0) against tol3z vn2^2.
            const double v1 = t1[q];
            double nv1 = v1, nv2 = t2[q];
            if (v1 != 0.0) {
                bool recompute;
                if (v1 < 1.0e150 && t2[q] < 1.0e150) {
                    const double rem = fmax(v1 * v1 - ai2, 0.0);   // = temp * vn1^2
                    recompute = rem <= tol3z * t2[q] * t2[q];
                    nv1 = sqrt(rem);
                } else {
                    const double tt = sqrt(ai2) / v1;
                    const double temp = fmax(1.0 - tt * tt, 0.0);
                    const double qq = v1 / t2[q];
                    recompute = !(temp * qq * qq > tol3z);
                    nv1 = v1 * sqrt(temp);
                }
                if (recompute) {
                    if (sumsq_unsafe(rest)) {
                        __syncwarp(seg8_mask());
                        nv1 = (i + 1 < n) ? seg8_colnorm(n, ld, A, j, i + 1, lane8) : 0.0;
                    } else {
                        nv1 = sqrt(rest);
                    }
                    nv2 = nv1;
                }
            }
            if (lane8 == 0) {
                s.vn1[j] = nv1;
                s.vn2[j] = nv2;
            }
        }
        __syncthreads();
    }
    // D = |diag R|, rows of the upper triangle scaled by 1/D
    for (int i = tid; i < n; i += blockDim.x) {
        const cplx a = A[i * ld + i];
        const double d = hypot(a.x, a.y);
        s.d[i] = d;
        s.vn1[i] = 1.0 / d;
    }
    __syncthreads();
    for (int e = tid; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - (e / n) * n;
        if (c >= r) {
            const double x = s.vn1[r];
            const cplx a = A[r * ld + c];
            A[r * ld + c] = cmk(a.x * x, a.y * x);
        }
    }
    for (int k = tid; k < n; k += blockDim.x) s.ipiv[s.piv[k]] = k;
    __syncthreads();
}

// C <- Q^H C (ZUNMQR 'L','C'): each segment holds its columns in registers.
template <int R8, int CPS>
COLD void apply_qh_left(int n, int ld, const cplx* F, const cplx* tau, cplx* C) {
    const int tid = threadIdx.x, lane8 = tid & 7, seg = tid >> 3, nseg = blockDim.x >> 3;
    cplx c[CPS][R8];
#pragma unroll
    for (int q = 0; q < CPS; ++q)
#pragma unroll
        for (int k = 0; k < R8; ++k) {
            const int j = seg + q * nseg, r = lane8 + 8 * k;
            c[q][k] = (j < n && r < n) ? C[r * ld + j] : cmk(0.0, 0.0);
        }
    for (int i = 0; i < n; ++i) {
        const cplx ct = cconj(tau[i]);
        cplx v[R8];
#pragma unroll
        for (int k = 0; k < R8; ++k) {
            const int r = lane8 + 8 * k;
            v[k] = (r == i) ? cmk(1.0, 0.0) : ((r > i && r < n) ? F[r * ld + i] : cmk(0.0, 0.0));
        }
#pragma unroll
        for (int q = 0; q < CPS; ++q) {
            cplx w = cmk(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < R8; ++k) w = cfmacj(v[k], c[q][k], w);
            w.x = seg8_sum(w.x);
            w.y = seg8_sum(w.y);
            const cplx f = cmul(ct, w);
#pragma unroll
            for (int k = 0; k < R8; ++k) c[q][k] = csub(c[q][k], cmul(v[k], f));
        }
    }
#pragma unroll
    for (int q = 0; q < CPS; ++q)
#pragma unroll
        for (int k = 0; k < R8; ++k) {
            const int j = seg + q * nseg, r = lane8 + 8 * k;
            if (j < n && r < n) C[r * ld + j] = c[q][k];
        }
    __syncthreads();
}

// C <- C Q (ZUNMQR 'R','N'): each segment holds its rows in registers.
template <int R8, int CPS>
COLD void apply_q_right(int n, int ld, const cplx* F, const cplx* tau, cplx* C) {
    const int tid = threadIdx.x, lane8 = tid & 7, seg = tid >> 3, nseg = blockDim.x >> 3;
    cplx c[CPS][R8];   // c[q][k] = C[row seg+q*nseg][col lane8+8k]
#pragma unroll
    for (int q = 0; q < CPS; ++q)
#pragma unroll
        for (int k = 0; k < R8; ++k) {
            const int r = seg + q * nseg, col = lane8 + 8 * k;
            c[q][k] = (r < n && col < n) ? C[r * ld + col] : cmk(0.0, 0.0);
        }
    for (int i = 0; i < n; ++i) {
        const cplx t = tau[i];
        cplx v[R8];
#pragma unroll
        for (int k = 0; k < R8; ++k) {
            const int col = lane8 + 8 * k;
            v[k] = (col == i) ? cmk(1.0, 0.0) : ((col > i && col < n) ? F[col * ld + i] : cmk(0.0, 0.0));
        }
#pragma unroll
        for (int q = 0; q < CPS; ++q) {
            cplx w = cmk(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < R8; ++k) w = cfma(c[q][k], v[k], w);
            w.x = seg8_sum(w.x);
            w.y = seg8_sum(w.y);
            const cplx f = cmul(t, w);
#pragma unroll
            for (int k = 0; k < R8; ++k) c[q][k] = csub(c[q][k], cmulcj(f, v[k]));
        }
    }
#pragma unroll
    for (int q = 0; q < CPS; ++q)
#pragma unroll
        for (int k = 0; k < R8; ++k) {
            const int r = seg + q * nseg, col = lane8 + 8 * k;
            if (r < n && col < n) C[r * ld + col] = c[q][k];
        }
    __syncthreads();
}

// Q = H_0 ... H_{n-1} (ZUNGQR), or Q^H with conjT, written to Q (no alias with F).
template <int R8, int CPS>
COLD void form_q(int n, int ld, const cplx* F, const cplx* tau, cplx* Q, bool conjT) {
    const int tid = threadIdx.x, lane8 = tid & 7, seg = tid >> 3, nseg = blockDim.x >> 3;
    cplx c[CPS][R8];
#pragma unroll
    for (int q = 0; q < CPS; ++q)
#pragma unroll
        for (int k = 0; k < R8; ++k) {
            const int j = seg + q * nseg, r = lane8 + 8 * k;
            c[q][k] = cmk((r == j) ? 1.0 : 0.0, 0.0);
        }
    for (int i = n - 1; i >= 0; --i) {
        const cplx t = tau[i];
        cplx v[R8];
#pragma unroll
        for (int k = 0; k < R8; ++k) {
            const int r = lane8 + 8 * k;
            v[k] = (r == i) ? cmk(1.0, 0.0) : ((r > i && r < n) ? F[r * ld + i] : cmk(0.0, 0.0));
        }
#pragma unroll
        for (int q = 0; q < CPS; ++q) {
            const int j = seg + q * nseg;
            if (j < i) continue;   // columns left of i are untouched by H_i (ZUNG2R), uniform per segment
            cplx w = cmk(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < R8; ++k) w = cfmacj(v[k], c[q][k], w);
            w.x = seg8_sum(w.x);
            w.y = seg8_sum(w.y);
            const cplx f = cmul(t, w);
#pragma unroll
            for (int k = 0; k < R8; ++k) c[q][k] = csub(c[q][k], cmul(v[k], f));
        }
    }
#pragma unroll
    for (int q = 0; q < CPS; ++q)
#pragma unroll
        for (int k = 0; k < R8; ++k) {
            const int j = seg + q * nseg, r = lane8 + 8 * k;
            if (j < n && r < n) {
                if (conjT) Q[j * ld + r] = cconj(c[q][k]);
                else Q[r * ld + j] = c[q][k];
            }
        }
    __syncthreads();
}

// Inverses of the diagonal of the upper triangle of F into rinv (n complex),
// and of the positive vector d into dinv (n reals), for the triangular solves.
COLD void diag_inverse(int n, int ld, const cplx* F, const double* d, cplx* rinv, double* dinv) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const cplx a = F[i * ld + i];
        const double id2 = 1.0 / (a.x * a.x + a.y * a.y);
        rinv[i] = cmk(a.x * id2, -a.y * id2);
        dinv[i] = 1.0 / d[i];
    }
    __syncthreads();
}

// C <- R^{-1} diag(rs) C (ZTRSM 'L','U','N','N' after scaling row r of C by
// rs[r]); rinv from diag_inverse.  Each segment holds its columns in
// registers; row i's value comes from lane i%8 by shuffle.
template <int R8, int CPS>
COLD void trsm_left_upper(int n, int ld, const cplx* F, const cplx* rinv, const double* rs, cplx* C) {
    const int tid = threadIdx.x, lane8 = tid & 7, seg = tid >> 3, nseg = blockDim.x >> 3;
    const unsigned m = seg8_mask();
    const int base = tid & 24;
    cplx c[CPS][R8];
#pragma unroll
    for (int q = 0; q < CPS; ++q)
#pragma unroll
        for (int k = 0; k < R8; ++k) {
            const int j = seg + q * nseg, r = lane8 + 8 * k;
            if (j < n && r < n) {
                const cplx x = C[r * ld + j];
                const double f = rs[r];
                c[q][k] = cmk(x.x * f, x.y * f);
            } else {
                c[q][k] = cmk(0.0, 0.0);
            }
        }
#pragma unroll
    for (int kk = R8 - 1; kk >= 0; --kk) {
        for (int l = 7; l >= 0; --l) {
            const int i = 8 * kk + l;
            if (i >= n) continue;   // uniform
            const cplx ri = rinv[i];
            cplx fcol[R8];
#pragma unroll
            for (int k = 0; k < R8; ++k) {
                const int r = lane8 + 8 * k;
                fcol[k] = (r < i) ? F[r * ld + i] : cmk(0.0, 0.0);
            }
#pragma unroll
            for (int q = 0; q < CPS; ++q) {
                cplx x;
                x.x = __shfl_sync(m, c[q][kk].x, base + l);
                x.y = __shfl_sync(m, c[q][kk].y, base + l);
                x = cmul(x, ri);
                if (lane8 == l) c[q][kk] = x;
#pragma unroll
                for (int k = 0; k < R8; ++k) c[q][k] = csub(c[q][k], cmul(fcol[k], x));   // fcol = 0 for rows >= i
            }
        }
    }
#pragma unroll
    for (int q = 0; q < CPS; ++q)
#pragma unroll
        for (int k = 0; k < R8; ++k) {
            const int j = seg + q * nseg, r = lane8 + 8 * k;
            if (j < n && r < n) C[r * ld + j] = c[q][k];
        }
    __syncthreads();
}

// C <- C diag(cs) R^{-H} (ZTRSM 'R','U','C','N' after scaling column c of C by
// cs[c]): X R^H = C diag(cs) solved for columns n-1..0.  Each segment holds
// its rows in registers; column c's value comes from lane c%8.
template <int R8, int CPS>
COLD void trsm_right_upperH(int n, int ld, const cplx* F, const cplx* rinv, const double* cs, cplx* C) {
    const int tid = threadIdx.x, lane8 = tid & 7, seg = tid >> 3, nseg = blockDim.x >> 3;
    const unsigned m = seg8_mask();
    const int base = tid & 24;
    cplx c[CPS][R8];   // c[q][k] = C[row seg+q*nseg][col lane8+8k]
#pragma unroll
    for (int q = 0; q < CPS; ++q)
#pragma unroll
        for (int k = 0; k < R8; ++k) {
            const int r = seg + q * nseg, col = lane8 + 8 * k;
            if (r < n && col < n) {
                const cplx x = C[r * ld + col];
                const double f = cs[col];
                c[q][k] = cmk(x.x * f, x.y * f);
            } else {
                c[q][k] = cmk(0.0, 0.0);
            }
        }
#pragma unroll
    for (int kk = R8 - 1; kk >= 0; --kk) {
        for (int l = 7; l >= 0; --l) {
            const int cc = 8 * kk + l;
            if (cc >= n) continue;
            const cplx ri = cconj(rinv[cc]);   // 1 / conj(R_cc)
            cplx frow[R8];                      // R[k][cc] for k < cc
#pragma unroll
            for (int k = 0; k < R8; ++k) {
                const int col = lane8 + 8 * k;
                frow[k] = (col < cc) ? F[col * ld + cc] : cmk(0.0, 0.0);
            }
#pragma unroll
            for (int q = 0; q < CPS; ++q) {
                cplx x;
                x.x = __shfl_sync(m, c[q][kk].x, base + l);
                x.y = __shfl_sync(m, c[q][kk].y, base + l);
                x = cmul(x, ri);
                if (lane8 == l) c[q][kk] = x;
#pragma unroll
                for (int k = 0; k < R8; ++k) c[q][k] = csub(c[q][k], cmulcj(x, frow[k]));
            }
        }
    }
#pragma unroll
    for (int q = 0; q < CPS; ++q)
#pragma unroll
        for (int k = 0; k < R8; ++k) {
            const int r = seg + q * nseg, col = lane8 + 8 * k;
            if (r < n && col < n) C[r * ld + col] = c[q][k];
        }
    __syncthreads();
}

// Row permutation in place.  forward: out[k][:] = in[piv[k]][:] (ZLAPMR .true.,
// i.e. P^T X); backward: out[piv[k]][:] = in[k][:] (ZLAPMR .false., i.e. P X).
template <int MAXE>
COLD void permute_rows(int n, int ld, cplx* C, const int* piv, const int* ipiv, bool forward) {
    cplx v[MAXE];
#pragma unroll
    for (int k = 0; k < MAXE; ++k) {
        const int e = threadIdx.x + k * blockDim.x;
        if (e < n * n) {
            const int r = e / n, c = e % n;
            v[k] = C[(forward ? piv[r] : ipiv[r]) * ld + c];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < MAXE; ++k) {
        const int e = threadIdx.x + k * blockDim.x;
        if (e < n * n) {
            const int r = e / n, c = e - (e / n) * n;
            C[r * ld + c] = v[k];
        }
    }
    __syncthreads();
}

// Column permutation in place.  forward: out[:, k] = in[:, piv[k]] (ZLAPMT
// .true., X P); backward: out[:, piv[k]] = in[:, k] (ZLAPMT .false., X P^T).
template <int MAXE>
COLD void permute_cols(int n, int ld, cplx* C, const int* piv, const int* ipiv, bool forward) {
    cplx v[MAXE];
#pragma unroll
    for (int k = 0; k < MAXE; ++k) {
        const int e = threadIdx.x + k * blockDim.x;
        if (e < n * n) {
            const int r = e / n, c = e % n;
            v[k] = C[r * ld + (forward ? piv[c] : ipiv[c])];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < MAXE; ++k) {
        const int e = threadIdx.x + k * blockDim.x;
        if (e < n * n) {
            const int r = e / n, c = e - (e / n) * n;
            C[r * ld + c] = v[k];
        }
    }
    __syncthreads();
}
