// CTA-level dense complex FP64 linear algebra on matrices resident in shared
// memory (row-major, leading dimension n).  Every routine is called by all
// threads of the block and returns with the block synchronised.
//
// These restate the LAPACK/BLAS operations the reference sweep calls
// (src/number_conserving/src/stabilization.f90:41-190 and
// src/common/mymats.f90:20-29): ZGEMM, ZTRMM, ZGEQP3 (unblocked ZLAQP2 path,
// which LAPACK takes for the matrix sizes here), ZUNGQR, ZUNMQR, ZTRSM,
// ZLAPMR/ZLAPMT.  They are written for the sweep's sizes (n <= 64): one CTA
// owns one matrix, so every step is a barrier-separated pass over shared
// memory instead of a blocked panel algorithm.
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
COLD void gemm_rs(int n, cplx* C, MatOp A, MatOp B, int tri = TRI_NONE) {
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
                if (r < n && c < n) C[r * n + c] = acc[i][j];
            }
    }
    __syncthreads();
}

// C = A * B with A, B, C n x n row-major in shared memory (C may alias A or
// B); the per-slice propagation products.
template <int TR, int TC>
DEVI void gemm_smem(int n, cplx* C, const cplx* A, const cplx* B) {
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
        for (int i = 0; i < TR; ++i) ra[i] = min(r0 + i, n - 1) * n;
#pragma unroll
        for (int j = 0; j < TC; ++j) cb[j] = min(c0 + j, n - 1);
        for (int k = 0; k < n; ++k) {
            cplx a[TR], b[TC];
#pragma unroll
            for (int i = 0; i < TR; ++i) a[i] = A[ra[i] + k];
#pragma unroll
            for (int j = 0; j < TC; ++j) b[j] = B[k * n + cb[j]];
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
                if (r < n && c < n) C[r * n + c] = acc[i][j];
            }
    }
    __syncthreads();
}

// dst = op(src) elementwise copy for an n x n matrix (dst must not alias src
// unless op is the identity view).
COLD void copy_op(int n, cplx* dst, MatOp src) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) dst[e] = src.at(e / n, e % n);
    __syncthreads();
}

// In-place conjugate transpose via register staging; MAXE >= ceil(n*n/blockDim).
template <int MAXE>
COLD void conj_transpose_inplace(int n, cplx* A) {
    cplx v[MAXE];
#pragma unroll
    for (int k = 0; k < MAXE; ++k) {
        const int e = threadIdx.x + k * blockDim.x;
        if (e < n * n) v[k] = cconj(A[(e % n) * n + e / n]);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < MAXE; ++k) {
        const int e = threadIdx.x + k * blockDim.x;
        if (e < n * n) A[e] = v[k];
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
DEVI double seg8_colnorm(int n, const cplx* A, int j, int r0, int lane8) {
    double m = 0.0;
    for (int r = r0 + lane8; r < n; r += 8) m = fmax(m, fmax(fabs(A[r * n + j].x), fabs(A[r * n + j].y)));
    m = seg8_max(m);
    if (m == 0.0) return 0.0;
    double s = 0.0;
    for (int r = r0 + lane8; r < n; r += 8) {
        double a = A[r * n + j].x / m, b = A[r * n + j].y / m;
        s += a * a + b * b;
    }
    s = seg8_sum(s);
    return m * sqrt(s);
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
COLD void qrp_inplace(int n, cplx* A, QRScratch s) {
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int lane8 = tid & 7, seg = tid >> 3, nseg = nthr >> 3;
    const double tol3z = 1.0536712127723509e-08;   // sqrt(2^-53), LAPACK's sqrt(dlamch('E'))
    // initial column norms
    for (int j = seg; j < n; j += nseg) {
        double v = seg8_colnorm(n, A, j, 0, lane8);
        if (lane8 == 0) { s.vn1[j] = v; s.vn2[j] = v; s.piv[j] = j; }
    }
    __syncthreads();
    for (int i = 0; i < n; ++i) {
        // pivot: first index of max vn1[i..n) (IDAMAX), by warp 0
        if (tid < 32) {
            double best = -1.0;
            int bi = n;
            for (int j = i + tid; j < n; j += 32) {
                double v = s.vn1[j];
                if (v > best) { best = v; bi = j; }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                double ob = __shfl_xor_sync(0xffffffffu, best, o);
                int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            if (tid == 0) s.ibcast[0] = (bi < n) ? bi : i;   // all-NaN norms: keep column i
        }
        __syncthreads();
        const int pvt = s.ibcast[0];
        if (pvt != i) {
            for (int r = tid; r < n; r += nthr) {
                cplx t = A[r * n + i];
                A[r * n + i] = A[r * n + pvt];
                A[r * n + pvt] = t;
            }
            if (tid == 0) {
                int t = s.piv[pvt]; s.piv[pvt] = s.piv[i]; s.piv[i] = t;
                s.vn1[pvt] = s.vn1[i];
                s.vn2[pvt] = s.vn2[i];
            }
        }
        __syncthreads();
        // Householder reflector for A[i:, i] (ZLARFG), by segment 0
        if (seg == 0) {
            double xn = seg8_colnorm(n, A, i, i + 1, lane8);
            cplx alpha = A[i * n + i];
            cplx tau = cmk(0.0, 0.0), beta = alpha;
            cplx scl = cmk(0.0, 0.0);
            bool doit = !(xn == 0.0 && alpha.y == 0.0);
            if (doit) {
                double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn * xn);
                double b = (alpha.x >= 0.0) ? -nrm : nrm;
                tau = cmk((b - alpha.x) / b, -alpha.y / b);
                scl = cdiv(cmk(1.0, 0.0), cmk(alpha.x - b, alpha.y));
                beta = cmk(b, 0.0);
            }
            if (doit) {
                for (int r = i + 1 + lane8; r < n; r += 8) A[r * n + i] = cmul(scl, A[r * n + i]);
            }
            if (lane8 == 0) { A[i * n + i] = beta; s.tau[i] = tau; }
        }
        __syncthreads();
        // apply H^H = I - conj(tau) v v^H to A[i:, i+1:], then downdate norms
        const cplx ctau = cconj(s.tau[i]);
        for (int j = i + 1 + seg; j < n; j += nseg) {
            cplx w = cmk(0.0, 0.0);
            for (int r = i + lane8; r < n; r += 8) {
                cplx v = (r == i) ? cmk(1.0, 0.0) : A[r * n + i];
                w = cfmacj(v, A[r * n + j], w);
            }
            w.x = seg8_sum(w.x);
            w.y = seg8_sum(w.y);
            cplx f = cmul(ctau, w);
            for (int r = i + lane8; r < n; r += 8) {
                cplx v = (r == i) ? cmk(1.0, 0.0) : A[r * n + i];
                A[r * n + j] = csub(A[r * n + j], cmul(v, f));
            }
            __syncwarp(seg8_mask());
            // norm downdate (ZLAQP2): lane 0 of the segment owns row i
            double v1 = s.vn1[j];
            int recompute = 0;
            double newv = v1;
            if (v1 != 0.0) {
                double t = cabsv(A[i * n + j]) / v1;
                double temp = fmax(1.0 - t * t, 0.0);
                double q = v1 / s.vn2[j];
                double temp2 = temp * q * q;
                if (temp2 <= tol3z) recompute = 1;
                else newv = v1 * sqrt(temp);
            }
            double nv = newv;
            if (recompute) nv = (i + 1 < n) ? seg8_colnorm(n, A, j, i + 1, lane8) : 0.0;
            __syncwarp(seg8_mask());
            if (lane8 == 0) {
                s.vn1[j] = nv;
                if (recompute) s.vn2[j] = nv;
            }
        }
        __syncthreads();
    }
    // QDRP post-step: D = |diag R|, scale the rows of the upper triangle
    for (int i = tid; i < n; i += nthr) s.d[i] = cabsv(A[i * n + i]);
    __syncthreads();
    for (int e = tid; e < n * n; e += nthr) {
        int r = e / n, c = e % n;
        if (c >= r) {
            double x = s.d[r];
            A[e] = cmk(A[e].x / x, A[e].y / x);
        }
    }
    for (int k = tid; k < n; k += nthr) s.ipiv[s.piv[k]] = k;
    __syncthreads();
}

// Q = H_0 H_1 ... H_{n-1} (ZUNGQR) from the reflectors stored below the
// diagonal of F, written to Q (must not alias F).  conjT writes Q^H instead.
template <int MAXE>
COLD void form_q(int n, const cplx* F, const cplx* tau, cplx* Q, bool conjT) {
    const int tid = threadIdx.x, lane8 = tid & 7, seg = tid >> 3, nseg = blockDim.x >> 3;
    for (int e = tid; e < n * n; e += blockDim.x) Q[e] = cmk((e / n) == (e % n) ? 1.0 : 0.0, 0.0);
    __syncthreads();
    for (int i = n - 1; i >= 0; --i) {
        const cplx t = tau[i];
        for (int j = i + seg; j < n; j += nseg) {
            cplx w = cmk(0.0, 0.0);
            for (int r = i + lane8; r < n; r += 8) {
                cplx v = (r == i) ? cmk(1.0, 0.0) : F[r * n + i];
                w = cfmacj(v, Q[r * n + j], w);
            }
            w.x = seg8_sum(w.x);
            w.y = seg8_sum(w.y);
            cplx f = cmul(t, w);
            for (int r = i + lane8; r < n; r += 8) {
                cplx v = (r == i) ? cmk(1.0, 0.0) : F[r * n + i];
                Q[r * n + j] = csub(Q[r * n + j], cmul(v, f));
            }
        }
        __syncthreads();
    }
    if (conjT) conj_transpose_inplace<MAXE>(n, Q);
}

// C <- Q^H C (ZUNMQR 'L','C'), reflectors in F.
COLD void apply_qh_left(int n, const cplx* F, const cplx* tau, cplx* C) {
    const int tid = threadIdx.x, lane8 = tid & 7, seg = tid >> 3, nseg = blockDim.x >> 3;
    for (int i = 0; i < n; ++i) {
        const cplx ct = cconj(tau[i]);
        for (int j = seg; j < n; j += nseg) {
            cplx w = cmk(0.0, 0.0);
            for (int r = i + lane8; r < n; r += 8) {
                cplx v = (r == i) ? cmk(1.0, 0.0) : F[r * n + i];
                w = cfmacj(v, C[r * n + j], w);
            }
            w.x = seg8_sum(w.x);
            w.y = seg8_sum(w.y);
            cplx f = cmul(ct, w);
            for (int r = i + lane8; r < n; r += 8) {
                cplx v = (r == i) ? cmk(1.0, 0.0) : F[r * n + i];
                C[r * n + j] = csub(C[r * n + j], cmul(v, f));
            }
        }
        __syncthreads();
    }
}

// C <- C Q (ZUNMQR 'R','N'), reflectors in F.
COLD void apply_q_right(int n, const cplx* F, const cplx* tau, cplx* C) {
    const int tid = threadIdx.x, lane8 = tid & 7, seg = tid >> 3, nseg = blockDim.x >> 3;
    for (int i = 0; i < n; ++i) {
        const cplx t = tau[i];
        for (int r = seg; r < n; r += nseg) {
            cplx w = cmk(0.0, 0.0);
            for (int k = i + lane8; k < n; k += 8) {
                cplx v = (k == i) ? cmk(1.0, 0.0) : F[k * n + i];
                w = cfma(C[r * n + k], v, w);
            }
            w.x = seg8_sum(w.x);
            w.y = seg8_sum(w.y);
            cplx f = cmul(t, w);
            for (int k = i + lane8; k < n; k += 8) {
                cplx v = (k == i) ? cmk(1.0, 0.0) : F[k * n + i];
                C[r * n + k] = csub(C[r * n + k], cmulcj(f, v));
            }
        }
        __syncthreads();
    }
}

// C <- R^{-1} C with R the upper triangle of F (ZTRSM 'L','U','N','N').
// Column-parallel back substitution: one 8-lane segment per column.
COLD void trsm_left_upper(int n, const cplx* F, cplx* C) {
    const int tid = threadIdx.x, lane8 = tid & 7, seg = tid >> 3, nseg = blockDim.x >> 3;
    for (int c = seg; c < n; c += nseg) {
        for (int i = n - 1; i >= 0; --i) {
            // x_i = C[i][c] / R_ii (every lane computes it), then rows k < i downdate
            cplx xi = cdiv(C[i * n + c], F[i * n + i]);
            __syncwarp(seg8_mask());
            if (lane8 == 0) C[i * n + c] = xi;
            for (int k = lane8; k < i; k += 8) C[k * n + c] = csub(C[k * n + c], cmul(F[k * n + i], xi));
            __syncwarp(seg8_mask());
        }
    }
    __syncthreads();
}

// C <- C R^{-H} with R the upper triangle of F (ZTRSM 'R','U','C','N').
// Row-parallel: X R^H = C, solved for columns n-1 .. 0.
COLD void trsm_right_upperH(int n, const cplx* F, cplx* C) {
    const int tid = threadIdx.x, lane8 = tid & 7, seg = tid >> 3, nseg = blockDim.x >> 3;
    for (int r = seg; r < n; r += nseg) {
        for (int c = n - 1; c >= 0; --c) {
            cplx xc = cdiv(C[r * n + c], cconj(F[c * n + c]));
            __syncwarp(seg8_mask());
            if (lane8 == 0) C[r * n + c] = xc;
            // C[r][k] -= x_c * conj(R[k][c]) for k < c
            for (int k = lane8; k < c; k += 8) C[r * n + k] = csub(C[r * n + k], cmulcj(xc, F[k * n + c]));
            __syncwarp(seg8_mask());
        }
    }
    __syncthreads();
}

// Row permutation in place.  forward: out[k][:] = in[piv[k]][:] (ZLAPMR .true.,
// i.e. P^T X); backward: out[piv[k]][:] = in[k][:] (ZLAPMR .false., i.e. P X).
template <int MAXE>
COLD void permute_rows(int n, cplx* C, const int* piv, const int* ipiv, bool forward) {
    cplx v[MAXE];
#pragma unroll
    for (int k = 0; k < MAXE; ++k) {
        const int e = threadIdx.x + k * blockDim.x;
        if (e < n * n) {
            const int r = e / n, c = e % n;
            v[k] = C[(forward ? piv[r] : ipiv[r]) * n + c];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < MAXE; ++k) {
        const int e = threadIdx.x + k * blockDim.x;
        if (e < n * n) C[e] = v[k];
    }
    __syncthreads();
}

// Column permutation in place.  forward: out[:, k] = in[:, piv[k]] (ZLAPMT
// .true., X P); backward: out[:, piv[k]] = in[:, k] (ZLAPMT .false., X P^T).
template <int MAXE>
COLD void permute_cols(int n, cplx* C, const int* piv, const int* ipiv, bool forward) {
    cplx v[MAXE];
#pragma unroll
    for (int k = 0; k < MAXE; ++k) {
        const int e = threadIdx.x + k * blockDim.x;
        if (e < n * n) {
            const int r = e / n, c = e % n;
            v[k] = C[r * n + (forward ? piv[c] : ipiv[c])];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < MAXE; ++k) {
        const int e = threadIdx.x + k * blockDim.x;
        if (e < n * n) C[e] = v[k];
    }
    __syncthreads();
}
