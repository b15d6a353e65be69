// Dense complex FP64 linear algebra for the largest size class (n up to 160),
// whose matrices live in a per-chain region of global memory because neither
// the shared memory of one SM (227 KB) nor its register file holds the five
// n x n complex matrices a chain works on.  While a chain runs, its region
// stays in L2.
//
// Same operations and conventions as linalg.cuh (ZGEMM/ZTRMM, ZGEQP3 in the
// ZLAQP2 form with the QDRP_decompose post-step, ZUNGQR, ZUNMQR, ZTRSM,
// ZLAPMR/ZLAPMT; row-major with leading dimension ld; called by all threads
// of the block, returning with the block synchronised).  One warp per column
// (or row) of the operand: lane l holds rows l, l+32, ... (RW >= ceil(n/32) of
// them) of the warp's current columns, the warp walks its columns in groups
// of CPW, and reductions are warp shuffles.  Products and permutations are out
// of place through a scratch matrix S.
#pragma once
#include "linalg.cuh"

DEVI double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Overflow-safe 2-norm of column j, rows [r0, n), by one warp (CM: A is stored
// column-major, element (r, j) at A[j * ld + r]).
template <bool CM = false>
DEVI double warp_colnorm(int n, int ld, const cplx* A, int j, int r0) {
    const int lane = threadIdx.x & 31;
    double m = 0.0;
    for (int r = r0 + lane; r < n; r += 32) m = fmax(m, fmax(fabs(A[CM ? j * ld + r : r * ld + j].x), fabs(A[CM ? j * ld + r : r * ld + j].y)));
    m = warp_max(m);
    if (m == 0.0) return 0.0;
    double s = 0.0;
    for (int r = r0 + lane; r < n; r += 32) {
        const double a = A[CM ? j * ld + r : r * ld + j].x / m, b = A[CM ? j * ld + r : r * ld + j].y / m;
        s += a * a + b * b;
    }
    return m * sqrt(warp_sum(s));
}

template <bool CM = false>
DEVI double warp_norm(int n, int ld, const cplx* A, int j, int r0) {
    const int lane = threadIdx.x & 31;
    double ss = 0.0;
    for (int r = r0 + lane; r < n; r += 32) {
        const cplx a = A[CM ? j * ld + r : r * ld + j];
        ss = fma(a.x, a.x, fma(a.y, a.y, ss));
    }
    ss = warp_sum(ss);
    if (!sumsq_unsafe(ss)) return sqrt(ss);
    return warp_colnorm<CM>(n, ld, A, j, r0);
}

// C = op(A) op(B), C distinct from A and B; tri as in gemm_rs.
// Work items are a warp's: with B untransposed (B.sc == 1) lanes take 32
// consecutive columns of C over kGW rows, so each B(k, :) load is one coalesced
// row segment and each A(r, k) load is the same address in every lane; with A
// conjugate-transposed (A.sr == 1) lanes take 32 consecutive rows over kGW
// columns, the mirror image.  The remaining case (A untransposed, B
// transposed) keeps per-thread TR x TC tiles.  Every element of C takes the
// same k-ordered cfma sequence in all three forms.
constexpr int kGW = 9;
template <int TR, int TC>
COLD void gemm_big(int n, int ld, cplx* C, MatOp A, MatOp B, int tri = TRI_NONE) {
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int nch = (n + 31) >> 5, items = nch * ((n + kGW - 1) / kGW);
    if (B.sc == 1) {
        for (int it = threadIdx.x >> 5; it < items; it += nw) {
            const int c = (it % nch) * 32 + lane, rb = (it / nch) * kGW, cc = min(c, n - 1);
            cplx acc[kGW];
#pragma unroll
            for (int i = 0; i < kGW; ++i) acc[i] = cmk(0.0, 0.0);
            for (int k = 0; k < n; ++k) {
                cplx bv = B.at(k, cc);
                if (tri == TRI_B_LOWER_FROM_C && k < cc) bv = cmk(0.0, 0.0);
#pragma unroll
                for (int i = 0; i < kGW; ++i) {
                    const int r = rb + i;
                    cplx av = A.at(min(r, n - 1), k);
                    if (tri == TRI_A_UPPER && k < r) av = cmk(0.0, 0.0);
                    acc[i] = cfma(av, bv, acc[i]);
                }
            }
#pragma unroll
            for (int i = 0; i < kGW; ++i)
                if (c < n && rb + i < n) C[(rb + i) * ld + c] = acc[i];
        }
    } else if (A.sr == 1) {
        for (int it = threadIdx.x >> 5; it < items; it += nw) {
            const int r = (it % nch) * 32 + lane, cb = (it / nch) * kGW, rr = min(r, n - 1);
            cplx acc[kGW];
#pragma unroll
            for (int j = 0; j < kGW; ++j) acc[j] = cmk(0.0, 0.0);
            for (int k = 0; k < n; ++k) {
                cplx av = A.at(rr, k);
                if (tri == TRI_A_UPPER && k < rr) av = cmk(0.0, 0.0);
#pragma unroll
                for (int j = 0; j < kGW; ++j) {
                    const int c = cb + j;
                    cplx bv = B.at(k, min(c, n - 1));
                    if (tri == TRI_B_LOWER_FROM_C && k < c) bv = cmk(0.0, 0.0);
                    acc[j] = cfma(av, bv, acc[j]);
                }
            }
#pragma unroll
            for (int j = 0; j < kGW; ++j)
                if (r < n && cb + j < n) C[r * ld + cb + j] = acc[j];
        }
    } else {
        const int ncg = (n + TC - 1) / TC, nrg = (n + TR - 1) / TR;
        for (int g = threadIdx.x; g < ncg * nrg; g += blockDim.x) {
            const int r0 = (g / ncg) * TR, c0 = (g % ncg) * TC;
            cplx acc[TR][TC];
#pragma unroll
            for (int i = 0; i < TR; ++i)
#pragma unroll
                for (int j = 0; j < TC; ++j) acc[i][j] = cmk(0.0, 0.0);
            for (int k = 0; k < n; ++k) {
                cplx a[TR], b[TC];
#pragma unroll
                for (int i = 0; i < TR; ++i) {
                    const int r = r0 + i;
                    a[i] = (r < n) ? A.at(r, k) : cmk(0.0, 0.0);
                    if (tri == TRI_A_UPPER && k < r) a[i] = cmk(0.0, 0.0);
                }
#pragma unroll
                for (int j = 0; j < TC; ++j) {
                    const int c = c0 + j;
                    b[j] = (c < n) ? B.at(k, c) : cmk(0.0, 0.0);
                    if (tri == TRI_B_LOWER_FROM_C && k < c) b[j] = cmk(0.0, 0.0);
                }
#pragma unroll
                for (int i = 0; i < TR; ++i)
#pragma unroll
                    for (int j = 0; j < TC; ++j) acc[i][j] = cfma(a[i], b[j], acc[i][j]);
            }
#pragma unroll
            for (int i = 0; i < TR; ++i)
#pragma unroll
                for (int j = 0; j < TC; ++j) {
                    const int r = r0 + i, c = c0 + j;
                    if (r < n && c < n) C[r * ld + c] = acc[i][j];
                }
        }
    }
    __syncthreads();
}

// C = A B with one real operand (RIGHT_REAL: B real), C distinct from A and B.
template <int TR, int TC, bool RIGHT_REAL>
COLD void gemm_big_real(int n, int ld, cplx* C, const void* Ap, const void* Bp) {
    const int ncg = (n + TC - 1) / TC, nrg = (n + TR - 1) / TR;
    for (int g = threadIdx.x; g < ncg * nrg; g += blockDim.x) {
        const int r0 = (g / ncg) * TR, c0 = (g % ncg) * TC;
        int ra[TR], cb[TC];
#pragma unroll
        for (int i = 0; i < TR; ++i) ra[i] = min(r0 + i, n - 1) * ld;
#pragma unroll
        for (int j = 0; j < TC; ++j) cb[j] = min(c0 + j, n - 1);
        cplx acc[TR][TC];
#pragma unroll
        for (int i = 0; i < TR; ++i)
#pragma unroll
            for (int j = 0; j < TC; ++j) acc[i][j] = cmk(0.0, 0.0);
        for (int k = 0; k < n; ++k) {
            if (RIGHT_REAL) {
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
            } else {
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

COLD void copy_mat(int n, int ld, cplx* dst, const cplx* src) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - (e / n) * n;
        dst[r * ld + c] = src[r * ld + c];
    }
    __syncthreads();
}

// A <- A^H through S.
COLD void conj_transpose_big(int n, int ld, cplx* A, cplx* S) {
    copy_op(n, ld, S, op_c(A, ld));
    copy_mat(n, ld, A, S);
}

// Row / column permutations as permute_rows / permute_cols, through S.
COLD void permute_rows_big(int n, int ld, cplx* C, const int* piv, const int* ipiv, bool forward, cplx* S) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - (e / n) * n;
        S[r * ld + c] = C[(forward ? piv[r] : ipiv[r]) * ld + c];
    }
    __syncthreads();
    copy_mat(n, ld, C, S);
}
COLD void permute_cols_big(int n, int ld, cplx* C, const int* piv, const int* ipiv, bool forward, cplx* S) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - (e / n) * n;
        S[r * ld + c] = C[r * ld + (forward ? piv[c] : ipiv[c])];
    }
    __syncthreads();
    copy_mat(n, ld, C, S);
}

// ZGEQP3 (ZLAQP2 recurrence) + QDRP_decompose post-step, as qrp_inplace.
// Per column: every warp finds the pivot and forms the reflector from the
// pivot column (barrier); the warps update the trailing columns one by one,
// column pvt from the old column i, with ZLAQP2's norm downdate (barrier);
// column i takes the reflector and beta, rows above i of columns i and pvt are
// swapped (barrier).
template <int RW, bool CM = false>
COLD void qrp_big(int n, int ld, cplx* A, QRScratch s) {
#define QA(r, c) A[CM ? (c) * ld + (r) : (r) * ld + (c)]
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5, nw = blockDim.x >> 5;
    const double tol3z = 1.0536712127723509e-08;   // sqrt(2^-53), LAPACK's sqrt(dlamch('E'))
    for (int j = wp; j < n; j += nw) {
        const double v = warp_norm<CM>(n, ld, A, j, 0);
        if (lane == 0) {
            s.vn1[j] = v;
            s.vn2[j] = v;
            s.piv[j] = j;
        }
    }
    __syncthreads();
    for (int i = 0; i < n; ++i) {
        double best = -1.0;
        int bi = n;
        for (int j = i + lane; j < n; j += 32) {
            const double v = s.vn1[j];
            if (v > best) {
                best = v;
                bi = j;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ob > best || (ob == best && oi < bi)) {
                best = ob;
                bi = oi;
            }
        }
        const int pvt = (bi < n) ? bi : i;
        cplx v[RW];
        double ss = 0.0;
#pragma unroll
        for (int k = 0; k < RW; ++k) {
            const int r = lane + 32 * k;
            v[k] = (r < n && r > i) ? QA(r, pvt) : cmk(0.0, 0.0);
            ss = fma(v[k].x, v[k].x, fma(v[k].y, v[k].y, ss));
        }
        ss = warp_sum(ss);
        const cplx alpha = QA(i, pvt);
        double xn = sqrt(ss);
        if (sumsq_unsafe(ss)) xn = warp_colnorm<CM>(n, ld, A, pvt, i + 1);
        cplx tau = cmk(0.0, 0.0), beta = alpha, scl = cmk(0.0, 0.0);
        if (!(xn == 0.0 && alpha.y == 0.0)) {
            const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn * xn);
            const double b = (alpha.x >= 0.0) ? -nrm : nrm;
            const double ib = 1.0 / b;
            tau = cmk((b - alpha.x) * ib, -alpha.y * ib);
            const cplx d = cmk(alpha.x - b, alpha.y);
            const double id2 = 1.0 / (d.x * d.x + d.y * d.y);
            scl = cmk(d.x * id2, -d.y * id2);
            beta = cmk(b, 0.0);
        }
#pragma unroll
        for (int k = 0; k < RW; ++k) {
            const int r = lane + 32 * k;
            v[k] = (r == i) ? cmk(1.0, 0.0) : cmul(scl, v[k]);
        }
        __syncthreads();
        // trailing columns; logical column pvt holds the old column i
        const cplx ctau = cconj(tau);
        for (int j = i + 1 + wp; j < n; j += nw) {
            const int src = (j == pvt) ? i : j;
            cplx a[RW];
#pragma unroll
            for (int k = 0; k < RW; ++k) {
                const int r = lane + 32 * k;
                a[k] = (r < n && r >= i) ? QA(r, src) : cmk(0.0, 0.0);
            }
            const double t1 = s.vn1[src], t2 = s.vn2[src];
            cplx w = cmk(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < RW; ++k) w = cfmacj(v[k], a[k], w);
            w.x = warp_sum(w.x);
            w.y = warp_sum(w.y);
            const cplx f = cmul(ctau, w);
            double ai2 = 0.0, rest = 0.0;
#pragma unroll
            for (int k = 0; k < RW; ++k) {
                const int r = lane + 32 * k;
                a[k] = csub(a[k], cmul(v[k], f));
                const double m2 = a[k].x * a[k].x + a[k].y * a[k].y;
                if (r == i) ai2 = m2;
                if (r > i && r < n) rest += m2;
                if (r < n && r >= i) QA(r, j) = a[k];
            }
            ai2 = warp_sum(ai2);
            rest = warp_sum(rest);
            double nv1 = t1, nv2 = t2;
            if (t1 != 0.0) {
                bool recompute;
                if (t1 < 1.0e150 && t2 < 1.0e150) {
                    const double rem = fmax(t1 * t1 - ai2, 0.0);
                    recompute = rem <= tol3z * t2 * t2;
                    nv1 = sqrt(rem);
                } else {
                    const double tt = sqrt(ai2) / t1;
                    const double temp = fmax(1.0 - tt * tt, 0.0);
                    const double qq = t1 / t2;
                    recompute = !(temp * qq * qq > tol3z);
                    nv1 = t1 * sqrt(temp);
                }
                if (recompute) {
                    if (sumsq_unsafe(rest)) {
                        __syncwarp();
                        nv1 = (i + 1 < n) ? warp_colnorm<CM>(n, ld, A, j, i + 1) : 0.0;
                    } else {
                        nv1 = sqrt(rest);
                    }
                    nv2 = nv1;
                }
            }
            __syncwarp();
            if (lane == 0) {
                s.vn1[j] = nv1;
                s.vn2[j] = nv2;
            }
        }
        __syncthreads();
        if (wp == 0) {
#pragma unroll
            for (int k = 0; k < RW; ++k) {
                const int r = lane + 32 * k;
                if (r < n && r > i) QA(r, i) = v[k];
            }
            if (lane == 0) {
                QA(i, i) = beta;
                s.tau[i] = tau;
            }
        }
        if (pvt != i && tid < i) {
            const cplx ui = QA(tid, i), up = QA(tid, pvt);
            QA(tid, i) = up;
            QA(tid, pvt) = ui;
        }
        if (tid == 0 && pvt != i) {
            const int t = s.piv[pvt];
            s.piv[pvt] = s.piv[i];
            s.piv[i] = t;
        }
        __syncthreads();
    }
    for (int i = tid; i < n; i += blockDim.x) {
        const cplx a = QA(i, i);
        const double d = hypot(a.x, a.y);
        s.d[i] = d;
        s.vn1[i] = 1.0 / d;
    }
    __syncthreads();
    for (int e = tid; e < n * n; e += blockDim.x) {
        const int q = e / n, t = e - q * n;   // consecutive threads walk the storage order
        const int r = CM ? t : q, c = CM ? q : t;
        if (c >= r) {
            const double x = s.vn1[r];
            const cplx a = QA(r, c);
            QA(r, c) = cmk(a.x * x, a.y * x);
        }
    }
    for (int k = tid; k < n; k += blockDim.x) s.ipiv[s.piv[k]] = k;
    __syncthreads();
#undef QA
}

// v[k] = row lane+32k of reflector i (unit at i, zero above), from column i of F.
// dst <- src stored column-major (dst[c * ld + r] = src[r * ld + c]).  The
// reflector and triangular-solve routines below read F one column per warp;
// with FCM they read such a copy, so each warp load is one contiguous segment.
COLD void copy_col_major(int n, int ld, cplx* dst, const cplx* src) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - r * n;
        dst[c * ld + r] = src[r * ld + c];
    }
    __syncthreads();
}

template <int RW, bool FCM = false>
DEVI void load_reflector_col(int n, int ld, const cplx* F, int i, cplx (&v)[RW]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < RW; ++k) {
        const int r = lane + 32 * k;
        v[k] = (r == i) ? cmk(1.0, 0.0) : ((r > i && r < n) ? F[FCM ? i * ld + r : r * ld + i] : cmk(0.0, 0.0));
    }
}

// C <- Q^H C (ZUNMQR 'L','C'): columns of C are independent.
template <int RW, int CPW, bool FCM = false>
COLD void apply_qh_left_big(int n, int ld, const cplx* F, const cplx* tau, cplx* C) {
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int j0 = wp * CPW; j0 < n; j0 += nw * CPW) {
        cplx c[CPW][RW];
#pragma unroll
        for (int q = 0; q < CPW; ++q)
#pragma unroll
            for (int k = 0; k < RW; ++k) {
                const int j = j0 + q, r = lane + 32 * k;
                c[q][k] = (j < n && r < n) ? C[r * ld + j] : cmk(0.0, 0.0);
            }
        for (int i = 0; i < n; ++i) {
            const cplx ct = cconj(tau[i]);
            cplx v[RW];
            load_reflector_col<RW, FCM>(n, ld, F, i, v);
#pragma unroll
            for (int q = 0; q < CPW; ++q) {
                cplx w = cmk(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < RW; ++k) w = cfmacj(v[k], c[q][k], w);
                w.x = warp_sum(w.x);
                w.y = warp_sum(w.y);
                const cplx f = cmul(ct, w);
#pragma unroll
                for (int k = 0; k < RW; ++k) c[q][k] = csub(c[q][k], cmul(v[k], f));
            }
        }
#pragma unroll
        for (int q = 0; q < CPW; ++q)
#pragma unroll
            for (int k = 0; k < RW; ++k) {
                const int j = j0 + q, r = lane + 32 * k;
                if (j < n && r < n) C[r * ld + j] = c[q][k];
            }
    }
    __syncthreads();
}

// C <- C Q (ZUNMQR 'R','N'): rows of C are independent.
template <int RW, int CPW, bool FCM = false>
COLD void apply_q_right_big(int n, int ld, const cplx* F, const cplx* tau, cplx* C) {
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int r0 = wp * CPW; r0 < n; r0 += nw * CPW) {
        cplx c[CPW][RW];   // c[q][k] = C[row r0+q][col lane+32k]
#pragma unroll
        for (int q = 0; q < CPW; ++q)
#pragma unroll
            for (int k = 0; k < RW; ++k) {
                const int r = r0 + q, col = lane + 32 * k;
                c[q][k] = (r < n && col < n) ? C[r * ld + col] : cmk(0.0, 0.0);
            }
        for (int i = 0; i < n; ++i) {
            const cplx t = tau[i];
            cplx v[RW];
            load_reflector_col<RW, FCM>(n, ld, F, i, v);
#pragma unroll
            for (int q = 0; q < CPW; ++q) {
                cplx w = cmk(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < RW; ++k) w = cfma(c[q][k], v[k], w);
                w.x = warp_sum(w.x);
                w.y = warp_sum(w.y);
                const cplx f = cmul(t, w);
#pragma unroll
                for (int k = 0; k < RW; ++k) c[q][k] = csub(c[q][k], cmulcj(f, v[k]));
            }
        }
#pragma unroll
        for (int q = 0; q < CPW; ++q)
#pragma unroll
            for (int k = 0; k < RW; ++k) {
                const int r = r0 + q, col = lane + 32 * k;
                if (r < n && col < n) C[r * ld + col] = c[q][k];
            }
    }
    __syncthreads();
}

// Q = H_0 ... H_{n-1} (ZUNGQR), or Q^H with conjT, into Q (no alias with F).
// Column j of Q is H_0 ... H_j e_j.
template <int RW, int CPW, bool FCM = false>
COLD void form_q_big(int n, int ld, const cplx* F, const cplx* tau, cplx* Q, bool conjT) {
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int j0 = wp * CPW; j0 < n; j0 += nw * CPW) {
        cplx c[CPW][RW];
#pragma unroll
        for (int q = 0; q < CPW; ++q)
#pragma unroll
            for (int k = 0; k < RW; ++k) c[q][k] = cmk((lane + 32 * k == j0 + q) ? 1.0 : 0.0, 0.0);
        for (int i = min(j0 + CPW - 1, n - 1); i >= 0; --i) {
            const cplx t = tau[i];
            cplx v[RW];
            load_reflector_col<RW, FCM>(n, ld, F, i, v);
#pragma unroll
            for (int q = 0; q < CPW; ++q) {
                if (j0 + q < i) continue;   // H_i leaves e_j, j < i, unchanged (ZUNG2R); uniform in the warp
                cplx w = cmk(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < RW; ++k) w = cfmacj(v[k], c[q][k], w);
                w.x = warp_sum(w.x);
                w.y = warp_sum(w.y);
                const cplx f = cmul(t, w);
#pragma unroll
                for (int k = 0; k < RW; ++k) c[q][k] = csub(c[q][k], cmul(v[k], f));
            }
        }
#pragma unroll
        for (int q = 0; q < CPW; ++q)
#pragma unroll
            for (int k = 0; k < RW; ++k) {
                const int j = j0 + q, r = lane + 32 * k;
                if (j < n && r < n) {
                    if (conjT) Q[j * ld + r] = cconj(c[q][k]);
                    else Q[r * ld + j] = c[q][k];
                }
            }
    }
    __syncthreads();
}

// C <- R^{-1} diag(rs) C (as trsm_left_upper): columns independent; row i's
// value comes from lane i % 32 by shuffle.
template <int RW, int CPW, bool FCM = false>
COLD void trsm_left_upper_big(int n, int ld, const cplx* F, const cplx* rinv, const double* rs, cplx* C) {
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int j0 = wp * CPW; j0 < n; j0 += nw * CPW) {
        cplx c[CPW][RW];
#pragma unroll
        for (int q = 0; q < CPW; ++q)
#pragma unroll
            for (int k = 0; k < RW; ++k) {
                const int j = j0 + q, r = lane + 32 * k;
                if (j < n && r < n) {
                    const cplx x = C[r * ld + j];
                    const double f = rs[r];
                    c[q][k] = cmk(x.x * f, x.y * f);
                } else {
                    c[q][k] = cmk(0.0, 0.0);
                }
            }
#pragma unroll
        for (int kk = RW - 1; kk >= 0; --kk) {
            for (int l = 31; l >= 0; --l) {
                const int i = 32 * kk + l;
                if (i >= n) continue;   // uniform
                const cplx ri = rinv[i];
                cplx fcol[RW];
#pragma unroll
                for (int k = 0; k < RW; ++k) {
                    const int r = lane + 32 * k;
                    fcol[k] = (r < i) ? F[FCM ? i * ld + r : r * ld + i] : cmk(0.0, 0.0);
                }
#pragma unroll
                for (int q = 0; q < CPW; ++q) {
                    cplx x;
                    x.x = __shfl_sync(0xffffffffu, c[q][kk].x, l);
                    x.y = __shfl_sync(0xffffffffu, c[q][kk].y, l);
                    x = cmul(x, ri);
                    if (lane == l) c[q][kk] = x;
#pragma unroll
                    for (int k = 0; k < RW; ++k) c[q][k] = csub(c[q][k], cmul(fcol[k], x));
                }
            }
        }
#pragma unroll
        for (int q = 0; q < CPW; ++q)
#pragma unroll
            for (int k = 0; k < RW; ++k) {
                const int j = j0 + q, r = lane + 32 * k;
                if (j < n && r < n) C[r * ld + j] = c[q][k];
            }
    }
    __syncthreads();
}

// C <- C diag(cs) R^{-H} (as trsm_right_upperH): rows independent; column c's
// value comes from lane c % 32.
template <int RW, int CPW, bool FCM = false>
COLD void trsm_right_upperH_big(int n, int ld, const cplx* F, const cplx* rinv, const double* cs, cplx* C) {
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int r0 = wp * CPW; r0 < n; r0 += nw * CPW) {
        cplx c[CPW][RW];   // c[q][k] = C[row r0+q][col lane+32k]
#pragma unroll
        for (int q = 0; q < CPW; ++q)
#pragma unroll
            for (int k = 0; k < RW; ++k) {
                const int r = r0 + q, col = lane + 32 * k;
                if (r < n && col < n) {
                    const cplx x = C[r * ld + col];
                    const double f = cs[col];
                    c[q][k] = cmk(x.x * f, x.y * f);
                } else {
                    c[q][k] = cmk(0.0, 0.0);
                }
            }
#pragma unroll
        for (int kk = RW - 1; kk >= 0; --kk) {
            for (int l = 31; l >= 0; --l) {
                const int cc = 32 * kk + l;
                if (cc >= n) continue;
                const cplx ri = cconj(rinv[cc]);
                cplx frow[RW];
#pragma unroll
                for (int k = 0; k < RW; ++k) {
                    const int col = lane + 32 * k;
                    frow[k] = (col < cc) ? F[FCM ? cc * ld + col : col * ld + cc] : cmk(0.0, 0.0);
                }
#pragma unroll
                for (int q = 0; q < CPW; ++q) {
                    cplx x;
                    x.x = __shfl_sync(0xffffffffu, c[q][kk].x, l);
                    x.y = __shfl_sync(0xffffffffu, c[q][kk].y, l);
                    x = cmul(x, ri);
                    if (lane == l) c[q][kk] = x;
#pragma unroll
                    for (int k = 0; k < RW; ++k) c[q][k] = csub(c[q][k], cmulcj(x, frow[k]));
                }
            }
        }
#pragma unroll
        for (int q = 0; q < CPW; ++q)
#pragma unroll
            for (int k = 0; k < RW; ++k) {
                const int r = r0 + q, col = lane + 32 * k;
                if (r < n && col < n) C[r * ld + col] = c[q][k];
            }
    }
    __syncthreads();
}
