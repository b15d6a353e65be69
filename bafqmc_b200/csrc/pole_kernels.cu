// Pole diagnostics of the bosonic Green's function on the device
// (PoleDiagnostics, src/number_conserving/src/pole_diagnostics.f90:15-123).
//
// Per number-conserving chain, from the current G:
//   * the eigenvalues lambda of G (ZGEEV, pole_diagnostics.f90:15-51) and the
//     poles z = 1/lambda (|lambda| <= tiny gives 1/tiny, :100-107);
//   * pole_distance = max(min |z|, tiny), pole_x = -log10(pole_distance),
//     green_spectral_radius = max |lambda| (:109-112);
//   * green_smax, the largest singular value of G (ZGESVD, :53-89), as the
//     square root of the largest eigenvalue of G^H G.
// log_weight (:119) combines the field norm with log|det G| from the sweep's
// last stabilised factorisation and is assembled by the host call.
//
// One warp per chain (one CTA of 32 threads), with the matrix in shared memory
// at an odd leading dimension (in a per-chain HBM scratch above n = 112, whose
// matrix does not fit in shared memory).  The eigenvalues come from a diagonal balancing
// (Parlett and Reinsch, radix 2), a Householder reduction to Hessenberg form
// and the complex single-shift QR iteration with Wilkinson shifts and
// deflation on negligible subdiagonals (Golub and Van Loan, Matrix
// Computations, sections 7.4-7.5), eigenvalues only: each bulge chase works
// on the active window.  The reference's ZGEEV runs the same sequence of
// steps with LAPACK's own shift and deflation strategy, so both are backward
// stable and the eigenvalues agree to rounding, but not their order in the
// output (ZGEEV's is the diagonal of its Schur form, as here).
#include "sweep.cuh"
#include "kernels.h"

namespace bq {

namespace {

constexpr double kUlp = 2.220446049250313e-16;       // 2^-52
constexpr double kTiny = 2.2250738585072014e-308;    // smallest normal double (Fortran tiny(1.d0))

extern __shared__ __align__(16) unsigned char pole_smem[];

DEVI double cabs1(cplx a) { return fabs(a.x) + fabs(a.y); }

// principal square root from |z| and the half-angle identities
DEVI cplx csqrt_principal(cplx z) {
    const double r = hypot(z.x, z.y);
    if (r == 0.0) return cmk(0.0, 0.0);
    if (z.x >= 0.0) {
        const double t = sqrt(0.5 * (r + z.x));
        return cmk(t, z.y / (2.0 * t));
    }
    const double t = sqrt(0.5 * (r - z.x));
    return cmk(fabs(z.y) / (2.0 * t), copysign(t, z.y));
}

// Eigenvalues of [[a, b], [c, d]] as d + mu with mu^2 - (a - d) mu - bc = 0:
// e1 takes the root of larger modulus, e2 = d - bc / (x + y) the one nearer d
// (the Wilkinson shift).  Scaled by the largest entry against overflow.
DEVI void eig2x2(cplx a, cplx b, cplx c, cplx d, cplx& e1, cplx& e2) {
    const double s = fmax(fmax(cabs1(a), cabs1(b)), fmax(cabs1(c), cabs1(d)));
    if (s == 0.0) {
        e1 = e2 = cmk(0.0, 0.0);
        return;
    }
    const double is = 1.0 / s;
    a = cscale(a, is);
    b = cscale(b, is);
    c = cscale(c, is);
    d = cscale(d, is);
    const cplx x = cscale(csub(a, d), 0.5), bc = cmul(b, c);
    cplx y = csqrt_principal(cadd(cmul(x, x), bc));
    if (x.x * y.x + x.y * y.y < 0.0) y = cmk(-y.x, -y.y);
    const cplx den = cadd(x, y);
    if (den.x == 0.0 && den.y == 0.0) {
        e1 = e2 = cscale(d, s);
        return;
    }
    e1 = cscale(cadd(d, den), s);
    e2 = cscale(csub(d, cdiv(bc, den)), s);
}

// Plane rotation [c s; -conj(s) c] with c real that maps (x, y) to (r, 0).
DEVI void givens(cplx x, cplx y, double& c, cplx& s, cplx& r) {
    const double ay = cabsv(y);
    if (ay == 0.0) {
        c = 1.0;
        s = cmk(0.0, 0.0);
        r = x;
        return;
    }
    const double ax = cabsv(x);
    if (ax == 0.0) {
        c = 0.0;
        s = cscale(cconj(y), 1.0 / ay);
        r = cmk(ay, 0.0);
        return;
    }
    const double nrm = hypot(ax, ay);
    const cplx ph = cscale(x, 1.0 / ax);
    c = ax / nrm;
    s = cscale(cmulcj(ph, y), 1.0 / nrm);
    r = cscale(ph, nrm);
}

// 1 / z without overflow in |z|^2
DEVI cplx crecip(cplx z) {
    const double m = fmax(fabs(z.x), fabs(z.y));
    const double im = 1.0 / m;
    const cplx w = cscale(z, im);
    return cscale(cconj(w), im / cabs2(w));
}

// Diagonal similarity H <- D^-1 H D with D a power of 2 per index, equalising
// the off-diagonal row and column 1-norms (Parlett-Reinsch balancing).
DEVI void balance_warp(int n, int ld, cplx* H) {
    const int lane = threadIdx.x & 31;
    for (int pass = 0; pass < 64; ++pass) {
        bool changed = false;
        for (int i = 0; i < n; ++i) {
            double c = 0.0, r = 0.0;
            for (int j = lane; j < n; j += 32)
                if (j != i) {
                    c += cabs1(H[j * ld + i]);
                    r += cabs1(H[i * ld + j]);
                }
            c = warp_sum(c);
            r = warp_sum(r);
            if (c == 0.0 || r == 0.0) continue;
            const double s = c + r;
            double f = 1.0, g = 0.5 * r;
            for (int t = 0; t < 1100 && c < g; ++t) {
                f *= 2.0;
                c *= 4.0;
            }
            g = 2.0 * r;
            for (int t = 0; t < 1100 && c >= g; ++t) {
                f *= 0.5;
                c *= 0.25;
            }
            if ((c + r) / f < 0.95 * s) {
                changed = true;
                const double fi = 1.0 / f;
                for (int j = lane; j < n; j += 32) {
                    H[i * ld + j] = cscale(H[i * ld + j], fi);
                    H[j * ld + i] = cscale(H[j * ld + i], f);
                }
                __syncwarp();
            }
        }
        if (!changed) break;
    }
}

// Householder reduction to upper Hessenberg form (H <- P H P per column).
// v: n complex of scratch.
DEVI void hessenberg_warp(int n, int ld, cplx* H, cplx* v) {
    const int lane = threadIdx.x & 31;
    for (int k = 0; k + 2 < n; ++k) {
        const int m = n - k - 1;   // x = H[k+1 .. n-1][k]
        double tail = 0.0;
        for (int r = 1 + lane; r < m; r += 32) tail += cabs2(H[(k + 1 + r) * ld + k]);
        tail = warp_sum(tail);
        if (tail == 0.0) continue;   // column already reduced
        const cplx x0 = H[(k + 1) * ld + k];
        const double ax0 = cabsv(x0), nx = sqrt(ax0 * ax0 + tail);
        const cplx ph = ax0 == 0.0 ? cmk(1.0, 0.0) : cscale(x0, 1.0 / ax0);
        // v = x - beta e1 with beta = -ph |x|: v0 = ph (|x0| + |x|)
        const double a = ax0 + nx, t = 2.0 / (a * a + tail);
        for (int r = lane; r < m; r += 32) v[r] = r == 0 ? cscale(ph, a) : H[(k + 1 + r) * ld + k];
        __syncwarp();
        // left: rows k+1.., columns k+1..
        for (int c = k + 1 + lane; c < n; c += 32) {
            cplx w = cmk(0.0, 0.0);
            for (int r = 0; r < m; ++r) w = cfmacj(v[r], H[(k + 1 + r) * ld + c], w);
            w = cscale(w, t);
            for (int r = 0; r < m; ++r) {
                cplx& h = H[(k + 1 + r) * ld + c];
                h = csub(h, cmul(v[r], w));
            }
        }
        __syncwarp();
        // right: all rows, columns k+1..
        for (int r = lane; r < n; r += 32) {
            cplx w = cmk(0.0, 0.0);
            for (int c = 0; c < m; ++c) w = cfma(H[r * ld + k + 1 + c], v[c], w);
            w = cscale(w, t);
            for (int c = 0; c < m; ++c) {
                cplx& h = H[r * ld + k + 1 + c];
                h = csub(h, cmulcj(w, v[c]));
            }
        }
        // column k becomes (beta, 0, ..., 0) below the diagonal
        for (int r = lane; r < m; r += 32) H[(k + 1 + r) * ld + k] = r == 0 ? cscale(ph, -nx) : cmk(0.0, 0.0);
        __syncwarp();
    }
}

// Eigenvalues of the upper Hessenberg H (destroyed) into ev[0..n-1].
// Returns 0, or 1 if the iteration count exceeded 30 n.
DEVI int hqr_warp(int n, int ld, cplx* H, cplx* ev) {
    const int lane = threadIdx.x & 31;
    for (int i = lane; i < n; i += 32) ev[i] = cmk(__longlong_as_double(0x7ff8000000000000LL), 0.0);
    __syncwarp();
    int hi = n - 1, its = 0, total = 0;
    while (hi >= 0) {
        // largest k in [1, hi] with a negligible subdiagonal H[k][k-1]
        int l = 0;
        for (int base = hi; base >= 1; base -= 32) {
            const int k = base - lane;
            bool neg = false;
            if (k >= 1)
                neg = cabs1(H[k * ld + k - 1]) <= kUlp * (cabs1(H[k * ld + k]) + cabs1(H[(k - 1) * ld + k - 1]));
            const unsigned b = __ballot_sync(0xffffffffu, neg);
            if (b) {
                l = base - (__ffs(b) - 1);
                break;
            }
        }
        __syncwarp();
        if (l == hi) {
            if (lane == 0) ev[hi] = H[hi * ld + hi];
            hi -= 1;
            its = 0;
            __syncwarp();
            continue;
        }
        if (hi - l == 1) {
            cplx e1, e2;
            eig2x2(H[l * ld + l], H[l * ld + hi], H[hi * ld + l], H[hi * ld + hi], e1, e2);
            if (lane == 0) {
                ev[l] = e1;
                ev[hi] = e2;
            }
            hi -= 2;
            its = 0;
            __syncwarp();
            continue;
        }
        if (++total > 30 * n) return 1;
        ++its;
        cplx sig;
        if (its % 10 == 0) {   // exceptional shift against a stalled window
            sig = cadd(H[hi * ld + hi], cmk(0.75 * cabs1(H[hi * ld + hi - 1]), 0.0));
        } else {
            cplx e1;
            eig2x2(H[(hi - 1) * ld + hi - 1], H[(hi - 1) * ld + hi], H[hi * ld + hi - 1], H[hi * ld + hi], e1, sig);
        }
        cplx x = csub(H[l * ld + l], sig), y = H[(l + 1) * ld + l];
        for (int k = l; k < hi; ++k) {
            if (k > l) {
                x = H[k * ld + k - 1];
                y = H[(k + 1) * ld + k - 1];
            }
            double c;
            cplx s, r;
            givens(x, y, c, s, r);
            __syncwarp();
            if (k > l && lane == 0) {
                H[k * ld + k - 1] = r;
                H[(k + 1) * ld + k - 1] = cmk(0.0, 0.0);
            }
            // rows k, k+1 from the left, columns k..hi
            for (int j = k + lane; j <= hi; j += 32) {
                const cplx a = H[k * ld + j], b = H[(k + 1) * ld + j];
                H[k * ld + j] = cadd(cscale(a, c), cmul(s, b));
                H[(k + 1) * ld + j] = csub(cscale(b, c), cmulcj(a, s));   // -conj(s) a + c b
            }
            __syncwarp();
            // columns k, k+1 from the right, rows l..min(k+2, hi)
            const int ilast = min(k + 2, hi);
            for (int i = l + lane; i <= ilast; i += 32) {
                const cplx a = H[i * ld + k], b = H[i * ld + k + 1];
                H[i * ld + k] = cadd(cscale(a, c), cmulcj(b, s));        // c a + conj(s) b
                H[i * ld + k + 1] = csub(cscale(b, c), cmul(s, a));      // -s a + c b
            }
            __syncwarp();
        }
    }
    return 0;
}

// out per chain: kPoleScalars doubles (pole_distance, pole_x, spectral radius,
// smax, status) and zstride complex poles.
__global__ void __launch_bounds__(32) pole_kernel(KernelArgs ka, int zstride, double* zout, double* sout, cplx* hmat,
                                                   long long hstride) {
    const int chain = blockIdx.x;
    if (chain >= ka.nchains) return;
    const ChainDev cd = ka.chains[chain];
    const PointDev* P = ka.pts + cd.point;
    if (P->pairing || (ka.sc[chain].status & 1)) return;   // no pole files for Nambu chains; quarantined chains
    const int n = P->N, ld = n | 1, lane = threadIdx.x;
    cplx* v = reinterpret_cast<cplx*>(pole_smem);
    cplx* ev = v + n;
    cplx* H = hmat ? hmat + (long long)chain * hstride : ev + n;
    const cplx* G = reinterpret_cast<const cplx*>(ka.arena) + cd.arena_off;

    for (int e = lane; e < n * n; e += 32) {
        const int r = e / n, c = e - r * n;
        H[r * ld + c] = G[e];
    }
    __syncwarp();
    balance_warp(n, ld, H);
    hessenberg_warp(n, ld, H, v);
    int status = hqr_warp(n, ld, H, ev);
    __syncwarp();

    double rho = 0.0, zmin = __longlong_as_double(0x7ff0000000000000LL);
    double* zc = zout + (size_t)chain * zstride * 2;
    for (int i = lane; i < n; i += 32) {
        const cplx e = ev[i];
        const double ae = cabsv(e);
        const cplx z = ae <= kTiny ? cmk(1.0 / kTiny, 0.0) : crecip(e);
        zc[2 * i] = z.x;
        zc[2 * i + 1] = z.y;
        rho = fmax(rho, ae);
        zmin = fmin(zmin, cabsv(z));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        rho = fmax(rho, __shfl_xor_sync(0xffffffffu, rho, o));
        zmin = fmin(zmin, __shfl_xor_sync(0xffffffffu, zmin, o));
    }
    __syncwarp();

    // G^H G (Hermitian, positive semidefinite): its largest eigenvalue is smax^2
    for (int e = lane; e < n * n; e += 32) {
        const int r = e / n, c = e - r * n;
        cplx a = cmk(0.0, 0.0);
        for (int k = 0; k < n; ++k) a = cfmacj(G[k * n + r], G[k * n + c], a);
        H[r * ld + c] = a;
    }
    __syncwarp();
    hessenberg_warp(n, ld, H, v);
    status |= hqr_warp(n, ld, H, ev) << 1;
    __syncwarp();
    double lmax = 0.0;
    for (int i = lane; i < n; i += 32) lmax = fmax(lmax, ev[i].x);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));

    if (lane == 0) {
        const double pd = fmax(zmin, kTiny);
        double* so = sout + (size_t)chain * kPoleScalars;
        so[0] = pd;
        so[1] = -log10(pd);
        so[2] = rho;
        so[3] = sqrt(lmax);
        so[4] = (double)status;
    }
}

}  // namespace

long long pole_hbm_elems(int nmax) { return nmax > kPoleSmemMaxN ? (long long)nmax * (nmax | 1) : 0; }

cudaError_t launch_pole(const KernelArgs& ka, int nmax, int zstride, double* zout, double* sout, double2* hmat,
                        cudaStream_t st) {
    if (ka.nchains <= 0) return cudaSuccess;
    const long long hs = pole_hbm_elems(nmax);
    if (hs > 0 && !hmat) return cudaErrorInvalidValue;
    const size_t sm = sizeof(cplx) * (2 * (size_t)nmax + (hs > 0 ? 0 : (size_t)nmax * (nmax | 1)));
    cudaError_t e = cudaFuncSetAttribute(pole_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    pole_kernel<<<ka.nchains, 32, sm, st>>>(ka, zstride, zout, sout, hs > 0 ? hmat : nullptr, hs);
    return cudaGetLastError();
}

}  // namespace bq
