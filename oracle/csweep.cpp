// C++ restatement of the number-conserving sweep of BAFQMC
// (src/number_conserving/src/{localU,multiply,stabilization,local_sweep,obser_equal}.f90),
// following oracle/oracle.py call for call.  Test infrastructure: the timed CPU
// baseline of the benchmark (one chain per thread) and a
// second restatement that tests check against oracle.py.  The product never
// loads it.  Chains run on nthreads std::threads, one chain at a time each.
//
// Matrices are row-major n x n, element (i, j) = G(i, j).  Complex arithmetic
// follows Fortran rules and no operations are fused (built with
// -fcx-fortran-rules -ffp-contract=off).  The factorisations restate LAPACK's
// published algorithms: ZGEQP3 in its unblocked ZLAQP2 form (pivot on the
// largest partial column norm, ZLARFG reflectors, the norm downdate with its
// recomputation threshold sqrt(eps)), ZUNGQR, ZUNMQR, ZTRSM and ZTRMM.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <thread>

using cd = std::complex<double>;
using Mat = std::vector<cd>;

namespace {

double ranf(int32_t& seed) {   // src/common/random.f90:1-11
    const long long v = (48828125LL * (long long)seed) % 2147483648LL;
    seed = (int32_t)(v < 0 ? v + 2147483648LL : v);
    return (double)seed / 2147483648.0;
}

cd cexp(cd z) {
    const double l = std::exp(z.real());
    return cd(l * std::cos(z.imag()), l * std::sin(z.imag()));
}

// Smith's algorithm for a / b
cd cdiv(cd a, cd b) {
    if (std::fabs(b.real()) >= std::fabs(b.imag())) {
        const double r = b.imag() / b.real(), den = b.real() + b.imag() * r;
        return cd((a.real() + a.imag() * r) / den, (a.imag() - a.real() * r) / den);
    }
    const double r = b.real() / b.imag(), den = b.real() * r + b.imag();
    return cd((a.real() * r + a.imag()) / den, (a.imag() * r - a.real()) / den);
}

double cabs(cd z) { return std::hypot(z.real(), z.imag()); }

// C = A B (C distinct from A and B)
void gemm(int n, const cd* A, const cd* B, cd* C) {
    for (int i = 0; i < n * n; ++i) C[i] = 0.0;
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k) {
            const cd a = A[i * n + k];
            const cd* b = B + k * n;
            cd* c = C + i * n;
            for (int j = 0; j < n; ++j) c[j] += a * b[j];
        }
}
void conj_transpose(int n, const cd* A, cd* B) {
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) B[j * n + i] = std::conj(A[i * n + j]);
}

double colnorm(int n, const cd* A, int j, int r0) {   // DZNRM2 of A(r0:n-1, j)
    double scale = 0.0, ssq = 1.0;
    for (int r = r0; r < n; ++r)
        for (double x : {A[r * n + j].real(), A[r * n + j].imag()})
            if (x != 0.0) {
                const double ax = std::fabs(x);
                if (scale < ax) {
                    ssq = 1.0 + ssq * (scale / ax) * (scale / ax);
                    scale = ax;
                } else {
                    ssq += (ax / scale) * (ax / scale);
                }
            }
    return scale * std::sqrt(ssq);
}

// ZGEQP3 (ZLAQP2) + QDRP_decompose (stabilization.f90:41-67): on exit A holds
// the scaled R (row i divided by |R_ii|) and the reflectors; d = |diag R|.
void qdrp(int n, cd* A, std::vector<int>& piv, std::vector<cd>& tau, std::vector<double>& d) {
    const double tol3z = std::sqrt(std::pow(2.0, -53));
    std::vector<double> vn1(n), vn2(n);
    for (int j = 0; j < n; ++j) {
        vn1[j] = vn2[j] = colnorm(n, A, j, 0);
        piv[j] = j;
    }
    for (int i = 0; i < n; ++i) {
        int pvt = i;
        for (int j = i + 1; j < n; ++j)
            if (vn1[j] > vn1[pvt]) pvt = j;
        if (pvt != i) {
            for (int r = 0; r < n; ++r) std::swap(A[r * n + pvt], A[r * n + i]);
            std::swap(piv[pvt], piv[i]);
            vn1[pvt] = vn1[i];
            vn2[pvt] = vn2[i];
        }
        // ZLARFG on A(i:n-1, i)
        const cd alpha = A[i * n + i];
        const double xnorm = i + 1 < n ? colnorm(n, A, i, i + 1) : 0.0;
        cd t = 0.0;
        if (!(xnorm == 0.0 && alpha.imag() == 0.0)) {
            const double nrm = std::sqrt(alpha.real() * alpha.real() + alpha.imag() * alpha.imag() + xnorm * xnorm);
            const double beta = alpha.real() >= 0.0 ? -nrm : nrm;
            t = cd((beta - alpha.real()) / beta, -alpha.imag() / beta);
            const cd scal = cdiv(cd(1.0, 0.0), alpha - beta);
            for (int r = i + 1; r < n; ++r) A[r * n + i] *= scal;
            A[i * n + i] = beta;
        }
        tau[i] = t;
        // H(i)^H applied to the trailing columns
        const cd ct = std::conj(t);
        for (int j = i + 1; j < n; ++j) {
            cd w = A[i * n + j];
            for (int r = i + 1; r < n; ++r) w += std::conj(A[r * n + i]) * A[r * n + j];
            const cd f = ct * w;
            A[i * n + j] -= f;
            for (int r = i + 1; r < n; ++r) A[r * n + j] -= A[r * n + i] * f;
        }
        // norm downdate (ZLAQP2)
        for (int j = i + 1; j < n; ++j) {
            if (vn1[j] == 0.0) continue;
            double temp = cabs(A[i * n + j]) / vn1[j];
            temp = std::fmax(1.0 - temp * temp, 0.0);
            const double q = vn1[j] / vn2[j];
            if (temp * q * q <= tol3z) {
                vn1[j] = i + 1 < n ? colnorm(n, A, j, i + 1) : 0.0;
                vn2[j] = vn1[j];
            } else {
                vn1[j] *= std::sqrt(temp);
            }
        }
    }
    for (int i = 0; i < n; ++i) {
        const double x = cabs(A[i * n + i]);
        d[i] = x;
        for (int c = i; c < n; ++c) A[i * n + c] = cd(A[i * n + c].real() / x, A[i * n + c].imag() / x);
    }
}

// v_i (unit at i, zero above) from column i of F
inline cd vref(int n, const cd* F, int i, int r) { return r == i ? cd(1.0, 0.0) : (r > i ? F[r * n + i] : cd(0.0)); }

void ungqr(int n, const cd* F, const std::vector<cd>& tau, cd* Q) {   // Q = H_0 ... H_{n-1}
    for (int j = 0; j < n; ++j) {
        std::vector<cd> c(n, 0.0);
        c[j] = 1.0;
        for (int i = j; i >= 0; --i) {
            cd w = 0.0;
            for (int r = i; r < n; ++r) w += std::conj(vref(n, F, i, r)) * c[r];
            const cd f = tau[i] * w;
            for (int r = i; r < n; ++r) c[r] -= vref(n, F, i, r) * f;
        }
        for (int r = 0; r < n; ++r) Q[r * n + j] = c[r];
    }
}
void unmqr_lc(int n, const cd* F, const std::vector<cd>& tau, cd* C) {   // C <- Q^H C
    for (int i = 0; i < n; ++i) {
        const cd ct = std::conj(tau[i]);
        for (int j = 0; j < n; ++j) {
            cd w = 0.0;
            for (int r = i; r < n; ++r) w += std::conj(vref(n, F, i, r)) * C[r * n + j];
            const cd f = ct * w;
            for (int r = i; r < n; ++r) C[r * n + j] -= vref(n, F, i, r) * f;
        }
    }
}
void unmqr_rn(int n, const cd* F, const std::vector<cd>& tau, cd* C) {   // C <- C Q
    for (int i = 0; i < n; ++i)
        for (int r = 0; r < n; ++r) {
            cd w = 0.0;
            for (int k = i; k < n; ++k) w += C[r * n + k] * vref(n, F, i, k);
            const cd f = tau[i] * w;
            for (int k = i; k < n; ++k) C[r * n + k] -= f * std::conj(vref(n, F, i, k));
        }
}

struct Chain {
    int n, L, nwrap, nst;
    Mat G, UUR, VUR, UUL, VUL;
    std::vector<double> DUR, DUL;
    std::vector<Mat> UR, VR, UL, VL;
    std::vector<std::vector<double>> DR, DL;
    Mat t1, t2, t3;
    Chain(int n_, int L_, int nwrap_) : n(n_), L(L_), nwrap(nwrap_), nst(L_ / nwrap_) {
        auto eye = [&] {
            Mat m((size_t)n * n, 0.0);
            for (int i = 0; i < n; ++i) m[i * n + i] = 1.0;
            return m;
        };
        G = UUR = VUR = UUL = VUL = eye();
        DUR.assign(n, 1.0);
        DUL.assign(n, 1.0);
        UR.assign(nst + 1, Mat()); VR = UL = VL = UR;
        DR.assign(nst + 1, {}); DL = DR;
        t1.resize((size_t)n * n); t2.resize((size_t)n * n); t3.resize((size_t)n * n);
    }
    void stab_UR() {   // stabilization.f90:69-93
        std::vector<int> piv(n);
        std::vector<cd> tau(n);
        std::vector<double> d(n);
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) t1[r * n + c] = UUR[r * n + c] * DUR[c];
        qdrp(n, t1.data(), piv, tau, d);
        DUR = d;
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) t2[r * n + c] = VUR[piv[r] * n + c];
        for (int i = 0; i < n; ++i)   // ZTRMM L,U,N: rows ascending use the rows below, not yet changed
            for (int c = 0; c < n; ++c) {
                cd s = 0.0;
                for (int k = i; k < n; ++k) s += t1[i * n + k] * t2[k * n + c];
                t2[i * n + c] = s;
            }
        VUR = t2;
        ungqr(n, t1.data(), tau, UUR.data());
    }
    void stab_UL() {   // stabilization.f90:95-119
        std::vector<int> piv(n);
        std::vector<cd> tau(n);
        std::vector<double> d(n);
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) t1[r * n + c] = std::conj(UUL[c * n + r]) * DUL[c];
        qdrp(n, t1.data(), piv, tau, d);
        DUL = d;
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) t2[r * n + c] = VUL[r * n + piv[c]];
        for (int c = 0; c < n; ++c)   // ZTRMM R,U,C: columns ascending use the columns to the right
            for (int r = 0; r < n; ++r) {
                cd s = 0.0;
                for (int k = c; k < n; ++k) s += t2[r * n + k] * std::conj(t1[c * n + k]);
                t2[r * n + c] = s;
            }
        VUL = t2;
        ungqr(n, t1.data(), tau, t3.data());
        conj_transpose(n, t3.data(), UUL.data());
    }
    // stab_green (stabilization.f90:121-190) into out
    void stab_green(int nt, Mat& out, double* logdet) {
        gemm(n, VUR.data(), VUL.data(), t1.data());                 // V_R V_L
        Mat a((size_t)n * n), b((size_t)n * n);
        conj_transpose(n, UUR.data(), a.data());
        conj_transpose(n, UUL.data(), b.data());
        gemm(n, a.data(), b.data(), t2.data());                      // U_R^H U_L^H
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) t2[r * n + c] -= DUR[r] * (t1[r * n + c] * DUL[c]);
        if (nt > L / 2) {
            conj_transpose(n, t2.data(), t3.data());
            t2 = t3;
        }
        std::vector<int> piv(n);
        std::vector<cd> tau(n);
        std::vector<double> dup(n);
        qdrp(n, t2.data(), piv, tau, dup);
        if (nt < L / 2 + 1) {
            Mat tmp = a;   // U_R^H
            unmqr_lc(n, t2.data(), tau, tmp.data());
            for (int r = 0; r < n; ++r)
                for (int c = 0; c < n; ++c) tmp[r * n + c] = cd(tmp[r * n + c].real() / dup[r], tmp[r * n + c].imag() / dup[r]);
            for (int c = 0; c < n; ++c)   // ZTRSM L,U,N
                for (int i = n - 1; i >= 0; --i) {
                    cd s = tmp[i * n + c];
                    for (int k = i + 1; k < n; ++k) s -= t2[i * n + k] * tmp[k * n + c];
                    tmp[i * n + c] = cdiv(s, t2[i * n + i]);
                }
            for (int r = 0; r < n; ++r)
                for (int c = 0; c < n; ++c) t3[piv[r] * n + c] = tmp[r * n + c];
            gemm(n, b.data(), t3.data(), out.data());                // U_L^H P X
        } else {
            Mat tmp = b;   // U_L^H
            unmqr_rn(n, t2.data(), tau, tmp.data());
            for (int r = 0; r < n; ++r)
                for (int c = 0; c < n; ++c) tmp[r * n + c] = cd(tmp[r * n + c].real() / dup[c], tmp[r * n + c].imag() / dup[c]);
            for (int r = 0; r < n; ++r)   // ZTRSM R,U,C
                for (int c = n - 1; c >= 0; --c) {
                    cd s = tmp[r * n + c];
                    for (int k = c + 1; k < n; ++k) s -= tmp[r * n + k] * std::conj(t2[c * n + k]);
                    tmp[r * n + c] = cdiv(s, std::conj(t2[c * n + c]));
                }
            for (int r = 0; r < n; ++r)
                for (int c = 0; c < n; ++c) t3[r * n + piv[c]] = tmp[r * n + c];
            gemm(n, t3.data(), a.data(), out.data());                // X P^T U_R^H
        }
        if (logdet) {
            double s = 0.0;
            for (int i = 0; i < n; ++i) s += std::log(dup[i]);
            *logdet = s;
        }
    }
};

struct Params {
    int n, L, nwrap;
    double shift, RT, U1, U2;
    cd alpha[2];
    int active[2];
    const cd *expP, *expM, *phase;
    const int* bonds;   // n x 3 neighbours
    int hasK;
};

struct Obs {   // the bin sums compared against oracle.py's ObserEqual
    double density_total = 0, energy_density = 0, kinetic = 0, doubleOcc = 0, numsquare_up = 0;
    cd sf_K = 0, dw_K = 0, psf_Gamma = 0;
};

void measure(const Params& p, const Mat& G, Obs& o) {   // obser_equal.f90:95-198
    const int n = p.n;
    const double lq = n;
    std::vector<cd> du(n), dd(n);
    for (int i = 0; i < n; ++i) {
        du[i] = G[i * n + i] - 1.0;
        dd[i] = std::conj(G[i * n + i]) - 1.0;
    }
    double dens = 0, dbl = 0, onsite_up = 0, onsite_do = 0, nsq = 0;
    for (int i = 0; i < n; ++i) {
        dens += (du[i] + dd[i]).real() / lq;
        dbl += (du[i] * dd[i]).real() / lq;
        onsite_up += (2.0 * du[i] * du[i] + du[i]).real();
        onsite_do += (2.0 * dd[i] * dd[i] + dd[i]).real();
    }
    cd psf = 0, sfk = 0, dwk = 0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const cd gup = G[i * n + j];
            cd gupc = G[j * n + i];                 // Grupc(i, j) = Grup(j, i) - delta
            if (i == j) gupc -= 1.0;
            const cd gdo = std::conj(gup), gdoc = std::conj(gupc);
            nsq += (du[i] * du[j] + gupc * gup).real();
            psf += gupc * gdoc;
            if (p.hasK) {
                const cd ph = p.phase[i * n + j];
                sfk += ph * (gupc + gdoc);
                dwk += ph * (du[i] * du[j] + gupc * gup + dd[i] * dd[j] + gdoc * gdo + du[i] * dd[j] + dd[i] * du[j]);
            }
        }
    double kin = 0;
    for (int nb = 0; nb < 3; ++nb)
        for (int i = 0; i < n; ++i) {
            const int j = p.bonds[i * 3 + nb];
            cd gij = G[j * n + i], gji = G[i * n + j];   // Grupc(i, j), Grupc(j, i)
            if (i == j) {
                gij -= 1.0;
                gji -= 1.0;
            }
            kin += p.RT * (gij + gji + std::conj(gij) + std::conj(gji)).real() / lq;
        }
    const double inter = (p.U1 + p.U2) * (onsite_up + onsite_do) / lq + 2.0 * (p.U2 - p.U1) * dbl;
    const double lq2 = lq * lq;
    o.density_total += dens;
    o.doubleOcc += dbl;
    o.numsquare_up += nsq;
    o.kinetic += kin;
    o.energy_density += kin + inter;
    o.psf_Gamma += psf / lq2;
    o.sf_K += sfk / lq2;
    o.dw_K += dwk / lq2;
}

struct Run {
    const Params& p;
    Chain ch;
    int32_t seed;
    double* phi;   // [L][n][2]
    long long nacc[2] = {0, 0}, nc[2] = {0, 0};
    double xmax = 0, xmean = 0;
    Obs obs;
    int nobs = 0;
    Run(const Params& p_, int32_t seed_, double* phi_) : p(p_), ch(p_.n, p_.L, p_.nwrap), seed(seed_), phi(phi_) {}

    cd expalpha(int nf, double ph, int nflag) const {
        const cd z(p.alpha[nf].real() * ph, p.alpha[nf].imag() * ph);
        return cexp(cd(z.real() * nflag, z.imag() * nflag));
    }
    void metro(int nf, int ii, int nt) {   // localU.f90:31-77
        const int n = p.n;
        double& ph = phi[((long)nt * n + ii) * 2 + nf];
        const double po = ph;
        const double xflip = ranf(seed);
        const double pn = po + (xflip - 0.5) * std::fabs(p.shift);
        const double gn = std::exp(-0.5 * pn * pn), go = std::exp(-0.5 * po * po);
        const cd ratio_exp = cdiv(cd(gn, 0.0), cd(go, 0.0));
        const cd delta = cdiv(expalpha(nf, pn, 1), expalpha(nf, po, 1)) - 1.0;
        cd rd = 1.0 + delta * (1.0 - ch.G[ii * n + ii]);
        rd = cdiv(cd(1.0, 0.0), rd);
        const double rabs = cabs(ratio_exp * rd * std::conj(rd));
        const double rnd = ranf(seed);
        ++nc[nf];
        if (rabs > rnd) {
            ++nacc[nf];
            const cd a = -rd * delta;
            std::vector<cd> col(n), vec(n);
            for (int r = 0; r < n; ++r) col[r] = ch.G[r * n + ii];
            for (int c = 0; c < n; ++c) vec[c] = -ch.G[ii * n + c];
            vec[ii] += 1.0;
            for (int r = 0; r < n; ++r) {
                const cd ac = a * col[r];
                for (int c = 0; c < n; ++c) ch.G[r * n + c] += ac * vec[c];
            }
            ph = pn;
        }
    }
    void prop_L(int nf, int nt) {   // localU.f90:79-95
        const int n = p.n;
        for (int ii = n - 1; ii >= 0; --ii) {
            metro(nf, ii, nt);
            const double ph = phi[((long)nt * n + ii) * 2 + nf];
            const cd ep = expalpha(nf, ph, 1), em = expalpha(nf, ph, -1);
            for (int r = 0; r < n; ++r) ch.G[r * n + ii] *= ep;
            for (int c = 0; c < n; ++c) ch.G[ii * n + c] *= em;
        }
        for (int ii = n - 1; ii >= 0; --ii) {
            const cd ep = expalpha(nf, phi[((long)nt * n + ii) * 2 + nf], 1);
            for (int r = 0; r < n; ++r) ch.UUL[r * n + ii] *= ep;
        }
    }
    void prop_R(int nf, int nt) {   // localU.f90:97-113
        const int n = p.n;
        for (int ii = 0; ii < n; ++ii) {
            const double ph = phi[((long)nt * n + ii) * 2 + nf];
            const cd ep = expalpha(nf, ph, 1), em = expalpha(nf, ph, -1);
            for (int c = 0; c < n; ++c) ch.G[ii * n + c] *= ep;
            for (int r = 0; r < n; ++r) ch.G[r * n + ii] *= em;
            metro(nf, ii, nt);
        }
        for (int ii = 0; ii < n; ++ii) {
            const cd ep = expalpha(nf, phi[((long)nt * n + ii) * 2 + nf], 1);
            for (int c = 0; c < n; ++c) ch.UUR[ii * n + c] *= ep;
        }
    }
    void mult(const cd* A, Mat& X, bool left) {   // X <- A X (left) or X A
        if (left) gemm(p.n, A, X.data(), ch.t3.data());
        else gemm(p.n, X.data(), A, ch.t3.data());
        X.swap(ch.t3);
    }
    void drift(Mat& gr) {
        double dif = 0;
        for (size_t k = 0; k < gr.size(); ++k) dif += cabs(gr[k] - ch.G[k]);
        if (dif > xmax) xmax = dif;
        xmean += dif;
        ch.G.swap(gr);
    }
    void pre() {   // local_sweep.f90:80-94
        const int n = p.n;
        ch.UR[0] = ch.UUR; ch.VR[0] = ch.VUR; ch.DR[0] = ch.DUR;
        for (int nt = 1; nt <= p.L; ++nt) {
            for (int nf = 0; nf < 2; ++nf) {
                if (!p.active[nf]) continue;
                for (int ii = 0; ii < n; ++ii) {
                    const cd ep = expalpha(nf, phi[((long)(nt - 1) * n + ii) * 2 + nf], 1);
                    for (int c = 0; c < n; ++c) ch.UUR[ii * n + c] *= ep;
                }
            }
            mult(p.expP, ch.UUR, true);
            if (nt % p.nwrap == 0) {
                const int st = nt / p.nwrap;
                ch.stab_UR();
                ch.UR[st] = ch.UUR; ch.VR[st] = ch.VUR; ch.DR[st] = ch.DUR;
                if (nt == p.L) {
                    Mat g((size_t)n * n);
                    ch.stab_green(nt, g, nullptr);
                    ch.G = g;
                }
            }
        }
    }
    void wrap_L(int nt) {
        const int st = nt / p.nwrap;
        ch.UUR = ch.UR[st]; ch.VUR = ch.VR[st]; ch.DUR = ch.DR[st];
        if (nt != p.L) {
            ch.stab_UL();
            Mat g((size_t)p.n * p.n);
            ch.stab_green(nt, g, nullptr);
            drift(g);
        }
        ch.UL[st] = ch.UUL; ch.VL[st] = ch.VUL; ch.DL[st] = ch.DUL;
    }
    void wrap_R(int nt) {
        const int st = nt / p.nwrap;
        ch.UUL = ch.UL[st]; ch.VUL = ch.VL[st]; ch.DUL = ch.DL[st];
        if (nt != 0) {
            ch.stab_UR();
            Mat g((size_t)p.n * p.n);
            ch.stab_green(nt, g, nullptr);
            drift(g);
        }
        ch.UR[st] = ch.UUR; ch.VR[st] = ch.VUR; ch.DR[st] = ch.DUR;
    }
    void sweep() {   // local_sweep.f90:96-134
        for (int nt = p.L; nt >= 1; --nt) {
            if (nt % p.nwrap == 0) wrap_L(nt);
            measure(p, ch.G, obs);
            ++nobs;
            mult(p.expP, ch.G, false);   // propT_L: G e^{-dK}, then e^{+dK} G, U_L e^{-dK}
            mult(p.expM, ch.G, true);
            mult(p.expP, ch.UUL, false);
            if (p.active[1]) prop_L(1, nt - 1);
            if (p.active[0]) prop_L(0, nt - 1);
        }
        wrap_L(0);
        wrap_R(0);
        for (int nt = 1; nt <= p.L; ++nt) {
            if (p.active[0]) prop_R(0, nt - 1);
            if (p.active[1]) prop_R(1, nt - 1);
            mult(p.expP, ch.G, true);    // propT_R: e^{-dK} G, then G e^{+dK}, e^{-dK} U_R
            mult(p.expM, ch.G, false);
            mult(p.expP, ch.UUR, true);
            if (nt % p.nwrap == 0) wrap_R(nt);
            measure(p, ch.G, obs);
            ++nobs;
        }
    }
};

}  // namespace

// Runs nchains chains of one point: bafqmc_pre's work, then nsweep sweeps.
// seeds and phi ([chain][L][n][2]) are updated in place.  Per chain out:
// obs[chain][12] = density_total, energy_density, kinetic, doubleOcc,
// numsquare_up, sf_K (re, im), dw_K (re, im), psf_Gamma (re, im) averaged over
// the last sweep's measurements, then accepted[2], proposals[2], Xmaxm;
// G[chain][n][n][2] (optional) the final Green's function.  sweep_seconds
// receives the longest time any thread spent in sweeps (after pre).
extern "C" int csweep_run(int n, int L, int nwrap, double shiftLoc, double RT, double U1, double U2,
                          const double* alpha /* [2][2] */, const int* active, const double* expP,
                          const double* expM, const double* phase, int hasK, const int* bonds, int nchains,
                          int32_t* seeds, double* phi, int nsweep, int nthreads, double* obs, double* G,
                          double* sweep_seconds) {
    Params p;
    p.n = n;
    p.L = L;
    p.nwrap = nwrap;
    p.shift = shiftLoc;
    p.RT = RT;
    p.U1 = U1;
    p.U2 = U2;
    for (int k = 0; k < 2; ++k) {
        p.alpha[k] = cd(alpha[2 * k], alpha[2 * k + 1]);
        p.active[k] = active[k];
    }
    p.expP = reinterpret_cast<const cd*>(expP);
    p.expM = reinterpret_cast<const cd*>(expM);
    p.phase = reinterpret_cast<const cd*>(phase);
    p.hasK = hasK;
    p.bonds = bonds;
    std::atomic<int> next(0);
    std::vector<double> tmax(std::max(nthreads, 1), 0.0);
    auto worker = [&](int tid) {
        for (int c = next++; c < nchains; c = next++) {
            Run r(p, seeds[c], phi + (long)c * L * n * 2);
            r.pre();
            const auto t0 = std::chrono::steady_clock::now();
            for (int s = 0; s < nsweep; ++s) {
                r.obs = Obs();
                r.nobs = 0;
                r.sweep();
            }
            const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            tmax[tid] = std::max(tmax[tid], dt);
            seeds[c] = r.seed;
            if (obs) {
                double* o = obs + (long)c * 15;
                const double z = 1.0 / r.nobs;
                const Obs& b = r.obs;
                const double v[15] = {b.density_total * z, b.energy_density * z, b.kinetic * z, b.doubleOcc * z,
                                      b.numsquare_up * z, b.sf_K.real() * z, b.sf_K.imag() * z, b.dw_K.real() * z,
                                      b.dw_K.imag() * z, b.psf_Gamma.real() * z, b.psf_Gamma.imag() * z,
                                      (double)r.nacc[0], (double)r.nacc[1], (double)r.nc[0], r.xmax};
                std::memcpy(o, v, sizeof v);
            }
            if (G) std::memcpy(G + (long)c * n * n * 2, r.ch.G.data(), sizeof(cd) * n * n);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) pool.emplace_back(worker, t);
    worker(0);
    for (auto& t : pool) t.join();
    double tm = 0.0;
    for (double v : tmax) tm = std::max(tm, v);
    if (sweep_seconds) *sweep_seconds = tm;
    return 0;
}
