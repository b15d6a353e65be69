// Complex x real slice products on the 5th-generation tensor cores (tcgen05,
// sm_100a) in 3xTF32-compensated FP32: the mixed-precision option of the
// slice propagation C = X R or C = R X (X complex n x n, R = e^{-+dtau K} real
// n x n), for the size class whose matrices live in HBM (n <= 144).
//
// R is close to the identity (dtau is small), so C = X + X (R - I) or
// C = X + (R - I) X: the tensor cores form only the correction, and the
// epilogue adds X in FP64, which keeps the FP32 error relative to the
// correction's size rather than to C's.  The correction is one GEMM
// D = A B^T of real FP32 operands with M = 2n rows:
//   right:  A[m][k] = Re X[m][k] (m < n), Im X[m-n][k] (m >= n),
//           B[j][k] = (R - I)[k][j],  C[m][j] = X[m][j] + D[m][j] + i D[m+n][j];
//   left:   A[m][k] = Re X[k][m], Im X[k][m-n],  B[j][k] = (R - I)[j][k],
//           C[j][m] = X[j][m] + D[m][j] + i D[m+n][j]   (transposed product).
// Each FP64 operand x splits into TF32 hi = rn(x) and lo = rn(x - hi), and
// D accumulates lo*hi + hi*lo + hi*hi per K step in FP32 in tensor memory
// (the lo*lo term is below FP32 resolution).  The product runs in place: a
// row of D needs only its row of A, and every chunk of X is staged before the
// epilogue writes X + D back into X.
//
// Layout (PTX ISA, tcgen05 shared-memory matrix descriptors, no swizzle,
// K-major): operands are staged in chunks of kTcKC K values; within a chunk,
// each group of 4 K values (16 bytes) is a block of rows x 16 bytes, so an
// 8-row x 16-byte core matrix is contiguous, core matrices along M (N) are
// 128 bytes apart (SBO) and along K one block apart (LBO).  One MMA covers
// M = 128 rows, N = the product's column count rounded up to 16, K = 8.  The
// accumulator of M tile t sits at tensor-memory columns t*N .. t*N+N-1.
#pragma once
#include "cplx.cuh"

namespace bq {

constexpr int kTcMT = 384;   // A rows staged: 2n <= 288 rounded up to the M tile (128)
constexpr int kTcNB = 144;   // B rows staged: n rounded up to 16
constexpr int kTcKC = 32;    // K values per staged chunk (4 MMAs)
constexpr int kTcCols = 512;   // tensor-memory columns allocated (3 tiles x 144 <= 512)
constexpr size_t kTcABytes = sizeof(uint32_t) * kTcMT * kTcKC;   // one of A hi / A lo
constexpr size_t kTcBBytes = sizeof(uint32_t) * kTcNB * kTcKC;   // one of B hi / B lo
constexpr int kTcSpin = 1 << 22;   // bound on mbarrier polls before a product is declared failed
constexpr int kTcPer = 9;          // staged elements per thread and chunk: 144 * 32 / 512

DEVI uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: start address, leading (K) and stride (M/N)
// byte offsets in 16-byte units, descriptor version 1 (bits 46-47), no swizzle.
DEVI uint64_t tc_sdesc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}
// Instruction descriptor, kind::tf32: F32 accumulator (bits 4-5 = 1), A and B
// TF32 (bits 7-9, 10-12 = 2), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t tc_idesc_tf32(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

DEVI void tc_mma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t"
        "}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z));
}
DEVI void tc_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}
DEVI void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
DEVI void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
DEVI void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

DEVI void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Waits for the completion of the phase with the given parity; false after `spin` polls.
DEVI bool mbar_wait(uint32_t mbar, uint32_t parity, int spin = kTcSpin) {
    for (int it = 0; it < spin; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t"
            "}"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Warp-wide: allocate ncols tensor-memory columns, base address to *dst (shared).
DEVI void tmem_alloc(uint32_t dst_saddr, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_saddr), "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
DEVI void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
// Warp-wide: 16 consecutive columns of the warp's 32 lanes (lane quarter = warp % 4).
DEVI void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

DEVI uint32_t to_tf32(float f) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(f));
    return r;
}
// x = hi + lo to about 21 bits: hi = rn_tf32(x), lo = rn_tf32(x - hi) (residual in FP64)
DEVI void split_tf32(double x, uint32_t& hi, uint32_t& lo) {
    hi = to_tf32((float)x);
    lo = to_tf32((float)(x - (double)__uint_as_float(hi)));
}

// Shared-memory staging and tensor-memory state of the products.
struct TcBufs {
    uint32_t* ahi;
    uint32_t* alo;
    uint32_t* bhi;
    uint32_t* blo;
    uint64_t* mbar;   // completion barrier of the MMAs of one staged chunk
    uint32_t tmem;    // accumulator base (lane 0, first allocated column)
};

// X <- X R (right) or X <- R X (left) as above, n <= 144, matrices row-major
// with leading dimension ld.  Called by all threads of the CTA (blockDim.x a
// multiple of 128); returns with the CTA synchronised.  *phase (shared
// memory) is the parity of the next completion of b.mbar.
// Returns false if an MMA group did not complete within the poll bound (X is
// then unchanged); a group that did not complete within a second bound either
// is left in flight, and *pending (shared memory) receives 2 + its parity, so
// that the caller waits for it before it releases the tensor memory.
// wait_test: issue no MMA and poll 1024 times, so that the wait expires with
// nothing in flight (the test of this give-up path).
DEVI bool tc_product(int n, int ld, cplx* X, const double* R, bool right, const TcBufs& b, uint32_t* phase,
                     bool wait_test, uint32_t* pending) {
    cplx* C = X;
    const int tid = threadIdx.x, T = blockDim.x;
    const int nb = (n + 15) & ~15;            // MMA N
    const int mt = (2 * n + 127) >> 7;        // M tiles of 128 rows
    const int kpad = (n + 7) & ~7;            // K rounded up to the MMA step
    const uint32_t idesc = tc_idesc_tf32(128, nb);
    const uint32_t a_hi = smem_u32(b.ahi), a_lo = smem_u32(b.alo), b_hi = smem_u32(b.bhi), b_lo = smem_u32(b.blo);
    const uint32_t mb = smem_u32(b.mbar);
    bool ok = true;
    for (int k0 = 0; k0 < kpad; k0 += kTcKC) {
        const int kc = min(kTcKC, kpad - k0);   // a multiple of 8
        // A: one complex element of X per thread and step, consecutive threads on
        // consecutive addresses (along k for right products, along the row index for
        // left ones); its real part goes to row r, its imaginary part to row r + n.
        // Every load of a thread is issued before the first split, so the L2
        // latencies overlap (kTcPer >= n * kTcKC / blockDim.x).
        {
            cplx z[kTcPer];
            int offs[kTcPer];
#pragma unroll
            for (int q = 0; q < kTcPer; ++q) {
                const int e = tid + q * T;
                offs[q] = -1;
                z[q] = cmk(0.0, 0.0);
                if (e < n * kc) {
                    int r, kk;
                    if (right) {
                        r = e / kc;
                        kk = e - r * kc;
                    } else {
                        kk = e / n;
                        r = e - kk * n;
                    }
                    const int k = k0 + kk;
                    if (k < n) z[q] = right ? X[r * ld + k] : X[k * ld + r];
                    offs[q] = (kk >> 2) * (kTcMT * 4) + r * 4 + (kk & 3);
                }
            }
#pragma unroll
            for (int q = 0; q < kTcPer; ++q) {
                if (offs[q] < 0) continue;
                uint32_t hr, lr, hi_, li_;
                split_tf32(z[q].x, hr, lr);
                split_tf32(z[q].y, hi_, li_);
                b.ahi[offs[q]] = hr;
                b.alo[offs[q]] = lr;
                b.ahi[offs[q] + n * 4] = hi_;
                b.alo[offs[q] + n * 4] = li_;
            }
        }
        // B = (R - I) along the contiguous index: j for right products (R[k][j]), k for left ones
        {
            double v[kTcPer];
            int offs[kTcPer];
#pragma unroll
            for (int q = 0; q < kTcPer; ++q) {
                const int e = tid + q * T;
                offs[q] = -1;
                v[q] = 0.0;
                if (e < nb * kc) {
                    int j, kk;
                    if (right) {
                        kk = e / nb;
                        j = e - kk * nb;
                    } else {
                        j = e / kc;
                        kk = e - j * kc;
                    }
                    const int k = k0 + kk;
                    if (k < n && j < n) v[q] = (right ? R[k * ld + j] : R[j * ld + k]) - (j == k ? 1.0 : 0.0);
                    offs[q] = (kk >> 2) * (kTcNB * 4) + j * 4 + (kk & 3);
                }
            }
#pragma unroll
            for (int q = 0; q < kTcPer; ++q) {
                if (offs[q] < 0) continue;
                uint32_t hi, lo;
                split_tf32(v[q], hi, lo);
                b.bhi[offs[q]] = hi;
                b.blo[offs[q]] = lo;
            }
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0 && !wait_test) {
            tc_fence_after();
            for (int s = 0; s < kc / 8; ++s) {
#pragma unroll
                for (int p = 0; p < 3; ++p) {   // lo*hi, hi*lo, hi*hi
                    const uint32_t ab = (p == 0) ? a_lo : a_hi;
                    const uint32_t bb = (p == 1) ? b_lo : b_hi;
                    const uint64_t bd = tc_sdesc(bb + 2 * s * (kTcNB * 16), kTcNB * 16, 128);
                    const uint32_t acc = (k0 > 0 || s > 0 || p > 0) ? 1u : 0u;
                    for (int t = 0; t < mt; ++t) {
                        const uint64_t ad = tc_sdesc(ab + 2 * s * (kTcMT * 16) + t * (128 * 16), kTcMT * 16, 128);
                        tc_mma_tf32(b.tmem + (uint32_t)(t * nb), ad, bd, idesc, acc);
                    }
                }
            }
            tc_commit(mb);
        }
        // every thread waits: the staging buffers are reused by the next chunk
        const uint32_t ph = *phase;
        if (!mbar_wait(mb, ph, wait_test ? 1024 : kTcSpin)) ok = false;
        const bool all = __syncthreads_and(ok ? 1 : 0) != 0;
        if (tid == 0) *phase = ph ^ 1u;
        if (!all) {   // give the group in flight one more bounded wait, then stop
            if (!wait_test) {
                const bool done = mbar_wait(mb, ph);
                if (tid == 0 && !done) *pending = 2u + ph;
            }
            ok = false;
            break;
        }
    }
    tc_fence_after();
    if (ok) {
        const int w = tid >> 5, lane = tid & 31, q = w & 3, g = w >> 2, ng = T >> 7;
        const int cchunks = nb >> 4;
        double* Cd = reinterpret_cast<double*>(C);
        for (int it = g; it < mt * cchunks; it += ng) {
            const int t = it / cchunks, cc = it - t * cchunks;
            uint32_t r[16];
            tmem_ld16(b.tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(t * nb + 16 * cc), r);
            const int m = 128 * t + 32 * q + lane;
            if (m < 2 * n) {
                const int row = m < n ? m : m - n, part = m < n ? 0 : 1;
                double xv[16];
#pragma unroll
                for (int jj = 0; jj < 16; ++jj) {   // all 16 loads in flight before the adds
                    const int j = 16 * cc + jj;
                    const long idx = right ? (long)row * ld + j : (long)j * ld + row;
                    xv[jj] = j < n ? Cd[2 * idx + part] : 0.0;
                }
#pragma unroll
                for (int jj = 0; jj < 16; ++jj) {
                    const int j = 16 * cc + jj;
                    if (j < n) {
                        const long idx = right ? (long)row * ld + j : (long)j * ld + row;
                        Cd[2 * idx + part] = xv[jj] + (double)__uint_as_float(r[jj]);
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    return ok;
}

}  // namespace bq
