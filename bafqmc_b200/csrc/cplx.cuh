// Complex FP64 helpers and CTA-level reductions for the BAFQMC sweep kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define DEVI __device__ __forceinline__

typedef double2 cplx;

DEVI cplx cmk(double r, double i) { return make_double2(r, i); }
DEVI cplx cadd(cplx a, cplx b) { return cmk(a.x + b.x, a.y + b.y); }
DEVI cplx csub(cplx a, cplx b) { return cmk(a.x - b.x, a.y - b.y); }
DEVI cplx cmul(cplx a, cplx b) { return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
// a * conj(b)
DEVI cplx cmulcj(cplx a, cplx b) { return cmk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); }
DEVI cplx cconj(cplx a) { return cmk(a.x, -a.y); }
DEVI cplx cscale(cplx a, double s) { return cmk(a.x * s, a.y * s); }
// acc + a*b
DEVI cplx cfma(cplx a, cplx b, cplx acc) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
    return acc;
}
// acc + conj(a)*b
DEVI cplx cfmacj(cplx a, cplx b, cplx acc) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(-a.y, b.x, acc.y);
    return acc;
}
DEVI double cabs2(cplx a) { return a.x * a.x + a.y * a.y; }
DEVI double cabsv(cplx a) { return hypot(a.x, a.y); }
// Smith's algorithm for a / b.
DEVI cplx cdiv(cplx a, cplx b) {
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, den = b.x + b.y * r;
        return cmk((a.x + a.y * r) / den, (a.y - a.x * r) / den);
    } else {
        double r = b.x / b.y, den = b.y + b.x * r;
        return cmk((a.x * r + a.y) / den, (a.y * r - a.x) / den);
    }
}
// exp(z) for complex z
DEVI cplx cexpz(cplx z) {
    double s, c;
    sincos(z.y, &s, &c);
    double e = exp(z.x);
    return cmk(e * c, e * s);
}

DEVI double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of NV values; result valid in every thread. scratch holds
// NV * (blockDim.x/32) doubles. Contains two __syncthreads.
template <int NV>
DEVI void block_sum(double (&v)[NV], double* scratch) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) scratch[k * nw + wid] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double s = 0.0;
        for (int w = 0; w < nw; ++w) s += scratch[k * nw + w];
        v[k] = s;
    }
    __syncthreads();
}
