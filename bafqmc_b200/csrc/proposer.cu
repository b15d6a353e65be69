// Learned global proposer: a 4-layer periodic 3x3x3 convolutional network
// over the (imaginary time x site) HS field of one lattice point, its training
// (Gaussian negative log-likelihood, Adam) and the exact Metropolis-Hastings
// move it proposes.  The reference has no such component; its only global
// move is the dead global_update.f90, whose accept rule (global_update.f90:
// 237-249) the move keeps with the Hastings term of a non-symmetric proposal.
//
// Network (the oracle's definition, oracle/proposer.py):
//   x0 = bf16(phi) (2 channels), x_l = bf16(relu(b_l + conv(x_{l-1}, W_l))) for
//   l = 1..3 (width channels), out = b_4 + conv(x_3, W_4) (mu_0, mu_1, lsig_0, lsig_1:
//   mean and log scale of the proposed field, whose displacement from phi is
//   the Gaussian mu - phi + exp(lsig) xi),
// with periodic neighbours in t, y and x, bf16 weights and float32 accumulation.
//
// Kernels here run on the CUDA cores and serve every layer shape; every layer
// of the forward pass and of the input-gradient pass also has a tensor-core
// path (conv_tc.cuh) for width 64, sites a multiple of 4 and L a multiple of 32.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/bafqmc_b200.h"
#include "conv_tc.cuh"
#include "net.h"
#include "sweep.cuh"

namespace bq {

NetShape make_net_shape(int Lx, int Ly, int L, int width) {
    NetShape s{};
    s.Lx = Lx;
    s.Ly = Ly;
    s.L = L;
    s.Ns = Lx * Ly;
    s.width = width;
    const int ci[kNetLayers] = {kNetIn, width, width, width};
    const int co[kNetLayers] = {width, width, width, kNetOut};
    long long off = 0;
    for (int l = 0; l < kNetLayers; ++l) {
        s.cin[l] = ci[l];
        s.cout[l] = co[l];
        // storage planes: a multiple of two (16 channels, one MMA K step)
        s.pin[l] = ((ci[l] + 15) / 16) * 2;
        s.pout[l] = ((co[l] + 15) / 16) * 2;
        s.woff[l] = off;
        off += (long long)kNetTaps * co[l] * ci[l];
        s.boff[l] = off;
        off += co[l];
    }
    s.nparams = off;
    return s;
}

namespace {

DEVI __nv_bfloat16* act_row(const NetShape& s, __nv_bfloat16* base, int planes, int b, int site, int q, int tp) {
    return base + ((((long long)b * s.Ns + site) * planes + q) * (s.L + 2) + tp) * 8;
}
DEVI const __nv_bfloat16* act_row(const NetShape& s, const __nv_bfloat16* base, int planes, int b, int site, int q,
                                  int tp) {
    return base + ((((long long)b * s.Ns + site) * planes + q) * (s.L + 2) + tp) * 8;
}
DEVI void unpack8(uint4 v, float (&f)[8]) {
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float2 t = __bfloat1622float2(h[k]);
        f[2 * k] = t.x;
        f[2 * k + 1] = t.y;
    }
}
DEVI uint4 pack8(const float (&f)[8]) {
    uint4 v;
    __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&v);
#pragma unroll
    for (int k = 0; k < 4; ++k) h[k] = __floats2bfloat162_rn(f[2 * k], f[2 * k + 1]);
    return v;
}
// the row of time slice t (0..L-1), and its halo copy when t is at an end
DEVI void store_row(const NetShape& s, __nv_bfloat16* base, int planes, int b, int site, int q, int t, uint4 v) {
    *reinterpret_cast<uint4*>(act_row(s, base, planes, b, site, q, t + 1)) = v;
    if (t == 0) *reinterpret_cast<uint4*>(act_row(s, base, planes, b, site, q, s.L + 1)) = v;
    if (t == s.L - 1) *reinterpret_cast<uint4*>(act_row(s, base, planes, b, site, q, 0)) = v;
}

// ---------------------------------------------------------------------------
// x0 from the fields: config b at src + off(b) (float64 ensemble fields or the
// float32 training set), [L][Ns][2] in the confin order
template <typename T>
__global__ void pack_kernel(NetShape s, const T* src, const ChainDev* chains, const int* idx, long long stride,
                            __nv_bfloat16* x0, int planes) {
    const int b = blockIdx.x;
    const long long off = chains ? chains[b].phi_off : (long long)(idx ? idx[b] : b) * stride;
    const T* phi = src + off;
    const int rows = s.Ns * s.L;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) {
        const int site = r / s.L, t = r - site * s.L;
        float f[8] = {(float)phi[((long long)t * s.Ns + site) * 2], (float)phi[((long long)t * s.Ns + site) * 2 + 1],
                      0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        store_row(s, x0, planes, b, site, 0, t, pack8(f));
        const float z[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        for (int q = 1; q < planes; ++q) store_row(s, x0, planes, b, site, q, t, pack8(z));
    }
}

// ---------------------------------------------------------------------------
// Reference convolution on the CUDA cores.  A block holds 32 consecutive time
// slices of one site of one chain; warp g produces channels g*JPT .. g*JPT+JPT-1.
//   FWD:  y[p][j] = bias[j] + sum_k sum_i x[nbr(p, +tap_k)][i] W[k][j][i]
//   BWD:  y[p][j] = (mask[p][j] > 0) sum_k sum_i g[nbr(p, -tap_k)][i] W[k][i][j]
// (BWD is the gradient w.r.t. the layer input, masked by the ReLU of the
// previous layer, whose output is `mask`).
enum ConvMode { CONV_HIDDEN = 0, CONV_OUT = 1, CONV_BWD = 2 };

struct ConvRefArgs {
    NetShape s;
    const __nv_bfloat16* in;
    int pin, ci;          // input planes, channels summed over
    __nv_bfloat16* outb;  // bf16 output (HIDDEN, BWD)
    int pout, co;         // output planes, channels produced
    float* outf;          // float32 output [b][t][site][4] (OUT)
    const float* wq;      // layer weights [27][layer cout][layer cin], bf16 values
    const float* bias;
    const __nv_bfloat16* mask;   // BWD: the layer's input activation (plane-major, pout planes)
    int mode;
};

template <int JPT>
__global__ void __launch_bounds__(128) conv_ref_kernel(ConvRefArgs a) {
    extern __shared__ float sW[];   // [ci][4 * JPT]
    const NetShape& s = a.s;
    const int tiles = (s.L + 31) / 32;
    const int blk = blockIdx.x;
    const int b = blk / (s.Ns * tiles);
    const int rem = blk - b * s.Ns * tiles;
    const int site = rem / tiles, tile = rem - site * tiles;
    const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
    const int t = tile * 32 + lane;
    const int y = site / s.Lx, x = site - y * s.Lx;
    const int cop = 4 * JPT;
    const int sgn = a.mode == CONV_BWD ? -1 : 1;
    float acc[JPT];
#pragma unroll
    for (int j = 0; j < JPT; ++j) acc[j] = 0.f;
    for (int k = 0; k < kNetTaps; ++k) {
        __syncthreads();
        for (int e = threadIdx.x; e < a.ci * cop; e += blockDim.x) {
            const int i = e / cop, j = e - i * cop;
            float w = 0.f;
            if (j < a.co)
                w = a.mode == CONV_BWD ? a.wq[((long long)k * a.ci + i) * a.co + j] : a.wq[((long long)k * a.co + j) * a.ci + i];
            sW[e] = w;
        }
        __syncthreads();
        if (t >= s.L) continue;
        const int tn = (t + sgn * tap_a(k) + s.L) % s.L;
        const int yn = (y + sgn * tap_b(k) + s.Ly) % s.Ly;
        const int xn = (x + sgn * tap_c(k) + s.Lx) % s.Lx;
        const int sn = yn * s.Lx + xn;
        for (int q = 0; q * 8 < a.ci; ++q) {
            float v[8];
            unpack8(*reinterpret_cast<const uint4*>(act_row(s, a.in, a.pin, b, sn, q, tn + 1)), v);
#pragma unroll
            for (int ii = 0; ii < 8; ++ii) {
                const int i = q * 8 + ii;
                if (i >= a.ci) break;
                const float* wr = sW + i * cop + g * JPT;
#pragma unroll
                for (int j = 0; j < JPT; ++j) acc[j] = fmaf(v[ii], wr[j], acc[j]);
            }
        }
    }
    if (t >= s.L) return;
    if (a.mode == CONV_OUT) {
#pragma unroll
        for (int j = 0; j < JPT; ++j) {
            const int jj = g * JPT + j;
            if (jj < a.co) a.outf[(((long long)b * s.L + t) * s.Ns + site) * kNetOut + jj] = acc[j] + a.bias[jj];
        }
        return;
    }
    if (JPT % 8 == 0) {
        for (int q8 = 0; q8 < JPT / 8; ++q8) {
            const int q = (g * JPT) / 8 + q8;
            if (q >= a.pout) break;   // a narrower layer stores fewer planes than 4 warps x JPT channels
            float f[8];
            float m[8];
            if (a.mode == CONV_BWD) unpack8(*reinterpret_cast<const uint4*>(act_row(s, a.mask, a.pout, b, site, q, t + 1)), m);
#pragma unroll
            for (int ii = 0; ii < 8; ++ii) {
                const int jj = q * 8 + ii;
                float v = acc[q8 * 8 + ii];
                if (a.mode == CONV_HIDDEN) v = fmaxf(v + a.bias[jj], 0.f);
                else v = m[ii] > 0.f ? v : 0.f;
                f[ii] = jj < a.co ? v : 0.f;
            }
            store_row(s, a.outb, a.pout, b, site, q, t, pack8(f));
        }
    }
}

// dW[k][o][i] += sum_p g[p][o] x[nbr(p, k)][i] over a chunk of points p
// (block (k, chunk)); thread (o = tid / 4, i0 = 16 * (tid % 4)).
struct WgradArgs {
    NetShape s;
    const __nv_bfloat16* x;   // layer input, pin planes
    int pin, cin;
    const __nv_bfloat16* g;   // gradient of the layer's pre-activation, pout planes
    int pout, cout;
    float* dw;                // [27][cout][cin]
    long long npts, per;      // points of the batch, points per chunk
};

__global__ void __launch_bounds__(256) wgrad_ref_kernel(WgradArgs a) {
    __shared__ float sg[32][65];
    __shared__ float sx[32][65];
    const NetShape& s = a.s;
    const int k = blockIdx.x;
    const long long p0 = (long long)blockIdx.y * a.per;
    const long long p1 = min(a.npts, p0 + a.per);
    const int o = threadIdx.x >> 2, i0 = (threadIdx.x & 3) * 16;
    float acc[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) acc[j] = 0.f;
    for (long long pb = p0; pb < p1; pb += 32) {
        // one 16-byte vector of g and of x per thread: point pb + tid / 8, plane tid % 8
        {
            const int pp = threadIdx.x >> 3, q = threadIdx.x & 7;
            const long long p = pb + pp;
            float fg[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, fx[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            if (p < p1) {
                const int t = (int)(p % s.L);
                const long long bs = p / s.L;
                const int site = (int)(bs % s.Ns), b = (int)(bs / s.Ns);
                if (q < a.pout) unpack8(*reinterpret_cast<const uint4*>(act_row(s, a.g, a.pout, b, site, q, t + 1)), fg);
                const int y = site / s.Lx, xx = site - y * s.Lx;
                const int tn = (t + tap_a(k) + s.L) % s.L;
                const int sn = ((y + tap_b(k) + s.Ly) % s.Ly) * s.Lx + (xx + tap_c(k) + s.Lx) % s.Lx;
                if (q < a.pin) unpack8(*reinterpret_cast<const uint4*>(act_row(s, a.x, a.pin, b, sn, q, tn + 1)), fx);
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                sg[pp][q * 8 + j] = fg[j];
                sx[pp][q * 8 + j] = fx[j];
            }
        }
        __syncthreads();
#pragma unroll 4
        for (int pp = 0; pp < 32; ++pp) {
            const float gv = sg[pp][o];
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[j] = fmaf(gv, sx[pp][i0 + j], acc[j]);
        }
        __syncthreads();
    }
    if (o >= a.cout) return;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const int i = i0 + j;
        if (i < a.cin) atomicAdd(a.dw + ((long long)k * a.cout + o) * a.cin + i, acc[j]);
    }
}

// db[o] += sum_p g[p][o] over a chunk of points
__global__ void bgrad_kernel(NetShape s, const __nv_bfloat16* g, int pout, int cout, float* db, long long npts,
                             long long per) {
    __shared__ float red[8][64];
    const long long p0 = (long long)blockIdx.x * per, p1 = min(npts, p0 + per);
    const int o = threadIdx.x & 63, lane8 = threadIdx.x >> 6;   // 4 point lanes x 64 channels
    float acc = 0.f;
    if (o < cout)
        for (long long p = p0 + lane8; p < p1; p += 4) {
            const int t = (int)(p % s.L);
            const long long bs = p / s.L;
            const int site = (int)(bs % s.Ns), b = (int)(bs / s.Ns);
            acc += __bfloat162float(act_row(s, g, pout, b, site, o >> 3, t + 1)[o & 7]);
        }
    red[lane8][o] = acc;
    __syncthreads();
    if (threadIdx.x < 64 && o < cout) atomicAdd(db + o, red[0][o] + red[1][o] + red[2][o] + red[3][o]);
}

// Loss of the pairs (input config pairs[b], target config pairs[B + b]) of the
// float32 set src: the Gaussian NLL of the target under N(mu, exp(lsig)^2) from
// the network at the input (in d_out), and the gradient of the output (bf16,
// plane-major, 2 planes).
__global__ void loss_kernel(NetShape s, const float* out, const float* src, const int* pairs, int B,
                            __nv_bfloat16* g4, double* loss, double inv_nf) {
    __shared__ double red[32];
    const int b = blockIdx.x;
    const long long cfg = (long long)s.L * s.Ns * 2;
    const float* tg = src + pairs[B + b] * cfg;
    double v[1] = {0.0};
    for (int r = threadIdx.x; r < s.L * s.Ns; r += blockDim.x) {
        const int t = r / s.Ns, site = r - t * s.Ns;
        const float* o = out + (((long long)b * s.L + t) * s.Ns + site) * kNetOut;
        float f[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        for (int a = 0; a < 2; ++a) {
            const double m = o[a], ls = o[2 + a];
            const double e = exp(-ls);
            const double z = ((double)tg[(long long)r * 2 + a] - m) * e;
            v[0] += 0.5 * z * z + ls;
            f[a] = (float)(-z * e * inv_nf);
            f[2 + a] = (float)((1.0 - z * z) * inv_nf);
        }
        store_row(s, g4, 2, b, site, 0, t, pack8(f));
        const float zf[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        store_row(s, g4, 2, b, site, 1, t, pack8(zf));
    }
    block_sum<1>(v, red);
    if (threadIdx.x == 0) atomicAdd(loss, v[0] * inv_nf);
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8) on the float32 master copy
__global__ void adam_kernel(float* p, const float* g, float* m, float* v, long long n, float lr, float c1, float c2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = 0.9f * m[i] + 0.1f * gi;
        const float vi = 0.999f * v[i] + 0.001f * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + 1e-8f);
    }
}

// bf16-rounded weights: float32 [27][cout][cin] for the CUDA-core kernels and
// the tensor-core operand layout [27][q][cout_pad][8] (K-major core matrices)
__global__ void requant_kernel(NetShape s, const float* p, float* wq, __nv_bfloat16* wt, int layer, long long wt_off,
                               int cpad) {
    const int ci = s.cin[layer], co = s.cout[layer];
    const long long n = (long long)kNetTaps * co * ci;
    const float* w = p + s.woff[layer];
    float* q = wq + s.woff[layer];
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        q[e] = __bfloat162float(__float2bfloat16_rn(w[e]));
    // operand layout, zero padded to cpad output rows and pin * 8 input channels
    const int qn = s.pin[layer];
    const long long nt = (long long)kNetTaps * qn * cpad * 8;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nt; e += (long long)gridDim.x * blockDim.x) {
        const int ii = (int)(e % 8);
        long long r = e / 8;
        const int o = (int)(r % cpad);
        r /= cpad;
        const int qq = (int)(r % qn);
        const int k = (int)(r / qn);
        const int i = qq * 8 + ii;
        const float val = (o < co && i < ci) ? w[((long long)k * co + o) * ci + i] : 0.f;
        wt[wt_off + e] = __float2bfloat16_rn(val);
    }
}

// Transposed weights for the gradient pass on the tensor cores: the layer's
// input channels become output rows and the taps are mirrored,
// Wb[k][q][i][8] = W[26 - k][o = 8q + .][i] (tap 26 - k is the negated offset).
__global__ void requant_bwd_kernel(NetShape s, const float* p, __nv_bfloat16* wt, int layer, long long wt_off, int cpad) {
    const int ci = s.cin[layer], co = s.cout[layer];
    const float* w = p + s.woff[layer];
    const int qn = s.pout[layer];   // K = the layer's output channels
    const long long nt = (long long)kNetTaps * qn * cpad * 8;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nt; e += (long long)gridDim.x * blockDim.x) {
        const int oo = (int)(e % 8);
        long long r = e / 8;
        const int i = (int)(r % cpad);
        r /= cpad;
        const int qq = (int)(r % qn);
        const int k = (int)(r / qn);
        const int o = qq * 8 + oo;
        const float val = (o < co && i < ci) ? w[((long long)(kNetTaps - 1 - k) * co + o) * ci + i] : 0.f;
        wt[wt_off + e] = __float2bfloat16_rn(val);
    }
}

// ---------------------------------------------------------------------------
// The move.  Proposal phi' = mu + exp(lsig) xi (mu, lsig: the network at phi)
// with xi from the chain's LCG (two draws per field in the field order, the
// Box-Muller cosine branch of fields.f90:280-288); lqf = log q(phi'|phi) =
// sum(-xi^2/2 - lsig).
__global__ void learned_propose_kernel(NetShape s, const float* out, KernelArgs ka, KernelArgs kp, double* lqf) {
    __shared__ double red[32];
    const int chain = blockIdx.x;
    const ChainDev cd = ka.chains[chain];
    ChainScalars* sc = ka.sc + chain;
    if (sc->status & 1) {   // quarantined: no draws, no proposal
        if (threadIdx.x == 0) lqf[chain] = 0.0;
        return;
    }
    const uint32_t seed0 = sc->seed;
    const int nf = s.L * s.Ns * 2;
    const uint32_t step = lcg_pow(2ull * blockDim.x);
    uint32_t sd = lcg_mul(lcg_pow(2ull * threadIdx.x + 1ull), seed0);
    double* prop = kp.phi + cd.phi_off;
    const float* o = out + (long long)chain * s.L * s.Ns * kNetOut;
    double v[1] = {0.0};
    for (int f = threadIdx.x; f < nf; f += blockDim.x) {
        const double u1 = lcg_u(sd);
        const double u2 = lcg_u(lcg_mul(kLcgA, sd));
        const double xi = sqrt(-2.0 * log(u1)) * cos(2.0 * 3.14159265358979323846 * u2);
        const double m = o[(f >> 1) * kNetOut + (f & 1)];
        const double ls = o[(f >> 1) * kNetOut + 2 + (f & 1)];
        prop[f] = m + exp(ls) * xi;
        v[0] += -0.5 * xi * xi - ls;
        sd = lcg_mul(step, sd);
    }
    block_sum<1>(v, red);
    if (threadIdx.x == 0) {
        lqf[chain] = v[0];
        sc->seed = lcg_mul(lcg_pow(2ull * nf), seed0);
        kp.sc[chain].status = 0;
    }
}

// hastings = log q(phi|phi') - log q(phi'|phi), out = the network at phi'
// (phi' enters log q(phi|phi') only through the network's output)
__global__ void learned_reverse_kernel(NetShape s, const float* out, KernelArgs ka, KernelArgs kp, const double* lqf,
                                       double* hastings) {
    __shared__ double red[32];
    const int chain = blockIdx.x;
    const ChainDev cd = ka.chains[chain];
    if (ka.sc[chain].status & 1) {
        if (threadIdx.x == 0) hastings[chain] = 0.0;
        return;
    }
    const int nf = s.L * s.Ns * 2;
    const double* phi = ka.phi + cd.phi_off;
    const float* o = out + (long long)chain * s.L * s.Ns * kNetOut;
    double v[1] = {0.0};
    for (int f = threadIdx.x; f < nf; f += blockDim.x) {
        const double m = o[(f >> 1) * kNetOut + (f & 1)];
        const double ls = o[(f >> 1) * kNetOut + 2 + (f & 1)];
        const double z = (phi[f] - m) * exp(-ls);
        v[0] += -0.5 * z * z - ls;
    }
    block_sum<1>(v, red);
    if (threadIdx.x == 0) hastings[chain] = v[0] - lqf[chain];
}

__global__ void pairs_kernel(int* pairs, int B, uint64_t seed, uint64_t counter, int chains, int slots, int lag) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (counter * (uint64_t)B + (uint64_t)b + 1ull);   // splitmix64
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const int c = (int)((z & 0xFFFFFFFFull) % (uint64_t)chains);
    const int t = (int)((z >> 32) % (uint64_t)(slots - lag));
    pairs[b] = t * chains + c;
    pairs[B + b] = (t + lag) * chains + c;
}

// training set slot `slot`: every chain's fields as float32, [chain][L][Ns][2]
__global__ void collect_kernel(KernelArgs ka, float* dst, long long per) {
    const int chain = blockIdx.x;
    const double* phi = ka.phi + ka.chains[chain].phi_off;
    float* d = dst + (long long)chain * per;
    for (long long k = threadIdx.x; k < per; k += blockDim.x) d[k] = (float)phi[k];
}

template <int JPT>
cudaError_t run_conv_ref(const ConvRefArgs& a, int chains, cudaStream_t st) {
    const int tiles = (a.s.L + 31) / 32;
    const size_t sm = sizeof(float) * a.ci * 4 * JPT;
    conv_ref_kernel<JPT><<<chains * a.s.Ns * tiles, 128, sm, st>>>(a);
    return cudaGetLastError();
}

}  // namespace

// ---------------------------------------------------------------------------
cudaError_t launch_pack_f64(bafqmc_net* n, const double* phi, int chains) {
    pack_kernel<double><<<chains, 256, 0, n->stream>>>(n->shape, phi, nullptr, nullptr,
                                                       (long long)n->shape.L * n->shape.Ns * 2, n->d_act[0],
                                                       n->shape.pin[0]);
    return cudaGetLastError();
}
cudaError_t launch_pack_chains(bafqmc_net* n, const KernelArgs& ka) {
    pack_kernel<double><<<ka.nchains, 256, 0, n->stream>>>(n->shape, ka.phi, ka.chains, nullptr, 0, n->d_act[0],
                                                           n->shape.pin[0]);
    return cudaGetLastError();
}
cudaError_t launch_pack_data(bafqmc_net* n, const float* src, const int* idx, int chains) {
    pack_kernel<float><<<chains, 256, 0, n->stream>>>(n->shape, src, nullptr, idx,
                                                      (long long)n->shape.L * n->shape.Ns * 2, n->d_act[0],
                                                      n->shape.pin[0]);
    return cudaGetLastError();
}

ConvRefArgs conv_args(bafqmc_net* n, int l, int mode) {
    const NetShape& s = n->shape;
    ConvRefArgs a{};
    a.s = s;
    a.wq = n->d_wq + s.woff[l];
    a.bias = n->d_params + s.boff[l];
    a.mode = mode;
    if (mode == CONV_BWD) {
        a.in = n->d_gact[l];
        a.pin = s.pout[l];
        a.ci = s.cout[l];
        a.outb = n->d_gact[l - 1];
        a.pout = s.pin[l];
        a.co = s.cin[l];
        a.mask = n->d_act[l];
    } else {
        a.in = n->d_act[l];
        a.pin = s.pin[l];
        a.ci = s.cin[l];
        a.co = s.cout[l];
        if (mode == CONV_OUT) a.outf = n->d_out;
        else {
            a.outb = n->d_act[l + 1];
            a.pout = s.pout[l];
        }
    }
    return a;
}

cudaError_t net_forward(bafqmc_net* n, int chains) {
    cudaError_t e = cudaSuccess;
    const NetShape& s = n->shape;
    for (int l = 0; l < kNetLayers && e == cudaSuccess; ++l) {
        const bool last = l == kNetLayers - 1;
        if (n->use_tc && conv_tc_applies(s, l, false))
            e = launch_conv_tc(n, l, false, chains);
        else if (last)
            e = run_conv_ref<1>(conv_args(n, l, CONV_OUT), chains, n->stream);
        else
            e = run_conv_ref<16>(conv_args(n, l, CONV_HIDDEN), chains, n->stream);
    }
    return e;
}

cudaError_t net_backward(bafqmc_net* n, int chains) {
    const NetShape& s = n->shape;
    cudaError_t e = cudaMemsetAsync(n->d_grad, 0, sizeof(float) * s.nparams, n->stream);
    const long long npts = (long long)chains * s.Ns * s.L;
    const int nchunk = (int)std::min<long long>(256, (npts + 2047) / 2048);
    const long long per = ((npts + nchunk - 1) / nchunk + 31) / 32 * 32;
    for (int l = kNetLayers - 1; l >= 0 && e == cudaSuccess; --l) {
        WgradArgs w{};
        w.s = s;
        w.x = n->d_act[l];
        w.pin = s.pin[l];
        w.cin = s.cin[l];
        w.g = n->d_gact[l];
        w.pout = s.pout[l];
        w.cout = s.cout[l];
        w.dw = n->d_grad + s.woff[l];
        w.npts = npts;
        w.per = per;
        wgrad_ref_kernel<<<dim3(kNetTaps, nchunk), 256, 0, n->stream>>>(w);
        e = cudaGetLastError();
        if (e != cudaSuccess) break;
        bgrad_kernel<<<nchunk, 256, 0, n->stream>>>(s, n->d_gact[l], s.pout[l], s.cout[l], n->d_grad + s.boff[l], npts,
                                                    per);
        e = cudaGetLastError();
        if (e != cudaSuccess || l == 0) break;
        if (n->use_tc && conv_tc_applies(s, l, true))
            e = launch_conv_tc(n, l, true, chains);
        else
            e = run_conv_ref<16>(conv_args(n, l, CONV_BWD), chains, n->stream);
    }
    return e;
}

// loss and gradient of `chains` pairs of the float32 configurations at src
// (d_pairs holds input and target indices); x0 must be packed from the inputs
cudaError_t net_loss_grad_src(bafqmc_net* n, int chains, const float* src) {
    const NetShape& s = n->shape;
    cudaError_t e = net_forward(n, chains);
    if (e == cudaSuccess) e = cudaMemsetAsync(n->d_loss, 0, sizeof(double), n->stream);
    if (e != cudaSuccess) return e;
    const double inv_nf = 1.0 / ((double)chains * s.L * s.Ns * 2);
    loss_kernel<<<chains, 256, 0, n->stream>>>(s, n->d_out, src, n->d_pairs, chains, n->d_gact[kNetLayers - 1], n->d_loss,
                                               inv_nf);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = net_backward(n, chains);
    return e;
}

cudaError_t net_adam(bafqmc_net* n, float lr) {
    n->adam_t += 1;
    const float c1 = 1.0f / (1.0f - powf(0.9f, (float)n->adam_t));
    const float c2 = 1.0f / (1.0f - powf(0.999f, (float)n->adam_t));
    adam_kernel<<<296, 256, 0, n->stream>>>(n->d_params, n->d_grad, n->d_adam_m, n->d_adam_v, n->shape.nparams, lr, c1,
                                            c2);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? net_requantize(n) : e;
}

cudaError_t net_requantize(bafqmc_net* n) {
    const NetShape& s = n->shape;
    for (int l = 0; l < kNetLayers; ++l) {
        const int cpad = s.pout[l] * 8;
        requant_kernel<<<148, 256, 0, n->stream>>>(s, n->d_params, n->d_wq, n->d_wt, l, n->wt_off[2 * l], cpad);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        requant_bwd_kernel<<<148, 256, 0, n->stream>>>(s, n->d_params, n->d_wt, l, n->wt_off[2 * l + 1], s.pin[l] * 8);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_pairs(bafqmc_net* n, int B, uint64_t seed, int lag) {
    pairs_kernel<<<(B + 127) / 128, 128, 0, n->stream>>>(n->d_pairs, B, seed, n->train_counter++, n->data_chains,
                                                          n->data_used, lag);
    return cudaGetLastError();
}

cudaError_t launch_collect(bafqmc_net* n, const KernelArgs& ka, int slot) {
    const long long per = (long long)n->shape.L * n->shape.Ns * 2;
    collect_kernel<<<ka.nchains, 256, 0, n->stream>>>(ka, n->d_data + (long long)slot * n->data_chains * per, per);
    return cudaGetLastError();
}

cudaError_t launch_learned_propose(bafqmc_net* n, const KernelArgs& ka, const KernelArgs& kp, double* lqf) {
    learned_propose_kernel<<<ka.nchains, 256, 0, n->stream>>>(n->shape, n->d_out, ka, kp, lqf);
    return cudaGetLastError();
}
cudaError_t launch_learned_reverse(bafqmc_net* n, const KernelArgs& ka, const KernelArgs& kp, const double* lqf,
                                   double* hastings) {
    learned_reverse_kernel<<<ka.nchains, 256, 0, n->stream>>>(n->shape, n->d_out, ka, kp, lqf, hastings);
    return cudaGetLastError();
}

}  // namespace bq

// ---------------------------------------------------------------------------
// tensor-core convolution: host side
namespace bq {

bool conv_tc_applies(const NetShape& s, int l, bool bwd) {
    if (s.width != 64 || s.Ns % 4 != 0 || s.L % 32 != 0) return false;
    return bwd ? l >= 1 : true;   // the first layer's input gradient is never needed
}

namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}
int sm_count(int device) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || v < 1) v = 148;
    return v;
}

template <int PIN, int NOUT, int MODE>
cudaError_t run_conv_tc(bafqmc_net* n, const CUtensorMap& map, const ConvTcArgs& a, int grid) {
    using C = ConvTcCfg<PIN, NOUT>;
    cudaError_t e = cudaFuncSetAttribute(conv_tc_kernel<PIN, NOUT, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)C::kSmem);
    if (e != cudaSuccess) return e;
    conv_tc_kernel<PIN, NOUT, MODE><<<grid, kConvThreads, C::kSmem, n->stream>>>(map, a);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_conv_tc(bafqmc_net* n, int l, bool bwd, int chains) {
    const NetShape& s = n->shape;
    if (!conv_tc_applies(s, l, bwd)) return cudaErrorInvalidValue;
    const __nv_bfloat16* A = bwd ? n->d_gact[l] : n->d_act[l];
    const int pin = bwd ? s.pout[l] : s.pin[l];   // planes of the A operand
    PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    // 5-D view of the plane-major tensor: (channel in plane, row in an 8-row group
    // [10: the group and its two halo rows], plane, group [stride 8 rows], site column)
    CUtensorMap map;
    const cuuint64_t dims[5] = {8, 10, (cuuint64_t)pin, (cuuint64_t)(s.L / 8), (cuuint64_t)chains * s.Ns};
    const cuuint64_t strides[4] = {16, (cuuint64_t)(s.L + 2) * 16, 8 * 16, (cuuint64_t)pin * (s.L + 2) * 16};
    const cuuint32_t box[5] = {8, 10, (cuuint32_t)pin, 4, 1};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    const CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<__nv_bfloat16*>(A), dims, strides,
                           box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    ConvTcArgs a{};
    a.s = s;
    a.chains = chains;
    a.wt = n->d_wt + n->wt_off[2 * l + (bwd ? 1 : 0)];
    a.bias = bwd ? nullptr : n->d_params + s.boff[l];
    a.nbias = s.cout[l];
    a.mask = bwd ? n->d_act[l] : nullptr;
    a.out = bwd ? n->d_gact[l - 1] : (l + 1 < kNetLayers ? n->d_act[l + 1] : nullptr);
    a.outf = n->d_out;
    a.err = n->d_err;
    a.spin = n->wait_test ? (1LL << 12) : kConvSpin;
    a.skip_mma = n->wait_test;
    const int ntiles = chains * (s.Ns / 4) * (s.L / 32);
    const int grid = std::min(ntiles, sm_count(n->device));
    if (!bwd && l == 0) return run_conv_tc<2, 64, CTC_HIDDEN>(n, map, a, grid);
    if (!bwd && l == kNetLayers - 1) return run_conv_tc<8, 16, CTC_OUT>(n, map, a, grid);
    if (!bwd) return run_conv_tc<8, 64, CTC_HIDDEN>(n, map, a, grid);
    if (l == kNetLayers - 1) return run_conv_tc<2, 64, CTC_BWD>(n, map, a, grid);
    return run_conv_tc<8, 64, CTC_BWD>(n, map, a, grid);
}

}  // namespace bq

// ---------------------------------------------------------------------------
// C ABI of the network (include/bafqmc_b200.h)
namespace {

#define NCK(call)                                                                                  \
    do {                                                                                           \
        cudaError_t _e = (call);                                                                   \
        if (_e != cudaSuccess)                                                                     \
            return bq::net_fail(BAFQMC_ECUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
    } while (0)

void free_bufs(bafqmc_net* n) {
    for (int l = 0; l < bq::kNetLayers; ++l) {
        if (n->d_act[l]) cudaFree(n->d_act[l]);
        if (n->d_gact[l]) cudaFree(n->d_gact[l]);
        n->d_act[l] = n->d_gact[l] = nullptr;
    }
    void* ps[] = {n->d_out, n->d_pairs};
    for (void* p : ps)
        if (p) cudaFree(p);
    n->d_out = nullptr;
    n->d_pairs = nullptr;
    n->cap = 0;
}

int check_status(bafqmc_net* n) {
    int st = 0;
    NCK(cudaMemcpyAsync(&st, n->d_err, sizeof(int), cudaMemcpyDeviceToHost, n->stream));
    NCK(cudaStreamSynchronize(n->stream));
    if (st) return bq::net_fail(BAFQMC_ETIMEOUT, "a bounded wait of the tensor-core convolution expired (status " +
                                                     std::to_string(st) + ")");
    return BAFQMC_OK;
}

int upload_configs(bafqmc_net* n, int count, const double* a, const double* b) {
    const long long per = (long long)n->shape.L * n->shape.Ns * 2;
    const long long need = per * count * (b ? 2 : 1);
    if (need > n->tin_cap) {
        if (n->d_tin) NCK(cudaFree(n->d_tin));
        n->d_tin = nullptr;
        NCK(cudaMalloc(&n->d_tin, sizeof(float) * need));
        n->tin_cap = need;
    }
    std::vector<float> h((size_t)need);
    for (long long k = 0; k < per * count; ++k) h[k] = (float)a[k];
    if (b)
        for (long long k = 0; k < per * count; ++k) h[per * count + k] = (float)b[k];
    NCK(cudaMemcpy(n->d_tin, h.data(), sizeof(float) * need, cudaMemcpyHostToDevice));
    return BAFQMC_OK;
}

}  // namespace

int bq::net_ensure_cap(bafqmc_net* n, int chains) {
    if (chains <= n->cap) return BAFQMC_OK;
    free_bufs(n);
    const NetShape& s = n->shape;
    for (int l = 0; l < kNetLayers; ++l) {
        const size_t a = sizeof(__nv_bfloat16) * (size_t)chains * act_chain_elems(s, s.pin[l]);
        const size_t g = sizeof(__nv_bfloat16) * (size_t)chains * act_chain_elems(s, s.pout[l]);
        NCK(cudaMalloc(&n->d_act[l], a));
        NCK(cudaMemsetAsync(n->d_act[l], 0, a, n->stream));
        NCK(cudaMalloc(&n->d_gact[l], g));
        NCK(cudaMemsetAsync(n->d_gact[l], 0, g, n->stream));
    }
    NCK(cudaMalloc(&n->d_out, sizeof(float) * (size_t)chains * s.L * s.Ns * kNetOut));
    NCK(cudaMalloc(&n->d_pairs, sizeof(int) * 2 * (size_t)chains));
    n->cap = chains;
    return BAFQMC_OK;
}

extern "C" {

int bafqmc_net_create(int Lx, int Ly, int Ltrot, int width, int device, bafqmc_net** out) {
    if (!out) return bq::net_fail(BAFQMC_EARG, "null output");
    *out = nullptr;
    if (Lx < 1 || Ly < 1 || Ltrot < 3) return bq::net_fail(BAFQMC_EARG, "lattice must be at least 1 x 1 x 3");
    if (width < 16 || width > bq::kNetMaxWidth || width % 16)
        return bq::net_fail(BAFQMC_EARG, "width must be 16, 32, 48 or 64");
    bafqmc_net* n = new bafqmc_net();
    n->device = device;
    n->shape = bq::make_net_shape(Lx, Ly, Ltrot, width);
    auto bail = [&](int rc) {
        bafqmc_net_destroy(n);
        return rc;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bail(bq::net_fail(BAFQMC_ECUDA, "cudaSetDevice"));
    if (cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(bq::net_fail(BAFQMC_ECUDA, "cudaStreamCreate"));
    const bq::NetShape& s = n->shape;
    const size_t np = sizeof(float) * (size_t)s.nparams;
    long long wt = 0;
    for (int l = 0; l < bq::kNetLayers; ++l) {
        n->wt_off[2 * l] = wt;
        wt += (long long)bq::kNetTaps * s.pin[l] * s.pout[l] * 8 * 8;
        n->wt_off[2 * l + 1] = wt;
        wt += (long long)bq::kNetTaps * s.pout[l] * s.pin[l] * 8 * 8;
    }
    float** bufs[] = {&n->d_params, &n->d_grad, &n->d_adam_m, &n->d_adam_v, &n->d_wq};
    for (float** b : bufs) {
        if (cudaMalloc(b, np) != cudaSuccess || cudaMemset(*b, 0, np) != cudaSuccess)
            return bail(bq::net_fail(BAFQMC_ECUDA, "cudaMalloc parameters"));
    }
    if (cudaMalloc(&n->d_wt, sizeof(__nv_bfloat16) * wt) != cudaSuccess ||
        cudaMemset(n->d_wt, 0, sizeof(__nv_bfloat16) * wt) != cudaSuccess ||
        cudaMalloc(&n->d_loss, sizeof(double)) != cudaSuccess || cudaMalloc(&n->d_err, sizeof(int)) != cudaSuccess ||
        cudaMemset(n->d_err, 0, sizeof(int)) != cudaSuccess)
        return bail(bq::net_fail(BAFQMC_ECUDA, "cudaMalloc network state"));
    n->use_tc = bq::conv_tc_applies(s, 1, false) ? 1 : 0;
    *out = n;
    return BAFQMC_OK;
}

void bafqmc_net_destroy(bafqmc_net* n) {
    if (!n) return;
    cudaSetDevice(n->device);
    if (n->stream) cudaStreamSynchronize(n->stream);
    free_bufs(n);
    void* ps[] = {n->d_params, n->d_grad, n->d_adam_m, n->d_adam_v, n->d_wq, n->d_wt, n->d_loss, n->d_losses,
                  n->d_tin, n->d_data, n->d_err, n->d_lqf, n->d_hastings};
    for (void* p : ps)
        if (p) cudaFree(p);
    if (n->stream) cudaStreamDestroy(n->stream);
    delete n;
}

long long bafqmc_net_num_params(const bafqmc_net* n) { return n ? n->shape.nparams : -1; }

int bafqmc_net_set_params(bafqmc_net* n, const float* params) {
    if (!n || !params) return bq::net_fail(BAFQMC_EARG, "null argument");
    NCK(cudaSetDevice(n->device));
    const size_t np = sizeof(float) * (size_t)n->shape.nparams;
    NCK(cudaMemcpyAsync(n->d_params, params, np, cudaMemcpyHostToDevice, n->stream));
    NCK(cudaMemsetAsync(n->d_adam_m, 0, np, n->stream));
    NCK(cudaMemsetAsync(n->d_adam_v, 0, np, n->stream));
    n->adam_t = 0;
    NCK(bq::net_requantize(n));
    NCK(cudaStreamSynchronize(n->stream));
    return BAFQMC_OK;
}

int bafqmc_net_get_params(bafqmc_net* n, float* params) {
    if (!n || !params) return bq::net_fail(BAFQMC_EARG, "null argument");
    NCK(cudaSetDevice(n->device));
    NCK(cudaMemcpyAsync(params, n->d_params, sizeof(float) * (size_t)n->shape.nparams, cudaMemcpyDeviceToHost,
                        n->stream));
    NCK(cudaStreamSynchronize(n->stream));
    return BAFQMC_OK;
}

int bafqmc_net_set_tensor_cores(bafqmc_net* n, int enable) {
    if (!n) return bq::net_fail(BAFQMC_EARG, "null network");
    if (enable && !bq::conv_tc_applies(n->shape, 1, false))
        return bq::net_fail(BAFQMC_EUNSUPPORTED,
                            "the tensor-core convolution needs width 64, sites a multiple of 4 and Ltrot a multiple of 32");
    n->use_tc = enable ? 1 : 0;
    return BAFQMC_OK;
}

int bafqmc_net_forward(bafqmc_net* n, int chains, const double* phi, float* out) {
    if (!n || !phi || !out || chains < 1) return bq::net_fail(BAFQMC_EARG, "bad forward arguments");
    NCK(cudaSetDevice(n->device));
    int rc = bq::net_ensure_cap(n, chains);
    if (rc != BAFQMC_OK) return rc;
    rc = upload_configs(n, chains, phi, nullptr);
    if (rc != BAFQMC_OK) return rc;
    NCK(bq::launch_pack_data(n, n->d_tin, nullptr, chains));
    NCK(bq::net_forward(n, chains));
    const bq::NetShape& s = n->shape;
    NCK(cudaMemcpyAsync(out, n->d_out, sizeof(float) * (size_t)chains * s.L * s.Ns * bq::kNetOut,
                        cudaMemcpyDeviceToHost, n->stream));
    return check_status(n);
}

int bafqmc_net_loss_grad(bafqmc_net* n, int chains, const double* phi, const double* target, double* loss,
                         float* grad) {
    if (!n || !phi || !target || chains < 1) return bq::net_fail(BAFQMC_EARG, "bad loss arguments");
    NCK(cudaSetDevice(n->device));
    int rc = bq::net_ensure_cap(n, chains);
    if (rc != BAFQMC_OK) return rc;
    rc = upload_configs(n, chains, phi, target);
    if (rc != BAFQMC_OK) return rc;
    std::vector<int> pairs(2 * (size_t)chains);
    for (int b = 0; b < chains; ++b) {
        pairs[b] = b;
        pairs[chains + b] = chains + b;
    }
    NCK(cudaMemcpy(n->d_pairs, pairs.data(), sizeof(int) * pairs.size(), cudaMemcpyHostToDevice));
    NCK(bq::launch_pack_data(n, n->d_tin, nullptr, chains));
    NCK(bq::net_loss_grad_src(n, chains, n->d_tin));
    if (loss) NCK(cudaMemcpyAsync(loss, n->d_loss, sizeof(double), cudaMemcpyDeviceToHost, n->stream));
    if (grad)
        NCK(cudaMemcpyAsync(grad, n->d_grad, sizeof(float) * (size_t)n->shape.nparams, cudaMemcpyDeviceToHost,
                            n->stream));
    return check_status(n);
}

int bafqmc_net_reserve_data(bafqmc_net* n, int chains, int slots) {
    if (!n || chains < 1 || slots < 2) return bq::net_fail(BAFQMC_EARG, "bad training-set size");
    NCK(cudaSetDevice(n->device));
    if (n->d_data) NCK(cudaFree(n->d_data));
    n->d_data = nullptr;
    const size_t bytes = sizeof(float) * (size_t)chains * slots * n->shape.L * n->shape.Ns * 2;
    NCK(cudaMalloc(&n->d_data, bytes));
    n->data_chains = chains;
    n->data_slots = slots;
    n->data_used = 0;
    return BAFQMC_OK;
}

int bafqmc_net_train(bafqmc_net* n, int steps, int batch, int lag, double lr, unsigned long long seed,
                     double* losses) {
    if (!n || steps < 1 || batch < 1 || lag < 1) return bq::net_fail(BAFQMC_EARG, "bad training arguments");
    if (n->data_used <= lag)
        return bq::net_fail(BAFQMC_ESTATE, "the training set holds " + std::to_string(n->data_used) +
                                               " collected sweeps, not more than the lag");
    NCK(cudaSetDevice(n->device));
    int rc = bq::net_ensure_cap(n, batch);
    if (rc != BAFQMC_OK) return rc;
    if (steps > n->losses_cap) {
        if (n->d_losses) NCK(cudaFree(n->d_losses));
        n->d_losses = nullptr;
        NCK(cudaMalloc(&n->d_losses, sizeof(double) * steps));
        n->losses_cap = steps;
    }
    for (int k = 0; k < steps; ++k) {
        NCK(bq::launch_pairs(n, batch, seed, lag));
        NCK(bq::launch_pack_data(n, n->d_data, n->d_pairs, batch));
        NCK(bq::net_loss_grad_src(n, batch, n->d_data));
        NCK(bq::net_adam(n, (float)lr));
        NCK(cudaMemcpyAsync(n->d_losses + k, n->d_loss, sizeof(double), cudaMemcpyDeviceToDevice, n->stream));
    }
    if (losses)
        NCK(cudaMemcpyAsync(losses, n->d_losses, sizeof(double) * steps, cudaMemcpyDeviceToHost, n->stream));
    return check_status(n);
}

int bafqmc_net_set_wait_test(bafqmc_net* n, int enable) {
    if (!n) return bq::net_fail(BAFQMC_EARG, "null network");
    NCK(cudaSetDevice(n->device));
    NCK(cudaStreamSynchronize(n->stream));
    n->wait_test = enable ? 1 : 0;
    NCK(cudaMemset(n->d_err, 0, sizeof(int)));   // a new test (or its end) starts from a clean status
    return BAFQMC_OK;
}

int bafqmc_net_time_layers(bafqmc_net* n, int chains, int reps, double* ms) {
    if (!n || !ms || chains < 1 || reps < 1) return bq::net_fail(BAFQMC_EARG, "bad timing arguments");
    NCK(cudaSetDevice(n->device));
    int rc = bq::net_ensure_cap(n, chains);
    if (rc != BAFQMC_OK) return rc;
    const bq::NetShape& s = n->shape;
    // inputs: whatever x0 holds (zeros or the last packed fields); the time does not depend on the values
    cudaEvent_t ev[bq::kNetLayers + 1];
    for (auto& e : ev) NCK(cudaEventCreate(&e));
    double acc[bq::kNetLayers] = {};
    for (int r = 0; r < reps + 1; ++r) {   // the first repetition warms up
        NCK(cudaEventRecord(ev[0], n->stream));
        for (int l = 0; l < bq::kNetLayers; ++l) {
            cudaError_t e;
            if (n->use_tc && bq::conv_tc_applies(s, l, false)) e = bq::launch_conv_tc(n, l, false, chains);
            else if (l == bq::kNetLayers - 1) e = bq::run_conv_ref<1>(bq::conv_args(n, l, bq::CONV_OUT), chains, n->stream);
            else e = bq::run_conv_ref<16>(bq::conv_args(n, l, bq::CONV_HIDDEN), chains, n->stream);
            NCK(e);
            NCK(cudaEventRecord(ev[l + 1], n->stream));
        }
        NCK(cudaEventSynchronize(ev[bq::kNetLayers]));
        if (r == 0) continue;
        for (int l = 0; l < bq::kNetLayers; ++l) {
            float t = 0.f;
            NCK(cudaEventElapsedTime(&t, ev[l], ev[l + 1]));
            acc[l] += t;
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    for (int l = 0; l < bq::kNetLayers; ++l) ms[l] = acc[l] / reps;
    return check_status(n);
}

int bafqmc_net_status(bafqmc_net* n, int* status) {
    if (!n || !status) return bq::net_fail(BAFQMC_EARG, "null argument");
    NCK(cudaSetDevice(n->device));
    NCK(cudaMemcpyAsync(status, n->d_err, sizeof(int), cudaMemcpyDeviceToHost, n->stream));
    NCK(cudaStreamSynchronize(n->stream));
    return BAFQMC_OK;
}

}  // extern "C"
