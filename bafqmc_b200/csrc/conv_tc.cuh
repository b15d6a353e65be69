// Periodic 3x3x3 convolutions of the proposer network on the tensor cores
// (tcgen05.mma kind::f16, bf16 operands, float32 accumulators in tensor
// memory), as an implicit GEMM: M = 128 output points, N = the layer's output
// channels (64, or 16 for the 4-channel output layer), K = 27 taps x the input
// channels (8 planes of 8, or 2 planes for the 2-channel input and the output
// layer's gradient).
//
// Tile: 4 consecutive sites x 32 consecutive time slices of one chain (M row
// m = 32 * segment + slice offset).  For each of the 9 spatial offsets (b, c)
// a stage holds, per segment s and 8-slice group g, the 10 rows t0 + 8g - 1 ..
// t0 + 8g + 8 of the neighbour site's column (all PIN channel planes), laid out
// [plane][row][16 bytes] (PIN * 160 bytes) at (4s + g) * PIN * 160.  One TMA
// copy brings a segment's four groups: the tensor map views the plane-major
// tensor as 5-D (channel in plane, row in group [10], plane, group [stride 8
// rows, overlapping the row dimension], site column), box 8 x 10 x PIN x 4 x 1.
// The three time offsets a of the stage are then the same rows read at a row
// offset 1 + a: a core matrix (8 rows x 16 bytes) starts at
// group + plane * 160 + (1 + a) * 16, so the A operand of tap (a, b, c) is the
// no-swizzle K-major layout with leading (K, next plane) offset 160 bytes and
// stride (M, next 8-row group) offset PIN * 160 bytes.  The stage's three taps
// of weights, [tap][plane][N rows][8], arrive by one bulk copy (K offset
// N * 16, N offset 128).
//
// Warp roles: warp 0 issues the copies (and owns the tensor memory), warp 1
// the MMAs, warps 2-5 the epilogue (warp w reads tensor-memory lanes
// 32 (w % 4) .. 32 (w % 4) + 31, i.e. rows of its lane quarter).  Stages are a
// ring with full / empty mbarriers; the accumulator is double buffered
// (2 x N columns), so a tile's epilogue overlaps the next tile's MMAs.
// Epilogues: bias + ReLU into 8 bf16 planes (hidden layers), bias into the
// float32 output [chain][t][site][4] (last layer), or the ReLU mask of the
// previous layer into 8 bf16 planes (gradient pass).  Every wait is bounded:
// on expiry the kernel records status 1 in *err, the other roles leave their
// loops, copies and MMAs in flight are drained with bounded waits, and the
// tensor memory is released.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

#include "net.h"
#include "tc.cuh"

namespace bq {

constexpr int kConvThreads = 192;
constexpr long long kConvSpin = 1LL << 22;
enum ConvTcMode { CTC_HIDDEN = 0, CTC_OUT = 1, CTC_BWD = 2 };

template <int PIN, int NOUT>
struct ConvTcCfg {
    static constexpr int kBoxBytes = PIN * 160;                      // 8 channels x 10 rows x PIN planes x 2 B
    static constexpr int kPitch = kBoxBytes;                         // one 8-row group; M stride of the operand
    static constexpr int kSeg = 4 * kPitch;                          // one TMA box: a segment's 4 row groups
    static constexpr int kA = 4 * kSeg;                              // 4 segments
    static constexpr int kTapB = PIN * NOUT * 16;                    // one tap's weights
    static constexpr int kB = 3 * kTapB;
    static constexpr int kStage = kA + kB;
    static constexpr int kTx = 16 * kBoxBytes + kB;                   // bytes the copies of a stage deliver
    static constexpr int kStages = (200 * 1024) / kStage < 8 ? (200 * 1024) / kStage : 8;
    static constexpr int kCols = 2 * NOUT < 32 ? 32 : 2 * NOUT;      // tensor-memory columns (power of 2)
    static constexpr size_t kSmem = (size_t)kStages * kStage + 1024;
    static_assert(kStage % 128 == 0 && kSeg % 128 == 0 && kStages >= 2, "stage layout (TMA boxes 128-byte aligned)");
    static_assert(NOUT == 16 || NOUT == 64, "N of the MMA");
    static_assert(PIN == 2 || PIN == 8, "input planes");
};

__host__ __device__ constexpr uint32_t tc_idesc_bf16(int M, int N) {
    // F32 accumulator (bits 4-5 = 1), A and B bf16 (bits 7-9, 10-12 = 1), K-major
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

struct ConvTcArgs {
    NetShape s;
    int chains;
    const __nv_bfloat16* wt;     // [27][PIN][NOUT][8] operand layout of this layer / direction
    const float* bias;           // forward: per output channel
    int nbias;                   // real output channels (bias entries)
    const __nv_bfloat16* mask;   // backward: the layer input (ReLU mask), 8 planes
    __nv_bfloat16* out;          // hidden / backward: 8 planes, plane-major with halos
    float* outf;                 // last layer: [chain][t][site][4]
    int* err;
    long long spin;   // poll bound of every wait
    int skip_mma;     // test hook: issue no MMA, so that the waits on them expire
};

namespace convtc {

DEVI bool wait_bounded(uint32_t mbar, uint32_t parity, volatile int* abort_flag, long long spin) {
    for (long long it = 0; it < spin; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 255) == 255 && *abort_flag) return false;
    }
    return false;
}
DEVI void arrive_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
DEVI void arrive(uint32_t mbar) { asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory"); }
DEVI void tma_load_5d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4, uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], "
        "[%7];" ::"r"(dst),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(mbar)
        : "memory");
}
DEVI void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"((uint64_t)src), "r"(bytes), "r"(mbar)
                 : "memory");
}
DEVI void mma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
// 32 consecutive float32 columns of the warp's 32 lanes
DEVI void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

DEVI int nbr_site(const NetShape& s, int site, int bc) {
    const int y = site / s.Lx, x = site - y * s.Lx;
    const int yn = (y + bc / 3 - 1 + s.Ly) % s.Ly, xn = (x + bc % 3 - 1 + s.Lx) % s.Lx;
    return yn * s.Lx + xn;
}

}  // namespace convtc

template <int PIN, int NOUT, int MODE>
__global__ void __launch_bounds__(kConvThreads, 1) conv_tc_kernel(const __grid_constant__ CUtensorMap amap, ConvTcArgs a) {
    using C = ConvTcCfg<PIN, NOUT>;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // 1024-byte aligned base for the stages
    uint8_t* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
    __shared__ uint64_t full[C::kStages], empty[C::kStages], tfull[2], tempty[2], drain;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;
    __shared__ float sbias[64];
    const NetShape& s = a.s;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles_t = s.L / 32, groups = s.Ns / 4;
    const int ntiles = a.chains * groups * tiles_t;

    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int i = 0; i < C::kStages; ++i) {
            mbar_init(smem_u32(&full[i]), 1);
            mbar_init(smem_u32(&empty[i]), 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(smem_u32(&tfull[i]), 1);
            mbar_init(smem_u32(&tempty[i]), 4);
        }
        mbar_init(smem_u32(&drain), 1);
    }
    if (threadIdx.x < 64)
        sbias[threadIdx.x] = (MODE != CTC_BWD && a.bias && (int)threadIdx.x < a.nbias) ? a.bias[threadIdx.x] : 0.f;
    if (warp == 0) tmem_alloc(smem_u32(&tmem_base), C::kCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;

    if (warp == 0) {
        // ---------------- producer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int issued = 0;
            for (int tile = blockIdx.x; tile < ntiles && !abort_flag; tile += gridDim.x) {
                const int tt = tile % tiles_t;
                const int rest = tile / tiles_t;
                const int sg = rest % groups, b = rest / groups;
                for (int bc = 0; bc < 9; ++bc) {
                    if (!convtc::wait_bounded(smem_u32(&empty[stage]), phase ^ 1u, &abort_flag, a.spin)) {
                        abort_flag = 1;
                        break;
                    }
                    const uint32_t fb = smem_u32(&full[stage]);
                    convtc::arrive_expect_tx(fb, C::kTx);
                    const uint32_t sa = smem_u32(smem + (size_t)stage * C::kStage);
                    for (int seg = 0; seg < 4; ++seg) {   // one box: the segment's 4 groups of 10 rows
                        const int col = b * s.Ns + convtc::nbr_site(s, 4 * sg + seg, bc);
                        convtc::tma_load_5d(sa + (uint32_t)(seg * C::kSeg), &amap, 0, 0, 0, tt * 4, col, fb);
                    }
                    convtc::bulk_load(sa + C::kA, a.wt + (size_t)bc * (C::kB / 2), C::kB, fb);
                    ++issued;
                    if (++stage == C::kStages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
            }
            // drain: every issued stage's copies complete before the block exits
            int st = stage;
            uint32_t ph = phase;
            for (int k = 0; k < min(issued, C::kStages); ++k) {
                if (--st < 0) {
                    st = C::kStages - 1;
                    ph ^= 1u;
                }
                volatile int never = 0;
                convtc::wait_bounded(smem_u32(&full[st]), ph, &never, a.spin);
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer
        if (lane == 0) {
            const uint32_t idesc = tc_idesc_bf16(128, NOUT);
            int stage = 0;
            uint32_t phase = 0;
            int acc = 0;
            uint32_t acc_phase = 0;
            for (int tile = blockIdx.x; tile < ntiles && !abort_flag; tile += gridDim.x) {
                if (!convtc::wait_bounded(smem_u32(&tempty[acc]), acc_phase ^ 1u, &abort_flag, a.spin)) {
                    abort_flag = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(acc * NOUT);
                bool ok = true;
                for (int bc = 0; bc < 9; ++bc) {
                    if (!convtc::wait_bounded(smem_u32(&full[stage]), phase, &abort_flag, a.spin)) {
                        abort_flag = 1;
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = smem_u32(smem + (size_t)stage * C::kStage);
                    const uint32_t sb = sa + C::kA;
                    for (int ta = 0; ta < 3 && !a.skip_mma; ++ta)
                        for (int kk = 0; kk < PIN / 2; ++kk) {
                            const uint64_t ad = tc_sdesc(sa + (uint32_t)(2 * kk * 160 + ta * 16), 160, C::kPitch);
                            const uint64_t bd =
                                tc_sdesc(sb + (uint32_t)(ta * C::kTapB + 2 * kk * NOUT * 16), NOUT * 16, 128);
                            convtc::mma_bf16(d, ad, bd, idesc, (bc | ta | kk) ? 1u : 0u);
                        }
                    if (!a.skip_mma) tc_commit(smem_u32(&empty[stage]));
                    if (++stage == C::kStages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                if (!ok) break;
                if (!a.skip_mma) tc_commit(smem_u32(&tfull[acc]));
                if (++acc == 2) {
                    acc = 0;
                    acc_phase ^= 1u;
                }
            }
            // every MMA issued by this thread has completed before the memory is released
            tc_commit(smem_u32(&drain));
            volatile int never = 0;
            if (!convtc::wait_bounded(smem_u32(&drain), 0, &never, a.spin)) atomicOr(a.err, 2);
        }
    } else {
        // ---------------- epilogue (warps 2-5)
        const int quarter = warp & 3;
        const int m = 32 * quarter + lane;
        const int seg = m >> 5, toff = m & 31;
        int acc = 0;
        uint32_t acc_phase = 0;
        for (int tile = blockIdx.x; tile < ntiles && !abort_flag; tile += gridDim.x) {
            const int tt = tile % tiles_t;
            const int rest = tile / tiles_t;
            const int sg = rest % groups, b = rest / groups;
            if (!convtc::wait_bounded(smem_u32(&tfull[acc]), acc_phase, &abort_flag, a.spin)) {
                abort_flag = 1;
                break;
            }
            tc_fence_after();
            const uint32_t taddr = tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(acc * NOUT);
            float v[NOUT];
            if constexpr (NOUT == 64) {
                float h[32];
                convtc::tmem_ld32(taddr, h);
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] = h[j];
                convtc::tmem_ld32(taddr + 32, h);
#pragma unroll
                for (int j = 0; j < 32; ++j) v[32 + j] = h[j];
            } else {
                uint32_t r[16];
                tmem_ld16(taddr, r);
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) convtc::arrive(smem_u32(&tempty[acc]));
            if (++acc == 2) {
                acc = 0;
                acc_phase ^= 1u;
            }
            const int site = 4 * sg + seg, t = tt * 32 + toff;
            if constexpr (MODE == CTC_OUT) {
                float4 o = make_float4(v[0] + sbias[0], v[1] + sbias[1], v[2] + sbias[2], v[3] + sbias[3]);
                *reinterpret_cast<float4*>(a.outf + (((long long)b * s.L + t) * s.Ns + site) * kNetOut) = o;
            } else {
                const long long rowbase = ((long long)b * s.Ns + site) * 8;   // plane 0 of the column
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    float f[8];
                    if constexpr (MODE == CTC_BWD) {
                        const uint4 mv =
                            *reinterpret_cast<const uint4*>(a.mask + ((rowbase + q) * (s.L + 2) + t + 1) * 8);
                        const __nv_bfloat162* mh = reinterpret_cast<const __nv_bfloat162*>(&mv);
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const float2 mm = __bfloat1622float2(mh[k]);
                            f[2 * k] = mm.x > 0.f ? v[8 * q + 2 * k] : 0.f;
                            f[2 * k + 1] = mm.y > 0.f ? v[8 * q + 2 * k + 1] : 0.f;
                        }
                    } else {
#pragma unroll
                        for (int k = 0; k < 8; ++k) f[k] = fmaxf(v[8 * q + k] + sbias[8 * q + k], 0.f);
                    }
                    uint4 o;
                    __nv_bfloat162* oh = reinterpret_cast<__nv_bfloat162*>(&o);
#pragma unroll
                    for (int k = 0; k < 4; ++k) oh[k] = __floats2bfloat162_rn(f[2 * k], f[2 * k + 1]);
                    __nv_bfloat16* col = a.out + (rowbase + q) * (s.L + 2) * 8;
                    *reinterpret_cast<uint4*>(col + (t + 1) * 8) = o;
                    if (t == 0) *reinterpret_cast<uint4*>(col + (s.L + 1) * 8) = o;
                    if (t == s.L - 1) *reinterpret_cast<uint4*>(col) = o;
                }
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && abort_flag) atomicOr(a.err, 1);
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, C::kCols);
}

}  // namespace bq
