// Launch interface between the C-ABI host code and the sweep kernels.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace bq {

struct PointDev;
struct ChainDev;
struct ChainScalars;

struct KernelArgs {
    const PointDev* pts;
    const ChainDev* chains;
    int nchains;
    int obs_stride;
    double2* arena;
    double* phi;
    double* obs;
    ChainScalars* sc;
    int timers;   // nonzero: accumulate per-phase SM cycles into ChainScalars::cyc
    int mixed;    // nonzero: slice products of the N <= 144 class on the tensor cores (3xTF32)
    int traverse = 0;   // sweep_kernel: 0 both traversals, 1 the left one only, 2 the right one only
    // time-displaced pass (tau_kernel): per-CTA matrix regions, per-chain drift
    // statistics (kTauStats doubles), optional probe of the four functions at slice
    // tau_probe_nt (kTauProbeElems complex values per chain)
    double2* tau_ws = nullptr;
    double* tau_stats = nullptr;
    double2* tau_probe = nullptr;
    int tau_probe_nt = 0;
};

// time-displaced pass of chains with N <= kTauMaxN (the Nambu chains' {b, c^dagger}
// block; 2N x 2N inverse in the N <= 72 or N <= 144 routines).  Per chain: drift
// max of G(0,tau), G(tau,0), G(tau,tau), their sums, passes run, non-finite
// recomputations.
constexpr int kTauMaxN = 72;
constexpr int kTauStats = 8;
constexpr long long kTauProbeElems = 4LL * kTauMaxN * kTauMaxN;   // G(0,0), G(0,tau), G(tau,0), G(tau,tau)
long long tau_region_elems();   // complex values of one CTA's matrix region
// grid: CTAs (one per SM); each walks chains idx[k], k = blockIdx.x (mod grid)
cudaError_t launch_tau(const KernelArgs& ka, const int* idx, int count, int grid, cudaStream_t st);

// kernel classes of the fused sweep: size (N <= 16, N <= 36, N <= 72) + 3 * sector
// (0 number-conserving, 1 Nambu), and class 6: number-conserving N <= 144
constexpr int kNumClasses = 7;
int class_nmax(int cls);
size_t smem_bytes(int cls);
int class_of(int n, int pairing);   // -1 if no class holds n
long long class_work_elems(int cls); // complex values of HBM workspace per chain

cudaError_t upload_pow_table(const uint32_t* tab, int count);
cudaError_t launch_sweep(int cls, const KernelArgs& ka, const int* idx, int count, cudaStream_t st);
cudaError_t launch_pre(int cls, const KernelArgs& ka, const int* idx, int count, cudaStream_t st);
cudaError_t launch_warmup(const KernelArgs& ka, int nwarm, cudaStream_t st);
cudaError_t launch_bin_reset(const KernelArgs& ka, cudaStream_t st);
cudaError_t launch_bin_finish(const KernelArgs& ka, cudaStream_t st);
cudaError_t launch_point_average(const KernelArgs& ka, int npts, const int* start, const int* list, double* out,
                                 cudaStream_t st);
cudaError_t launch_field_norm(const KernelArgs& ka, double* out, cudaStream_t st);
cudaError_t launch_field_check(const KernelArgs& ka, int* bad, cudaStream_t st);   // bad[chain]: non-finite field
// global shift move: proposal into kp's state, then the exact decision (kp's pre run in between)
cudaError_t launch_global_propose(const KernelArgs& ka, const KernelArgs& kp, const double* shift, cudaStream_t st);
// hastings (optional): log q(phi|phi') - log q(phi'|phi) per chain of a non-symmetric proposal
cudaError_t launch_global_accept(const KernelArgs& ka, const KernelArgs& kp, const double* fn, const double* fn2,
                                 const double* hastings, int* accepted, cudaStream_t st);
// block statistics over n = npts * obs_stride values: accumulate one bin, finish blocks, final mean / sem
cudaError_t launch_stats_add(const double* pout, double* cur, double* blk, int n, int finish, int block_size,
                             cudaStream_t st);
cudaError_t launch_stats_final(const double* blk, int nb, int n, double* mean, double* sem, cudaStream_t st);

// pole diagnostics of the number-conserving chains' G: per chain kPoleScalars
// doubles (pole_distance, pole_x, spectral radius, largest singular value,
// status) at sout, the poles 1/lambda at zout (zstride complex per chain);
// nmax bounds N over those chains
// above kPoleSmemMaxN the matrix lives in hmat: pole_hbm_elems(nmax) complex
// values per chain
constexpr int kPoleScalars = 5;
constexpr int kPoleSmemMaxN = 112;
long long pole_hbm_elems(int nmax);
cudaError_t launch_pole(const KernelArgs& ka, int nmax, int zstride, double* zout, double* sout, double2* hmat,
                        cudaStream_t st);

}  // namespace bq
