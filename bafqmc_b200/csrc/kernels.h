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
};

// size classes of the fused sweep kernel: 0 -> N <= 16, 1 -> N <= 36
constexpr int kNumClasses = 2;
int class_nmax(int cls);
size_t smem_bytes(int cls);

cudaError_t upload_pow_table(const uint32_t* tab, int count);
cudaError_t launch_sweep(int cls, const KernelArgs& ka, const int* idx, int count, cudaStream_t st);
cudaError_t launch_pre(int cls, const KernelArgs& ka, const int* idx, int count, cudaStream_t st);
cudaError_t launch_warmup(const KernelArgs& ka, int nwarm, cudaStream_t st);
cudaError_t launch_bin_reset(const KernelArgs& ka, cudaStream_t st);
cudaError_t launch_bin_finish(const KernelArgs& ka, cudaStream_t st);
cudaError_t launch_point_average(const KernelArgs& ka, int npts, const int* start, const int* list, double* out,
                                 cudaStream_t st);
cudaError_t launch_field_norm(const KernelArgs& ka, double* out, cudaStream_t st);

}  // namespace bq
