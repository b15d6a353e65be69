// Learned global proposer: the convolutional network over the (imaginary time
// x site) HS field of one lattice point, its training state, and the launch
// interface shared by proposer.cu (kernels, the network's C ABI) and capi.cu
// (the move on an ensemble).
//
// Activation layout ("plane-major"): a tensor of C channels (C a multiple of
// 8) for B chains of Ns sites and L slices is
//     act[b][site][q][tp][8]   bf16,  q = channel / 8,  tp = t + 1 in [0, L + 2)
// so each group of 8 channels of one site is a column of L + 2 rows of 16
// bytes along imaginary time, with halo rows tp = 0 (a copy of t = L - 1) and
// tp = L + 1 (a copy of t = 0) that make the periodic neighbours t +- 1 plain
// row offsets.  This is the operand layout of the tensor-core convolution: a
// box of 8 channels x 10 rows x all planes is one TMA copy, and a core matrix
// of the MMA (8 rows x 16 bytes) is contiguous at every row offset.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "kernels.h"

namespace bq {

constexpr int kNetTaps = 27;
constexpr int kNetLayers = 4;
constexpr int kNetIn = 2;    // channels in: the two auxiliary fields
constexpr int kNetOut = 4;   // channels out: m_0, m_1, lsig_0, lsig_1
constexpr int kNetMaxWidth = 64;

// tap k = 3 * ((b + 1) * 3 + (c + 1)) + (a + 1): offsets (a, b, c) in (t, y, x)
__host__ __device__ inline int tap_a(int k) { return k % 3 - 1; }
__host__ __device__ inline int tap_b(int k) { return (k / 3) / 3 - 1; }
__host__ __device__ inline int tap_c(int k) { return (k / 3) % 3 - 1; }

struct NetShape {
    int Lx, Ly, L, Ns;   // Ns = Lx * Ly
    int width;
    int cin[kNetLayers], cout[kNetLayers];
    int pin[kNetLayers], pout[kNetLayers];   // storage planes of each layer's input / output
    long long woff[kNetLayers], boff[kNetLayers];   // offsets into the flat parameter vector
    long long nparams;
};

NetShape make_net_shape(int Lx, int Ly, int L, int width);

// rows (sites x (L + 2)) x 8 bf16 per plane and chain
inline long long act_chain_elems(const NetShape& s, int planes) {
    return (long long)s.Ns * planes * (s.L + 2) * 8;
}

}  // namespace bq

// The network's device state (opaque to C callers: include/bafqmc_b200.h).
struct bafqmc_net {
    int device = 0;
    cudaStream_t stream = nullptr;
    bq::NetShape shape{};
    int cap = 0;   // chains the activation buffers hold
    float* d_params = nullptr;   // float32 master copy (flat, the oracle's layout)
    float* d_grad = nullptr;
    float* d_adam_m = nullptr;
    float* d_adam_v = nullptr;
    float* d_wq = nullptr;       // bf16-rounded weights as float32, [27][cout][cin] per layer
    // bf16 weights in the tensor-core operand layout [27][q][rows][8]: per
    // layer the forward form (rows = output channels) at wt_off[2l] and the
    // mirrored, transposed form of the gradient pass at wt_off[2l + 1]
    __nv_bfloat16* d_wt = nullptr;
    long long wt_off[2 * bq::kNetLayers] = {};
    long long adam_t = 0;
    __nv_bfloat16* d_act[bq::kNetLayers] = {};   // x0 (input) .. x3
    __nv_bfloat16* d_gact[bq::kNetLayers] = {};  // gradients of the pre-activations of layers 1 .. 4 (index l - 1)
    float* d_out = nullptr;      // [cap][L][Ns][4] network output
    double* d_loss = nullptr;
    double* d_losses = nullptr;  // per training step
    int losses_cap = 0;
    float* d_tin = nullptr;      // host-supplied configurations (float32) of the test entry points
    long long tin_cap = 0;
    // training set: configurations of the plain sampler, float32 [slot][chain][L][Ns][2]
    float* d_data = nullptr;
    int data_chains = 0, data_slots = 0, data_used = 0;
    int* d_pairs = nullptr;      // [2 * cap] (input, target) configuration indices of a training batch
    uint64_t train_counter = 0;
    int use_tc = 1;              // convolutions on the tensor cores (where conv_tc_applies)
    int* d_err = nullptr;        // status of the tensor-core kernels (bounded waits that expired)
    int wait_test = 0;           // bafqmc_net_set_wait_test: MMAs skipped, short wait bound
    // proposal bookkeeping of the move: log q(phi'|phi) and the Hastings term per chain
    double* d_lqf = nullptr;
    double* d_hastings = nullptr;
    int move_cap = 0;
};

namespace bq {

int net_fail(int code, const std::string& msg);   // sets bafqmc_last_error's message
int net_ensure_cap(bafqmc_net* n, int chains);     // activation buffers for `chains`

// input pack into x0 (plane-major bf16 with halos) from fields in the confin
// order: `chains` configurations back to back (float64), the chains of an
// ensemble (ka.phi + ka.chains[c].phi_off), or configurations idx[] of a
// float32 set
cudaError_t launch_pack_f64(bafqmc_net* n, const double* phi, int chains);
cudaError_t launch_pack_chains(bafqmc_net* n, const KernelArgs& ka);
cudaError_t launch_pack_data(bafqmc_net* n, const float* src, const int* idx, int chains);
// forward pass of `chains` chains from x0 to d_out
cudaError_t net_forward(bafqmc_net* n, int chains);
// parameter gradient into d_grad from the gradient of the output in d_gact[3]
cudaError_t net_backward(bafqmc_net* n, int chains);
// forward, loss (into d_loss) and gradient for the pairs d_pairs of the
// float32 configurations at src; x0 must hold the packed inputs
cudaError_t net_loss_grad_src(bafqmc_net* n, int chains, const float* src);
cudaError_t net_adam(bafqmc_net* n, float lr);
cudaError_t net_requantize(bafqmc_net* n);
// B random (input, target) pairs `lag` collected sweeps apart into d_pairs
cudaError_t launch_pairs(bafqmc_net* n, int B, uint64_t seed, int lag);
// copy every chain's fields of ka into training-set slot `slot`
cudaError_t launch_collect(bafqmc_net* n, const KernelArgs& ka, int slot);
// tensor-core convolution of layer l (forward, or the gradient pass if bwd)
cudaError_t launch_conv_tc(bafqmc_net* n, int l, bool bwd, int chains);
bool conv_tc_applies(const NetShape& s, int l, bool bwd);

// the move on an ensemble: propose from ka's fields into kp's (seed advanced in ka),
// then, after the forward pass at the proposal, the Hastings term
cudaError_t launch_learned_propose(bafqmc_net* n, const KernelArgs& ka, const KernelArgs& kp, double* lqf);
cudaError_t launch_learned_reverse(bafqmc_net* n, const KernelArgs& ka, const KernelArgs& kp, const double* lqf,
                                   double* hastings);

}  // namespace bq
