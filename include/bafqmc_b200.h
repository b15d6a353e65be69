/*
 * bafqmc_b200.h -- C ABI of the B200 implementation of the BAFQMC
 * finite-temperature auxiliary-field sweep (number-conserving solver and
 * Nambu pairing solver).
 *
 * The reference exposes this path as a process/file contract: a driver writes
 * paramC_sets.txt, confin.txt and seeds.txt into a run directory and launches
 * `mpirun -np N build/bosonDQMC.out` (src/number_conserving/run_paper.py:113,162;
 * the pairing program src/pairing/src/main.f90 likewise), one Markov chain per
 * MPI rank.  Each entry point below replaces one step of that program
 * (src/number_conserving/src/main.f90:22-85, src/pairing/src/main.f90:19-83);
 * the comment names the reference routine it stands in for.  A "chain" here is
 * one MPI rank of the reference; a "point" is one paramC_sets.txt parameter
 * set.  One handle may mix points of both sectors and of several sizes.
 *
 * Conventions
 *   - Every function returns 0 on success or a negative BAFQMC_E* code;
 *     bafqmc_last_error() gives a message for the calling thread.
 *   - Host buffers are caller-owned; device memory belongs to the handle.
 *   - A handle owns one CUDA stream; calls are asynchronous on that stream
 *     unless they return host data.  A handle is not thread-safe.
 *   - Complex matrices are row-major, element (i,j) = <b_i b_j^dagger>,
 *     stored as interleaved (re, im) doubles.
 *   - Fields are stored per chain as phi[nt][site][aux] (aux fastest), the
 *     order of confin.txt / confout.txt (fields.f90:81-103, 265-273).
 */
#ifndef BAFQMC_B200_H
#define BAFQMC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BAFQMC_OK 0
#define BAFQMC_EARG (-1)        /* invalid argument (calc_basic.f90:61-62,103 `stop`) */
#define BAFQMC_ECUDA (-2)       /* CUDA runtime error */
#define BAFQMC_EUNSUPPORTED (-3)/* size or sector not built in this library */
#define BAFQMC_ESTATE (-4)      /* call out of order (e.g. sweep before pre) */
#define BAFQMC_ENUMERIC (-5)    /* non-finite Green's function detected */
#define BAFQMC_ETIMEOUT (-6)    /* a bounded device-side wait expired (the call's results are not valid) */

/* Number of scalar observable slots per chain before the site densities. */
#define BAFQMC_OBS_SCALARS 32

/* One parameter point: the seven lines of paramC_sets.txt
 * (calc_basic.f90:52-59) plus the sector.  `delta` is the pairing amplitude
 * RDelta of the Nambu solver (src/pairing/src/calc_basic.f90:51) and must be
 * 0 for sector 0.  t is fixed to 1 as in the reference (calc_basic.f90:94). */
typedef struct bafqmc_point {
    int sector;              /* 0 = number-conserving (Ndim = Lx*Ly); 1 = Nambu pairing (stored block 2*Lx*Ly) */
    int Lx, Ly, Ltrot;
    double beta, U1, U2, mu, delta;
    int Nwrap;
    double shiftLoc;
    int iniType;             /* 1 uniform, 2 Gaussian, 3 |Gaussian| (fields.f90:115-154) */
    double iniAmpl, iniBias1, iniBias2;
    int LxTherm, LyTherm, LtrotTherm;   /* size of the seeded/confin field, tiled (fields.f90:156-234) */
} bafqmc_point;

typedef struct bafqmc_handle bafqmc_handle;

/* Model_init + Prop%make + WrList%make + Stabilize_init (model.f90:14-39,
 * main.f90:28-34): lattice tables, e^{-+dtau K}, HS factors and device state
 * for `nchains` chains, chain c using point chain_point[c]. */
int bafqmc_create(const bafqmc_point* pts, int npts, const int32_t* chain_point, int nchains, int device,
                  bafqmc_handle** out);
void bafqmc_destroy(bafqmc_handle* h);

/* Kernel classes and their autotuner (no counterpart in the reference).  A
 * kernel class is one tile configuration of the sweep kernels: threads per
 * CTA, CTAs per SM, GEMM micro-tile, register layout of the factorisations and
 * where the workspaces live.  Classes 0-2 hold Ndim <= 16 / 36 / 72
 * (number-conserving), 3-5 the same sizes for Nambu points, 6 number-
 * conserving Ndim <= 144.  bafqmc_create gives every point the smallest class
 * that holds it.  bafqmc_autotune times one sweep of trial_chains chains (0:
 * four per SM) of each distinct (Ndim, sector) among pts in every class that
 * can hold it, on scratch handles (nothing of a later run is touched), and
 * writes the fastest class per point to classes[npts]; ms_per_chain_sweep
 * (optional, [npts][7]) receives the measured time per chain-sweep of each
 * candidate (NaN where a class does not apply).  bafqmc_create_tuned takes
 * such a table (or -1 per point for the default). */
#define BAFQMC_NUM_CLASSES 7
int bafqmc_autotune(const bafqmc_point* pts, int npts, int device, int trial_chains, int* classes,
                    double* ms_per_chain_sweep);
int bafqmc_create_tuned(const bafqmc_point* pts, int npts, const int32_t* chain_point, int nchains, int device,
                        const int* classes, bafqmc_handle** out);
const char* bafqmc_last_error(void);

/* Sizes: dimension of a point's stored Green's function (Lx*Ly, or 2*Lx*Ly
 * for a Nambu point), and the per-chain observable stride. */
int bafqmc_point_dim(const bafqmc_handle* h, int point, int* ndim, int* lq, int* ltrot, int* nst);
int bafqmc_obs_stride(const bafqmc_handle* h);
int bafqmc_num_chains(const bafqmc_handle* h);

/* conf_set + conf_transfer (fields.f90:115-234): fields of each chain
 * ([Ltrot][Lx*Ly][2] doubles in both sectors) from its
 * seed (seeds.txt row), the seed advanced past the draws as in conf_therm_in. */
int bafqmc_fields_from_seeds(bafqmc_handle* h, const int32_t* seeds);

/* confin path of conf_therm_in (fields.f90:81-103): explicit seed and field
 * (already of the full Ltrot x Ns size) per chain.  get_state is conf_out's
 * payload (fields.f90:236-278).  Setting a state clears every chain's counters
 * and status; a NaN or infinite field value returns BAFQMC_EARG naming the
 * chain (and leaves the handle without fields). */
int bafqmc_set_state(bafqmc_handle* h, const int32_t* seeds, const double* phi);
int bafqmc_get_state(bafqmc_handle* h, int32_t* seeds, double* phi);

/* Local_sweep_therm x nwarm (local_sweep.f90:64-78): prior-only warm-up. */
int bafqmc_warmup_prior(bafqmc_handle* h, int nwarm);

/* Local_sweep_pre (local_sweep.f90:80-94): right UDV slots and G(beta). */
int bafqmc_pre(bafqmc_handle* h);

/* One measurement bin: Local_sweep%sweep (local_sweep.f90:136-161) with
 * nsweep left+right sweeps, then Obs_equal_ave and the acceptance ratio.
 * The bin's launches (accumulator reset, one persistent sweep launch per
 * kernel class and sweep, bin averages) are captured into a CUDA graph on the
 * first call and replayed by later calls with the same nsweep and timer
 * setting. */
int bafqmc_sweep(bafqmc_handle* h, int nsweep);

/* Observables of the last bin.  chain_obs: [nchains][stride] (per chain, the
 * values each rank holds before MPI_REDUCE); point_obs: [npts][stride], the
 * chain average that m_process_obs_equal writes (fourier_trans.f90:350-457).
 * Layout: BAFQMC_OBS_SCALARS slots (see bafqmc_b200/observables.py) then Lq
 * site densities. */
int bafqmc_bin_chain_obs(bafqmc_handle* h, double* chain_obs);
int bafqmc_bin_point_obs(bafqmc_handle* h, double* point_obs);

/* On-device block statistics of the per-bin chain averages.  The reference's
 * solver has none; its analysis scripts block the appended per-bin files
 * (benchmarks/paper/analysis.py:52-64).  After bafqmc_stats_reset, every bin's
 * point averages (the values bafqmc_bin_point_obs returns) are summed in bin
 * order into blocks of block_size bins, up to max_blocks blocks.  bafqmc_stats
 * writes, per point and slot ([npts][stride]), the mean of the completed block
 * means and its standard error sqrt(sum_b (m_b - mean)^2 / (nb - 1) / nb), each
 * sum taken in order as the analysis script does; nblocks receives nb.  Bins
 * of an unfinished block are not counted. */
int bafqmc_stats_reset(bafqmc_handle* h, int block_size, int max_blocks);
int bafqmc_stats(bafqmc_handle* h, double* mean, double* sem, int* nblocks);

/* Prop%Gr of one chain (row-major complex, ndim x ndim as bafqmc_point_dim
 * reports).  For a Nambu chain this is the {b, c^dagger} block of the
 * reference's 4Ns Green's function, rows/columns b_1..b_Ns, c^dagger_1..
 * c^dagger_Ns; the full matrix in the sector order b, c, b^dagger, c^dagger
 * (src/pairing/src/lattice.f90:26-35) has this block on {b, c^dagger}, its
 * complex conjugate on {c, b^dagger} and zeros elsewhere. */
int bafqmc_get_green(bafqmc_handle* h, int chain, double* G);

/* log_weight = -1/2 sum phi^2 + 2 log|det G| per chain
 * (pole_diagnostics.f90:119; log|det G| from the last stabilised
 * (I - B(beta,0)) factorisation).  The pairing program has no such output:
 * NaN for Nambu chains. */
int bafqmc_log_weight(bafqmc_handle* h, double* out);

/* PoleDiagnostics (pole_diagnostics.f90:91-123) of each number-conserving
 * chain's current G, computed on the device.
 *   z        optional, [nchains][zstride][2] doubles: the Ndim poles
 *            z = 1/lambda over the eigenvalues lambda of G (1/tiny where
 *            |lambda| <= tiny), the chain's row of the pole_z file; zstride >=
 *            Ndim of every number-conserving chain.  Eigenvalues come in the
 *            order of the diagonal of this library's Schur form, which need
 *            not be ZGEEV's order.
 *   scalars  [nchains][BAFQMC_POLE_SCALARS]: pole_distance, pole_x,
 *            green_spectral_radius, green_smax, log_weight (the five
 *            one-column files).
 * Nambu chains (the pairing program writes no pole files) and quarantined
 * chains (status bit 0, see bafqmc_counters) get NaN.  Returns
 * BAFQMC_ENUMERIC if a chain's eigenvalue iteration did not converge (the
 * reference stops on ZGEEV info != 0, pole_diagnostics.f90:41-46). */
#define BAFQMC_POLE_SCALARS 5
int bafqmc_pole_diagnostics(bafqmc_handle* h, double* z, int zstride, double* scalars);

/* Global moves.  The reference's global update (global_update.f90, not in its
 * build) pairs a Wolff cluster flip, built on neighbour couplings of an older
 * field action, with a uniform shift of each auxiliary channel.  Under this
 * model's weight w = exp(-sum phi^2 / 2) |det G|^2 (the exponent
 * bafqmc_log_weight reports) the fields have no neighbour couplings, so the
 * shift is the move that carries over.  bafqmc_global_shift proposes, per
 * chain, phi' = phi + X_ns on every field of channel ns, X_ns = (u - 1/2)
 * |shift[ns]| with u the chain's next two draws (ns = 0, 1), rebuilds G(beta)
 * and log|det(I - B)| of the proposal from scratch (bafqmc_pre's work, in a
 * second per-chain state allocated on first use), and accepts with
 * w'/w >= u' for the chain's third draw u' (global_update.f90:237-249).  An
 * accepted chain continues from the proposal's fields and UDV factors.
 * accepted (optional, [nchains]) receives 0 or 1.  Quarantined chains are
 * skipped.  Requires a built G (bafqmc_pre or a sweep).  The weight's
 * determinant factor is |det(I - B)|^-2 for a number-conserving chain and
 * |det(I - B_1)|^-1 for a Nambu chain (its 4Ns determinant to the power -1/2,
 * src/pairing/src/localU.f90:33-113, is the squared modulus of the
 * {b, c^dagger} block's). */
int bafqmc_global_shift(bafqmc_handle* h, const double* shift, int* accepted);

/* Learned global proposer.  The reference has none: its only global move is
 * the dead global_update.f90 (accept rule global_update.f90:237-249, kept
 * below with the Hastings term of a non-symmetric proposal).
 *
 * The network is a 4-layer periodic 3x3x3 convolution over the (imaginary
 * time x site) field of one lattice (Lx x Ly sites, Ltrot slices): 2 -> width
 * -> width -> width -> 4 channels, ReLU between layers, bf16 weights and
 * activations with float32 accumulation.  Its output per field (t, site, aux)
 * is the mean mu and log scale lsig of a Gaussian proposal
 * phi' = mu(phi) + exp(lsig(phi)) xi, whose displacement from phi is the
 * Gaussian mu - phi + exp(lsig) xi (with a zero last layer: the prior N(0, 1),
 * independently of phi).  Parameters are one float32 vector
 * (per layer W[27][cout][cin] then b[cout]; tap k = 3((b+1)3 + (c+1)) + (a+1)
 * for offsets (a, b, c) in (t, y, x)), the layout of the CPU oracle
 * oracle/proposer.py.  With width 64, Lx*Ly a multiple of 4 and Ltrot a
 * multiple of 32, the 64-channel layers run on the tensor cores (tcgen05,
 * operands staged by TMA); bafqmc_net_set_tensor_cores(n, 0) selects the
 * CUDA-core kernels for the same layers (a cross-check).  A network is not
 * thread-safe; it runs on its own stream, and on the ensemble's stream inside
 * bafqmc_learned_move and bafqmc_net_collect. */
typedef struct bafqmc_net bafqmc_net;
int bafqmc_net_create(int Lx, int Ly, int Ltrot, int width, int device, bafqmc_net** out);
void bafqmc_net_destroy(bafqmc_net* n);
long long bafqmc_net_num_params(const bafqmc_net* n);
/* set_params also resets the optimiser state */
int bafqmc_net_set_params(bafqmc_net* n, const float* params);
int bafqmc_net_get_params(bafqmc_net* n, float* params);
int bafqmc_net_set_tensor_cores(bafqmc_net* n, int enable);
/* Host buffers: phi [chains][Ltrot][Lx*Ly][2] doubles (the confin order, rounded
 * to bf16 on input), out [chains][Ltrot][Lx*Ly][4] floats (mu_0, mu_1, lsig_0, lsig_1). */
int bafqmc_net_forward(bafqmc_net* n, int chains, const double* phi, float* out);
/* Training loss of pairs (phi[b], target[b]): the mean over fields of the
 * Gaussian negative log-likelihood z^2/2 + lsig, z = (target - mu) e^{-lsig}
 * (inputs stored as float32), and its gradient (grad: num_params floats). */
int bafqmc_net_loss_grad(bafqmc_net* n, int chains, const double* phi, const double* target, double* loss,
                         float* grad);
/* Training set on the device: `slots` snapshots of the fields of a handle
 * with `chains` chains; bafqmc_net_collect appends the handle's current
 * fields as the next snapshot (call it after each sweep of the plain sampler). */
int bafqmc_net_reserve_data(bafqmc_net* n, int chains, int slots);
int bafqmc_net_collect(bafqmc_net* n, bafqmc_handle* h);
/* `steps` Adam steps (lr; beta 0.9, 0.999) on batches of `batch` pairs, each a
 * snapshot of one chain and the same chain `lag` snapshots later, drawn from
 * the training set by a counter-based generator seeded with `seed`.
 * losses (optional, [steps]) receives each batch's loss. */
int bafqmc_net_train(bafqmc_net* n, int steps, int batch, int lag, double lr, unsigned long long seed,
                     double* losses);
/* Status word of the tensor-core kernels: 0, or bit 0 (a wait of the copy /
 * MMA / epilogue pipeline expired and the kernel left its tiles) and bit 1
 * (the final wait for the MMAs in flight expired before the tensor memory was
 * released).  A call that sees a nonzero status returns BAFQMC_ETIMEOUT. */
int bafqmc_net_status(bafqmc_net* n, int* status);
/* Device time of each layer of the forward pass (ms[4], milliseconds per
 * launch), averaged over `reps` passes of `chains` chains after one warm-up
 * pass, timed with CUDA events on the network's stream.  A profiling aid: the
 * inputs are whatever the network last held. */
int bafqmc_net_time_layers(bafqmc_net* n, int chains, int reps, double* ms);
/* Test hook of the bounded waits: with enable set, the tensor-core kernels
 * issue no MMA and poll each wait only 4096 times, so every wait expires and
 * the kernel takes its give-up path (nothing is left in flight, the tensor
 * memory is released); enable = 0 restores normal operation.  Both clear the
 * status word. */
int bafqmc_net_set_wait_test(bafqmc_net* n, int enable);
/* One learned move of every chain of h (number-conserving chains on the
 * network's lattice): the network at phi gives the proposal phi' (xi from the
 * chain's LCG, two draws per field in the field order, the Box-Muller cosine
 * branch of fields.f90:280-288), the network at phi' gives
 * hastings = log q(phi|phi') - log q(phi'|phi), phi' is rebuilt from scratch
 * (bafqmc_pre's work, in the second per-chain state of bafqmc_global_shift),
 * and the chain's next draw u accepts when
 * exp(log w(phi') - log w(phi) + hastings) >= u.  accepted and hastings
 * (optional, [nchains]) receive the decisions and Hastings terms; with either
 * given the call synchronises.  Quarantined chains are skipped. */
int bafqmc_learned_move(bafqmc_handle* h, bafqmc_net* n, int* accepted, double* hastings);

/* Per chain, 14 doubles: acc_sum[2], therm_acc_sum[2], Xmaxm, Xmeanm,
 * status (bit 0: the chain's Green's function became non-finite, at a
 * stabilisation or in bafqmc_pre: the chain is quarantined, i.e. later sweeps
 * skip it and bafqmc_bin_point_obs averages over the other chains, until its
 * state is set again; bit 2: a tensor-core product did not complete within
 * its wait bound and the chain continued in FP64; bit 3: such a product's MMAs
 * had still not completed when the sweep released its tensor memory), seed, nobs, accepted global moves, proposals[2], accepted[2] (AccCounter,
 * Prop%Xmaxm/Xmeanm; the last four are PhaseCounter%count_proposed and
 * %count_accepted over all bins, src/pairing/src/operator_Hubbard.f90:269-284.
 * The Nambu weight ratio is real and positive here, so PhaseCounter's phase
 * sums are zero). */
#define BAFQMC_COUNTERS 14
int bafqmc_counters(bafqmc_handle* h, double* out);

/* Arithmetic of the slice propagation (multiply.f90:72-86, propT_L/R; the
 * reference computes it in FP64 with ZGEMM).  BAFQMC_PRECISION_MIXED runs the
 * slice products of chains with 72 < Ndim <= 144 (number-conserving, up to
 * 12x12) on the tensor cores in 3xTF32-compensated FP32 (the products
 * X e^{-+dtau K} and e^{-+dtau K} X with FP32 accumulation), in bafqmc_pre and
 * the sweeps; the stabilisation, (I - B)^{-1}, ratios and acceptance stay
 * FP64, and chains of the other size classes always run FP64.  Decisions of
 * a mixed chain are not bit-identical to the FP64 chain's.  Takes effect from
 * the next bafqmc_pre / bafqmc_sweep.  Default BAFQMC_PRECISION_FP64. */
#define BAFQMC_PRECISION_FP64 0
#define BAFQMC_PRECISION_MIXED 1
/* Test hook of the products' bounded wait: as MIXED, but the products issue
 * no MMA and poll their barrier 1024 times, so every chain's first product
 * gives up (status bit 2, nothing left in flight) and the chain continues in
 * FP64, bit-identical to a BAFQMC_PRECISION_FP64 run. */
#define BAFQMC_PRECISION_WAIT_TEST 2
int bafqmc_set_precision(bafqmc_handle* h, int mode);

/* Time-displaced Green's functions, the is_tau option (calc_basic.f90:36,56;
 * main.f90:50 enables it after Nthermal bins).  With enable set, each sweep of
 * bafqmc_sweep runs Dyn_reset + Dyn_sweep_R (dynamics.f90:37-57) between its
 * left and right traversals (local_sweep.f90:119-123): from G(0,0) the pass
 * propagates G(tau,0), G(0,tau) and G(tau,tau) slice by slice and every Nwrap
 * slices recomputes them from the stabilised factors (Wrap_tau,
 * stabilization.f90:368-404), recording the L1 drift of each.  The Markov chain
 * is unchanged (the pass works on copies).  Chains with N <= 72 (for a Nambu
 * chain N is its stored {b, c^dagger} block, 2 Lx Ly, and the pass works on
 * that block of the reference's 4Ns matrices; BAFQMC_EUNSUPPORTED above).  The
 * reference's L1 drifts on the 4Ns matrices are twice the block's (the
 * {c, b^dagger} block is its complex conjugate).  The U2 operator uses the U2
 * field and the 2N x 2N matrix the bosonic sign; dynamics.f90:52 passes the U1
 * field to the U2 operator and stabilization.f90:206-209 use the fermion sign,
 * both of which this library does not reproduce.
 * probe_nt in 1..Ltrot keeps the four functions of slice probe_nt of the last
 * pass for bafqmc_time_displaced_probe; 0 keeps none. */
int bafqmc_set_time_displaced(bafqmc_handle* h, int enable, int probe_nt);
/* out (optional): [nchains][8] = drift max of G(0,tau), G(tau,0), G(tau,tau)
 * (Wrap_tau's Xmaxm(1..3)), drift sums of the same (Xmeanm before the
 * division), passes run, non-finite recomputations; reset zeroes them after
 * the copy. */
int bafqmc_time_displaced_stats(bafqmc_handle* h, double* out, int reset);
/* out: 4 row-major N x N complex matrices (interleaved re, im) of the chain:
 * G(0,0), G(0,tau), G(tau,0), G(tau,tau) at the probe slice of the last pass
 * (a Nambu chain: their {b, c^dagger} blocks). */
int bafqmc_time_displaced_probe(bafqmc_handle* h, int chain, double* out);

/* Per-phase SM cycle counters of the sweep kernel (the reference has only a
 * total wall time, main.f90:26-27,67-71).  enable switches counting for the
 * following sweeps; out (optional) receives [nchains][4] accumulated cycles:
 * local updates, slice products, measurement, wraps/stabilisation. */
int bafqmc_phase_timers(bafqmc_handle* h, int enable, double* out);

int bafqmc_synchronize(bafqmc_handle* h);
/* The handle's cudaStream_t, for event timing by the caller. */
void* bafqmc_stream(bafqmc_handle* h);

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory once they run (another runtime's caching allocator owns the device,
 * or the driver sizes all memory before a campaign): bafqmc_pre followed by
 * one bin of nsweep sweeps for nchains chains of one point, with all scratch
 * in a fixed device array of BAFQMC_NOALLOC_MAX_BYTES that every GPU loading
 * the library holds until exit.  No cudaMalloc/cudaFree is called.
 *   seeds     [nchains] int32, device memory: in = start seeds, out = advanced
 *   phi       [nchains][Ltrot][Ns][2] doubles, device memory: fields, updated
 *   chain_obs [nchains][BAFQMC_OBS_SCALARS + Lx*Ly] doubles, device memory: the
 *             bin averages, laid out as bafqmc_bin_chain_obs for that point
 *   stream    cudaStream_t to run on (NULL = legacy default stream)
 * Sizes beyond the array return BAFQMC_EARG with the bytes needed, and a
 * NaN or infinite field value returns BAFQMC_EARG naming the chain (as
 * bafqmc_set_state).  The first call on a device sets it up once (the array's
 * device address and the LCG table in constant memory, a synchronous copy);
 * make that first call before any stream capture.  Every call copies
 * host-side set-up data to the array and reads the fields' check and the
 * chains' status back, synchronising the stream twice, so a call made while
 * the stream is capturing returns BAFQMC_ESTATE.  cudaDeviceReset between
 * calls is not supported (the device address is looked up once).  Every call
 * reuses the same array, so calls that overlap on the GPU (other streams,
 * other host threads) race and must not be issued; the call clears the
 * accumulators it reads.  Returns the number of quarantined chains (>= 0;
 * their Green's function became non-finite and their chain_obs row is NaN)
 * or a negative BAFQMC_E* code. */
#define BAFQMC_NOALLOC_MAX_BYTES (64u << 20)
int bafqmc_sweep_noalloc(const bafqmc_point* pt, int nchains, int32_t* seeds, double* phi, int nsweep,
                         double* chain_obs, void* stream);

#ifdef __cplusplus
}
#endif
#endif
