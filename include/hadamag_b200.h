/*
 * hadamag_b200.h -- C ABI of libhadamag_b200.so, the sm_100a (B200) implementation of
 * HadaMAG.jl's exact stabilizer-Renyi-entropy hot path, its MC_SRE Pauli sampler and
 * its qutrit Mana phase-space transforms.
 *
 * Plain C: pointers and sizes only.  A Julia backend reaches every entry point with
 * ccall; Python reaches them with ctypes.  Each entry point names the reference
 * interface it replaces (paths are relative to the HadaMAG.jl repository).
 *
 * Conventions
 *   - Complex arrays are interleaved (re, im) doubles, the memory layout of Julia's
 *     Vector{ComplexF64} and of numpy complex128.  Device pointers must be 16-byte
 *     aligned.
 *   - A state of n qubits has 2^n amplitudes; a state of L qutrits has 3^L.
 *   - Every call returns HM_OK (0) or a negative HM_ERR_* code; hm_last_error()
 *     describes the last failure on that context.
 *   - A context owns one CUDA device, one stream and grow-only device buffers.  Calls
 *     on one context are serialised by the caller (one context per host thread).
 *   - Results are returned to host memory; every call synchronises its stream before
 *     returning unless the name ends in _async.
 */
#ifndef HADAMAG_B200_H
#define HADAMAG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HM_ABI_VERSION 1

/* status codes */
#define HM_OK 0
#define HM_ERR_ARG -1     /* null pointer, bad enum, bad range                       */
#define HM_ERR_SIZE -2    /* length not q^n, n outside the supported range           */
#define HM_ERR_Q -3       /* unsupported Renyi index q                                */
#define HM_ERR_CUDA -4    /* a CUDA runtime call failed (message in hm_last_error)    */
#define HM_ERR_OOM -5     /* device allocation failed                                 */
#define HM_ERR_TIMEOUT -6 /* a bounded wait of the queue sweep gave up; no valid result */
#define HM_ERR_ALIGN -7   /* device pointer not 16-byte aligned                      */

/* precision / algorithm selector for the exact-SRE entry points */
#define HM_FP64 0  /* FP64 butterflies, FP64 double-double reduction            */
#define HM_FP32 1  /* FP32 butterflies, FP64 powers and reduction               */
#define HM_PLAIN 2 /* the reference CUDA backend's launch structure, FP64       */

typedef struct hm_ctx hm_ctx;

/* Library ABI version (HM_ABI_VERSION). */
int hm_abi_version(void);

/* Create a context on CUDA device `device`.  Replaces the per-call workspace of
 * ext/HadaMAGCUDAExt.jl:19-34 (SREChunkWorkspace), which is rebuilt on every SRE call. */
int hm_create(hm_ctx **ctx, int device);

/* Free every device buffer and the stream of the context. */
int hm_destroy(hm_ctx *ctx);

/* Text of the last error on this context ("" when none).  Valid until the next call. */
const char *hm_last_error(hm_ctx *ctx);

/* Run the context's work on an external cudaStream_t (NULL restores the context's own
 * stream).  Lets a caller time the kernels with events on that stream. */
int hm_set_stream(hm_ctx *ctx, void *cuda_stream);

/* Tuning knobs of the exact-SRE multi-pass sweeps (n >= 12); the autotuner sets them,
 * defaults apply otherwise.  HM_PARAM_BATCH: X-strings per batch (1..4096; the queue
 * sweep rounds it down to a power of two; 0 = derive it from HM_PARAM_UNITS);
 * HM_PARAM_RING: budget of the two-batch intermediate ring in MiB (8..4096; it should
 * stay L2 resident); HM_PARAM_UNITS: warp units per pass the automatic batch size aims
 * for (256..2^20); HM_PARAM_GRAPH: stage kernels captured per CUDA graph (1..1024,
 * default 128; sweeps of at most 32 stages launch them directly); HM_PARAM_ADJ_BATCH:
 * X-strings per batch of hm_sre_grad's stage kernels (power of two, 1..1024).  Value 0
 * restores the default.  Process-wide; returns HM_ERR_ARG for an unknown knob or value. */
#define HM_PARAM_BATCH 1
#define HM_PARAM_RING 2
#define HM_PARAM_UNITS 3
#define HM_PARAM_GRAPH 4
#define HM_PARAM_ADJ_BATCH 5
/* Knobs of the persistent queue sweep, which runs hm_sre_batched (and, when chosen, the
 * two-pass sizes 12 <= n <= 21 of the single-state entry points): HM_PARAM_ENGINE selects
 * the single-state sweep, 0 = automatic (the engine hm_autotune recorded for that size
 * and precision, else the stage kernels), 1 = stage kernels, 2 = queue sweep;
 * HM_PARAM_QUEUE_SLOTS: ring slots (2..64,
 * default 4); HM_PARAM_QUEUE_SLOT_MIB: size of a ring slot when no batch size is set or
 * tuned (1..4096 MiB, default 16); HM_PARAM_QUEUE_CHUNK: work units a warp claims at a
 * time (1..64, default 1); HM_PARAM_QUEUE_CTAS: CTAs per SM (1..32, 0 = as many as fit).
 * HM_PARAM_BATCH sets the queue's X-strings per batch of the largest state as well. */
#define HM_PARAM_ENGINE 6
#define HM_PARAM_QUEUE_SLOTS 7
#define HM_PARAM_QUEUE_SLOT_MIB 8
#define HM_PARAM_QUEUE_CHUNK 9
#define HM_PARAM_QUEUE_CTAS 10
/* Test of the queue sweep's bounded waits: with value 1 the pass-2 units of the first
 * batch wait for one pass-1 unit more than exist, each wait gives up after a few
 * thousand polls, and the call returns HM_ERR_TIMEOUT with the context still usable.
 * Value 0 (default) restores normal operation. */
#define HM_PARAM_QUEUE_STALL_TEST 11
/* HM_PARAM_QUEUE_LEAD: batches between a batch's pass 1 and its pass 2 in the queue
 * (1..16, default 2; the ring keeps at least lead + 1 slots). */
#define HM_PARAM_QUEUE_LEAD 12
/* HM_PARAM_BATCH_SPLIT_N: hm_sre_batched runs states with n below this (1..22, default
 * 15) in one queue launch and the others one state per call (22: every state up to n = 21
 * in the queue). */
#define HM_PARAM_BATCH_SPLIT_N 14
int hm_set_param(int param, int value);

/* Autotuner of the two-pass sweep (no reference counterpart): times the sweep of an n-qubit
 * state on a sample of Gray indices with the stage kernels (X = 1, 2, 3, 4, 5, 6, 8, 10,
 * 12, ... X-strings per stage: each power of two and 1.25 and 1.5 times it) and with the
 * queue sweep (X = 1, 2, 4, ... X-strings per ring slot, at full
 * occupancy and at one CTA per SM), records the fastest engine, batch size and CTAs per
 * SM for this (n, precision) in a process-wide table that later calls use unless a knob
 * forces another choice, and returns the batch size with the measured microseconds per
 * X-string.  12 <= n <= 21, precision HM_FP64 or HM_FP32.  Takes a second or two. */
int hm_autotune(hm_ctx *ctx, int n, int precision, int *best_x, double *best_us_per_x);

/* The choice hm_autotune recorded for (n, precision): engine 0 (not tuned), 1 (stage
 * kernels) or 2 (queue sweep), its batch size, and CTAs per SM (0 = as many as fit). */
int hm_autotune_choice(int n, int precision, int *engine, int *batch, int *ctas_per_sm);

/* Number of kernels the last call launched on the device (graph nodes included). */
int hm_last_launch_count(hm_ctx *ctx, long long *count);

/* Measured FP64 add throughput of the device, in operations per second (a register-
 * resident DADD kernel of about 10 ms).  Measurement utility for roofline reports; no
 * reference counterpart. */
int hm_probe_fp64_peak(hm_ctx *ctx, double *ops_per_s);

/* The FP32 counterpart (register-resident FADD chains): FP32 add operations per second,
 * the roofline of the FP32 butterflies of HM_FP32. */
int hm_probe_fp32_peak(hm_ctx *ctx, double *ops_per_s);

/* Device time in milliseconds of the main kernels of the last call (CUDA events on the
 * context's stream, recorded around the launches that do the transform work). */
int hm_last_kernel_ms(hm_ctx *ctx, double *ms);

/* ---------------------------------------------------------------------------------- */
/* Exact SRE                                                                            */
/* ---------------------------------------------------------------------------------- */

/* Exact stabilizer Renyi entropy over all 4^n Pauli strings.
 * Replaces SRE(psi, q; backend=:cuda) of ext/HadaMAGCUDAExt.jl:1381-1410 (and the CPU
 * backends src/Backends/Serial.jl:7-51, src/Backends/Threads.jl:108-159): for each q in
 * qs[0..nq), out_sre[i] = -log2(m_q / 2^n) with m_q = sum over x, k of (F_x(k)^2)^q, and
 * out_lost[0] = |1 - p2 / 2^n| with p2 = sum F^2.  As in the reference, for q != 2 the
 * value is (q-1) times the textbook M_q.
 * psi: host pointer, 2^n interleaved complex doubles.  1 <= n <= 24 (n <= 11 one fused
 * pass, 12 <= n <= 21 two passes, 22 <= n <= 24 three passes).  1 <= nq <= 4, each q in
 * [1, 16] (non-integer q allowed). */
int hm_sre(hm_ctx *ctx, const double *psi, int n, const double *qs, int nq, int precision, double *out_sre,
           double *out_lost);

/* Same as hm_sre with psi already resident in device memory (16-byte aligned). */
int hm_sre_dev(hm_ctx *ctx, const double *psi_dev, int n, const double *qs, int nq, int precision,
               double *out_sre, double *out_lost);

/* Raw sums over the Gray-code indices k in [k_begin, k_end) (X-string x = k ^ (k>>1)),
 * returned as double-double pairs so that partial ranges combine order-independently:
 * p2_dd[0] + p2_dd[1] = sum F^2, m_dd[2i] + m_dd[2i+1] = sum (F^2)^{qs[i]}.
 * Replaces compute_chunk_sre(istart, iend, ...) of src/SRE.jl:338-496 and the per-rank
 * Gray split of ext/HadaMAGMPICUDAExt.jl:49-56.  psi is a host pointer. */
int hm_sre_range(hm_ctx *ctx, const double *psi, int n, uint64_t k_begin, uint64_t k_end, const double *qs,
                 int nq, int precision, double *p2_dd, double *m_dd);

/* Device-pointer variant of hm_sre_range. */
int hm_sre_range_dev(hm_ctx *ctx, const double *psi_dev, int n, uint64_t k_begin, uint64_t k_end,
                     const double *qs, int nq, int precision, double *p2_dd, double *m_dd);

/* Exact SRE on several GPUs in one call (replaces the :mpi_cuda backend's per-rank work,
 * SRE of ext/HadaMAGMPICUDAExt.jl:30-99): the Gray range is split into ndev nearly equal
 * contiguous ranges (split_ranges, ext/HadaMAGMPICUDAExt.jl:8-28: the first N mod ndev
 * one longer), devices[i] sweeps range i from its own host thread with its own context,
 * and the double-double sums are added in list order.  A device may appear more than
 * once: its parts then run one after another on its thread.  Contexts are created on first use and kept until hm_multi_release().  Calls are
 * serialised process-wide; errors are described by hm_multi_last_error() (per thread).
 * psi: host pointer; other arguments and results as hm_sre. */
int hm_sre_multi(const int *devices, int ndev, const double *psi, int n, const double *qs, int nq, int precision,
                 double *out_sre, double *out_lost);

/* Range form of hm_sre_multi: the Gray indices [k_begin, k_end) of one process (an MPI
 * rank's share) split over its GPUs; double-double sums as hm_sre_range, to be reduced
 * across processes by the caller. */
int hm_sre_range_multi(const int *devices, int ndev, const double *psi, int n, uint64_t k_begin, uint64_t k_end,
                       const double *qs, int nq, int precision, double *p2_dd, double *m_dd);

/* Text of the last error of a multi-GPU call on this thread ("" when none). */
const char *hm_multi_last_error(void);

/* Destroy the contexts the multi-GPU calls keep. */
int hm_multi_release(void);

/* Batched exact SRE of many states of possibly different qubit counts (no reference
 * counterpart; the reference handles one state per call): one upload of every state, one
 * persistent queue launch for the states below HM_PARAM_BATCH_SPLIT_N, one call's kernels
 * per larger state.  psis[s] points to 2^ns[s] interleaved complex doubles (host).  For
 * each state s and each q: out_sre[s*nq + i]; out_lost[s]. */
int hm_sre_batched(hm_ctx *ctx, int nstates, const double *const *psis, const int *ns, const double *qs, int nq,
                   int precision, double *out_sre, double *out_lost);

/* Adjoint (no reference counterpart): value and gradient of SRE_q w.r.t. the real and
 * imaginary parts of psi.  grad is interleaved: grad[2r] = dSRE/dRe psi_r,
 * grad[2r+1] = dSRE/dIm psi_r.  The forward transform F_x is recomputed per x, never
 * stored.  psi host pointer, 1 <= n <= 21, q integer in [1, 8]. */
int hm_sre_grad(hm_ctx *ctx, const double *psi, int n, double q, double *out_sre, double *grad);

/* Exact SRE for callers that cannot allocate device memory.  No counterpart in the
 * reference.  Some hosts cannot call cudaMalloc at all: code running inside another
 * framework's memory pool, plugins that must not grow the device footprint after start-
 * up, processes whose device memory is fully reserved by an allocator they do not own.
 * This entry point allocates nothing: no context, no cudaMalloc / cudaFree, no pinned
 * host buffers.  Its scratch (the device copy of the state, per-warp partial sums, the
 * folded result; about 400 KB) is a fixed array inside the library, which every GPU that
 * loads the library keeps until the process exits.
 *   psi: host pointer, 2^n interleaved complex doubles, 1 <= n <= HM_NOALLOC_MAX_N (11);
 *   larger n returns HM_ERR_SIZE and computes nothing.  qs[0..nq), 1 <= nq <= 4, q in
 *   [1, 16].  Results as hm_sre (FP64): out_sre[i], out_lost[0], in host memory.
 *   cuda_stream: the stream to run on (NULL = the legacy default stream); the call
 *   returns after synchronising it.  Runs on the calling thread's current device.
 * The first call on a device looks up the scratch array's device address; make that
 * first call before any stream capture.  The address is looked up again after the
 * device's context changes (cudaDeviceReset, a recreated primary context); the first call
 * after such a change is again a set-up call.  Every call on a device shares the one
 * array and it keeps the last call's contents, so calls that overlap on the GPU (other
 * threads, other streams) race: serialise them. */
#define HM_NOALLOC_MAX_N 11
int hm_sre_noalloc(const double *psi, int n, const double *qs, int nq, double *out_sre, double *out_lost,
                   void *cuda_stream);

/* ---------------------------------------------------------------------------------- */
/* MC_SRE                                                                               */
/* ---------------------------------------------------------------------------------- */

/* Metropolis estimate of SRE_q (replaces MC_SRE of src/Backends/Threads.jl:161-221 with
 * mc_sre_beta! of src/SRE.jl:110-192).  Chain i runs at beta_i = i / (nbeta - 1).  The
 * proposal stream is an input: prop_delta[i*nsamples + t] is the XOR of the site bits the
 * reference draws for step t of chain i (src/SRE.jl:164-170), rs[i*nsamples + t] its
 * uniform acceptance draw (src/SRE.jl:145).  Outputs: out_m2 = -log2(2^-I + I_add)
 * (Simpson), per-chain means M2[i], M2ADD[i] = m0/2^n, P2[i]; final_mask[i] (optional,
 * may be NULL) the chain's current X-string after the last step.  nbeta odd, 3 <= nbeta
 * <= HM_MC_MAX_NBETA (the reference takes any odd count; nbeta = 1 divides by zero in its
 * beta grid).  1 <= n <= 21. */
#define HM_MC_MAX_NBETA 4095
int hm_mc_sre(hm_ctx *ctx, const double *psi, int n, double q, int nbeta, int nsamples, const uint64_t *prop_delta,
              const double *rs, double *out_m2, double *M2, double *M2ADD, double *P2, uint64_t *final_mask);

/* Chains chain_begin .. chain_end-1 of the nbeta-point grid of hm_mc_sre (chain i at
 * beta_i = i / (nbeta - 1)), for running the chains on several GPUs.  The chains are
 * independent (src/Backends/Threads.jl:175-205).  prop_delta / rs hold those chains'
 * streams (nsamples each, in chain order); M2, M2ADD, P2 (and final_mask, optional)
 * receive chain_end - chain_begin values.  The caller gathers every chain and combines
 * them with Simpson's rule as hm_mc_sre does (hadamag_b200.shard.mc_sharded). */
int hm_mc_sre_chains(hm_ctx *ctx, const double *psi, int n, double q, int nbeta, int chain_begin, int chain_end,
                     int nsamples, const uint64_t *prop_delta, const double *rs, double *M2, double *M2ADD,
                     double *P2, uint64_t *final_mask);

/* ---------------------------------------------------------------------------------- */
/* Mana                                                                                 */
/* ---------------------------------------------------------------------------------- */

/* Mana of a pure L-qutrit state (3^L interleaved complex doubles, host).
 * Replaces Mana(psi::StateVec{T,3}) of src/Backends/Threads.jl:223-271 with
 * compute_chunk_mana_qutrits of src/Mana.jl:19-92: log2(sum |W|) / log2(3).  1 <= L <= 12. */
int hm_mana_pure(hm_ctx *ctx, const double *psi, int L, double *out_mana);

/* Sum of |W| over the ternary X-strings x_begin .. x_end-1 (natural order, 0 <= x_begin <
 * x_end <= 3^L) as a double-double sum_dd[0] + sum_dd[1].  The sum over every X-string
 * S gives Mana = log2(S) / log2(3), so ranges can run on several GPUs and be added
 * (hadamag_b200.shard.mana_sharded; the reference's threads split their X-string range
 * the same way, src/Backends/Threads.jl:236-262). */
int hm_mana_pure_range(hm_ctx *ctx, const double *psi, int L, int64_t x_begin, int64_t x_end, double *sum_dd);

/* Mana of an N-qutrit density matrix (3^N x 3^N, column-major, interleaved complex
 * doubles, host).  Replaces Mana(rho::DensityMatrix) of src/Mana.jl:305-314:
 * log2(sum |M^{(x)N} vec9(rho)| / 3^N).  1 <= N <= 8. */
int hm_mana_mixed(hm_ctx *ctx, const double *rho, int N, double *out_mana);

/* ---------------------------------------------------------------------------------- */
/* Gray tables (parity checks of the device-side X-string enumeration)                 */
/* ---------------------------------------------------------------------------------- */

/* Binary Gray table computed on the device, as generate_binary of src/Basis.jl:14-27:
 * codes[k] = k ^ (k >> 1) (2^n entries), flips[k] = 1-based bit that flips between
 * codes[k] and codes[k+1] (2^n - 1 entries).  0 <= n <= 30. */
int hm_gray_table(hm_ctx *ctx, int n, uint64_t *codes, int64_t *flips);

/* q-ary Gray table computed on the device, as generate_general of src/Basis.jl:146-164:
 * xtab is n x q^n column-major (column k = integer_to_gray(k)), flips has q^n - 1
 * 1-based digit positions.  2 <= q <= 16, q^n <= 2^26. */
int hm_gray_table_general(hm_ctx *ctx, int n, int q, int64_t *xtab, int64_t *flips);

/* Rank `rank`'s slice of the Gray table split over P processes, computed on the device,
 * as generate_binary_splitted / generate_general_splitted of src/Basis.jl:76-106 and
 * 206-250 (the enumeration of the reference's MPI backends): the global indices
 * code_off .. code_off + code_cnt - 1 of the partition_counts split (src/Helpers.jl:18-23).
 * q = 2: codes[j] = i ^ (i >> 1) (as uint64 bits); q > 2: codes is n x code_cnt
 * column-major (column j = integer_to_gray(code_off + j)).  flips: the code_cnt - 1
 * 1-based bit / digit positions inside the slice.  The caller sizes codes and flips for
 * the slice (at most ceil(q^n / P) columns).  q^n <= 2^30. */
int hm_gray_table_split(hm_ctx *ctx, int n, int q, int rank, int P, int64_t *codes, int64_t *flips,
                        int64_t *code_off, int64_t *code_cnt);

/* ---------------------------------------------------------------------------------- */
/* State files                                                                          */
/* ---------------------------------------------------------------------------------- */

/* Read a state file into page-locked host memory (replaces load_state of
 * src/State.jl:388-404): ".npy" (a complex128 vector, or float64 read as real amplitudes)
 * with one read straight into the buffer, any other name as whitespace-separated real /
 * imaginary pairs.  ".jld2" (HDF5) returns HM_ERR_ARG: this library reads no HDF5.
 * *psi_pinned receives 2 *len doubles (interleaved complex) from cudaMallocHost, to be
 * released with hm_free_state; *len must be a power of q (HM_ERR_SIZE otherwise, as the
 * reference's StateVec check).  Errors are described by hm_io_last_error() (per thread). */
int hm_load_state(const char *path, int q, double **psi_pinned, uint64_t *len);

/* Release a buffer from hm_load_state. */
int hm_free_state(double *psi_pinned);

/* Text of the last error of hm_load_state on this thread ("" when none). */
const char *hm_io_last_error(void);

/* ---------------------------------------------------------------------------------- */
/* State preparation (inputs of the SRE and Mana paths)                                 */
/* ---------------------------------------------------------------------------------- */
/* States are q^n interleaved complex doubles on the host, q in {2, 3}, 1 <= n <= 30
 * (q = 2) or 19 (q = 3).  Sites are 1-based with site 1 the least significant digit;
 * a two-site gate is q^2 x q^2, column-major, interleaved complex, with row / column
 * index o1 q + o2 / d1 q + d2 (d1 the digit of site s1). */

/* Apply a two-site gate to sites s1 != s2 in place.  Replaces apply_2gate! of
 * src/State.jl:254-345 (apply_2gate_qubit! 279-309, apply_2gate_qudit! 311-344). */
int hm_apply_2gate(hm_ctx *ctx, double *psi, int n, int q, const double *gate, int s1, int s2);

/* Brick-wall circuit in place: layers 1..depth, odd layers on sites (1,2),(3,4),...,
 * even layers on (2,3),(4,5),...; `gates` holds one q^2 x q^2 gate per site pair in
 * layer order (ngates must equal that count).  Replaces the loop of
 * apply_brick_wall_haar! (src/State.jl:200-221) and apply_brick_wall_cliff! (146-183);
 * the caller draws the gates (haar_random_unitary, src/Helpers.jl:102-132). */
int hm_brick_wall(hm_ctx *ctx, double *psi, int n, int q, int depth, const double *gates, int ngates);

/* Reduced density matrix rho_A = Tr_B |psi><psi| of a contiguous block of NA sites
 * (0 <= NA <= n, q^NA <= 16384): side 0 keeps sites 1..NA (`:left`), side 1 keeps
 * sites n-NA+1..n (`:right`).  rho: q^NA x q^NA, column-major, interleaved complex.
 * Replaces reduced_density_matrix of src/DensityMatrix.jl:94-123. */
int hm_reduced_density_matrix(hm_ctx *ctx, const double *psi, int n, int q, int NA, int side, double *rho);

#ifdef __cplusplus
}
#endif

#endif /* HADAMAG_B200_H */
