/*
 * mqw.h — C ABI of the B200-native multi-stage quantum-walk simulator.
 *
 * The reference (Asa-Hopkins/MultiStageQW) has no library API: its whole
 * product is the command `MultiQW n m filename [start problems]`
 * (MultiQW.cpp:241-458). This header exposes that path as plain C entry
 * points — plain pointers and sizes, no CUDA or torch types — so that a host
 * program in any language can bind it (ctypes, cgo, JNI, N-API). The
 * `MultiQW` binary built from multistageqw_b200/csrc/multiqw_cli.cpp is the
 * drop-in replacement of the reference command and sits on top of this ABI.
 *
 * Conventions
 *  - Every call returns an mqw_status; nothing aborts the process.
 *  - The caller owns host buffers; a context owns its device buffers.
 *  - One context per host thread. Calls on one context are serialised by the
 *    caller, and plan executions of one context must also be ordered on the
 *    device (one stream, or a synchronisation between them): the plans share
 *    the context's scratch buffers.
 *  - Instance layout (MultiQW.cpp:270-323): per instance n(n+1)/2 float64
 *    values; first the n(n-1)/2 couplings J(i,j) for i = 1..n-1, j = 0..i-1
 *    in that loop order, then the n fields h(0..n-1).
 *  - Ground-state probabilities are reported per instance as the mean over
 *    the evaluated time samples (MultiQW.cpp:454).
 */
#ifndef MQW_H
#define MQW_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MQW_ABI_VERSION 3  /* 3: mqw_chain_pass_timing reports chains per launch */
#define MQW_SAMPLES 100  /* time samples per stage, MultiQW.cpp:257 */
#define MQW_MAX_N 30     /* 2^30 amplitudes; the reference overflows at n >= 31 (MultiQW.cpp:246) */
#define MQW_MAX_M 64     /* stages per walk */

typedef enum mqw_status {
  MQW_OK = 0,
  MQW_ERR_INVALID = 1,     /* bad argument (n, m, count, null pointer, ...) */
  MQW_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  MQW_ERR_NOMEM = 3,       /* device or host allocation failed */
  MQW_ERR_IO = 4,          /* instance file missing, unreadable or too short */
  MQW_ERR_TIMEOUT = 5,     /* a device-side bounded wait gave up */
  MQW_ERR_UNSUPPORTED = 6, /* configuration not supported by this build */
  MQW_ERR_NO_DEVICE = 7    /* no CUDA device, or the device is not sm_100 */
} mqw_status;

typedef enum mqw_precision {
  MQW_FP32 = 0, /* complex64 state, FP32 recurrence (the reference's precision) */
  MQW_FP64 = 1, /* complex128 state, FP64 recurrence (the GPU oracle) */
  MQW_FP32_COMPENSATED = 2 /* complex64 state, FP32 recurrence whose n-term
                              partner sums are compensated (TwoSum): about one
                              rounding per sum; grid path only (n >= 6), no
                              stage-1 basis */
} mqw_precision;

typedef struct mqw_options {
  int precision;   /* mqw_precision, default MQW_FP32 */
  int samples;     /* samples evaluated per instance, 1..100, default 100.
                      The time draws are always the reference's 100 per
                      stage; fewer samples evaluates the first ones. */
  double cheb_tol; /* Chebyshev tail tolerance, default 1e-6 (MultiQW.cpp:440) */
  int group;       /* trajectories per grid-path launch, 0 = autotuned */
  int resident_max_n; /* largest n run with a whole state in one CTA's shared
                         memory, 0 = default (13 for FP32, 12 for FP64) */
  const float* stage_scale; /* optional (gamma_i, t_i) multipliers, two
                               floats per stage, instance after instance
                               (m_0 + m_1 + ... pairs, caller order): a
                               learned schedule; NULL = the paper heuristic */
  int tile_log;    /* grid-path tile (log2 amplitudes), 0 = autotuned */
  int graph;       /* 1 (default): a plan's second execution captures a
                      CUDA graph of its whole device pipeline and the later
                      ones replay it (a plan executed once pays no capture);
                      0: launch kernels one by one every time */
  int lanes;       /* grid-path walk groups in flight at once, each on its
                      own stream (1..4), 0 = autotuned */
  int threads;     /* CTA threads of the grid path at its widest tile: 512
                      or 256 (twice the amplitudes per thread), 0 = autotuned */
  int lane_smem;   /* grid-path partners along the warp-lane axes: 1 from
                      shared memory, -1 by warp shuffles, 0 = autotuned */
  int tma;         /* grid-path tile staging (FP32): 1 bulk copies (TMA)
                      completing on an mbarrier, 2 per-thread cp.async with
                      a second exchange tile (shapes with 8 amplitude pairs
                      per thread), -1 per-thread cp.async, 0 = autotuned */
  int stage1_basis; /* 1 (default): FP32 walks of an instance share one
                       Chebyshev basis for their first stage (built once,
                       recombined per walk); 0: every walk runs its own
                       first-stage recurrence */
  int final_projection; /* 1 (default): FP32 walks of an instance get their
                       last-stage P by projection onto one basis built from
                       e_{E_loc} (the output norm is taken as the input norm,
                       exact up to the 1e-6 Chebyshev tail); 0: every walk
                       runs its own last-stage recurrence */
  int cluster;     /* where the widest grid-path tile leaves axes to neither
                      tiling (n > 20 in FP32): 1 tiles spanning a thread-block
                      cluster, -1 single-CTA tiles with those axes read from
                      global memory, 0 = autotuned (clusters when the other
                      shape fields are all fixed) */
} mqw_options;

typedef struct mqw_diag_info {
  double e0;     /* lowest energy (reference arithmetic)           */
  double emax;   /* highest energy                                  */
  double mid;    /* (emax + e0) / 2, subtracted from H_P            */
  float e_abs;   /* (emax - e0) / 2, the spectral half-width        */
  uint32_t e_loc;/* ground-state index, first minimum in Gray order */
} mqw_diag_info;

typedef struct mqw_run_stats {
  long long instances;
  long long trajectories;   /* instance x sample walks */
  long long terms;          /* summed Chebyshev degree over all stages */
  double term_amps;         /* sum over trajectories and stages of K * 2^n */
  long long launches;       /* kernels launched by the library */
  long long term_launches;  /* grid-path Clenshaw-term launches */
  double kernel_ms;         /* device time of the propagation phase (CUDA
                               events on the launching stream) */
  double h2d_bytes;         /* host-to-device bytes copied by the plan */
  double d2h_bytes;         /* device-to-host bytes copied by the plan */
  double pass_amps;         /* term x amplitudes the grid-path Clenshaw passes
                               actually executed (the shared bases replace
                               the per-walk first and last stages, so this
                               can be well below term_amps) */
  double aux_bytes;         /* device bytes the shared-basis kernels move:
                               basis stores, recombination and projection
                               reads and writes */
} mqw_run_stats;

typedef struct mqw_ctx mqw_ctx;
typedef struct mqw_plan mqw_plan;

/* ---- context --------------------------------------------------------- */

/* Create a context on CUDA device `device`. Fails with MQW_ERR_NO_DEVICE if
 * the device is absent or not a Blackwell sm_100 part. */
mqw_status mqw_create(mqw_ctx** ctx, int device);
void mqw_destroy(mqw_ctx* ctx);
/* Message of the last failing call on this context (never NULL). */
const char* mqw_last_error(const mqw_ctx* ctx);
const char* mqw_status_string(mqw_status s);
void mqw_default_options(mqw_options* opt);
int mqw_abi_version(void);

/* ---- host-side pieces (no GPU needed) ------------------------------------ */

/* Upper-tail normal quantile Phi^{-1}(1-p) as float.
 * Replaces my_normcdfinvf (MultiQW.cpp:80-86). */
float mqw_inv_norm_upper(float p);

/* Couplings (n*n, symmetric, halved: J(i,j) = float(raw)/2) and fields.
 * Replaces the instance unpacking of MultiQW.cpp:306-323. */
mqw_status mqw_load_instance(int n, const double* raw, float* J, float* h);

/* Per-stage hopping rates gamma[m], first-stage-exact time lower bounds
 * short_t[m], the 100 time samples per stage times[m][100] (libstdc++
 * std::mt19937 seeded 29552825458725, re-seeded per instance) and
 * total_t = sum(short_t). For m == 1 the times are sorted and differenced
 * (cumulative evolution). Replaces MultiQW.cpp:365-430. */
mqw_status mqw_schedule(int n, int m, const double* raw, float* gammas,
                        float* short_t, float* times, float* total_t);

/* Read `problems` instances starting at instance `start` from a reference
 * instance file. Unlike the reference (which silently repeats the previous
 * instance past the end of the file, MultiQW.cpp:303), a short file is an
 * MQW_ERR_IO. Replaces MultiQW.cpp:268-271, 303-304. */
mqw_status mqw_read_instances(const char* filename, int n, long long start,
                              long long problems, double* raw_out);

/* Host build of the same coefficient routine the GPU runs (mqw_cheb_coeffs):
 * bit-identical results, for callers without a GPU and for checking. */
mqw_status mqw_cheb_coeffs_host(int count, const double* s, double tol,
                                int max_k, float* coeffs, int* degrees);

/* ---- device pieces ------------------------------------------------------- */

/* Ising diagonal of one instance on the GPU with the reference's arithmetic
 * (float Gray-code increments accumulated in double, MultiQW.cpp:325-362):
 * hp[2^n] = float(E) - float(mid) (nullable), energies[2^n] in double
 * (nullable), and the ground-state index / spectral bounds in *info. */
mqw_status mqw_build_diag(mqw_ctx* ctx, int n, const double* raw, float* hp,
                          double* energies, mqw_diag_info* info);

/* Raw moments mean(H_P^k), k = 1..4, of the shifted float diagonal (the
 * H_P of MultiQW.cpp:361), reduced on the GPU in FP64 in a fixed order; the
 * skewness and kurtosis that the reference's comment at MultiQW.cpp:379-383
 * considers for a higher-moment heuristic are M3/M2^1.5 and M4/M2^2. info
 * (nullable) receives the diagonal's spectral data as in mqw_build_diag. */
mqw_status mqw_diag_moments(mqw_ctx* ctx, int n, const double* raw,
                            double* moments, mqw_diag_info* info);

/* Chebyshev coefficients of exp(i s x) on [-1,1] computed on the GPU in FP64
 * (Jacobi–Anger, tail-sum truncation at `tol`), cast to float:
 * coeffs[count][max_k], degrees[count]. Replaces the call to
 * Chebyshev<double>::RCF_odd_even(f, 1e-6) at MultiQW.cpp:436-440. */
mqw_status mqw_cheb_coeffs(mqw_ctx* ctx, int count, const double* s,
                           double tol, int max_k, float* coeffs, int* degrees);

/* One Clenshaw propagation out = sum_k c_k T_k(H~) psi on the GPU, with
 * H~ = (hp - gamma * sum_q X_q) / scale, real c_k for even k and imaginary
 * for odd k, 6 <= n <= 30 (grid path). psi/out are interleaved complex
 * (re, im) of 2^n amplitudes
 * (float for MQW_FP32, double for MQW_FP64 in `precision`); hp is float.
 * Replaces Clenshaw (MultiQW.cpp:177-236). */
mqw_status mqw_clenshaw(mqw_ctx* ctx, int precision, int n, int K,
                        const float* coeffs, const float* hp, float gamma,
                        float scale, const void* psi, void* out);

/* ---- propagation without allocation ---------------------------------- */

/* Largest n accepted by mqw_clenshaw_noalloc (its fixed working space). */
#define MQW_NOALLOC_MAX_N 16

/* No counterpart in the reference (which has no library API). The same
 * propagation as mqw_clenshaw, for callers that cannot allocate device
 * memory — code that must not synchronise the device (cudaMalloc and cudaFree
 * can), or hosts whose own allocator or fixed memory budget owns all device
 * memory. All pointers are DEVICE pointers owned by the caller: d_coeffs[K],
 * d_hp[2^n], d_psi[2^n] and d_out[2^n] complex (float for MQW_FP32, double
 * for MQW_FP64); d_out must not alias d_psi and receives the result. Work is
 * queued on `stream` (a cudaStream_t, NULL = the legacy default stream) of the
 * current device; the call returns without waiting for it.
 * Working space is a fixed device array of about 1 MiB inside the library
 * (held by every GPU that loads it until exit); n > MQW_NOALLOC_MAX_N returns
 * MQW_ERR_UNSUPPORTED and 6 <= n is required. The first call on each device
 * looks up that array's device address (and makes the kernels' shared-memory
 * opt-in on that device); make it before any stream capture. The address is
 * kept for the life of the process: after a cudaDeviceReset of a device this
 * entry point must not be called on it again. Calls that overlap on the GPU
 * share the array and race: order them on one stream. After any status other
 * than MQW_OK the contents of d_out are undefined. Calls no cudaMalloc,
 * cudaFree or other allocating routine. */
mqw_status mqw_clenshaw_noalloc(int precision, int n, int K,
                                const float* d_coeffs, const float* d_hp,
                                float gamma, float scale, const void* d_psi,
                                void* d_out, void* stream);

/* ---- the whole path -------------------------------------------------- */

/* For `count` instances of n spins and m stages in the reference's layout
 * (raw = count * n(n+1)/2 doubles, host memory): ground-state probability
 * per instance (p_out, double), total_t per instance (nullable) and the
 * ground-state index per instance (nullable). opt may be NULL (defaults).
 * Replaces the problem loop of MultiQW.cpp:296-456. */
mqw_status mqw_run_problems(mqw_ctx* ctx, int n, int m, const double* raw,
                            int count, const mqw_options* opt, double* p_out,
                            float* total_t_out, uint32_t* e_loc_out,
                            mqw_run_stats* stats);

/* Plans separate host preparation from device execution so a batch can be
 * executed repeatedly with its inputs resident in device memory. Instances
 * may have different n and m: n[i], m[i], and raw holds each instance's
 * n_i(n_i+1)/2 values back to back. */
mqw_status mqw_plan_create(mqw_ctx* ctx, int count, const int* n,
                           const int* m, const double* raw,
                           const mqw_options* opt, mqw_plan** plan);
/* Run the batch on `stream` (a cudaStream_t, NULL = the context's stream);
 * returns after the work is queued and the degree read-back it needs. */
mqw_status mqw_plan_execute(mqw_plan* plan, void* stream);
/* Copy results to the host (waits for the plan's stream). Any pointer may be
 * NULL. p_sample (nullable) receives count*samples per-sample values. */
mqw_status mqw_plan_results(mqw_plan* plan, double* p_out, float* total_t,
                            uint32_t* e_loc, double* p_sample);
mqw_status mqw_plan_stats(const mqw_plan* plan, mqw_run_stats* stats);
void mqw_plan_destroy(mqw_plan* plan);

/* Failure-path self-test of the device-side bounded waits: runs one pass
 * whose tile copies can never complete (its mbarrier expects bytes nobody
 * sends), so every CTA's wait gives up after 5 ms, records the error and
 * returns. Returns MQW_ERR_TIMEOUT when the kernel reported it as designed
 * (the context stays usable); any other status is a failure. */
mqw_status mqw_selftest_wait_timeout(mqw_ctx* ctx);

/* Measured bandwidth of the memory tiers a walk's working set can live in,
 * GB/s: L2 (a 32 MB buffer read, and copied 16 MB to 16 MB, with L1-bypassing
 * loads), shared memory (conflict-free 16-byte loads, 4 blocks per SM), HBM
 * (a 1 GB to 1 GB copy). The roofline denominators for L2- and shared-memory-
 * resident workloads. Allocates ~2 GB for the duration of the call. */
typedef struct mqw_tier_peaks {
  double l2_read_gbs, l2_copy_gbs, smem_gbs, hbm_copy_gbs;
} mqw_tier_peaks;
mqw_status mqw_measure_peaks(mqw_ctx* ctx, mqw_tier_peaks* out);

/* The grid-path shape the autotuner picks for n-spin walks in `precision`
 * on this context (tuning now if it has not yet): tile of 2^tile_log
 * amplitudes per CTA, spread over 2^cluster_log CTAs; global_axes axes whose
 * partners are read from global memory; group walks per launch; lanes
 * launches in flight; us_per_walk_pass the timed cost of one walk-term. */
typedef struct mqw_grid_shape {
  int tile_log, cluster_log, global_axes, group, lanes;
  int threads;     /* threads per CTA */
  int lane_smem;   /* 1: lane-axis partners from shared memory */
  int tma;         /* 1: tiles staged by bulk copies, 2: cp.async with a
                      second exchange tile, 0: per-thread cp.async */
  double us_per_walk_pass;
} mqw_grid_shape;
mqw_status mqw_grid_shape_for(mqw_ctx* ctx, int precision, int n,
                              mqw_grid_shape* out);

/* Device time of the grid-path pass kernel alone, in the autotuned shape for
 * (precision, n): `reps` passes (alternating tilings) over zero-filled walks,
 * the shape's walks per launch on each of its concurrent lanes, bracketed by
 * CUDA events on the context's stream. us_per_launch = elapsed / (reps x
 * lanes) — with several lanes in flight this is the launch-to-launch time,
 * not one launch's latency; us_per_walk_pass = us_per_launch / walks per
 * launch. Any output pointer may be NULL. No counterpart in the reference
 * (the measurement behind the roofline of Clenshaw_step, MultiQW.cpp:88). */
mqw_status mqw_pass_timing(mqw_ctx* ctx, int precision, int n, int reps,
                           double* us_per_launch, double* us_per_walk_pass,
                           int* walks_per_launch, int* lanes);
/* The same for the real chain pass (FP32 shared-basis chains: 20 B per
 * amplitude), with the tuned tile of n and the plan's launches of the
 * product-basis chains: 8 chains per launch at n = 17-18 (MQW_CHAIN_BATCH
 * if set) on the tuned walk lanes, else one chain per launch on 4 lanes from
 * n = 19 (MQW_CHAIN_LANES if set) or the tuned walk lanes below (at n <= 16
 * a plan runs whole chains per launch instead; this times their passes
 * launched one by one). `reps` launches per lane on zero-filled vectors,
 * captured in a CUDA graph as a plan's pipeline is, the second replay timed
 * with CUDA events on the context's stream; us_per_launch = elapsed /
 * (reps * lanes) (the launch-to-launch time with `lanes` in flight), each
 * launch one pass of `chains_per_launch` chains. Tiles spread over a
 * cluster are MQW_ERR_UNSUPPORTED (the chains never use them). */
mqw_status mqw_chain_pass_timing(mqw_ctx* ctx, int n, int reps, double* us_per_launch,
                                 int* lanes, int* tile_log, int* chains_per_launch);

/* ---- learned stage schedule (no counterpart in the reference) ---------- */
/* Building blocks of the MLP that proposes per-stage (gamma, t) multipliers
 * (multistageqw_b200/learned.py): BF16 weights, FP32 activations and
 * accumulation. All pointers are DEVICE pointers; work is queued on `stream`
 * (a cudaStream_t, NULL = legacy default stream) of the current device.
 * W_bf16 is row-major [out][in] (bfloat16 bit patterns); X [batch][in];
 * Y, dY [batch][out]. */

/* Y = X W^T + b, then ReLU when relu != 0. b may be NULL. */
mqw_status mqw_mlp_linear_forward(int batch, int in, int out,
                                  const uint16_t* W_bf16, const float* b,
                                  const float* X, float* Y, int relu,
                                  void* stream);
/* With dZ = dY (masked by Y > 0 when relu != 0): dW = dZ^T X [out][in],
 * db = column sums of dZ [out], and dX = dZ W [batch][in] when dX != NULL.
 * Y is the layer's forward output (needed only when relu != 0). */
mqw_status mqw_mlp_linear_backward(int batch, int in, int out,
                                   const uint16_t* W_bf16, const float* X,
                                   const float* Y, const float* dY, float* dX,
                                   float* dW, float* db, int relu,
                                   void* stream);
/* One Adam step on FP32 master weights w with moments m, v (step >= 1), then
 * w_bf16 = bf16(w) when w_bf16 != NULL. */
mqw_status mqw_mlp_adam(int count, float* w, uint16_t* w_bf16, const float* g,
                        float* m, float* v, float lr, float beta1, float beta2,
                        float eps, float weight_decay, int step, void* stream);
/* w_bf16 = bf16(w), round to nearest even. */
mqw_status mqw_mlp_to_bf16(int count, const float* w, uint16_t* w_bf16,
                           void* stream);

/* ---- the reference command -------------------------------------------- */

/* Equivalent of `MultiQW n m filename [start problems]` (MultiQW.cpp:241-458):
 * reads the instances, runs them, prints "total_t P" per problem to stdout
 * (when print != 0) and appends one float32 per problem to
 * <out_dir>/output_<n>_<m> (out_dir NULL = current directory). */
mqw_status mqw_multiqw(mqw_ctx* ctx, int n, int m, const char* filename,
                       long long start, long long problems,
                       const char* out_dir, int print);

#ifdef __cplusplus
}
#endif

#endif /* MQW_H */
