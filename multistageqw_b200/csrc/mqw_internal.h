// Internal declarations shared by the host runtime (mqw_host.cpp) and the
// CUDA kernels (mqw_diag.cu, mqw_coeffs.cu, mqw_propagate.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace mqw {

constexpr int kSamples = 100;          // MultiQW.cpp:257
constexpr int kMaxN = 30;
constexpr int kMaxGroup = 8;           // trajectories per grid-path launch
constexpr int kMaxTileLog = 13;        // grid-path tile: up to 2^13 amplitudes
constexpr int kDiagChunkLog = 12;      // Gray ranks per diagonal chunk
constexpr int kMaxChebTop = 16384;     // Miller start-index bound

// Per-instance device-side description (one per instance in a plan).
struct InstanceDesc {
  int n, m;
  int stages;            // m, or 100 cumulative steps when m == 1
  int raw_off;           // offset of the instance's raw doubles
  long long hp_off;      // offset of its 2^n diagonal in the hp pool
  int sched_off;         // offset into gamma[] (m entries)
  int times_off;         // offset into times[] (m * 100 entries)
  int traj_off;          // first trajectory index (samples or 1 walk)
};

// Reference-arithmetic spectral data of one instance.
struct DiagOut {
  double e0, emax, mid;
  float e_abs;
  uint32_t e_loc;
};

// Chunk partials of the Gray-code scan.
struct ChunkPartial {
  double total;     // sum of the chunk's increments
  double vmin;      // min over the chunk of the running (chunk-local) sum
  double vmax;
  uint32_t rmin;    // Gray rank of the first minimum
  uint32_t pad;
};

// ---- diagonal -------------------------------------------------------------
// Builds hp (float, shifted) and optionally energies (double) for `count`
// instances of the same n. raw: device pointer to count*n(n+1)/2 doubles.
// scratch: device buffer of diag_scratch_bytes(n, count) bytes.
size_t diag_scratch_bytes(int n, int count);
cudaError_t launch_diag(int n, int count, const double* raw, float* hp,
                        double* energies, DiagOut* out, void* scratch,
                        cudaStream_t stream);

// Bandwidth probes (GB/s) of L2 (read; copy), shared memory (read) and HBM
// (copy); allocates and frees ~2 GB of probe buffers.
cudaError_t measure_tiers(cudaStream_t st, int sm_count, double* l2_read_gbs,
                          double* l2_copy_gbs, double* smem_gbs, double* hbm_copy_gbs);

// Moments mean(hp^k), k = 1..4, of a 2^n diagonal into the last four
// doubles of `scratch` (moments_scratch_bytes()).
size_t moments_scratch_bytes();
cudaError_t launch_moments(int n, const float* hp, void* scratch, cudaStream_t stream);

// ---- Chebyshev coefficients --------------------------------------------
// One entry per (instance, stage, sample) "coefficient job".
struct CoefJob {
  int inst;        // instance index (DiagOut / n)
  int n;
  float gamma;     // hopping rate of the stage
  float t;         // evolution time of the sample
};
// Pass 1: degree of each job (s = fl(fl(e_abs + gamma*n) * t)).
cudaError_t launch_cheb_degree(const CoefJob* jobs, int count,
                               const DiagOut* diag, double tol, int* degree,
                               float* onenorm, cudaStream_t stream);
// Pass 2: float coefficients at coef + offset[job].
cudaError_t launch_cheb_coeffs(const CoefJob* jobs, int count,
                               const DiagOut* diag, double tol,
                               const long long* offset, float* coef,
                               cudaStream_t stream);
// Direct: coefficients for explicit s values (API helper).
cudaError_t launch_cheb_from_s(const double* s, int count, double tol,
                               int max_k, float* coef, int* degree,
                               cudaStream_t stream);

// ---- propagation --------------------------------------------------------
// Trajectory-stage data for the resident (one-CTA-per-walk) kernel.
struct ResidentWalk {
  int inst;            // instance
  int n;
  int stages;          // number of Clenshaw stages in the walk
  int record_each;     // 1: record P after every stage (m == 1 walks)
  int stage_desc_off;  // first entry in StageDesc table
  int p_off;           // where P values go (p_sample index)
  long long hp_off;
};
struct StageDesc {
  long long coef_off;  // offset into the coefficient pool
  int K;
  float gamma;
  float onenorm;       // stored by the degree pass
};

int resident_max_n(int precision);
cudaError_t launch_resident(int precision, const ResidentWalk* walks,
                            int count, int max_n, const StageDesc* stages,
                            const float* coef, const float* hp,
                            const DiagOut* diag, double* p_sample,
                            cudaStream_t stream);

// Grid path: one fused pass over tiles for up to kMaxGroup walks of the same
// n. Pass r completes b_r (from the partial P_r and the axes the previous
// pass could not see) and starts b_{r-1} (the partial P_{r-1} over the axes
// internal to this pass's tiling). Passes alternate between two tilings:
//   T1: 2^L consecutive amplitudes (axes [0, L));
//   T2: 2^(L-a) rows of 2^a consecutive amplitudes, one row per value of the
//       top L-a axes (axes [0, a) and [n-L+a, n)).
// Axes in neither tiling ([L, n-L+a), when n > 2L-a) are read from global
// memory during the finish. With C > 0 a tiling's tile of 2^(L+C)
// amplitudes is spread over a cluster of 2^C CTAs (each holds 2^L, the CTA's
// cluster rank supplies the top C tile bits) and L above stands for L + C;
// partners along the rank bits are read from the other CTAs' shared memory.
struct PassWalk {
  const void* bin;     // b_{r+1}; may equal bout only when no axis is read
                       // from global memory (nu == 0)
  void* bout;          // b_r
  void* part;          // P_r in, P_{r-1} out (in place)
  const void* psi;     // stage input state
  const float* hp;     // shifted diagonal
  const float* coef;   // coefficient list of this walk-stage (index r)
  const double* kappa; // 1/||psi|| of the stage input (nullptr = 1)
  double* norm_part;   // r == 0: per-tile |b_0|^2 partials
  float gamma;
  float scale;         // onenorm
  int r;               // term completed by this pass
  int K;               // degree of this walk-stage
  int psi_uniform;     // psi is the uniform state (psi0, 0): not read
  int active;
  float psi0;          // float(1/sqrt(2^n)), the uniform amplitude
  float* real_out;     // basis passes (FP32): also store Re(b_r) here as a
                       // real vector (nullptr: no)
};
struct PassParams {
  int n, L, a;
  int C;               // cluster log: a tile spans 2^C CTAs (0 = one CTA)
  int threads;         // CTA threads at the widest single-CTA tile: 512 (0)
                       // or 256 (more pairs per thread)
  int lane_smem;       // 1: lane-axis partners from shared memory (FP32,
                       // tiles of 2^12 and 2^13), 0: warp shuffles
  int tma;             // 2: a second exchange tile (8 pairs per thread).
                       // 1: the tile's b, P, psi and D arrive by bulk
                       // copies
                       // (TMA) on an mbarrier, FP32 single-CTA tiles
  int comp;            // 1: compensated partner sums (FP32-compensated mode)
  int tiling;          // 1 or 2
  int count;
  unsigned* err;       // device error word (bit 0: a bounded wait gave up)
  unsigned long long wait_ns;  // limit of each bounded wait (0: 200 ms)
  int test_stall;      // test hook: expect bytes that never arrive
  PassWalk walk[kMaxGroup];
};
struct PassGeomHost {
  int L, a, nu;        // CTA tile log, row log, axes read from global memory
  int C;               // cluster log (tile of 2^(L+C) amplitudes over 2^C CTAs)
  int threads;         // CTA threads (0: default 512)
  int lane_smem;       // lane axes through shared memory instead of shuffles
  int tma;             // tile staging: 0 cp.async, 1 bulk copies (TMA), 2
                       // cp.async with a second exchange tile
};
// Geometry for n; lmax > 0 caps the tile (log2 amplitudes), else the
// precision's default cap (or MQW_PASS_TILE_LOG) applies.
PassGeomHost pass_geom(int precision, int n, int lmax = 0, int threads = 0,
                        int lane_smem = 0, int tma = 0, int cluster = 1);
cudaError_t launch_pass(int precision, const PassParams& p,
                        cudaStream_t stream);
// Chain launch: every term of one walk-stage per walk in one launch, a
// thread-block cluster of 2^(n-L) <= 16 CTAs per walk with cluster barriers
// between the passes (n small enough that no axis is read from global
// memory). chain_tile_log gives its tile log L for (precision, n), or 0 when
// it does not apply (also with MQW_CHAIN=0). p: as for launch_pass with
// p.L = chain_tile_log, per walk K (its degree) and active = K > 0; p.tiling
// and the walks' r are not read.
int chain_tile_log(int precision, int n);
cudaError_t launch_pass_chain(int precision, const PassParams& p, cudaStream_t stream);

// Stage-1 shared basis. Every walk of an instance starts from the uniform
// state psi0 and its first stage applies the same operator H~ (one gamma and
// onenorm per instance stage), only with its own time, i.e. its own
// coefficients. The basis w_j = U_j(H~) psi0 (Chebyshev polynomials of the
// second kind: w_0 = psi0, w_1 = 2 H~ psi0, w_{j+1} = 2 H~ w_j - w_{j-1},
// real vectors stored as interleaved complex with zero imaginary part) is
// built once per instance by pass_kernel launches with one unit coefficient,
// and each walk's stage output sum_k c_k T_k(H~) psi0 is recombined from it:
// with T_0 = U_0, T_1 = U_1 / 2, T_k = (U_k - U_{k-2}) / 2,
//   sum_k c_k T_k = sum_j d_j U_j,  d_0 = c_0 - c_2/2,  d_j = (c_j - c_{j+2})/2,
// d_j real for even j and imaginary for odd j, like c_j.
struct CombineWalk {
  const float* coef;   // the walk's stage-1 coefficients c_0 .. c_{K-1}
  int K;
  void* out;           // stage output (interleaved complex, 2^n amplitudes)
  double* norm_part;   // per-block |out|^2 partials (2^(n-L) blocks)
};
struct CombineParams {
  const void* basis;   // Kb real FP32 vectors of 2^n amplitudes
  int n, L, Kb, count;
  CombineWalk walk[kMaxGroup];
};
constexpr int kMaxBasis = 1024;  // basis vectors (stage-1 degree bound)
constexpr int kRecombineLog = 10;  // amplitudes per recombination block (log2, at most)
// Last-stage projection. Only |psi_out[E_loc]|^2 of a walk's last stage is
// used, and H~ is real symmetric, so
//   psi_out[E_loc] = sum_k c_k (T_k(H~) psi)[E_loc] = sum_j d_j <w_j, psi>
// with the basis w_j = U_j(H~) e_loc built once per instance (the same
// pass_kernel recurrence started from the unit vector at E_loc) and d_j the
// stage-1 recombination weights of the walk's last-stage coefficients. The
// output norm is taken as the input norm: |f_K(x)| = 1 +- the 1e-6 tail on
// [-1, 1], so P moves by at most 2e-6 relative. With w_j real,
// sum_j d_j <w_j, psi> = <v, psi> for v = sum_j d_j w_j: the projection is
// the stage-1 recombination of v followed by one dot product with psi.
struct ProjectWalk {
  const float* coef;   // the walk's last-stage coefficients c_0 .. c_{K-1}
  int K;
  const void* psi;     // last-stage input (interleaved complex, unnormalised)
  const double* kappa; // 1/||psi||
  double* p_out;       // receives |psi_out[E_loc]|^2 kappa^2
};
struct ProjectParams {
  const float* basis;  // Kb real FP32 vectors of 2^n amplitudes
  int n, L, Kb, count;
  double* part;        // scratch: [count][2^(n-L) blocks][2] partial <v, psi>
  ProjectWalk walk[kMaxGroup];
};
cudaError_t launch_project(const ProjectParams& p, cudaStream_t stream);
// psi = the unit vector at E_loc of instance `inst` (complex FP32, 2^n).
cudaError_t launch_unit_eloc(void* psi, int n, const DiagOut* diag, cudaStream_t stream);

// Real unit-coefficient chains (FP32). The shared-basis chains — the
// stage-1 basis from the uniform state, the last-stage basis from
// e_{E_loc}, the stage-2 product basis from the real stage-1 basis vectors —
// apply a real operator to a real start vector with real unit coefficients,
// so every vector of the recurrence is real. real_pass_kernel runs one pass
// of such a chain on real vectors (4 bytes per amplitude instead of a
// complex 8) with the same tilings, thread layout and partner-sum order as
// pass_kernel, so its outputs equal the real parts of the complex chain's
// bit for bit. Pass j of a chain with top index R (r = R - j >= 1, a =
// 2/scale): j == 0 writes b_R = v to bout and starts P_{R-1} = a (D v -
// gamma X_Z v); j > 0 finishes b_r = P_r - a gamma X_F b_{r+1} (b_{r+1} in
// bin, the previous pass's bout), writes it to bout and starts P_{r-1} =
// a (D b_r - gamma X_Z b_r) - b_{r+1}. Single-CTA tiles (C = 0) only.
struct RealChainParams {
  int n, L, a;
  int tiling;          // 1 or 2 (odd r: 2)
  int first;           // j == 0
  const float* bin;    // b_{r+1} (j > 0)
  float* bout;         // b_r, written (the basis vector itself)
  float* part;         // P, real, in place
  const float* start;  // v (j == 0; unused when start_uniform)
  int start_uniform;   // v is the uniform state psi0
  float psi0;
  const float* hp;
  float gamma, scale;
  // Single-pass launches: this pass finishes / starts its term with
  // a = 1/onenorm (the second and first pass of a first-kind chain).
  int half_finish, half_start;
  // Chain and batch launches only (launch_real_chain, launch_real_batch;
  // tiling, first, bin, bout, part and start are taken per chain from
  // RealChainDesc): passes j = 0 .. K-1 of terms r = R - j, pass j writing
  // b_r to out_base[j & 1] + (j >> 1) * out_stride floats. tbasis: the
  // chains' vectors are first-kind, T_j(H~) v (T_1 = H~ v), instead of
  // U_j(H~) v.
  int K, R;
  long long out_stride;
  int tbasis;
};
cudaError_t launch_real_pass(const RealChainParams& p, cudaStream_t stream);
// Whole chains in one launch: per chain a cluster of 2^(n-L) CTAs with
// cluster barriers between the passes, L = chain_tile_log(0, n) (FP32);
// the chains of a launch share n, K, R, the operator and out_stride.
constexpr int kMaxChainBatch = 64;
struct RealChainDesc {
  const float* start;   // v (unused when start_uniform)
  float* part;          // the chain's own partial P (real, 2^n floats)
  float* out_base[2];   // outputs of even / odd j
};
struct RealChainBatch {
  RealChainParams p;
  int chains;
  RealChainDesc chain[kMaxChainBatch];
};
cudaError_t launch_real_chain(const RealChainBatch& b, cudaStream_t stream);
// Pass j (term r = R - j) of each of the b.chains chains in one launch
// (single-CTA tiles of 2^L, L = p.L; any n, axes beyond both tilings read
// from global memory).
cudaError_t launch_real_batch(const RealChainBatch& b, int j, cudaStream_t stream);
// v = e_{E_loc} as a real vector of 2^n floats.
cudaError_t launch_unit_eloc_real(float* v, int n, const DiagOut* diag, cudaStream_t stream);
cudaError_t launch_combine(int precision, const CombineParams& p,
                           cudaStream_t stream);

// Stage-2 product basis (FP32; mqw_stage2.cu). The vectors
// Y_jk = U_k(H~_2) w_j (j < Kb stage-1 basis vectors, k < K2) are stored in
// two parity classes, (j + k) even first, then odd; within a class in
// row-major (j, k) order. S2Layout maps between (j, k) and the row q of its
// class.
struct S2Layout {
  int Kb, K2;
  // First k of class h for stage-1 index j (k = h - j mod 2).
  __host__ __device__ int k0(int h, int j) const { return (h ^ j) & 1; }
  // Number of k < K2 with k = first (mod 2).
  __host__ __device__ int cnt(int first) const { return first == 0 ? (K2 + 1) / 2 : K2 / 2; }
  __host__ __device__ int rows(int h) const {
    return ((Kb + 1) / 2) * cnt(k0(h, 0)) + (Kb / 2) * cnt(k0(h, 1));
  }
  __host__ __device__ int index(int j, int k) const {
    const int h = (j + k) & 1;
    return ((j + 1) / 2) * cnt(k0(h, 0)) + (j / 2) * cnt(k0(h, 1)) + (k - k0(h, j)) / 2;
  }
  __host__ __device__ void pair(int h, int q, int* j, int* k) const {
    const int ce = cnt(k0(h, 0));  // a pair of j (even, odd) spans ce + co = K2 rows
    const int jp = q / K2, rem = q - jp * K2;
    if (rem < ce) {
      *j = 2 * jp;
      *k = k0(h, *j) + 2 * rem;
    } else {
      *j = 2 * jp + 1;
      *k = k0(h, *j) + 2 * (rem - ce);
    }
  }
};
// Coefficient matrices of one instance's walks: walk `col` (< walks) has its
// stage-s job at job0 + col * m + s. Row (j, k) of class h weighs basis
// vector j with the walk's stage-sj coefficients and chain step k with its
// stage-sk ones (the stage-2 product basis: sj = 0, sk = 1; the product
// basis of the last two stages: sj = m - 1, sk = m - 2).
struct S2CoefParams {
  const StageDesc* stages;
  const float* coef;
  int job0, m, walks;
  int sj, sk;
  int tbasis;  // first-kind basis vectors: the weights are the coefficients
               // c themselves (else the second-kind weights d)
  int col_stride;      // columns per row (a multiple of s2_tile_cols(walks))
  S2Layout lay;
  int rows_pad[2];     // rows of C0 / C1 (zero-padded to multiples of 8)
  float* C0;           // class 0 (real part): [rows_pad[0]][col_stride]
  float* C1;           // class 1 (imaginary part)
};
struct S2GemmParams {
  const float* Y;      // class-0 rows, then class-1 rows, 2^n floats each
  const float* C0;
  const float* C1;
  int rows[2], rows_pad[2];
  int col_stride;
  int n, walks;
  int out_walks;       // walk capacity of `out`
  float* out;          // planar: Re of walk w at out + w 2^n, Im at
                       // out + (out_walks + w) 2^n
};
struct UnpackWalk {
  const float* re;
  const float* im;
  void* out;           // interleaved complex state
  double* norm_part;   // per-block |psi|^2 partials
};
struct UnpackParams {
  int n, L, count;
  UnpackWalk walk[kMaxGroup];
};
// Projection onto the product basis of the last two stages (m = 4): per
// walk P = |sum_i V_i psi_i|^2 / |psi|^2 with V (the walk's recombined
// last-two-stage vector) and psi (its stage-2 state) planar: Re of walk w at
// base + w 2^n, Im at base + (stride + w) 2^n. Blocks of 2^L amplitudes
// (L = min(n, 12)) leave FP64 partials in `part` (last2_part_bytes).
struct Last2Params {
  const float* V;
  const float* psi;
  int n, L, walks;
  int v_walks, psi_walks;  // walk strides of V and psi
  double* part;
  double* p_out;           // P of walk w at p_out[w]
};
cudaError_t launch_last2(const Last2Params& p, cudaStream_t stream);
size_t last2_part_bytes(int n, int walks);
cudaError_t launch_real_to_complex(void* dst, const float* src, int n, cudaStream_t stream);
cudaError_t launch_s2_coef(const S2CoefParams& p, cudaStream_t stream);
// Columns of one GEMM tile for `walks` walks (C's row stride is a multiple).
int s2_tile_cols(int walks);
cudaError_t launch_s2_gemm(const S2GemmParams& p, cudaStream_t stream);
// The same GEMM on the tensor cores (tcgen05 kind::tf32, three-product TF32
// split, mqw_stage2_tc.cu): writes the K-major hi/lo coefficient copies into
// Ct (s2_tc_coef_floats floats; cp gives the coefficients, its C0/C1 are not
// used) and then the planar outputs g.out. Walks <= 128, n >= 8. err: the
// device error word (bit 1 set when a bounded wait expired).
int s2_tc_np(int walks);
int s2_tc_kp(const S2Layout& lay);
size_t s2_tc_coef_floats(int walks, const S2Layout& lay);
cudaError_t launch_s2_gemm_tc(const S2CoefParams& cp, float* Ct, const S2GemmParams& g,
                              unsigned* err, cudaStream_t stream);
// The GEMM alone, on given K-major hi/lo coefficient copies Ct ([4 Np][Kp]:
// class-0 hi, class-0 lo, class-1 hi, class-1 lo rows of Np walks each).
cudaError_t launch_s2_gemm_tc_raw(const float* Y, const int rows[2], const float* Ct, int Np,
                                  int Kp, int n, int walks, int out_walks, float* out,
                                  unsigned* err, cudaStream_t stream);
cudaError_t launch_unpack(const UnpackParams& p, cudaStream_t stream);

// Finalisation after a stage: kappa[g] = 1/sqrt(sum of partials); when
// record != 0 also p_out[g] = |out[e_loc]|^2 * kappa^2.
struct FinalTraj {
  const double* norm_part;
  int tiles;
  double* kappa;
  const void* out;     // stage output state
  uint32_t e_loc;      // read on device from DiagOut when diag != nullptr
  const DiagOut* diag;
  double* p_out;       // nullptr = no record
};
struct FinalParams {
  int count;
  FinalTraj traj[kMaxGroup];
};
cudaError_t launch_finalize(int precision, const FinalParams& p,
                            cudaStream_t stream);

// Mean of p_sample rows (fixed order) into p_mean.
cudaError_t launch_mean(const double* p_sample, const int* p_off,
                        const int* p_cnt, int count, double* p_mean,
                        cudaStream_t stream);

}  // namespace mqw
