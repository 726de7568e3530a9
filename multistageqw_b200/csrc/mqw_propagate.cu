// Chebyshev/Clenshaw propagation of the multi-stage walk (the hot path).
//
// One Clenshaw term (MultiQW.cpp:88-173, the reference's Clenshaw_step on the
// real and imaginary halves) is, per amplitude i of the complex state,
//   b_r[i] = c_r psi[i] + a (D[i] b_{r+1}[i] - gamma sum_q b_{r+1}[i ^ 2^q])
//            - b_{r+2}[i]
// with a = 2/onenorm (1/onenorm for the last term r = 0, MultiQW.cpp:232),
// c_r real for even r and imaginary for odd r (MultiQW.cpp:206-212), and
// D the shifted float diagonal. The state is interleaved complex
// (float2 / double2); the Hamiltonian is real, so one complex multiply-add
// does what the reference does with two real calls.
//
// Normalisation (MultiQW.cpp:443) is lazy: instead of dividing the stage
// output by its norm, the next stage's coefficients are scaled by
// kappa = 1/||psi|| (the Clenshaw sum is linear in psi), and the final
// ground-state probability is |psi[E_loc]|^2 * kappa^2. Norms are accumulated
// in double with a fixed reduction order, so results are run-to-run
// deterministic.
//
// Two execution shapes:
//  * resident_kernel: one CTA owns a whole walk (instance x sample) with
//    b_{r+1}, b_{r+2}, psi and D in shared memory (n <= 13 in FP32, n <= 12 in
//    FP64) and runs all stages and terms in one launch.
//  * term_kernel: one launch per term for up to 8 walks of the same n; each
//    CTA stages a 2^11-amplitude tile of b_{r+1} in shared memory for the low
//    axes and reads high-axis partners straight from global memory (a warp's
//    partners are 32 consecutive amplitudes, so every load is coalesced).
#include "mqw_internal.h"

namespace mqw {
namespace {

template <typename R> struct Cplx;
template <> struct Cplx<float> { using T = float2; };
template <> struct Cplx<double> { using T = double2; };

template <typename R>
__device__ __forceinline__ typename Cplx<R>::T mk(R x, R y) {
  typename Cplx<R>::T v;
  v.x = x;
  v.y = y;
  return v;
}

// c * psi with c real (even term) or imaginary (odd term).
template <typename R>
__device__ __forceinline__ typename Cplx<R>::T coef_psi(R c, bool odd,
                                                        typename Cplx<R>::T p) {
  return odd ? mk<R>(-c * p.y, c * p.x) : mk<R>(c * p.x, c * p.y);
}

// One amplitude of a Clenshaw term given the partner sum acc.
template <typename R>
__device__ __forceinline__ typename Cplx<R>::T term_update(
    typename Cplx<R>::T cpsi, typename Cplx<R>::T b1, typename Cplx<R>::T acc,
    typename Cplx<R>::T b2, R d, R gamma, R a) {
  const R ux = fma(d, b1.x, -gamma * acc.x);
  const R uy = fma(d, b1.y, -gamma * acc.y);
  return mk<R>(fma(a, ux, cpsi.x - b2.x), fma(a, uy, cpsi.y - b2.y));
}

template <typename R>
__device__ __forceinline__ double block_sum(double v, double* s_red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) s_red[warp] = v;
  __syncthreads();
  double r = 0.0;
  const int nw = (blockDim.x + 31) >> 5;
  for (int w = 0; w < nw; w++) r += s_red[w];
  return r;
}

// ---------------------------------------------------------------------------
// Resident kernel: a whole walk in one CTA.
// ---------------------------------------------------------------------------
struct ResidentArgs {
  const ResidentWalk* walks;
  const StageDesc* stages;
  const float* coef;
  const float* hp;
  const DiagOut* diag;
  double* p_sample;
};

template <typename R>
__global__ void __launch_bounds__(512) resident_kernel(ResidentArgs args) {
  using C2 = typename Cplx<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const ResidentWalk w = args.walks[blockIdx.x];
  const int n = w.n;
  const int N = 1 << n;
  C2* sb1 = reinterpret_cast<C2*>(smem_raw);
  C2* sb2 = sb1 + N;
  C2* spsi = sb2 + N;
  R* sd = reinterpret_cast<R*>(spsi + N);
  double* s_red = reinterpret_cast<double*>(sd + N + (N & 1));
  const int tid = threadIdx.x, T = blockDim.x;
  const float* hp = args.hp + w.hp_off;
  const R psi0 = (R)(float)(1.0 / sqrt((double)N));
  for (int i = tid; i < N; i += T) {
    sd[i] = (R)hp[i];
    spsi[i] = mk<R>(psi0, (R)0);
  }
  const uint32_t e_loc = args.diag[w.inst].e_loc;
  double kappa = 1.0;
  __syncthreads();
  for (int st = 0; st < w.stages; st++) {
    const StageDesc sdsc = args.stages[w.stage_desc_off + st];
    const int K = sdsc.K;
    const float* coef = args.coef + sdsc.coef_off;
    const R gamma = (R)sdsc.gamma;
    const R scale = (R)sdsc.onenorm;
    const R a_mid = (R)2 / scale;
    const R a_fin = (R)2 / ((R)2 * scale);
    double nrm = 0.0;
    for (int r = K - 1; r >= 0; r--) {
      const R c = (R)((double)coef[r] * kappa);
      const bool odd = r & 1;
      const R a = r == 0 ? a_fin : a_mid;
      for (int i = tid; i < N; i += T) {
        const C2 cpsi = coef_psi<R>(c, odd, spsi[i]);
        C2 out;
        if (r == K - 1) {
          out = cpsi;
        } else {
          const C2 b1 = sb1[i];
          C2 acc = mk<R>((R)0, (R)0);
          for (int q = 0; q < n; q++) {
            const C2 v = sb1[i ^ (1 << q)];
            acc.x += v.x;
            acc.y += v.y;
          }
          const C2 b2 = (r == K - 2) ? mk<R>((R)0, (R)0) : sb2[i];
          out = term_update<R>(cpsi, b1, acc, b2, sd[i], gamma, a);
        }
        sb2[i] = out;
        if (r == 0) nrm += (double)out.x * out.x + (double)out.y * out.y;
      }
      __syncthreads();
      C2* t = sb1;
      sb1 = sb2;
      sb2 = t;
    }
    // The stage output is in sb1; it becomes the next stage's psi.
    const double norm2 = block_sum<R>(nrm, s_red);
    kappa = 1.0 / sqrt(norm2);
    C2* t = spsi;
    spsi = sb1;
    sb1 = t;
    if (w.record_each || st == w.stages - 1) {
      if (tid == 0) {
        const C2 v = spsi[e_loc];
        const double p = ((double)v.x * v.x + (double)v.y * v.y) * kappa * kappa;
        args.p_sample[w.p_off + (w.record_each ? st : 0)] = p;
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Grid path: one Clenshaw term.
// ---------------------------------------------------------------------------
constexpr int kTermThreads = 256;

template <typename R>
__global__ void __launch_bounds__(kTermThreads) term_kernel(TermParams p) {
  using C2 = typename Cplx<R>::T;
  __shared__ C2 s_b1[1 << kMaxTileLog];
  __shared__ double s_red[32];
  const TermTraj& T = p.traj[blockIdx.y];
  const int mode = T.mode;
  if (mode == kSkip) return;
  const int n = p.n, lt = p.lt;
  const int tile = 1 << lt;
  const size_t base = (size_t)blockIdx.x << lt;
  const C2* __restrict__ b1 = reinterpret_cast<const C2*>(T.b1);
  C2* __restrict__ b2 = reinterpret_cast<C2*>(T.b2);
  const C2* __restrict__ psi = reinterpret_cast<const C2*>(T.psi);
  const float* __restrict__ hp = T.hp;
  const double kap = T.kappa ? *T.kappa : 1.0;
  const R c = (R)((double)T.coef[0] * kap);
  const bool odd = T.odd;
  const R scale = (R)T.scale;
  const R a = T.final_term ? (R)2 / ((R)2 * scale) : (R)2 / scale;
  const R gamma = (R)T.gamma;
  if (mode != kFirst) {
    for (int i = threadIdx.x; i < tile; i += blockDim.x) s_b1[i] = b1[base + i];
    __syncthreads();
  }
  double nrm = 0.0;
  for (int i = threadIdx.x; i < tile; i += blockDim.x) {
    const size_t gi = base + i;
    const C2 cpsi = coef_psi<R>(c, odd, psi[gi]);
    C2 out;
    if (mode == kFirst) {
      out = cpsi;
    } else {
      C2 acc = mk<R>((R)0, (R)0);
      for (int q = 0; q < lt; q++) {
        const C2 v = s_b1[i ^ (1 << q)];
        acc.x += v.x;
        acc.y += v.y;
      }
      for (int q = lt; q < n; q++) {
        const C2 v = b1[gi ^ ((size_t)1 << q)];
        acc.x += v.x;
        acc.y += v.y;
      }
      const C2 b2v = mode == kSecond ? mk<R>((R)0, (R)0) : b2[gi];
      out = term_update<R>(cpsi, s_b1[i], acc, b2v, (R)hp[gi], gamma, a);
    }
    b2[gi] = out;
    if (T.final_term) nrm += (double)out.x * out.x + (double)out.y * out.y;
  }
  if (T.final_term) {
    const double s = block_sum<R>(nrm, s_red);
    if (threadIdx.x == 0) T.norm_part[blockIdx.x] = s;
  }
}

template <typename R>
__global__ void finalize_kernel(FinalParams p) {
  using C2 = typename Cplx<R>::T;
  const int g = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (g >= p.count) return;
  const FinalTraj& F = p.traj[g];
  double s = 0.0;
  for (int t = lane; t < F.tiles; t += 32) s += F.norm_part[t];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) {
    const double kap = 1.0 / sqrt(s);
    *F.kappa = kap;
    if (F.p_out) {
      const uint32_t e = F.diag ? F.diag->e_loc : F.e_loc;
      const C2 v = reinterpret_cast<const C2*>(F.out)[e];
      *F.p_out = ((double)v.x * v.x + (double)v.y * v.y) * kap * kap;
    }
  }
}

template <typename R>
__global__ void uniform_kernel(typename Cplx<R>::T* psi, int n) {
  const size_t N = (size_t)1 << n;
  const R v = (R)(float)(1.0 / sqrt((double)N));
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N;
       i += (size_t)gridDim.x * blockDim.x)
    psi[i] = mk<R>(v, (R)0);
}

__global__ void mean_kernel(const double* p_sample, const int* p_off,
                            const int* p_cnt, int count, double* p_mean) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  double s = 0.0;
  const int o = p_off[i], c = p_cnt[i];
  for (int k = 0; k < c; k++) s += p_sample[o + k];
  p_mean[i] = s / c;
}

template <typename R>
size_t resident_smem(int n) {
  const size_t N = (size_t)1 << n;
  return N * (3 * sizeof(typename Cplx<R>::T) + sizeof(R)) +
         ((N & 1) ? sizeof(R) : 0) + 32 * sizeof(double);
}

}  // namespace

int resident_max_n(int precision) { return precision == 0 ? 13 : 12; }

cudaError_t launch_resident(int precision, const ResidentWalk* walks,
                            int count, int max_n, const StageDesc* stages,
                            const float* coef, const float* hp,
                            const DiagOut* diag, double* p_sample,
                            cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  ResidentArgs a{walks, stages, coef, hp, diag, p_sample};
  const int T = (1 << max_n) < 512 ? (1 << max_n) : 512;
  const int threads = T < 32 ? 32 : T;
  if (precision == 0) {
    const size_t sm = resident_smem<float>(max_n);
    cudaError_t e = cudaFuncSetAttribute(resident_kernel<float>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    resident_kernel<float><<<count, threads, sm, stream>>>(a);
  } else {
    const size_t sm = resident_smem<double>(max_n);
    cudaError_t e = cudaFuncSetAttribute(resident_kernel<double>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    resident_kernel<double><<<count, threads, sm, stream>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t launch_term(int precision, const TermParams& p,
                        cudaStream_t stream) {
  dim3 grid((unsigned)(((size_t)1 << p.n) >> p.lt), p.count);
  const int threads = (1 << p.lt) < kTermThreads ? (1 << p.lt) : kTermThreads;
  const int th = threads < 32 ? 32 : threads;
  if (precision == 0)
    term_kernel<float><<<grid, th, 0, stream>>>(p);
  else
    term_kernel<double><<<grid, th, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_finalize(int precision, const FinalParams& p,
                            cudaStream_t stream) {
  if (precision == 0)
    finalize_kernel<float><<<1, 32 * kMaxGroup, 0, stream>>>(p);
  else
    finalize_kernel<double><<<1, 32 * kMaxGroup, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_uniform(int precision, void* psi, int n,
                           cudaStream_t stream) {
  const size_t N = (size_t)1 << n;
  const int T = 256;
  const unsigned blocks = (unsigned)((N + T - 1) / T < 4096 ? (N + T - 1) / T : 4096);
  if (precision == 0)
    uniform_kernel<float><<<blocks, T, 0, stream>>>((float2*)psi, n);
  else
    uniform_kernel<double><<<blocks, T, 0, stream>>>((double2*)psi, n);
  return cudaGetLastError();
}

cudaError_t launch_mean(const double* p_sample, const int* p_off,
                        const int* p_cnt, int count, double* p_mean,
                        cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  mean_kernel<<<(count + 127) / 128, 128, 0, stream>>>(p_sample, p_off, p_cnt,
                                                      count, p_mean);
  return cudaGetLastError();
}

}  // namespace mqw
