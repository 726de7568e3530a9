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
//  * pass_kernel: one launch per term for up to 8 walks of the same n,
//    alternating between two tilings of the state so that every term streams
//    its vectors once as coalesced tile rows (see the grid-path section).
#include <stdlib.h>

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
// Grid path: fused two-tiling passes.
//
// Clenshaw term r splits as b_r = P_r - a_r*gamma*X_F b_{r+1}, where the
// partial
//   P_r = c_r psi + a_r (D b_{r+1} - gamma X_Z b_{r+1}) - b_{r+2}
// sums the axes Z internal to the tiling of the pass that produced b_{r+1},
// and F = all axes \ Z. Pass r therefore (1) loads the b_{r+1} tile, finishes
// b_r over F (internal to this pass's tiling, plus the few axes of neither
// tiling read from global memory), keeps the b_r tile in shared memory, and
// (2) starts P_{r-1} over all axes of this tiling. Each pass reads b_{r+1},
// P_r, psi and D and writes b_r and P_{r-1}: 44 bytes per amplitude in FP32,
// all as coalesced tile rows, with no partner gathers across tiles.
// Threads own pairs of neighbouring amplitudes (axis 0 lives in registers).
// ---------------------------------------------------------------------------
constexpr int kPassThreads = 512;

template <typename R> struct V4 { R x, y, z, w; };

template <typename R> __device__ __forceinline__ V4<R> ld4(const R* p);
template <> __device__ __forceinline__ V4<float> ld4<float>(const float* p) {
  const float4 t = *reinterpret_cast<const float4*>(p);
  return {t.x, t.y, t.z, t.w};
}
template <> __device__ __forceinline__ V4<double> ld4<double>(const double* p) {
  const double2 a = reinterpret_cast<const double2*>(p)[0];
  const double2 b = reinterpret_cast<const double2*>(p)[1];
  return {a.x, a.y, b.x, b.y};
}
template <typename R> __device__ __forceinline__ void st4(R* p, const V4<R>& v);
template <> __device__ __forceinline__ void st4<float>(float* p, const V4<float>& v) {
  *reinterpret_cast<float4*>(p) = make_float4(v.x, v.y, v.z, v.w);
}
template <> __device__ __forceinline__ void st4<double>(double* p, const V4<double>& v) {
  reinterpret_cast<double2*>(p)[0] = make_double2(v.x, v.y);
  reinterpret_cast<double2*>(p)[1] = make_double2(v.z, v.w);
}
template <typename R>
__device__ __forceinline__ void add4(V4<R>& a, const V4<R>& b) {
  a.x += b.x;
  a.y += b.y;
  a.z += b.z;
  a.w += b.w;
}
// c * psi for a pair, c real (even term) or imaginary (odd term).
template <typename R>
__device__ __forceinline__ V4<R> cpsi4(R c, bool odd, const V4<R>& p) {
  return odd ? V4<R>{-c * p.y, c * p.x, -c * p.w, c * p.z}
             : V4<R>{c * p.x, c * p.y, c * p.z, c * p.w};
}

struct TileMap {
  int n, L, a, tiling;
  size_t tile;
  // Global amplitude index of in-tile position pos (an even position for a
  // pair; the pair's second amplitude is index + 1).
  __device__ __forceinline__ size_t index(int pos) const {
    if (tiling == 1) return (tile << L) | (size_t)pos;
    const int amask = (1 << a) - 1;
    return (size_t)(pos & amask) | (tile << a) |
           ((size_t)(pos >> a) << (n - L + a));
  }
};

// Asynchronous global->shared copies (cp.async, sm_80+): the loads of a
// whole tile are in flight at once without holding registers.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}
template <typename R>
__device__ __forceinline__ void cp_async_pair(R* smem, const R* gmem) {
  cp_async16(smem, gmem);
  if (sizeof(R) == 8) cp_async16(smem + 2, gmem + 2);
}

template <typename R>
__device__ __forceinline__ V4<R> shfl4(const V4<R>& v, int lane_mask) {
  return {__shfl_xor_sync(0xffffffffu, v.x, lane_mask),
          __shfl_xor_sync(0xffffffffu, v.y, lane_mask),
          __shfl_xor_sync(0xffffffffu, v.z, lane_mask),
          __shfl_xor_sync(0xffffffffu, v.w, lane_mask)};
}

// Sum over tile axes [q0, q1) of the partners of register pair j, where pair
// index pp = tid | (j << logT): tile bit 0 is inside the pair, bits 1..5 are
// lane bits (shuffles), bits 6..logT are warp bits (shared memory sx), and
// the top bits index the thread's own registers v[].
template <typename R, int RP>
__device__ __forceinline__ V4<R> axis_sum(const V4<R> (&v)[RP], int j,
                                          const R* sx, int logT, int q0,
                                          int q1, int tid) {
  V4<R> acc{0, 0, 0, 0};
  if (q0 <= 0 && 0 < q1) add4<R>(acc, V4<R>{v[j].z, v[j].w, v[j].x, v[j].y});
  const int l1 = min(q1, 6);
  for (int q = max(q0, 1); q < l1; q++) add4<R>(acc, shfl4<R>(v[j], 1 << (q - 1)));
  const int w1 = min(q1, logT + 1);
  const int pp = tid | (j << logT);
  for (int q = max(q0, 6); q < w1; q++) add4<R>(acc, ld4<R>(sx + 4 * (pp ^ (1 << (q - 1)))));
#pragma unroll
  for (int k = 0; (1 << k) < RP; k++) {
    const int q = logT + 1 + k;
    if (q >= q0 && q < q1) add4<R>(acc, v[j ^ (1 << k)]);
  }
  return acc;
}

template <typename R, int RP, int NU>
__global__ void __launch_bounds__(kPassThreads, 2) pass_kernel(PassParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double s_red[32];
  const PassWalk& W = p.walk[blockIdx.y];
  if (!W.active) return;
  const int n = p.n, L = p.L, a = p.a;
  const int T = blockDim.x, tid = threadIdx.x;
  const int logT = 31 - __clz(T);
  const int npairs = T * RP;
  R* sx = reinterpret_cast<R*>(smem_raw);    // exchange tile: 2^L complex
  R* sp = sx + 4 * (size_t)npairs;          // staged P_r, [j][tid] pairs
  R* ss = sp + 4 * (size_t)npairs;          // staged psi
  float2* sd = reinterpret_cast<float2*>(ss + 4 * (size_t)npairs);  // staged D
  const TileMap tm{n, L, a, p.tiling, (size_t)blockIdx.x};
  // bin and bout may be the same buffer (in-place update when NU == 0: this
  // CTA is then the only reader and writer of its tile's positions).
  const R* bin = reinterpret_cast<const R*>(W.bin);
  R* bout = reinterpret_cast<R*>(W.bout);
  R* __restrict__ part = reinterpret_cast<R*>(W.part);
  const R* __restrict__ psi = reinterpret_cast<const R*>(W.psi);
  const float* __restrict__ hp = W.hp;
  const int r = W.r, K = W.K;
  const bool first = r == K - 1;
  const bool uni = W.psi_uniform;
  // Finish axes (tile bits): T1 -> [a, min(L, n-L+a)), T2 -> [max(2L-n, a), L);
  // axes [L, L+NU) are in neither tiling and come from global memory.
  const int fb0 = p.tiling == 1 ? a : max(2 * L - n, a);
  const int fb1 = p.tiling == 1 ? min(L, n - L + a) : L;

  // Stage P_r, psi and D for this thread's own pairs.
#pragma unroll
  for (int j = 0; j < RP; j++) {
    const size_t gi = tm.index(2 * (tid | (j << logT)));
    const int o = j * T + tid;
    if (!first) cp_async_pair<R>(sp + 4 * o, part + 2 * gi);
    if (!uni) cp_async_pair<R>(ss + 4 * o, psi + 2 * gi);
    cp_async8(sd + o, hp + gi);
  }
  V4<R> va[RP];  // b_{r+1}
#pragma unroll
  for (int j = 0; j < RP; j++)
    va[j] = first ? V4<R>{0, 0, 0, 0}
                  : ld4<R>(bin + 2 * tm.index(2 * (tid | (j << logT))));
  const double kap = W.kappa ? *W.kappa : 1.0;
  const R scale = (R)W.scale;
  const R gamma = (R)W.gamma;
  const R a_mid = (R)2 / scale, a_fin = (R)2 / ((R)2 * scale);
  const R psi0 = (R)(float)(1.0 / sqrt((double)((size_t)1 << n)));
  V4<R> vb[RP];  // b_r
  if (first) {
    const R cr = (R)((double)W.coef[r] * kap);
    cp_async_wait_all();
#pragma unroll
    for (int j = 0; j < RP; j++) {
      const V4<R> pv = uni ? V4<R>{psi0, 0, psi0, 0} : ld4<R>(ss + 4 * (j * T + tid));
      vb[j] = cpsi4<R>(cr, r & 1, pv);
    }
  } else {
    const R ag = (r == 0 ? a_fin : a_mid) * gamma;
#pragma unroll
    for (int j = 0; j < RP; j++) st4<R>(sx + 4 * (tid | (j << logT)), va[j]);
    __syncthreads();
    cp_async_wait_all();
#pragma unroll
    for (int j = 0; j < RP; j++) {
      V4<R> acc = axis_sum<R, RP>(va, j, sx, logT, fb0, fb1, tid);
      if (NU > 0) {
        const size_t gi = tm.index(2 * (tid | (j << logT)));
        V4<R> gv[NU > 0 ? NU : 1];
#pragma unroll
        for (int u = 0; u < NU; u++) gv[u] = ld4<R>(bin + 2 * (gi ^ ((size_t)1 << (L + u))));
#pragma unroll
        for (int u = 0; u < NU; u++) add4<R>(acc, gv[u]);
      }
      const V4<R> pr = ld4<R>(sp + 4 * (j * T + tid));
      vb[j] = V4<R>{fma(-ag, acc.x, pr.x), fma(-ag, acc.y, pr.y),
                    fma(-ag, acc.z, pr.z), fma(-ag, acc.w, pr.w)};
    }
  }
#pragma unroll
  for (int j = 0; j < RP; j++)
    st4<R>(bout + 2 * tm.index(2 * (tid | (j << logT))), vb[j]);
  if (r == 0) {
    double nrm = 0.0;
#pragma unroll
    for (int j = 0; j < RP; j++)
      nrm += (double)vb[j].x * vb[j].x + (double)vb[j].y * vb[j].y +
             (double)vb[j].z * vb[j].z + (double)vb[j].w * vb[j].w;
    const double sum = block_sum<R>(nrm, s_red);
    if (tid == 0) W.norm_part[blockIdx.x] = sum;
    return;
  }
  // Start P_{r-1} = c psi + a (D b_r - gamma X_Z b_r) - b_{r+1} over all tile axes.
  __syncthreads();
#pragma unroll
  for (int j = 0; j < RP; j++) st4<R>(sx + 4 * (tid | (j << logT)), vb[j]);
  __syncthreads();
  const int rm = r - 1;
  const R am = rm == 0 ? a_fin : a_mid;
  const R cm = (R)((double)W.coef[rm] * kap);
#pragma unroll
  for (int j = 0; j < RP; j++) {
    const V4<R> acc = axis_sum<R, RP>(vb, j, sx, logT, 0, L, tid);
    const int o = j * T + tid;
    const V4<R> pv = uni ? V4<R>{psi0, 0, psi0, 0} : ld4<R>(ss + 4 * o);
    const float2 d = sd[o];
    V4<R> out = cpsi4<R>(cm, rm & 1, pv);
    const R d0 = (R)d.x, d1 = (R)d.y;
    out.x = fma(am, fma(d0, vb[j].x, -gamma * acc.x), out.x - va[j].x);
    out.y = fma(am, fma(d0, vb[j].y, -gamma * acc.y), out.y - va[j].y);
    out.z = fma(am, fma(d1, vb[j].z, -gamma * acc.z), out.z - va[j].z);
    out.w = fma(am, fma(d1, vb[j].w, -gamma * acc.w), out.w - va[j].w);
    st4<R>(part + 2 * tm.index(2 * (tid | (j << logT))), out);
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

PassGeomHost pass_geom(int precision, int n) {
  // Tile: 2^L amplitudes of b_{r+1} and 2^L of b_r in shared memory
  // (64 KB at L = 12 in FP32, 3 CTAs per SM). Rows of 2^a = 16 amplitudes
  // (128 bytes in FP32) keep T2 loads coalesced. L is chosen so the two
  // tilings cover every axis when possible (2L - a >= n).
  static int env = -2;
  if (env == -2) {
    const char* e = getenv("MQW_PASS_TILE_LOG");
    env = e ? atoi(e) : -1;
  }
  int Lmax = precision == 0 ? 12 : 11;
  if (env >= 2 && env <= 13) Lmax = env;
  // Threads own pairs along the top tile axes, lanes cover tile axes 1..5,
  // so a tile has at least 6 axes (n >= 6 on the grid path).
  PassGeomHost g;
  g.a = 4;
  int L = (n + g.a + 1) / 2;
  if (L < 6) L = 6;
  if (L > Lmax) L = Lmax;
  if (L > n) L = n;
  g.L = L;
  g.nu = n - (2 * L - g.a);
  if (g.nu < 0) g.nu = 0;
  return g;
}

namespace {
template <typename R, int RP, int NU>
cudaError_t launch_pass_k(const PassParams& p, dim3 grid, int threads,
                          size_t smem, cudaStream_t stream) {
  static size_t configured = 0;
  if (smem > 48 * 1024 && smem > configured) {
    cudaError_t e = cudaFuncSetAttribute(pass_kernel<R, RP, NU>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    configured = smem;
  }
  pass_kernel<R, RP, NU><<<grid, threads, smem, stream>>>(p);
  return cudaGetLastError();
}

template <typename R, int RP>
cudaError_t launch_pass_rp(const PassParams& p, dim3 grid, int threads,
                           size_t smem, int nu, cudaStream_t stream) {
  switch (nu) {
#define MQW_NU(k) \
  case k:         \
    return launch_pass_k<R, RP, k>(p, grid, threads, smem, stream);
    MQW_NU(0) MQW_NU(1) MQW_NU(2) MQW_NU(3) MQW_NU(4) MQW_NU(5) MQW_NU(6)
    MQW_NU(7) MQW_NU(8) MQW_NU(9) MQW_NU(10) MQW_NU(11) MQW_NU(12) MQW_NU(13)
    MQW_NU(14)
#undef MQW_NU
    default:
      return cudaErrorInvalidValue;
  }
}

template <typename R>
cudaError_t launch_pass_t(const PassParams& p, cudaStream_t stream) {
  const int nu = p.n - (2 * p.L - p.a) > 0 ? p.n - (2 * p.L - p.a) : 0;
  dim3 grid((unsigned)((size_t)1 << (p.n - p.L)), p.count);
  const int npairs = 1 << (p.L - 1);
  // 512 threads when the tile has enough pairs; never fewer than one warp
  // (L >= 6 guarantees >= 32 pairs).
  const int threads = npairs < kPassThreads ? npairs : kPassThreads;
  const int rp = npairs / threads;
  const size_t smem = (size_t)npairs * (3 * 4 * sizeof(R) + sizeof(float2));
  switch (rp) {
    case 1: return launch_pass_rp<R, 1>(p, grid, threads, smem, nu, stream);
    case 2: return launch_pass_rp<R, 2>(p, grid, threads, smem, nu, stream);
    case 4: return launch_pass_rp<R, 4>(p, grid, threads, smem, nu, stream);
    default: return cudaErrorInvalidValue;
  }
}
}  // namespace

cudaError_t launch_pass(int precision, const PassParams& p,
                        cudaStream_t stream) {
  if (p.n < 6 || p.L < 6 || p.L > p.n || p.a < 1 || p.a >= p.L ||
      (p.tiling != 1 && p.tiling != 2) || p.count < 1 || p.count > kMaxGroup)
    return cudaErrorInvalidValue;
  return precision == 0 ? launch_pass_t<float>(p, stream)
                        : launch_pass_t<double>(p, stream);
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
