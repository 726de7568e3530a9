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

#include <algorithm>
#include <map>
#include <mutex>
#include <utility>

#include "mqw_internal.h"

namespace mqw {
namespace {

// Dynamic shared-memory opt-ins. cudaFuncSetAttribute applies to the current
// device only, so the size a kernel has been opted in to is recorded per
// (device, kernel); contexts on several devices and several host threads may
// launch concurrently, hence the lock. The first launch of a kernel on a
// device makes the call (before any stream capture that uses it).
std::mutex g_optin_mu;
std::map<std::pair<int, const void*>, size_t> g_optin;

cudaError_t ensure_smem_optin(const void* fn, size_t bytes, bool nonportable_cluster) {
  if (bytes <= 48 * 1024 && !nonportable_cluster) return cudaSuccess;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_optin_mu);
  size_t& done = g_optin[std::make_pair(dev, fn)];
  if (bytes <= done) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return e;
  if (nonportable_cluster) {
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
  }
  done = bytes;
  return cudaSuccess;
}

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
// c * psi for a pair, c real (even term) or imaginary (odd term).
template <typename R>
__device__ __forceinline__ V4<R> cpsi4(R c, bool odd, const V4<R>& p) {
  return odd ? V4<R>{-c * p.y, c * p.x, -c * p.w, c * p.z}
             : V4<R>{c * p.x, c * p.y, c * p.z, c * p.w};
}

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


// A pair of neighbouring amplitudes as the hot loops carry it. FP32: two
// 64-bit registers, each a packed (re, im), accumulated with sm_100's
// add.rn.f32x2 and exchanged with 64-bit shuffles; FP64: two double2.
template <typename R> struct Pair;
template <> struct Pair<float> { unsigned long long a, b; };
template <> struct Pair<double> { double2 a, b; };

__device__ __forceinline__ Pair<float> pld(const float* p) {
  const ulonglong2 t = *reinterpret_cast<const ulonglong2*>(p);
  return {t.x, t.y};
}
__device__ __forceinline__ Pair<double> pld(const double* p) {
  return {reinterpret_cast<const double2*>(p)[0], reinterpret_cast<const double2*>(p)[1]};
}
__device__ __forceinline__ void pst(float* p, const Pair<float>& v) {
  *reinterpret_cast<ulonglong2*>(p) = make_ulonglong2(v.a, v.b);
}
__device__ __forceinline__ void pst(double* p, const Pair<double>& v) {
  reinterpret_cast<double2*>(p)[0] = v.a;
  reinterpret_cast<double2*>(p)[1] = v.b;
}
__device__ __forceinline__ Pair<float> pshfl(const Pair<float>& v, int m) {
  return {__shfl_xor_sync(0xffffffffu, v.a, m), __shfl_xor_sync(0xffffffffu, v.b, m)};
}
__device__ __forceinline__ Pair<double> pshfl(const Pair<double>& v, int m) {
  return {make_double2(__shfl_xor_sync(0xffffffffu, v.a.x, m), __shfl_xor_sync(0xffffffffu, v.a.y, m)),
          make_double2(__shfl_xor_sync(0xffffffffu, v.b.x, m), __shfl_xor_sync(0xffffffffu, v.b.y, m))};
}
__device__ __forceinline__ void padd(Pair<float>& acc, const Pair<float>& v) {
  asm("add.rn.f32x2 %0, %0, %1;" : "+l"(acc.a) : "l"(v.a));
  asm("add.rn.f32x2 %0, %0, %1;" : "+l"(acc.b) : "l"(v.b));
}
__device__ __forceinline__ void padd(Pair<double>& acc, const Pair<double>& v) {
  acc.a.x += v.a.x;
  acc.a.y += v.a.y;
  acc.b.x += v.b.x;
  acc.b.y += v.b.y;
}
template <typename R> __device__ __forceinline__ Pair<R> pzero();
template <> __device__ __forceinline__ Pair<float> pzero<float>() { return {0ull, 0ull}; }
template <> __device__ __forceinline__ Pair<double> pzero<double>() {
  return {make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
}
template <typename R>
__device__ __forceinline__ Pair<R> pswap(const Pair<R>& v) { return {v.b, v.a}; }

// Register-pair views (no data movement).
__device__ __forceinline__ V4<float> to4(const Pair<float>& v) {
  float x, y, z, w;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(x), "=f"(y) : "l"(v.a));
  asm("mov.b64 {%0, %1}, %2;" : "=f"(z), "=f"(w) : "l"(v.b));
  return {x, y, z, w};
}
__device__ __forceinline__ V4<double> to4(const Pair<double>& v) {
  return {v.a.x, v.a.y, v.b.x, v.b.y};
}
__device__ __forceinline__ Pair<float> from4(const V4<float>& v) {
  unsigned long long a, b;
  asm("mov.b64 %0, {%1, %2};" : "=l"(a) : "f"(v.x), "f"(v.y));
  asm("mov.b64 %0, {%1, %2};" : "=l"(b) : "f"(v.z), "f"(v.w));
  return {a, b};
}
__device__ __forceinline__ Pair<double> from4(const V4<double>& v) {
  return {make_double2(v.x, v.y), make_double2(v.z, v.w)};
}

// Distributed shared memory (thread-block clusters): the shared-window
// address of the same variable in the CTA of cluster rank `rank`, loads from
// it, and the cluster-wide barrier (release/acquire: orders this CTA's shared
// memory writes before the other CTAs' reads after the barrier).
__device__ __forceinline__ unsigned cluster_addr(const void* smem, unsigned rank) {
  const unsigned local = (unsigned)__cvta_generic_to_shared(smem);
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
  return r;
}
__device__ __forceinline__ Pair<float> pld_cluster(const float*, unsigned addr) {
  unsigned long long a, b;
  asm volatile("ld.shared::cluster.v2.u64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "r"(addr) : "memory");
  return {a, b};
}
__device__ __forceinline__ Pair<double> pld_cluster(const double*, unsigned addr) {
  double x, y, z, w;
  asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(x), "=d"(y) : "r"(addr) : "memory");
  asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(z), "=d"(w) : "r"(addr + 16) : "memory");
  return {make_double2(x, y), make_double2(z, w)};
}
__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n"
               "barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
// Bulk copies (TMA, no multicast) into this CTA's shared memory, completing
// on an mbarrier, and bounded waits on it: a wait gives up after `limit_ns`
// of %globaltimer time so that a copy that never lands cannot hang the GPU.
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  unsigned long long limit_ns) {
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > limit_ns) return false;
  return true;
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes,
                                          unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// The block barrier, or the cluster barrier when the tile spans a cluster.
template <int CL>
__device__ __forceinline__ void tile_barrier() {
  if constexpr (CL > 0) cluster_barrier();
  else __syncthreads();
}

// Sum over tile axes q in [q0, q1) of the partners of register pair j. The
// pair index of register j is pp = tid | (j << LOGT): tile bit 0 is inside
// the pair, bits 1..5 are lane bits (shuffles), bits 6..LOGT are warp bits
// (exchange tile sx in shared memory), and bits above index the thread's own
// registers v[]. Every loop is unrolled at compile time; [q0, q1) only
// predicates whole axes.
// Accumulator of an amplitude pair's bit-flip partners. Plain: packed adds.
// Compensated (FP32, COMP): each component is a TwoSum (Knuth's error-free
// addition) pair (s, e) whose error term e collects the rounding of every
// addition, so the partner sum is accurate to about one rounding instead of
// about sqrt(n) of them.
template <typename R, bool COMP> struct PartnerSum {
  Pair<R> acc = pzero<R>();
  __device__ __forceinline__ void add(const Pair<R>& v) { padd(acc, v); }
  __device__ __forceinline__ Pair<R> value() const { return acc; }
};
__device__ __forceinline__ void two_sum(float& s, float& e, float v) {
  const float t = __fadd_rn(s, v);
  const float bp = __fsub_rn(t, s);
  e = __fadd_rn(e, __fadd_rn(__fsub_rn(s, __fsub_rn(t, bp)), __fsub_rn(v, bp)));
  s = t;
}
template <> struct PartnerSum<float, true> {
  V4<float> s{0.0f, 0.0f, 0.0f, 0.0f}, e{0.0f, 0.0f, 0.0f, 0.0f};
  __device__ __forceinline__ void add(const Pair<float>& p) {
    const V4<float> v = to4(p);
    two_sum(s.x, e.x, v.x);
    two_sum(s.y, e.y, v.y);
    two_sum(s.z, e.z, v.z);
    two_sum(s.w, e.w, v.w);
  }
  __device__ __forceinline__ Pair<float> value() const {
    return from4(V4<float>{__fadd_rn(s.x, e.x), __fadd_rn(s.y, e.y), __fadd_rn(s.z, e.z),
                           __fadd_rn(s.w, e.w)});
  }
};

// LS: the lane axes are read from the exchange tile too (one 16-byte shared
// load per partner pair instead of four 32-bit shuffles: the same bytes
// through the shared-memory pipe, a quarter of the instructions).
template <typename R, int LT, int LOGT, int RP, bool LS = false, bool COMP = false>
__device__ __forceinline__ PartnerSum<R, COMP> axis_sum(const Pair<R> (&v)[RP], int j,
                                                       const R* sx, int q0, int q1,
                                                       int tid) {
  PartnerSum<R, COMP> acc;
  if (q0 <= 0) acc.add(pswap<R>(v[j]));
  const int pp = tid | (j << LOGT);
#pragma unroll
  for (int q = 1; q <= 5 && q < LT; q++)
    if (q >= q0 && q < q1) {
      if constexpr (LS) acc.add(pld(sx + 4 * (pp ^ (1 << (q - 1)))));
      else acc.add(pshfl(v[j], 1 << (q - 1)));
    }
#pragma unroll
  for (int q = 6; q <= LOGT && q < LT; q++)
    if (q >= q0 && q < q1) acc.add(pld(sx + 4 * (pp ^ (1 << (q - 1)))));
#pragma unroll
  for (int k = 0; (1 << k) < RP; k++) {
    const int q = LOGT + 1 + k;
    if (q >= q0 && q < q1) acc.add(v[j ^ (1 << k)]);
  }
  return acc;
}

// CTA shape of a tile of 2^LT amplitudes with at most TB threads: each
// thread owns RP pairs. Fewer threads own more pairs, so more tile axes are
// register axes (free) and fewer go through shuffles or shared memory.
template <int LT, int TB = kPassThreads> struct PassShape {
  static constexpr int kPairs = 1 << (LT - 1);
  static constexpr int kThreads = kPairs < TB ? kPairs : TB;
  static constexpr int kRP = kPairs / kThreads;
  static constexpr int kLogT = kThreads >= 512 ? 9 : kThreads >= 256 ? 8 : kThreads >= 128 ? 7 : kThreads >= 64 ? 6 : 5;
  // With RP >= 8 a thread has the registers to keep P_r (the partial read by
  // the finish) in registers; smaller RP stages it in shared memory.
  static constexpr bool kStageP = kRP < 8;
  template <typename R, bool StageP = kStageP>
  static constexpr size_t smem() {
    return (size_t)kPairs * ((StageP ? 3 : 2) * 4 * sizeof(R) + sizeof(float2));
  }
};

// Two CTAs per SM in FP32 (64 registers); FP64 pairs need twice the
// registers, so FP64 allows one CTA per SM at up to 128 registers.
// CL > 0: the tiling's tile spans a cluster of 2^CL CTAs (tile bits
// [LT, LT + CL) are the CTA's cluster rank); partners along those bits are
// read from the other CTAs' exchange tiles, and every barrier that guards the
// exchange tile is a cluster barrier. All CTAs of a cluster belong to the
// same walk and term, so they take the same path through every barrier.
// Register budget: 64 per thread when P is staged in shared memory (two
// 512-thread CTAs per SM), 128 when it is kept in registers; FP64 and cluster
// tiles take one CTA per SM.
template <int LT, int TB, bool FP32, int CL>
constexpr int pass_min_blocks() {
  using S = PassShape<LT, TB>;
  if (!FP32 || CL > 0) return 1;
  const int per_cta = S::kThreads * (S::kStageP ? 64 : 128);
  return 65536 / per_cta > 1 ? 65536 / per_cta : 1;
}

// TMA: in T1 passes (contiguous tiles) the tile's b_{r+1} (straight into the
// exchange tile), P_r, psi and D arrive by four bulk copies issued by one
// thread on one mbarrier, instead of per-thread loads and cp.async; P is then
// always staged in shared memory. T2 tiles (2^(LT-4) rows of 16 amplitudes)
// keep the per-thread path: one bulk copy per 64-128 byte row measured 2.6x
// slower than cp.async.
// COMP: the partner sums are compensated (PartnerSum<float, true>): the
// FP32-compensated precision mode.
// X2: a second exchange tile: b_r is written to its own tile without first
// waiting for every reader of b_{r+1}'s tile (one block barrier fewer per
// pass) at the cost of 16 B of shared memory per amplitude. Shapes with P in
// registers (8 pairs per thread) only, where it still leaves two CTAs per
// SM at the 2^12 tile.
// pass_tile is one CTA's share of one pass: term r of walk W in tiling
// `tiling` (1 or 2), on the CTA's tile `bx` (the x block index: tile and,
// with CL > 0, cluster rank).
template <typename R, int LT, int CL, int TB, bool LS = false, bool TMA = false,
          bool COMP = false, bool X2 = false>
__device__ __forceinline__ void pass_tile(const PassParams& p, const PassWalk& W, const int r,
                                          const int tiling, const unsigned bx) {
  using S = PassShape<LT, TB>;
  constexpr int RP = S::kRP, LOGT = S::kLogT, T = S::kThreads;
  constexpr bool kStageP = S::kStageP || TMA;
  static_assert(!TMA || CL == 0, "bulk-copy staging is for single-CTA tiles");
  static_assert(!X2 || (!kStageP && CL == 0 && !TMA && !LS),
                "the second exchange tile is for shapes with P in registers and a single-CTA tile");
  constexpr int LL = LT + CL;  // tile bits of the tiling
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double s_red[32];
  __shared__ __align__(8) unsigned long long tma_bar;
  const int n = p.n, a = p.a;
  const int tid = threadIdx.x;
  R* sx = reinterpret_cast<R*>(smem_raw);  // exchange tile: 2^LT complex
  R* sp = sx + 4 * S::kPairs;              // staged P_r, [j][tid] pairs
  R* ss = kStageP ? sp + 4 * S::kPairs : sp;  // staged psi
  float2* sd = reinterpret_cast<float2*>(ss + 4 * S::kPairs);  // staged D
  // X2: b_r's exchange tile, after the staged D
  R* sx2 = X2 ? reinterpret_cast<R*>(sd + S::kPairs) : sx;
  // Global amplitude index of register pair j: g0 + j * gstride (32-bit: n <= 30).
  // For a 1-D cluster the cluster rank is bx mod 2^CL.
  const unsigned rank = CL > 0 ? (bx & ((1u << CL) - 1u)) : 0u;
  const int nu = n - (2 * LL - a) > 0 ? n - (2 * LL - a) : 0;
  // Launch order of the tiles: the tile bits of the nu axes read from global
  // memory come first, so that the tiles whose amplitudes a tile reads are
  // processed at about the same time and those reads hit L2. In T1 they are
  // the lowest tile bits already; in T2 they are the top nu of the n - LL
  // tile bits, rotated down here.
  unsigned tile = bx >> CL;
  if (tiling == 2 && nu > 0) {
    const int tb = n - LL;
    tile = ((tile & ((1u << nu) - 1u)) << (tb - nu)) | (tile >> nu);
  }
  const unsigned pos0 = (rank << LT) | (2u * tid);  // tile position of pair 0
  unsigned g0, gstride;
  if (tiling == 1) {
    g0 = (tile << LL) | pos0;
    gstride = 1u << (LOGT + 1);
  } else {
    const unsigned amask = (1u << a) - 1u;
    g0 = (pos0 & amask) | (tile << a) | ((pos0 >> a) << (n - LL + a));
    gstride = 1u << (LOGT + 1 + n - LL);
  }
  // Exchange tiles of the cluster's other CTAs, one per rank bit.
  unsigned peer_sx[CL > 0 ? CL : 1];
#pragma unroll
  for (int k = 0; k < CL; k++) peer_sx[k] = cluster_addr(sx, rank ^ (1u << k));
  const R* bin = reinterpret_cast<const R*>(W.bin);  // may alias bout (nu == 0)
  R* bout = reinterpret_cast<R*>(W.bout);
  R* __restrict__ part = reinterpret_cast<R*>(W.part);
  const R* __restrict__ psi = reinterpret_cast<const R*>(W.psi);
  const float* __restrict__ hp = W.hp;
  const int K = W.K;
  const bool first = r == K - 1;
  const bool uni = W.psi_uniform;
  // Finish axes (tile bits): T1 -> [a, min(L, n-L+a)), T2 -> [max(2L-n, a), L)
  // with L = LL; axes [LL, LL+nu) are in neither tiling and come from global
  // memory.
  const int fb0 = tiling == 1 ? a : max(2 * LL - n, a);
  const int fb1 = tiling == 1 ? min(LL, n - LL + a) : LL;
  // Partners along the rank bits [LT, LL) that lie in [q0, q1): all of a
  // pair's remote loads are issued together (before the local partner sums,
  // which hide their latency) and added afterwards.
  struct Remote {
    Pair<R> v[CL > 0 ? CL : 1];
  };
  auto cluster_load = [&](int j, int q0, int q1) {
    Remote rv;
    const unsigned off = (unsigned)(4 * sizeof(R)) * (unsigned)(tid | (j << LOGT));
#pragma unroll
    for (int k = 0; k < CL; k++)
      if (LT + k >= q0 && LT + k < q1) rv.v[k] = pld_cluster((const R*)nullptr, peer_sx[k] + off);
    return rv;
  };
  auto cluster_add = [&](PartnerSum<R, COMP>& acc, const Remote& rv, int q0, int q1) {
#pragma unroll
    for (int k = 0; k < CL; k++)
      if (LT + k >= q0 && LT + k < q1) acc.add(rv.v[k]);
  };

  Pair<R> va[RP];  // b_{r+1}
  Pair<R> pv[kStageP ? 1 : RP];  // P_r when kept in registers
  const bool bulk = TMA && tiling == 1;
  if (bulk) {
    // The tile as rows of contiguous amplitudes (T1: one row of 2^LT).
    const int row_log = tiling == 1 ? LT : a;
    const unsigned rows = 1u << (LT - row_log);
    const unsigned row_amps = 1u << row_log;
    const unsigned vec_bytes = row_amps * 2u * (unsigned)sizeof(R);
    const unsigned d_bytes = row_amps * (unsigned)sizeof(float);
    if (tid == 0) mbar_init(&tma_bar, 1);
    __syncthreads();
    if (tid < 32) {
      if (tid == 0) {
        const unsigned per_row = (first ? 0u : 2u * vec_bytes) + (uni ? 0u : vec_bytes) + d_bytes;
        mbar_arrive_expect_tx(&tma_bar, rows * per_row + (p.test_stall ? 16u : 0u));
      }
      __syncwarp();
      for (unsigned k = tid; k < rows; k += 32) {
        const unsigned g = tiling == 1 ? (tile << LT)
                                         : ((tile << a) | (k << (n - LT + a)));
        const unsigned pos = k * row_amps;
        if (!first) {
          bulk_load(sx + 2 * (size_t)pos, bin + 2 * (size_t)g, vec_bytes, &tma_bar);
          bulk_load(sp + 2 * (size_t)pos, part + 2 * (size_t)g, vec_bytes, &tma_bar);
        }
        if (!uni) bulk_load(ss + 2 * (size_t)pos, psi + 2 * (size_t)g, vec_bytes, &tma_bar);
        bulk_load(reinterpret_cast<float*>(sd) + pos, hp + g, d_bytes, &tma_bar);
      }
    }
    const unsigned long long limit = p.wait_ns ? p.wait_ns : 200000000ull;
    const bool ok = mbar_wait_bounded(&tma_bar, 0, limit);
    if (__syncthreads_or(!ok)) {
      // Give up on this tile: report, wait (bounded) for any copy still in
      // flight into this CTA's shared memory, and leave.
      if (tid == 0 && p.err) atomicOr(p.err, 1u);
      mbar_wait_bounded(&tma_bar, 0, limit);
      __syncthreads();
      return;
    }
#pragma unroll
    for (int j = 0; j < RP; j++) va[j] = first ? pzero<R>() : pld(sx + 4 * (tid | (j << LOGT)));
  } else {
    // Stage P_r (unless it goes to registers), psi and D for this thread's
    // own pairs.
#pragma unroll
    for (int j = 0; j < RP; j++) {
      const unsigned gi = g0 + j * gstride;
      const int o = j * T + tid;
      if (kStageP && !first) cp_async_pair<R>(sp + 4 * o, part + 2 * (size_t)gi);
      if (!uni) cp_async_pair<R>(ss + 4 * o, psi + 2 * (size_t)gi);
      cp_async8(sd + o, hp + gi);
    }
#pragma unroll
    for (int j = 0; j < RP; j++) {
      va[j] = first ? pzero<R>() : pld(bin + 2 * (size_t)(g0 + j * gstride));
      if constexpr (!kStageP) pv[j] = first ? pzero<R>() : pld(part + 2 * (size_t)(g0 + j * gstride));
    }
  }
  const double kap = W.kappa ? *W.kappa : 1.0;
  const R scale = (R)W.scale;
  const R gamma = (R)W.gamma;
  const R a_mid = (R)2 / scale, a_fin = (R)2 / ((R)2 * scale);
  const R psi0 = (R)W.psi0;
  Pair<R> vb[RP];  // b_r
  if (first) {
    const R cr = (R)((double)W.coef[r] * kap);
    if (!bulk) cp_async_wait_all();
#pragma unroll
    for (int j = 0; j < RP; j++) {
      const V4<R> pv = uni ? V4<R>{psi0, 0, psi0, 0} : ld4<R>(ss + 4 * (j * T + tid));
      vb[j] = from4(cpsi4<R>(cr, r & 1, pv));
    }
  } else {
    const R ag = (r == 0 ? a_fin : a_mid) * gamma;
    if (!bulk) {  // (with bulk copies the exchange tile already holds b_{r+1})
#pragma unroll
      for (int j = 0; j < RP; j++) pst(sx + 4 * (tid | (j << LOGT)), va[j]);
      tile_barrier<CL>();
      cp_async_wait_all();
    }
#pragma unroll
    for (int j = 0; j < RP; j++) {
      const Remote rv = cluster_load(j, fb0, fb1);
      PartnerSum<R, COMP> accp = axis_sum<R, LT, LOGT, RP, LS, COMP>(va, j, sx, fb0, fb1, tid);
      cluster_add(accp, rv, fb0, fb1);
      const unsigned gi = g0 + j * gstride;
      for (int u0 = 0; u0 < nu; u0 += 4) {
        Pair<R> gv[4];
#pragma unroll
        for (int u = 0; u < 4; u++)
          if (u0 + u < nu) gv[u] = pld(bin + 2 * (size_t)(gi ^ (1u << (LL + u0 + u))));
#pragma unroll
        for (int u = 0; u < 4; u++)
          if (u0 + u < nu) accp.add(gv[u]);
      }
      const V4<R> acc = to4(accp.value());
      V4<R> pr;
      if constexpr (kStageP) pr = ld4<R>(sp + 4 * (j * T + tid));
      else pr = to4(pv[kStageP ? 0 : j]);
      vb[j] = from4(V4<R>{fma(-ag, acc.x, pr.x), fma(-ag, acc.y, pr.y),
                          fma(-ag, acc.z, pr.z), fma(-ag, acc.w, pr.w)});
    }
  }
#pragma unroll
  for (int j = 0; j < RP; j++) pst(bout + 2 * (size_t)(g0 + j * gstride), vb[j]);
  if constexpr (sizeof(R) == 4) {
    if (W.real_out) {  // basis passes: the real parts as a real vector too
#pragma unroll
      for (int j = 0; j < RP; j++) {
        const V4<R> v = to4(vb[j]);
        *reinterpret_cast<float2*>(W.real_out + (g0 + j * gstride)) = make_float2(v.x, v.z);
      }
    }
  }
  if (r == 0) {
    double nrm = 0.0;
#pragma unroll
    for (int j = 0; j < RP; j++) {
      const V4<R> v = to4(vb[j]);
      nrm += (double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z + (double)v.w * v.w;
    }
    const double sum = block_sum<R>(nrm, s_red);
    if (tid == 0) W.norm_part[bx] = sum;
    if constexpr (CL > 0) cluster_barrier();  // peers may still read sx
    return;
  }
  // Start P_{r-1} = c psi + a (D b_r - gamma X_Z b_r) - b_{r+1} over all tile axes.
  // (X2: b_r goes to its own exchange tile, so no reader of b_{r+1}'s tile
  // has to be waited for.)
  if constexpr (!X2) tile_barrier<CL>();  // every reader of sx (this CTA and its peers) is done
#pragma unroll
  for (int j = 0; j < RP; j++) pst(sx2 + 4 * (tid | (j << LOGT)), vb[j]);
  tile_barrier<CL>();
  const int rm = r - 1;
  const R am = rm == 0 ? a_fin : a_mid;
  const R cm = (R)((double)W.coef[rm] * kap);
#pragma unroll
  for (int j = 0; j < RP; j++) {
    const Remote rv = cluster_load(j, 0, LL);
    PartnerSum<R, COMP> accp = axis_sum<R, LT, LOGT, RP, LS, COMP>(vb, j, sx2, 0, LT, tid);
    cluster_add(accp, rv, 0, LL);
    const V4<R> acc = to4(accp.value());
    const int o = j * T + tid;
    const V4<R> pv = uni ? V4<R>{psi0, 0, psi0, 0} : ld4<R>(ss + 4 * o);
    const float2 d = sd[o];
    const V4<R> b = to4(vb[j]);
    const V4<R> b1 = to4(va[j]);
    V4<R> out = cpsi4<R>(cm, rm & 1, pv);
    const R d0 = (R)d.x, d1 = (R)d.y;
    out.x = fma(am, fma(d0, b.x, -gamma * acc.x), out.x - b1.x);
    out.y = fma(am, fma(d0, b.y, -gamma * acc.y), out.y - b1.y);
    out.z = fma(am, fma(d1, b.z, -gamma * acc.z), out.z - b1.z);
    out.w = fma(am, fma(d1, b.w, -gamma * acc.w), out.w - b1.w);
    st4<R>(part + 2 * (size_t)(g0 + j * gstride), out);
  }
  // A CTA's shared memory must outlive its peers' reads of it.
  if constexpr (CL > 0) cluster_barrier();
}

// One pass (term W.r) for each walk of the launch: blockIdx.y is the walk,
// blockIdx.x the tile (and cluster rank).
template <typename R, int LT, int CL, int TB, bool LS = false, bool TMA = false,
          bool COMP = false, bool X2 = false>
__global__ void __launch_bounds__(PassShape<LT, TB>::kThreads,
                                  pass_min_blocks<LT, TB, sizeof(R) == 4, CL>())
    pass_kernel(PassParams p) {
  const PassWalk& W = p.walk[blockIdx.y];
  if (!W.active) return;
  pass_tile<R, LT, CL, TB, LS, TMA, COMP, X2>(p, W, W.r, p.tiling, blockIdx.x);
}

// Chain launch (small n, no axis read from global memory): a thread-block
// cluster of 2^(n-LT) CTAs, one per tile, runs all K terms of one walk-stage
// (blockIdx.y the walk, b and P updated in place), passes r = K-1 .. 0 in
// tilings 1 (even r) and 2 (odd r). A cluster barrier (arrive.release /
// wait.acquire at cluster scope, which orders the global-memory writes of
// every thread of the cluster) separates consecutive passes, so that each
// pass reads the tiles its peers wrote in the one before. One launch
// replaces K single-pass launches; the arithmetic is the same.
template <typename R, int LT>
__global__ void __launch_bounds__(PassShape<LT>::kThreads,
                                  pass_min_blocks<LT, kPassThreads, sizeof(R) == 4, 0>())
    pass_chain_kernel(PassParams p) {
  const PassWalk& W = p.walk[blockIdx.y];
  if (!W.active) return;  // every CTA of the cluster has the same walk
  for (int r = W.K - 1; r >= 0; r--) {
    pass_tile<R, LT, 0, kPassThreads>(p, W, r, (r & 1) ? 2 : 1, blockIdx.x);
    if (r > 0) cluster_barrier();
  }
}

// The shared bases are streamed (hundreds of MB per walk group at n = 20)
// with evict-first loads (__ldcs), so that they do not push the walks'
// L2-resident states out of the cache for the passes running beside them.

// Recombination from a shared basis for G walks (FP32). Block b covers
// amplitudes [b 2^L, (b+1) 2^L) and forms, per walk, v = sum_j d_j w_j
// (d_0 = c_0 - c_2/2, d_j = (c_j - c_{j+2})/2; real for even j, imaginary for
// odd j) from the real basis vectors w_j, each read once for all G walks
// with eight vectors in flight per thread.
//  * Stage-1 recombination (kProject false): v is the walk's stage output;
//    it is written and the block's |v|^2 is left in norm_part[b].
//  * Last-stage projection (kProject true): the walk's psi_out[E_loc] =
//    sum_j d_j <w_j, psi> = <v, psi> (w_j real), so v is dotted with the
//    walk's stage input psi in FP64 and the block's sum is left in
//    part[g][b] (re, im); project_final_kernel adds the blocks.
// All sums run in a fixed order (deterministic), and per walk the
// arithmetic does not depend on G.
template <int G, bool kProject, typename Params>
__global__ void __launch_bounds__(256) recombine_kernel(Params p) {
  __shared__ float sd[G][kMaxBasis];
  __shared__ double s_red[32];
  const int Kb = p.Kb;
  for (int e = threadIdx.x; e < G * Kb; e += blockDim.x) {
    const int g = e / Kb, j = e % Kb;
    const auto& W = p.walk[g];
    const float cj = j < W.K ? W.coef[j] : 0.0f;
    const float cj2 = j + 2 < W.K ? W.coef[j + 2] : 0.0f;
    sd[g][j] = j == 0 ? cj - 0.5f * cj2 : 0.5f * (cj - cj2);
  }
  __syncthreads();
  const size_t N = (size_t)1 << p.n;
  const size_t chunk = (size_t)1 << p.L;
  const size_t base = (size_t)blockIdx.x * chunk;
  const float* __restrict__ basis = reinterpret_cast<const float*>(p.basis);
  double acc[G][2];  // |v|^2 (stage 1) or <v, psi> (re, im; projection)
#pragma unroll
  for (int g = 0; g < G; g++) acc[g][0] = acc[g][1] = 0.0;
  for (size_t i = base + 4 * threadIdx.x; i < base + chunk; i += 4 * blockDim.x) {
    float re[G][4], im[G][4];
#pragma unroll
    for (int g = 0; g < G; g++)
#pragma unroll
      for (int k = 0; k < 4; k++) re[g][k] = im[g][k] = 0.0f;
    auto accumulate = [&](const float4& w, int j, bool odd) {
#pragma unroll
      for (int g = 0; g < G; g++) {
        const float d = sd[g][j];
        float* a = odd ? im[g] : re[g];
        a[0] = fmaf(d, w.x, a[0]);
        a[1] = fmaf(d, w.y, a[1]);
        a[2] = fmaf(d, w.z, a[2]);
        a[3] = fmaf(d, w.w, a[3]);
      }
    };
    int j = 0;
    for (; j + 8 <= Kb; j += 8) {
      float4 w[8];
#pragma unroll
      for (int u = 0; u < 8; u++)
        w[u] = __ldcs(reinterpret_cast<const float4*>(basis + (size_t)(j + u) * N + i));
#pragma unroll
      for (int u = 0; u < 8; u++) accumulate(w[u], j + u, u & 1);  // j is even
    }
    for (; j < Kb; j++)
      accumulate(__ldcs(reinterpret_cast<const float4*>(basis + (size_t)j * N + i)), j, j & 1);
#pragma unroll
    for (int g = 0; g < G; g++) {
      if constexpr (kProject) {
        const float* psi = reinterpret_cast<const float*>(p.walk[g].psi) + 2 * i;
        const float4 a = __ldcs(reinterpret_cast<const float4*>(psi));
        const float4 b = __ldcs(reinterpret_cast<const float4*>(psi + 4));
        const float pr[4] = {a.x, a.z, b.x, b.z}, pi[4] = {a.y, a.w, b.y, b.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {  // (re + i im)(pr + i pi)
          acc[g][0] = fma((double)re[g][k], (double)pr[k], acc[g][0]);
          acc[g][0] = fma(-(double)im[g][k], (double)pi[k], acc[g][0]);
          acc[g][1] = fma((double)re[g][k], (double)pi[k], acc[g][1]);
          acc[g][1] = fma((double)im[g][k], (double)pr[k], acc[g][1]);
        }
      } else {
        float4* out = reinterpret_cast<float4*>(reinterpret_cast<float*>(p.walk[g].out) + 2 * i);
        out[0] = make_float4(re[g][0], im[g][0], re[g][1], im[g][1]);
        out[1] = make_float4(re[g][2], im[g][2], re[g][3], im[g][3]);
#pragma unroll
        for (int k = 0; k < 4; k++)
          acc[g][0] += (double)re[g][k] * re[g][k] + (double)im[g][k] * im[g][k];
      }
    }
  }
#pragma unroll
  for (int g = 0; g < G; g++) {
    if constexpr (kProject) {
      const size_t blocks = N >> p.L;
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const double sum = block_sum<float>(acc[g][c], s_red);
        if (threadIdx.x == 0) p.part[((size_t)g * blocks + blockIdx.x) * 2 + c] = sum;
        __syncthreads();  // s_red is reused by the next sum
      }
    } else {
      const double sum = block_sum<float>(acc[g][0], s_red);
      if (threadIdx.x == 0) p.walk[g].norm_part[blockIdx.x] = sum;
      __syncthreads();  // s_red is reused by the next walk's sum
    }
  }
}

// Last-stage projection, final: one block per walk sums the walk's block
// partials of <v, psi> in a fixed order (strided per thread, then the block
// sum) and writes P = |<v, psi>|^2 kappa^2.
__global__ void __launch_bounds__(256) project_final_kernel(ProjectParams p) {
  __shared__ double s_red[32];
  const int g = blockIdx.x;
  const ProjectWalk& W = p.walk[g];
  const size_t blocks = ((size_t)1 << p.n) >> p.L;
  const double* part = p.part + (size_t)g * blocks * 2;
  double re = 0.0, im = 0.0;
  for (size_t b = threadIdx.x; b < blocks; b += blockDim.x) {
    re += part[2 * b];
    im += part[2 * b + 1];
  }
  re = block_sum<float>(re, s_red);
  __syncthreads();  // s_red is reused
  im = block_sum<float>(im, s_red);
  if (threadIdx.x == 0) {
    const double kap = W.kappa ? *W.kappa : 1.0;
    *W.p_out = (re * re + im * im) * kap * kap;
  }
}

// psi = e_{E_loc} (complex FP32): the start vector of the last-stage basis.
__global__ void unit_eloc_kernel(float2* psi, const DiagOut* diag) {
  psi[diag->e_loc] = make_float2(1.0f, 0.0f);
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


__global__ void mean_kernel(const double* p_sample, const int* p_off,
                            const int* p_cnt, int count, double* p_mean) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  double s = 0.0;
  const int o = p_off[i], c = p_cnt[i];
  for (int k = 0; k < c; k++) s += p_sample[o + k];
  p_mean[i] = s / c;
}

// ---------------------------------------------------------------------------
// Real unit-coefficient chains (see RealChainParams): pass_kernel's tilings,
// thread layout and partner-sum order on real vectors. A register "pair" is
// two neighbouring real amplitudes packed in 64 bits (summed with
// add.rn.f32x2, exchanged with one 64-bit shuffle); the exchange tiles hold
// 2^LT floats. 256 threads, P in registers, D staged by cp.async, two
// exchange tiles (b_{r+1}'s and b_r's) so that no barrier separates the
// last read of one from the first write of the other.
template <int LT, int TB = 256> struct RealShape {
  static constexpr int kPairs = 1 << (LT - 1);
  static constexpr int kThreads = kPairs < TB ? kPairs : TB;
  static constexpr int kRP = kPairs / kThreads;
  static constexpr int kLogT = kThreads >= 1024  ? 10
                               : kThreads >= 512 ? 9
                               : kThreads >= 256 ? 8
                               : kThreads >= 128 ? 7
                               : kThreads >= 64  ? 6
                                                 : 5;
  static constexpr size_t smem() { return (size_t)kPairs * (2 * 8 + 8); }
};

__device__ __forceinline__ unsigned long long rpair_swap(unsigned long long v) {
  return (v >> 32) | (v << 32);
}
__device__ __forceinline__ void rpair_add(unsigned long long& acc, unsigned long long v) {
  asm("add.rn.f32x2 %0, %0, %1;" : "+l"(acc) : "l"(v));
}

// Partner sum over tile axes [q0, q1) of register pair j (pass_kernel's
// axis_sum on real pairs: the same axes in the same order).
template <int LT, int LOGT, int RP>
__device__ __forceinline__ unsigned long long real_axis_sum(const unsigned long long (&v)[RP],
                                                            int j, const unsigned long long* sx,
                                                            int q0, int q1, int tid) {
  unsigned long long acc = 0ull;
  if (q0 <= 0) rpair_add(acc, rpair_swap(v[j]));
  const int pp = tid | (j << LOGT);
#pragma unroll
  for (int q = 1; q <= 5 && q < LT; q++)
    if (q >= q0 && q < q1) rpair_add(acc, __shfl_xor_sync(0xffffffffu, v[j], 1 << (q - 1)));
#pragma unroll
  for (int q = 6; q <= LOGT && q < LT; q++)
    if (q >= q0 && q < q1) rpair_add(acc, sx[pp ^ (1 << (q - 1))]);
#pragma unroll
  for (int k = 0; (1 << k) < RP; k++) {
    const int q = LOGT + 1 + k;
    if (q >= q0 && q < q1) rpair_add(acc, v[j ^ (1 << k)]);
  }
  return acc;
}

__device__ __forceinline__ float2 u2f(unsigned long long v) {
  float2 f;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(f.x), "=f"(f.y) : "l"(v));
  return f;
}
__device__ __forceinline__ unsigned long long f2u(float2 f) {
  unsigned long long v;
  asm("mov.b64 %0, {%1, %2};" : "=l"(v) : "f"(f.x), "f"(f.y));
  return v;
}

// real_tile is one CTA's share of one real pass: tiling `tiling`, the
// chain's first pass when `first`, b_{r+1} read from `bin_` and b_r written
// to `bout_`, the partial P in place at `part_`, the start vector `start_`,
// on the CTA's tile `bx`. `half_finish` / `half_start`: the term this pass
// finishes / starts uses a = 1/onenorm instead of 2/onenorm (a chain of
// first-kind vectors T_j v: T_1 = H~ v).
template <int LT, int TB = 256>
__device__ __forceinline__ void real_tile(const RealChainParams& p, const int tiling,
                                          const bool first, const float* bin_, float* bout_,
                                          float* part_, const float* start_, const unsigned bx,
                                          const bool half_finish = false,
                                          const bool half_start = false) {
  using S = RealShape<LT, TB>;
  constexpr int RP = S::kRP, LOGT = S::kLogT, T = S::kThreads;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned long long* sx1 = reinterpret_cast<unsigned long long*>(smem_raw);  // b_{r+1}
  unsigned long long* sx2 = sx1 + S::kPairs;                                  // b_r
  float2* sd = reinterpret_cast<float2*>(sx2 + S::kPairs);                    // staged D
  const int n = p.n, a = p.a, tid = threadIdx.x;
  const int nu = n - (2 * LT - a) > 0 ? n - (2 * LT - a) : 0;
  unsigned tile = bx;
  if (tiling == 2 && nu > 0) {
    const int tb = n - LT;
    tile = ((tile & ((1u << nu) - 1u)) << (tb - nu)) | (tile >> nu);
  }
  const unsigned pos0 = 2u * tid;
  unsigned g0, gstride;
  if (tiling == 1) {
    g0 = (tile << LT) | pos0;
    gstride = 1u << (LOGT + 1);
  } else {
    const unsigned amask = (1u << a) - 1u;
    g0 = (pos0 & amask) | (tile << a) | ((pos0 >> a) << (n - LT + a));
    gstride = 1u << (LOGT + 1 + n - LT);
  }
  const int fb0 = tiling == 1 ? a : max(2 * LT - n, a);
  const int fb1 = tiling == 1 ? min(LT, n - LT + a) : LT;
  const float* __restrict__ hp = p.hp;
  const float* __restrict__ bin = bin_;
  float* __restrict__ part = part_;
#pragma unroll
  for (int j = 0; j < RP; j++) cp_async8(sd + (j * T + tid), hp + g0 + j * gstride);
  unsigned long long va[RP], vb[RP];
  const float am = 2.0f / p.scale;
  const float afin = half_finish ? 1.0f / p.scale : am;  // the term finished here
  const float ast = half_start ? 1.0f / p.scale : am;    // the term started here
  const float gamma = p.gamma;
  if (first) {
#pragma unroll
    for (int j = 0; j < RP; j++) {
      va[j] = 0ull;
      vb[j] = p.start_uniform ? f2u(make_float2(p.psi0, p.psi0))
                              : *reinterpret_cast<const unsigned long long*>(start_ + g0 + j * gstride);
    }
    cp_async_wait_all();
  } else {
    unsigned long long pv[RP];
#pragma unroll
    for (int j = 0; j < RP; j++) {
      va[j] = *reinterpret_cast<const unsigned long long*>(bin + g0 + j * gstride);
      pv[j] = *reinterpret_cast<const unsigned long long*>(part + g0 + j * gstride);
    }
#pragma unroll
    for (int j = 0; j < RP; j++) sx1[tid | (j << LOGT)] = va[j];
    __syncthreads();
    cp_async_wait_all();
    const float ag = afin * gamma;
#pragma unroll
    for (int j = 0; j < RP; j++) {
      unsigned long long acc = real_axis_sum<LT, LOGT, RP>(va, j, sx1, fb0, fb1, tid);
      const unsigned gi = g0 + j * gstride;
      for (int u0 = 0; u0 < nu; u0 += 4) {
        unsigned long long gv[4];
#pragma unroll
        for (int u = 0; u < 4; u++)
          if (u0 + u < nu)
            gv[u] = *reinterpret_cast<const unsigned long long*>(bin + (gi ^ (1u << (LT + u0 + u))));
#pragma unroll
        for (int u = 0; u < 4; u++)
          if (u0 + u < nu) rpair_add(acc, gv[u]);
      }
      const float2 s = u2f(acc), pr = u2f(pv[j]);
      vb[j] = f2u(make_float2(fmaf(-ag, s.x, pr.x), fmaf(-ag, s.y, pr.y)));
    }
  }
#pragma unroll
  for (int j = 0; j < RP; j++)
    *reinterpret_cast<unsigned long long*>(bout_ + g0 + j * gstride) = vb[j];
  // Start P_{r-1} = a (D b_r - gamma X_Z b_r) - b_{r+1} over all tile axes.
#pragma unroll
  for (int j = 0; j < RP; j++) sx2[tid | (j << LOGT)] = vb[j];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < RP; j++) {
    const float2 s = u2f(real_axis_sum<LT, LOGT, RP>(vb, j, sx2, 0, LT, tid));
    const float2 d = sd[j * T + tid];
    const float2 b = u2f(vb[j]), b1 = u2f(va[j]);
    // pass_kernel's arithmetic with a zero coefficient: (0 - b1) + a (...)
    const float2 out = make_float2(fmaf(ast, fmaf(d.x, b.x, -gamma * s.x), 0.0f - b1.x),
                                   fmaf(ast, fmaf(d.y, b.y, -gamma * s.y), 0.0f - b1.y));
    *reinterpret_cast<unsigned long long*>(part + g0 + j * gstride) = f2u(out);
  }
}

// One real pass (p.tiling, p.first, p.bin -> p.bout); blockIdx.x is the tile.
// TB caps the CTA's threads (128 to 1024; see real_threads).
template <int LT, int TB = 256>
__global__ void __launch_bounds__(RealShape<LT, TB>::kThreads)
    real_pass_kernel(RealChainParams p) {
  real_tile<LT, TB>(p, p.tiling, p.first != 0, p.bin, p.bout, p.part, p.start, blockIdx.x,
                    p.half_finish != 0, p.half_start != 0);
}

// Chain launch of whole real chains (small n, no axis read from global
// memory): per chain (blockIdx.y; b.chain[] gives its start vector, partial
// P and outputs) a thread-block cluster of 2^(n-LT) CTAs, one per tile, runs
// the passes j = 0 .. K-1 (term r = R - j, tiling 2 for odd r), pass j
// writing b_r to out_base[j & 1] + (j >> 1) out_stride and reading b_{r+1}
// from the previous pass's output; cluster barriers separate the passes (see
// pass_chain_kernel). The chains of a launch share n, K, R and the operator.
template <int LT>
__global__ void __launch_bounds__(RealShape<LT>::kThreads) real_chain_kernel(RealChainBatch b) {
  const RealChainParams& p = b.p;
  const RealChainDesc& c = b.chain[blockIdx.y];
  for (int j = 0; j < p.K; j++) {
    const int r = p.R - j;
    const float* bin =
        j > 0 ? c.out_base[(j - 1) & 1] + (size_t)((j - 1) >> 1) * (size_t)p.out_stride : nullptr;
    float* bout = c.out_base[j & 1] + (size_t)(j >> 1) * (size_t)p.out_stride;
    real_tile<LT>(p, (r & 1) ? 2 : 1, j == 0, bin, bout, c.part, c.start, blockIdx.x,
                  p.tbasis && j == 1, p.tbasis && j == 0);
    if (j + 1 < p.K) cluster_barrier();
  }
}

// One pass (term r = R - j) of each of b.chains real chains: blockIdx.y is
// the chain (its start vector, partial P and outputs from b.chain[]),
// blockIdx.x the tile. Axes in neither tiling are read from global memory as
// in real_pass_kernel (b_{r+1} and b_r are different vectors).
template <int LT, int TB = 256>
__global__ void __launch_bounds__(RealShape<LT, TB>::kThreads)
    real_batch_kernel(RealChainBatch b, int j) {
  const RealChainParams& p = b.p;
  const RealChainDesc& c = b.chain[blockIdx.y];
  const int r = p.R - j;
  const float* bin =
      j > 0 ? c.out_base[(j - 1) & 1] + (size_t)((j - 1) >> 1) * (size_t)p.out_stride : nullptr;
  float* bout = c.out_base[j & 1] + (size_t)(j >> 1) * (size_t)p.out_stride;
  real_tile<LT, TB>(p, (r & 1) ? 2 : 1, j == 0, bin, bout, c.part, c.start, blockIdx.x,
                p.tbasis && j == 1, p.tbasis && j == 0);
}

__global__ void unit_eloc_real_kernel(float* v, const DiagOut* diag) { v[diag->e_loc] = 1.0f; }

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
  // The shared-memory opt-in is made per device on the first launch of each
  // size (never while a stream is being captured after the first eager
  // launch).
  if (precision == 0) {
    const size_t sm = resident_smem<float>(max_n);
    cudaError_t e = ensure_smem_optin((const void*)resident_kernel<float>, sm, false);
    if (e != cudaSuccess) return e;
    resident_kernel<float><<<count, threads, sm, stream>>>(a);
  } else {
    const size_t sm = resident_smem<double>(max_n);
    cudaError_t e = ensure_smem_optin((const void*)resident_kernel<double>, sm, false);
    if (e != cudaSuccess) return e;
    resident_kernel<double><<<count, threads, sm, stream>>>(a);
  }
  return cudaGetLastError();
}

namespace {
// Largest cluster log (<= 4) whose pass kernel can be resident on this
// device, for the precision's widest tile; 0 when clusters are unavailable.
template <typename R, int LT, int CL>
int cluster_fits() {
  using S = PassShape<LT>;
  const size_t smem = S::template smem<R>();
  if (ensure_smem_optin((const void*)pass_kernel<R, LT, CL, kPassThreads>, smem, CL > 3) !=
      cudaSuccess)
    return 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(1u << CL, 1, 1);
  cfg.blockDim = dim3(S::kThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 1u << CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, pass_kernel<R, LT, CL, kPassThreads>, &cfg) !=
      cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  return clusters > 0;
}

template <typename R, int LT>
int max_cluster_log() {
  // Per precision, probed once (one device type per process); the static's
  // initialisation is thread-safe.
  static const int cached = [] {
    int c = 0;
    if (cluster_fits<R, LT, 1>()) c = 1;
    if (c == 1 && cluster_fits<R, LT, 2>()) c = 2;
    if (c == 2 && cluster_fits<R, LT, 3>()) c = 3;
    if (c == 3 && cluster_fits<R, LT, 4>()) c = 4;
    return c;
  }();
  return cached;
}
}  // namespace

PassGeomHost pass_geom(int precision, int n, int lmax, int threads, int lane_smem, int tma,
                        int cluster) {
  // Tile: 2^L amplitudes of b_{r+1} and 2^L of b_r in shared memory
  // (64 KB at L = 12 in FP32, 3 CTAs per SM). Rows of 2^a = 16 amplitudes
  // (128 bytes in FP32) keep T2 loads coalesced. L is chosen so the two
  // tilings cover every axis when possible (2L - a >= n); above that, at the
  // widest compiled tile, a tiling's tile spans a cluster of 2^C CTAs
  // (2(L+C) - a >= n up to C = 4) before any axis is left to global memory;
  // cluster = 0 keeps single-CTA tiles there and reads the remaining axes
  // from global memory.
  static const int env = [] {  // read once; thread-safe initialisation
    const char* e = getenv("MQW_PASS_TILE_LOG");
    return e ? atoi(e) : -1;
  }();
  int Lmax = precision == 0 ? 12 : 11;
  if (env >= 6 && env <= 13) Lmax = env;
  if (lmax >= 6 && lmax <= 13) Lmax = lmax;
  // Compiled tile sizes: up to 2^13 in FP32 (the 2^13 tile is one 512-thread
  // CTA per SM with 8 pairs per thread), 2^11 in FP64. Clusters and the
  // 256-thread shape exist at the default widest tile `cap`.
  const int top = precision == 0 ? 13 : 11;
  const int cap = precision == 0 ? 12 : 11;
  if (Lmax > top) Lmax = top;
  // Threads own pairs along the top tile axes, lanes cover tile axes 1..5,
  // so a tile has at least 6 axes (n >= 6 on the grid path).
  PassGeomHost g;
  g.a = 4;
  g.C = 0;
  int L = (n + g.a + 1) / 2;
  if (L < 6) L = 6;
  if (L > Lmax) L = Lmax;
  if (L > n) L = n;
  g.L = L;
  g.nu = n - (2 * L - g.a);
  if (g.nu > 0 && L == cap && cluster) {
    const int cmax = precision == 0 ? max_cluster_log<float, 12>() : max_cluster_log<double, 11>();
    g.C = (g.nu + 1) / 2;
    if (g.C > cmax) g.C = cmax;
    g.nu = n - (2 * (L + g.C) - g.a);
  }
  if (g.nu < 0) g.nu = 0;
  // The 256-thread CTA exists for the widest single-CTA tile only.
  g.threads = (threads == 256 && L == cap && g.C == 0) ? 256 : 0;
  // Lane axes through shared memory: FP32 single-CTA tiles of 2^12 or 2^13.
  g.lane_smem = (lane_smem && precision == 0 && g.C == 0 && L >= cap) ? 1 : 0;
  // Staging: bulk copies (1) on FP32 single-CTA tiles; cp.async with a
  // second exchange tile (2) on FP32 single-CTA tiles with 8 pairs per thread
  // (the 256-thread 2^12 tile or the 2^13 tile) and shuffled lane axes.
  g.tma = 0;
  if (tma == 1 && precision == 0 && g.C == 0) g.tma = 1;
  if (tma == 2 && precision == 0 && g.C == 0 && !g.lane_smem &&
      ((L == cap && g.threads == 256) || L == 13))
    g.tma = 2;
  return g;
}

namespace {
template <typename R, int LT, int CL, int TB = kPassThreads, bool LS = false, bool TMA = false,
          bool COMP = false, bool X2 = false>
cudaError_t launch_pass_lt(const PassParams& p, cudaStream_t stream) {
  using S = PassShape<LT, TB>;
  // X2: a second exchange tile after the staged D.
  const size_t smem = S::template smem<R, S::kStageP || TMA>() +
                      (X2 ? (size_t)S::kPairs * 4 * sizeof(R) : 0);
  {
    cudaError_t e = ensure_smem_optin((const void*)pass_kernel<R, LT, CL, TB, LS, TMA, COMP, X2>,
                                      smem, CL > 3);
    if (e != cudaSuccess) return e;
  }
  const dim3 grid((unsigned)((size_t)1 << (p.n - LT)), p.count);
  if constexpr (CL == 0) {
    pass_kernel<R, LT, 0, TB, LS, TMA, COMP, X2><<<grid, S::kThreads, smem, stream>>>(p);
    return cudaGetLastError();
  } else {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(S::kThreads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1u << CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, pass_kernel<R, LT, CL, TB, LS, TMA, COMP>, p);
  }
}

// FP32 single-CTA tile variants: threads (512/256), lane axes (shuffles or
// shared memory) and staging (cp.async or bulk copies).
// p.tma: 0 cp.async staging, 1 bulk copies, 2 cp.async staging with a
// second exchange tile (shapes with 8 pairs per thread, shuffled lane axes).
template <typename R, int LT, int TB>
cudaError_t launch_pass_variant(const PassParams& p, cudaStream_t stream) {
  if (p.tma == 2) {
    if constexpr (!PassShape<LT, TB>::kStageP) {
      if (p.lane_smem) return cudaErrorInvalidValue;
      return launch_pass_lt<R, LT, 0, TB, false, false, false, true>(p, stream);
    }
    return cudaErrorInvalidValue;
  }
  if (p.lane_smem) {
    if (p.tma) return launch_pass_lt<R, LT, 0, TB, true, true>(p, stream);
    return launch_pass_lt<R, LT, 0, TB, true, false>(p, stream);
  }
  if (p.tma) return launch_pass_lt<R, LT, 0, TB, false, true>(p, stream);
  return launch_pass_lt<R, LT, 0, TB, false, false>(p, stream);
}

// The widest tile with a cluster of 2^C CTAs.
template <typename R, int LT>
cudaError_t launch_pass_cluster(const PassParams& p, cudaStream_t stream) {
  switch (p.C) {
    case 0:
      if constexpr (sizeof(R) == 4) {
        if (p.threads == 256) return launch_pass_variant<R, LT, 256>(p, stream);
        return launch_pass_variant<R, LT, kPassThreads>(p, stream);
      }
      if (p.threads == 256) return launch_pass_lt<R, LT, 0, 256>(p, stream);
      return launch_pass_lt<R, LT, 0>(p, stream);
    case 1: return launch_pass_lt<R, LT, 1>(p, stream);
    case 2: return launch_pass_lt<R, LT, 2>(p, stream);
    case 3: return launch_pass_lt<R, LT, 3>(p, stream);
    case 4: return launch_pass_lt<R, LT, 4>(p, stream);
    default: return cudaErrorInvalidValue;
  }
}

template <typename R>
cudaError_t launch_pass_t(const PassParams& p, cudaStream_t stream) {
  constexpr int cap = sizeof(R) == 4 ? 12 : 11;
  if constexpr (sizeof(R) == 4) {
    if (p.comp) {  // compensated partner sums: the default shape only
      if (p.C != 0 || p.threads == 256 || p.lane_smem || p.tma) return cudaErrorInvalidValue;
      switch (p.L) {
        case 6: return launch_pass_lt<R, 6, 0, kPassThreads, false, false, true>(p, stream);
        case 7: return launch_pass_lt<R, 7, 0, kPassThreads, false, false, true>(p, stream);
        case 8: return launch_pass_lt<R, 8, 0, kPassThreads, false, false, true>(p, stream);
        case 9: return launch_pass_lt<R, 9, 0, kPassThreads, false, false, true>(p, stream);
        case 10: return launch_pass_lt<R, 10, 0, kPassThreads, false, false, true>(p, stream);
        case 11: return launch_pass_lt<R, 11, 0, kPassThreads, false, false, true>(p, stream);
        case 12: return launch_pass_lt<R, 12, 0, kPassThreads, false, false, true>(p, stream);
        default: return cudaErrorInvalidValue;
      }
    }
  } else {
    if (p.comp) return cudaErrorInvalidValue;
  }
  if (p.C != 0 && p.L != cap) return cudaErrorInvalidValue;
  if (p.threads == 256 && p.L != cap) return cudaErrorInvalidValue;
  if (p.lane_smem && (sizeof(R) != 4 || p.C != 0 || p.L < cap)) return cudaErrorInvalidValue;
  if (p.tma && (sizeof(R) != 4 || p.C != 0)) return cudaErrorInvalidValue;
  if (p.tma == 2 && p.L < cap) return cudaErrorInvalidValue;  // 8 pairs per thread only
  if constexpr (sizeof(R) == 4) {
    if (p.tma && p.L < cap) {
      switch (p.L) {
        case 6: return launch_pass_lt<R, 6, 0, kPassThreads, false, true>(p, stream);
        case 7: return launch_pass_lt<R, 7, 0, kPassThreads, false, true>(p, stream);
        case 8: return launch_pass_lt<R, 8, 0, kPassThreads, false, true>(p, stream);
        case 9: return launch_pass_lt<R, 9, 0, kPassThreads, false, true>(p, stream);
        case 10: return launch_pass_lt<R, 10, 0, kPassThreads, false, true>(p, stream);
        case 11: return launch_pass_lt<R, 11, 0, kPassThreads, false, true>(p, stream);
        default: return cudaErrorInvalidValue;
      }
    }
  }
  switch (p.L) {
    case 6: return launch_pass_lt<R, 6, 0>(p, stream);
    case 7: return launch_pass_lt<R, 7, 0>(p, stream);
    case 8: return launch_pass_lt<R, 8, 0>(p, stream);
    case 9: return launch_pass_lt<R, 9, 0>(p, stream);
    case 10: return launch_pass_lt<R, 10, 0>(p, stream);
    case 11:
      if constexpr (sizeof(R) == 8) return launch_pass_cluster<R, 11>(p, stream);
      return launch_pass_lt<R, 11, 0>(p, stream);
    case 12:
      if constexpr (sizeof(R) == 4) return launch_pass_cluster<R, 12>(p, stream);
      return cudaErrorInvalidValue;  // FP64 tiles stop at 2^11
    case 13:
      if constexpr (sizeof(R) == 4) {
        if (p.C != 0 || p.threads == 256) return cudaErrorInvalidValue;
        return launch_pass_variant<R, 13, kPassThreads>(p, stream);
      }
      return cudaErrorInvalidValue;
    default: return cudaErrorInvalidValue;
  }
}
}  // namespace

cudaError_t launch_pass(int precision, const PassParams& p,
                        cudaStream_t stream) {
  if (p.n < 6 || p.n > kMaxN || p.L < 6 || p.L > p.n || p.a != 4 || p.C < 0 || p.C > 4 ||
      p.n - p.L < p.C || (p.tiling != 1 && p.tiling != 2) || p.count < 1 ||
      p.count > kMaxGroup || (p.threads != 0 && p.threads != 256 && p.threads != 512) ||
      (p.threads == 256 && (p.C != 0 || p.L != (precision == 0 ? 12 : 11))))
    return cudaErrorInvalidValue;
  return precision == 0 ? launch_pass_t<float>(p, stream)
                        : launch_pass_t<double>(p, stream);
}

namespace {
// Chain launches: a cluster of `tiles` CTAs per walk (non-portable sizes
// above 8 are allowed: the attribute is set on every opt-in).
template <typename R, int LT>
cudaLaunchConfig_t chain_config(int tiles, int count, size_t* smem, cudaLaunchAttribute* attr) {
  using S = PassShape<LT>;
  *smem = S::template smem<R>();
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)tiles, (unsigned)count, 1);
  cfg.blockDim = dim3(S::kThreads, 1, 1);
  cfg.dynamicSmemBytes = *smem;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)tiles;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

template <typename R, int LT>
cudaError_t launch_chain_lt(const PassParams& p, cudaStream_t stream) {
  size_t smem = 0;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = chain_config<R, LT>(1 << (p.n - LT), p.count, &smem, attr);
  cfg.stream = stream;
  cudaError_t e = ensure_smem_optin((const void*)pass_chain_kernel<R, LT>, smem, true);
  if (e != cudaSuccess) return e;
  return cudaLaunchKernelEx(&cfg, pass_chain_kernel<R, LT>, p);
}

// Whether clusters of `tiles` CTAs of the chain kernel can be resident.
template <typename R, int LT>
bool chain_fits(int tiles) {
  size_t smem = 0;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = chain_config<R, LT>(tiles, 1, &smem, attr);
  if (ensure_smem_optin((const void*)pass_chain_kernel<R, LT>, smem, true) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, pass_chain_kernel<R, LT>, &cfg) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return clusters > 0;
}

template <typename R>
bool chain_fits_t(int L, int tiles) {
  switch (L) {
    case 9: return chain_fits<R, 9>(tiles);
    case 10: return chain_fits<R, 10>(tiles);
    case 11: return chain_fits<R, 11>(tiles);
    case 12:
      if constexpr (sizeof(R) == 4) return chain_fits<R, 12>(tiles);
      return false;
    default: return false;
  }
}
}  // namespace

int chain_tile_log(int precision, int n) {
  const char* e = getenv("MQW_CHAIN");
  if (e && atoi(e) == 0) return 0;
  const int cap = precision == 0 ? 12 : 11;
  // Up to 16 tiles per walk (the largest cluster), none of its axes read
  // from global memory (2L - 4 >= n), and at least the single-pass tile.
  // MQW_CHAIN_TILE_LOG asks for wider tiles (fewer CTAs per walk).
  int L = std::max(pass_geom(precision, n).L, n - 4);
  if (const char* t = getenv("MQW_CHAIN_TILE_LOG")) L = std::max(L, std::min(atoi(t), cap));
  if (L < 9 || L > cap || L > n || 2 * L - 4 < n) return 0;
  const int tiles = 1 << (n - L);
  // Residency of a cluster of that size, probed once per (device, shape).
  static std::mutex mu;
  static std::map<std::pair<int, int>, bool> fits;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  std::lock_guard<std::mutex> lk(mu);
  const auto key = std::make_pair(dev, precision * 64 + L * 4 + (n - L));
  auto it = fits.find(key);
  if (it == fits.end())
    it = fits.emplace(key, precision == 0 ? chain_fits_t<float>(L, tiles)
                                          : chain_fits_t<double>(L, tiles)).first;
  return it->second ? L : 0;
}

cudaError_t launch_pass_chain(int precision, const PassParams& p, cudaStream_t stream) {
  const int cap = precision == 0 ? 12 : 11;
  if (p.a != 4 || p.L < 9 || p.L > cap || p.L > p.n || p.n - p.L > 4 || 2 * p.L - 4 < p.n ||
      p.C != 0 || p.comp || p.count < 1 || p.count > kMaxGroup)
    return cudaErrorInvalidValue;
  if (precision == 0) {
    switch (p.L) {
      case 9: return launch_chain_lt<float, 9>(p, stream);
      case 10: return launch_chain_lt<float, 10>(p, stream);
      case 11: return launch_chain_lt<float, 11>(p, stream);
      case 12: return launch_chain_lt<float, 12>(p, stream);
      default: return cudaErrorInvalidValue;
    }
  }
  switch (p.L) {
    case 9: return launch_chain_lt<double, 9>(p, stream);
    case 10: return launch_chain_lt<double, 10>(p, stream);
    case 11: return launch_chain_lt<double, 11>(p, stream);
    default: return cudaErrorInvalidValue;
  }
}

template <bool kProject, typename Params>
void launch_recombine(const Params& p, cudaStream_t stream) {
  const unsigned blocks = (unsigned)((size_t)1 << (p.n - p.L));
  switch (p.count) {
    case 1: recombine_kernel<1, kProject><<<blocks, 256, 0, stream>>>(p); break;
    case 2: recombine_kernel<2, kProject><<<blocks, 256, 0, stream>>>(p); break;
    case 3: recombine_kernel<3, kProject><<<blocks, 256, 0, stream>>>(p); break;
    case 4: recombine_kernel<4, kProject><<<blocks, 256, 0, stream>>>(p); break;
    case 5: recombine_kernel<5, kProject><<<blocks, 256, 0, stream>>>(p); break;
    case 6: recombine_kernel<6, kProject><<<blocks, 256, 0, stream>>>(p); break;
    case 7: recombine_kernel<7, kProject><<<blocks, 256, 0, stream>>>(p); break;
    default: recombine_kernel<8, kProject><<<blocks, 256, 0, stream>>>(p); break;
  }
}

cudaError_t launch_combine(int precision, const CombineParams& p,
                           cudaStream_t stream) {
  if (precision != 0 || p.n < 6 || p.n > kMaxN || p.L < 6 || p.L > p.n || p.Kb < 1 ||
      p.Kb > kMaxBasis || p.count < 1 || p.count > kMaxGroup || !p.basis)
    return cudaErrorInvalidValue;
  for (int g = 0; g < p.count; g++)
    if (p.walk[g].K < 1 || p.walk[g].K > p.Kb || !p.walk[g].coef || !p.walk[g].out ||
        !p.walk[g].norm_part)
      return cudaErrorInvalidValue;
  launch_recombine<false>(p, stream);
  return cudaGetLastError();
}

cudaError_t launch_project(const ProjectParams& p, cudaStream_t stream) {
  if (p.n < 6 || p.n > kMaxN || p.L < 6 || p.L > p.n || p.Kb < 1 || p.Kb > kMaxBasis ||
      p.count < 1 || p.count > kMaxGroup || !p.basis || !p.part)
    return cudaErrorInvalidValue;
  for (int g = 0; g < p.count; g++)
    if (p.walk[g].K < 1 || p.walk[g].K > p.Kb || !p.walk[g].coef || !p.walk[g].psi ||
        !p.walk[g].p_out)
      return cudaErrorInvalidValue;
  launch_recombine<true>(p, stream);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  project_final_kernel<<<p.count, 256, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_unit_eloc(void* psi, int n, const DiagOut* diag, cudaStream_t stream) {
  if (n < 1 || n > kMaxN || !psi || !diag) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(psi, 0, ((size_t)1 << n) * sizeof(float2), stream);
  if (e != cudaSuccess) return e;
  unit_eloc_kernel<<<1, 1, 0, stream>>>(reinterpret_cast<float2*>(psi), diag);
  return cudaGetLastError();
}

cudaError_t launch_unit_eloc_real(float* v, int n, const DiagOut* diag, cudaStream_t stream) {
  if (n < 1 || n > kMaxN || !v || !diag) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(v, 0, ((size_t)1 << n) * sizeof(float), stream);
  if (e != cudaSuccess) return e;
  unit_eloc_real_kernel<<<1, 1, 0, stream>>>(v, diag);
  return cudaGetLastError();
}

namespace {
// CTA threads of the per-pass real chain launches (real_pass_kernel,
// real_batch_kernel) for tile log LT: 128 (eight pairs per thread, two
// shared-memory axes) up to 2^11 tiles, 256 above — measured per launch:
// 8-chain batches at n = 18 (2^11 tiles) 6.38 against 6.84 us, single
// chains at n = 20 (2^12 tiles) 3.41 against 3.95 us; 512 and 1024 threads
// (more warps, more shared-memory axes) were slower at both. The order of
// every partner sum is the same in all of them, so the results are too.
// MQW_REAL_THREADS (128, 256, 512, 1024) fixes it; read once.
int real_threads(int LT) {
  static const int t = [] {
    const char* e = getenv("MQW_REAL_THREADS");
    const int v = e ? atoi(e) : 0;
    return v == 128 || v == 256 || v == 512 || v == 1024 ? v : 0;
  }();
  return t ? t : LT <= 11 ? 128 : 256;
}
template <int LT, int TB>
cudaError_t launch_real_lt_tb(const RealChainParams& p, cudaStream_t stream) {
  using S = RealShape<LT, TB>;
  const size_t smem = S::smem();
  cudaError_t e = ensure_smem_optin((const void*)real_pass_kernel<LT, TB>, smem, false);
  if (e != cudaSuccess) return e;
  real_pass_kernel<LT, TB>
      <<<(unsigned)((size_t)1 << (p.n - LT)), S::kThreads, smem, stream>>>(p);
  return cudaGetLastError();
}
template <int LT>
cudaError_t launch_real_lt(const RealChainParams& p, cudaStream_t stream) {
  switch (real_threads(LT)) {
    case 128: return launch_real_lt_tb<LT, 128>(p, stream);
    case 512: return launch_real_lt_tb<LT, 512>(p, stream);
    case 1024: return launch_real_lt_tb<LT, 1024>(p, stream);
    default: return launch_real_lt_tb<LT, 256>(p, stream);
  }
}
}  // namespace

namespace {
template <int LT>
cudaError_t launch_real_chain_lt(const RealChainBatch& p, cudaStream_t stream) {
  using S = RealShape<LT>;
  const size_t smem = S::smem();
  cudaError_t e = ensure_smem_optin((const void*)real_chain_kernel<LT>, smem, true);
  if (e != cudaSuccess) return e;
  const unsigned tiles = 1u << (p.p.n - LT);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(tiles, (unsigned)p.chains, 1);
  cfg.blockDim = dim3(S::kThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = tiles;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, real_chain_kernel<LT>, p);
}
}  // namespace

cudaError_t launch_real_chain(const RealChainBatch& b, cudaStream_t stream) {
  const RealChainParams& p = b.p;
  if (p.n < 6 || p.n > kMaxN || p.L < 9 || p.L > 12 || p.L > p.n || p.n - p.L > 4 ||
      2 * p.L - 4 < p.n || p.a != 4 || p.K < 1 || p.R < p.K ||
      p.out_stride < ((long long)1 << p.n) || !p.hp || !(p.scale > 0.0f) || b.chains < 1 ||
      b.chains > kMaxChainBatch)
    return cudaErrorInvalidValue;
  for (int c = 0; c < b.chains; c++) {
    const RealChainDesc& d = b.chain[c];
    if (!d.out_base[0] || (p.K > 1 && !d.out_base[1]) || !d.part ||
        (!p.start_uniform && !d.start))
      return cudaErrorInvalidValue;
  }
  switch (p.L) {
    case 9: return launch_real_chain_lt<9>(b, stream);
    case 10: return launch_real_chain_lt<10>(b, stream);
    case 11: return launch_real_chain_lt<11>(b, stream);
    case 12: return launch_real_chain_lt<12>(b, stream);
    default: return cudaErrorInvalidValue;
  }
}

namespace {
template <int LT, int TB>
cudaError_t launch_real_batch_lt_tb(const RealChainBatch& b, int j, cudaStream_t stream) {
  using S = RealShape<LT, TB>;
  const size_t smem = S::smem();
  cudaError_t e = ensure_smem_optin((const void*)real_batch_kernel<LT, TB>, smem, false);
  if (e != cudaSuccess) return e;
  const dim3 grid((unsigned)((size_t)1 << (b.p.n - LT)), (unsigned)b.chains);
  real_batch_kernel<LT, TB><<<grid, S::kThreads, smem, stream>>>(b, j);
  return cudaGetLastError();
}
template <int LT>
cudaError_t launch_real_batch_lt(const RealChainBatch& b, int j, cudaStream_t stream) {
  switch (real_threads(LT)) {
    case 128: return launch_real_batch_lt_tb<LT, 128>(b, j, stream);
    case 512: return launch_real_batch_lt_tb<LT, 512>(b, j, stream);
    case 1024: return launch_real_batch_lt_tb<LT, 1024>(b, j, stream);
    default: return launch_real_batch_lt_tb<LT, 256>(b, j, stream);
  }
}
}  // namespace

cudaError_t launch_real_batch(const RealChainBatch& b, int j, cudaStream_t stream) {
  const RealChainParams& p = b.p;
  if (p.n < 6 || p.n > kMaxN || p.L < 6 || p.L > 13 || p.L > p.n || p.a != 4 || j < 0 ||
      j >= p.K || p.R < p.K || p.out_stride < ((long long)1 << p.n) || !p.hp ||
      !(p.scale > 0.0f) || b.chains < 1 || b.chains > kMaxChainBatch)
    return cudaErrorInvalidValue;
  for (int c = 0; c < b.chains; c++) {
    const RealChainDesc& d = b.chain[c];
    if (!d.out_base[0] || (p.K > 1 && !d.out_base[1]) || !d.part ||
        (j == 0 && !p.start_uniform && !d.start))
      return cudaErrorInvalidValue;
  }
  switch (p.L) {
    case 6: return launch_real_batch_lt<6>(b, j, stream);
    case 7: return launch_real_batch_lt<7>(b, j, stream);
    case 8: return launch_real_batch_lt<8>(b, j, stream);
    case 9: return launch_real_batch_lt<9>(b, j, stream);
    case 10: return launch_real_batch_lt<10>(b, j, stream);
    case 11: return launch_real_batch_lt<11>(b, j, stream);
    case 12: return launch_real_batch_lt<12>(b, j, stream);
    case 13: return launch_real_batch_lt<13>(b, j, stream);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_real_pass(const RealChainParams& p, cudaStream_t stream) {
  if (p.n < 6 || p.n > kMaxN || p.L < 6 || p.L > 13 || p.L > p.n || p.a != 4 ||
      (p.tiling != 1 && p.tiling != 2) || !p.bout || !p.part || !p.hp || !(p.scale > 0.0f) ||
      (p.first && !p.start_uniform && !p.start) || (!p.first && !p.bin) || p.bin == p.bout)
    return cudaErrorInvalidValue;
  switch (p.L) {
    case 6: return launch_real_lt<6>(p, stream);
    case 7: return launch_real_lt<7>(p, stream);
    case 8: return launch_real_lt<8>(p, stream);
    case 9: return launch_real_lt<9>(p, stream);
    case 10: return launch_real_lt<10>(p, stream);
    case 11: return launch_real_lt<11>(p, stream);
    case 12: return launch_real_lt<12>(p, stream);
    case 13: return launch_real_lt<13>(p, stream);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_finalize(int precision, const FinalParams& p,
                            cudaStream_t stream) {
  if (precision == 0)
    finalize_kernel<float><<<1, 32 * kMaxGroup, 0, stream>>>(p);
  else
    finalize_kernel<double><<<1, 32 * kMaxGroup, 0, stream>>>(p);
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
