// Stage-2 product-basis GEMM on the tensor cores (tcgen05, kind::tf32) with
// a three-product TF32 split, for FP32 accuracy.
//
// The product basis (mqw_stage2.cu) gives every walk's stage-2 output as one
// column of a real GEMM per parity class h:
//   out_h[walk][amp] = sum_q Y_h[q][amp] C_h[q][walk]
// (q the (j, k) pairs of the class, K_h of them; Y the basis vectors, 2^n
// floats each; C the walks' coefficient products). Here the amplitudes are
// the MMA's M dimension (M = 128 per CTA), the walks its N dimension (padded
// to a multiple of 16, at most 128) and the pairs its K dimension, in chunks
// of 32.
//
// TF32 keeps 10 mantissa bits. Each FP32 operand is split as x = hi + lo
// with hi = x rounded to TF32 (exact in TF32) and lo = x - hi (exact in
// FP32, |lo| <= 2^-11 |x|), and the product is accumulated as
//   A_hi B_hi + A_hi B_lo + A_lo B_hi
// in the FP32 TMEM accumulator; the dropped A_lo B_lo term and the TF32
// rounding of the lo parts are ~2^-21 relative, the level of FP32 rounding.
// The coefficient matrix is split once (s2_coef_tc_kernel, K-major hi and lo
// copies); the basis tile is split in shared memory as it arrives.
//
// The tensor cores' FP32 accumulation is not round-to-nearest: summed over
// the whole K dimension in TMEM, the result drifts toward zero by ~0.3 ulp
// per accumulation step (measured: P of the last-two-stage projection 2e-5
// low after ~500 steps). So the TMEM accumulator is restarted every
// kTcGroup chunks (a ring of kTcBufs buffers) and the accumulate warps add
// each group's result into FP32 registers with round-to-nearest.
//
// Data movement: Y tiles (MN-major: 32 amplitudes x 32 pairs per box, eight
// boxes per chunk) and the C tiles (K-major: 32 pairs x N walks) arrive by
// TMA (cp.async.bulk.tensor, no multicast) on an mbarrier per pipeline
// stage. An MN-major tf32 operand has one shared-memory layout the MMA
// accepts: 128-byte rows along M with the swizzle applied to 32-byte units
// (atoms of 4 rows; the TMA's 128B_ATOM_32B swizzle writes it); the K-major
// C tiles use the ordinary 128-byte swizzle. The kernel is persistent (one
// CTA per SM walks its share of the tiles); warp roles per CTA (320 threads):
//   warp 0      TMA producer (one thread);
//   warp 1      TMEM allocator and MMA issuer (one thread issues tcgen05.mma);
//   warps 2-5   split the Y tile into hi (in place) and lo;
//   warps 6-9   read each accumulation group (tcgen05.ld), add it into FP32
//               registers, and after a tile's last group store the tile to
//               the planar outputs (each warp reads its TMEM lane quarter:
//               32 amplitudes; a store covers 32 consecutive amplitudes of
//               one walk) while the MMAs of the next tile run.
// Every wait is bounded (%globaltimer): on expiry the CTA sets bit 1 of the
// device error word, the other roles see the abort flag and stop, in-flight
// copies and MMAs are waited for (bounded), the TMEM is freed and the CTA
// returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <map>
#include <mutex>

#include "mqw_internal.h"

namespace mqw {
namespace {

constexpr int kTcM = 128;            // amplitudes per MMA (TMEM lanes)
constexpr int kTcAmps = kTcM;        // amplitudes per CTA
constexpr int kTcBK = 32;            // pairs per chunk: one 128-byte row of tf32
constexpr int kTcStages = 3;
constexpr int kTcThreads = 320;
constexpr int kTcMaxN = 128;         // walks (MMA N) per CTA
constexpr int kTcGroup = 2;          // chunks per TMEM accumulation group
constexpr int kTcBufs = 4;           // TMEM accumulator buffers (a ring over groups)
constexpr unsigned kTcTmemCols = kTcBufs * kTcMaxN;  // 512: the whole TMEM
constexpr unsigned long long kTcWaitNs = 200000000ull;  // 200 ms

// Shared-memory layout (offsets from a 1024-byte aligned base).
constexpr unsigned kTcATile = kTcAmps * kTcBK * 4;        // 16 KB: four 4 KB boxes
constexpr unsigned kTcBTile = kTcMaxN * kTcBK * 4;        // 16 KB
constexpr unsigned kTcStage = 2 * kTcATile + 2 * kTcBTile;  // A(hi), A lo, B hi, B lo
constexpr unsigned kTcBarOff = kTcStages * kTcStage;
constexpr unsigned kTcSmem = kTcBarOff + 256 + 1024;     // barriers + alignment slack
static_assert(8 * (3 * kTcStages + 1 + 2 * kTcBufs) <= 256, "barrier space");

struct TcArgs {
  float* out;          // planar outputs: class 0 at out, class 1 at out + out_walks 2^n
  unsigned* err;       // device error word (bit 1: a bounded wait expired)
  int n, walks, out_walks;
  int Np;              // MMA N: walks padded to a multiple of 16
  int tiles;           // 2 x 2^n / 128: (block of 128 amplitudes, class) pairs
  int chunks[2];       // K chunks of 32 per class
  int crow[2];         // first row of the class's hi copy in the C map (lo: + Np)
};

__device__ __forceinline__ unsigned saddr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ unsigned long long gtime() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void bar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ bool bar_try(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bar_arrive(unsigned bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void bar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
// Waits for phase `parity` of `bar`; false when the CTA is aborting or the
// wait ran out of time (which starts the abort). The clock and the abort
// flag are read every 64 polls only: hundreds of polling threads reading
// %globaltimer on every poll saturate the SM's XU pipe, which the working
// warps share.
__device__ __forceinline__ bool bar_wait(unsigned bar, unsigned parity, volatile int* abort_flag,
                                         unsigned* err) {
  if (bar_try(bar, parity)) return true;
  const unsigned long long t0 = gtime();
  for (unsigned i = 1;; i++) {
    if (bar_try(bar, parity)) return true;
    if ((i & 63u) == 0) {
      if (*abort_flag) return false;
      if (gtime() - t0 > kTcWaitNs) {
        *abort_flag = 1;
        if (err) atomicOr(err, 2u);
        return false;
      }
    }
  }
}
// The same without the abort flag, for the teardown's drains.
__device__ __forceinline__ void bar_drain(unsigned bar, unsigned parity) {
  if (bar_try(bar, parity)) return;
  const unsigned long long t0 = gtime();
  for (unsigned i = 1;; i++) {
    if (bar_try(bar, parity)) return;
    if ((i & 63u) == 0 && gtime() - t0 > kTcWaitNs) return;
  }
}
__device__ __forceinline__ void tma_load_2d(unsigned dst, const CUtensorMap* map, int x, int y,
                                            unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

// UMMA shared-memory descriptor (sm_100 version bits); lbo/sbo in bytes;
// layout 2 = 128-byte swizzle, 1 = 128-byte swizzle with 32-byte atoms.
__device__ __forceinline__ unsigned long long umma_desc(unsigned addr, unsigned lbo, unsigned sbo,
                                                        unsigned layout) {
  unsigned long long d = 0;
  d |= (unsigned long long)((addr >> 4) & 0x3FFFu);
  d |= (unsigned long long)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (unsigned long long)((sbo >> 4) & 0x3FFFu) << 32;
  d |= 1ull << 46;  // descriptor version (sm_100)
  d |= (unsigned long long)layout << 61;
  return d;
}
// Instruction descriptor: D f32, A and B tf32, A MN-major, B K-major,
// M = 128, N = Np.
__device__ __forceinline__ unsigned umma_idesc(int Np) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (1u << 15) | ((unsigned)(Np >> 3) << 17) |
         ((unsigned)(kTcM >> 4) << 24);
}
__device__ __forceinline__ void umma_tf32(unsigned d_tmem, unsigned long long a,
                                          unsigned long long b, unsigned idesc, bool acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"((unsigned)acc)
      : "memory");
}
__device__ __forceinline__ void umma_commit(unsigned bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
      : "memory");
}

// 32 consecutive TMEM columns of this warp's lane quarter, one lane per
// thread (wait with tcgen05.wait::ld before use).
__device__ __forceinline__ void tmem_ld32(unsigned addr, unsigned (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
      "%28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(addr)
      : "memory");
}

// x = hi + lo: hi rounded to TF32 (nearest, ties away; 10 mantissa bits),
// lo = x - hi exactly.
__device__ __forceinline__ void split_tf32(float x, float& hi, float& lo) {
  const unsigned u = (__float_as_uint(x) + 0x1000u) & 0xFFFFE000u;
  hi = __uint_as_float(u);
  lo = x - hi;
}

// Persistent: one CTA per SM takes the tiles t = blockIdx.x, blockIdx.x +
// gridDim.x, ... (t & 1 the parity class, t >> 1 the block of 128
// amplitudes). Every role walks the same sequence of (tile, chunk) steps, so
// the stage ring (index `it`, all chunks of all the CTA's tiles) and the
// accumulator ring (index `gi`, all groups) run on across tiles: the MMAs of
// tile t + 1 proceed while the accumulate warps still add and store tile t.
__global__ void __launch_bounds__(kTcThreads, 1)
    s2_gemm_tc_kernel(const __grid_constant__ CUtensorMap mapY0,
                      const __grid_constant__ CUtensorMap mapY1,
                      const __grid_constant__ CUtensorMap mapC, TcArgs p) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ unsigned tmem_base_sh;
  __shared__ int abort_sh;
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const unsigned sbase = saddr(smem);
  const unsigned bars = sbase + kTcBarOff;
  auto full = [&](int s) { return bars + 8u * s; };
  auto conv = [&](int s) { return bars + 8u * (kTcStages + s); };
  auto empty = [&](int s) { return bars + 8u * (2 * kTcStages + s); };
  const unsigned accf = bars + 8u * (3 * kTcStages);  // every MMA done (teardown)
  // accumulation group gi lives in TMEM buffer gi % kTcBufs: full once its
  // MMAs completed, free once the accumulate warps have read it
  auto accfull = [&](int b) { return bars + 8u * (3 * kTcStages + 1 + b); };
  auto accfree = [&](int b) { return bars + 8u * (3 * kTcStages + 1 + kTcBufs + b); };
  auto a_tile = [&](int s) { return sbase + s * kTcStage; };
  auto alo_tile = [&](int s) { return sbase + s * kTcStage + kTcATile; };
  auto bhi_tile = [&](int s) { return sbase + s * kTcStage + 2 * kTcATile; };
  auto blo_tile = [&](int s) { return sbase + s * kTcStage + 2 * kTcATile + kTcBTile; };

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  volatile int* abort_flag = &abort_sh;

  if (threadIdx.x == 0) {
    abort_sh = 0;
    for (int s = 0; s < kTcStages; s++) {
      bar_init(full(s), 1);
      bar_init(conv(s), 128);
      bar_init(empty(s), 1);
    }
    bar_init(accf, 1);
    for (int b = 0; b < kTcBufs; b++) {
      bar_init(accfull(b), 1);
      bar_init(accfree(b), 128);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     saddr(&tmem_base_sh)),
                 "r"(kTcTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = tmem_base_sh;
  const unsigned b_bytes = (unsigned)p.Np * kTcBK * 4u;

  if (warp == 0) {
    if (lane == 0) {
      // TMA producer.
      int it = 0, issued = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < p.tiles && ok; t += gridDim.x) {
        const int h = t & 1, m0 = (t >> 1) * kTcAmps;
        const CUtensorMap* mY = h ? &mapY1 : &mapY0;
        for (int c = 0; c < p.chunks[h]; c++, it++) {
          const int s = it % kTcStages;
          if (it >= kTcStages &&
              !bar_wait(empty(s), ((it / kTcStages) - 1) & 1, abort_flag, p.err)) {
            ok = false;
            break;
          }
          bar_expect_tx(full(s), kTcATile + 2 * b_bytes);
          const int k0 = c * kTcBK;
          for (int b = 0; b < kTcAmps / 32; b++)
            tma_load_2d(a_tile(s) + b * 4096u, mY, m0 + 32 * b, k0, full(s));
          tma_load_2d(bhi_tile(s), &mapC, k0, p.crow[h], full(s));
          tma_load_2d(blo_tile(s), &mapC, k0, p.crow[h] + p.Np, full(s));
          issued = it + 1;
        }
      }
      if (*abort_flag) {
        // Copies issued but never consumed must land before the CTA's shared
        // memory is released; only the last kTcStages chunks can be pending
        // (a stage is reissued only after its previous chunk was consumed).
        for (int c = issued > kTcStages ? issued - kTcStages : 0; c < issued; c++)
          bar_drain(full(c % kTcStages), (c / kTcStages) & 1);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer.
      const unsigned idesc = umma_idesc(p.Np);
      int it = 0, gi = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < p.tiles && ok; t += gridDim.x) {
        const int chunks = p.chunks[t & 1];
        unsigned d = tmem;
        for (int c = 0; c < chunks; c++, it++) {
          const int s = it % kTcStages;
          const bool first = c % kTcGroup == 0;
          if (first) {
            // A group's buffer is reused once the accumulate warps have read
            // the group kTcBufs before it.
            const int b = gi % kTcBufs;
            if (gi >= kTcBufs &&
                !bar_wait(accfree(b), ((gi / kTcBufs) - 1) & 1, abort_flag, p.err)) {
              ok = false;
              break;
            }
            d = tmem + (unsigned)(b * kTcMaxN);
          }
          if (!bar_wait(conv(s), (it / kTcStages) & 1, abort_flag, p.err)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
          for (int kk = 0; kk < kTcBK / 8; kk++) {
            // A (MN-major, 32-byte-atom swizzle): blocks of 32 amplitudes 4 KB
            // apart (LBO), groups of 4 pair rows 512 B apart (SBO); the MMA's
            // 8 pairs start 1 KB further per step. B (K-major, 128-byte
            // swizzle): groups of 8 walk rows 1 KB apart (SBO); the MMA's 8
            // pairs start 32 B further per step.
            const unsigned long long ahi = umma_desc(a_tile(s) + kk * 1024u, 4096u, 512u, 1u);
            const unsigned long long alo = umma_desc(alo_tile(s) + kk * 1024u, 4096u, 512u, 1u);
            const unsigned long long bhi = umma_desc(bhi_tile(s) + kk * 32u, 16u, 1024u, 2u);
            const unsigned long long blo = umma_desc(blo_tile(s) + kk * 32u, 16u, 1024u, 2u);
            umma_tf32(d, ahi, bhi, idesc, !(first && kk == 0));
            umma_tf32(d, ahi, blo, idesc, true);
            umma_tf32(d, alo, bhi, idesc, true);
          }
          umma_commit(empty(s));  // the stage's tiles are free once these MMAs finish
          if (c % kTcGroup == kTcGroup - 1 || c == chunks - 1) {
            umma_commit(accfull(gi % kTcBufs));
            gi++;
          }
        }
      }
      // Every MMA issued has completed when accf flips (waited for on every
      // path, so that no commit is left to arrive after the CTA exits).
      umma_commit(accf);
      bar_drain(accf, 0);
    }
    __syncwarp();
  } else if (warp < 6) {
    // Warps 2-5: split each Y tile into hi (in place) and lo.
    const int ct = threadIdx.x - 64;  // 0..127
    int it = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < p.tiles && ok; t += gridDim.x) {
      const int chunks = p.chunks[t & 1];
      for (int c = 0; c < chunks; c++, it++) {
        const int s = it % kTcStages;
        if (!bar_wait(full(s), (it / kTcStages) & 1, abort_flag, p.err)) {
          ok = false;
          break;
        }
        float4* a = reinterpret_cast<float4*>(smem + s * kTcStage);
        float4* alo = reinterpret_cast<float4*>(smem + s * kTcStage + kTcATile);
#pragma unroll 4
        for (int e = ct; e < (int)(kTcATile / 16); e += 128) {
          const float4 v = a[e];
          float4 hi, lo;
          split_tf32(v.x, hi.x, lo.x);
          split_tf32(v.y, hi.y, lo.y);
          split_tf32(v.z, hi.z, lo.z);
          split_tf32(v.w, hi.w, lo.w);
          a[e] = hi;
          alo[e] = lo;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        bar_arrive(conv(s));
      }
    }
  } else {
    // Warps 6-9: add each accumulation group's result into FP32 registers
    // with round-to-nearest (this warp's TMEM lane quarter: 32 amplitudes,
    // one per thread, all walks), then store the tile's planar outputs (a
    // store covers 32 consecutive amplitudes of one walk).
    const int q = warp & 3;
    const size_t N = (size_t)1 << p.n;
    int gi = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < p.tiles && ok; t += gridDim.x) {
      const int h = t & 1, m0 = (t >> 1) * kTcAmps;
      const int groups = (p.chunks[h] + kTcGroup - 1) / kTcGroup;
      float acc[kTcMaxN];
#pragma unroll
      for (int j = 0; j < kTcMaxN; j++) acc[j] = 0.0f;
      for (int g = 0; g < groups; g++, gi++) {
        const int b = gi % kTcBufs;
        if (!bar_wait(accfull(b), (gi / kTcBufs) & 1, abort_flag, p.err)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const unsigned base = tmem + ((unsigned)(32 * q) << 16) + (unsigned)(b * kTcMaxN);
#pragma unroll
        for (int c0 = 0; c0 < kTcMaxN; c0 += 32) {
          if (c0 < p.Np) {
            unsigned r[32];
            tmem_ld32(base + (unsigned)c0, r);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int j = 0; j < 32; j++)
              acc[c0 + j] = __fadd_rn(acc[c0 + j], __uint_as_float(r[j]));
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        bar_arrive(accfree(b));
      }
      if (!ok || *abort_flag) break;
      float* out = p.out + (size_t)h * p.out_walks * N;
      const size_t amp = (size_t)m0 + 32 * q + lane;
#pragma unroll
      for (int j = 0; j < kTcMaxN; j++)
        if (j < p.walks) out[(size_t)j * N + amp] = acc[j];
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTcTmemCols)
                 : "memory");
  }
}

// K-major hi/lo copies of the coefficient matrices: row (2h + part) Np + w,
// column q (the class's pair index), Kp columns per row; zero outside the
// class's rows and walks.
__global__ void s2_coef_tc_kernel(S2CoefParams p, float* Ct, int Np, int Kp) {
  const size_t total = (size_t)2 * Np * Kp;  // (class, walk, q)
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int h = (int)(e / ((size_t)Np * Kp));
    const size_t r = e - (size_t)h * Np * Kp;
    const int w = (int)(r / Kp), q = (int)(r % Kp);
    float v = 0.0f;
    if (q < p.lay.rows(h) && w < p.walks) {
      int j, k;
      p.lay.pair(h, q, &j, &k);
      const StageDesc s1 = p.stages[p.job0 + w * p.m + p.sj];
      const StageDesc s2 = p.stages[p.job0 + w * p.m + p.sk];
      auto weight = [](const float* c, int K, int i) {
        const double ci = i < K ? (double)c[i] : 0.0;
        const double ci2 = i + 2 < K ? (double)c[i + 2] : 0.0;
        return i == 0 ? ci - 0.5 * ci2 : 0.5 * (ci - ci2);
      };
      const float* c1 = p.coef + s1.coef_off;
      const float* c2 = p.coef + s2.coef_off;
      const double d1 = p.tbasis ? (j < s1.K ? (double)c1[j] : 0.0) : weight(c1, s1.K, j);
      const double d2 = p.tbasis ? (k < s2.K ? (double)c2[k] : 0.0) : weight(c2, s2.K, k);
      const double sg = (h == 0 && (j & 1) && (k & 1)) ? -1.0 : 1.0;
      v = (float)(sg * d1 * d2);
    }
    float hi, lo;
    split_tf32(v, hi, lo);
    Ct[((size_t)(2 * h) * Np + w) * Kp + q] = hi;
    Ct[((size_t)(2 * h + 1) * Np + w) * Kp + q] = lo;
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  return fn;
}

// 2-D float32 tensor map: dims {inner, outer}, row pitch in bytes, box
// {bx, by}, the given swizzle.
bool make_map(CUtensorMap* m, const float* base, unsigned long long inner,
              unsigned long long outer, unsigned long long pitch, unsigned bx, unsigned by,
              CUtensorMapSwizzle swz) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (!enc) return false;
  const cuuint64_t dims[2] = {inner, outer};
  const cuuint64_t strides[1] = {pitch};
  const cuuint32_t box[2] = {bx, by};
  const cuuint32_t es[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box,
             es, CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

std::mutex g_tc_mu;
std::map<int, int> g_tc_sms;  // per device: SM count, once the shared-memory opt-in is made

}  // namespace

int s2_tc_np(int walks) { return (walks + 15) / 16 * 16; }
int s2_tc_kp(const S2Layout& lay) {
  const int r = lay.rows(0) > lay.rows(1) ? lay.rows(0) : lay.rows(1);
  return (r + kTcBK - 1) / kTcBK * kTcBK;
}
size_t s2_tc_coef_floats(int walks, const S2Layout& lay) {
  return (size_t)4 * s2_tc_np(walks) * s2_tc_kp(lay);
}

cudaError_t launch_s2_gemm_tc_raw(const float* Y, const int rows[2], const float* Ct, int Np,
                                  int Kp, int n, int walks, int out_walks, float* out,
                                  unsigned* err, cudaStream_t stream) {
  if (n < 8 || n > kMaxN || !Y || !out || !Ct || walks < 1 || Np != s2_tc_np(walks) ||
      Np > kTcMaxN || out_walks < walks || rows[0] < 1 || rows[1] < 1 || Kp % kTcBK != 0 ||
      Kp < rows[0] || Kp < rows[1] || !encode_fn())
    return cudaErrorInvalidValue;
  const unsigned long long N = 1ull << n;
  CUtensorMap mY0, mY1, mC;
  if (!make_map(&mY0, Y, N, (unsigned long long)rows[0], N * 4, 32, kTcBK,
                CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B) ||
      !make_map(&mY1, Y + (size_t)rows[0] * N, N, (unsigned long long)rows[1], N * 4, 32, kTcBK,
                CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B) ||
      !make_map(&mC, Ct, (unsigned long long)Kp, 4ull * Np, (unsigned long long)Kp * 4, kTcBK,
                (unsigned)Np, CU_TENSOR_MAP_SWIZZLE_128B))
    return cudaErrorInvalidValue;
  TcArgs a{};
  a.out = out;
  a.err = err;
  a.n = n;
  a.walks = walks;
  a.out_walks = out_walks;
  a.Np = Np;
  a.tiles = (int)(2 * (N / kTcAmps));
  for (int h = 0; h < 2; h++) {
    a.chunks[h] = (rows[h] + kTcBK - 1) / kTcBK;
    a.crow[h] = 2 * h * Np;
  }
  int sms = 0;
  {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(g_tc_mu);
    int& known = g_tc_sms[dev];
    if (known <= 0) {
      e = cudaFuncSetAttribute(s2_gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kTcSmem);
      if (e != cudaSuccess) return e;
      int count = 0;
      e = cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return e;
      known = count;
    }
    sms = known;
  }
  // Persistent: one CTA per SM (its shared memory admits no second one).
  const unsigned grid = (unsigned)(a.tiles < sms ? a.tiles : sms);
  s2_gemm_tc_kernel<<<grid, kTcThreads, kTcSmem, stream>>>(mY0, mY1, mC, a);
  return cudaGetLastError();
}

cudaError_t launch_s2_gemm_tc(const S2CoefParams& cp, float* Ct, const S2GemmParams& g,
                              unsigned* err, cudaStream_t stream) {
  const int Np = s2_tc_np(g.walks);
  const int Kp = s2_tc_kp(cp.lay);
  if (g.walks < 1 || Np > kTcMaxN || !Ct || cp.walks != g.walks ||
      cp.lay.rows(0) != g.rows[0] || cp.lay.rows(1) != g.rows[1])
    return cudaErrorInvalidValue;
  // Coefficients: K-major hi/lo copies.
  {
    const size_t total = (size_t)2 * Np * Kp;
    const size_t want = (total + 255) / 256;
    s2_coef_tc_kernel<<<(unsigned)(want < 8192 ? want : 8192), 256, 0, stream>>>(cp, Ct, Np, Kp);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return launch_s2_gemm_tc_raw(g.Y, g.rows, Ct, Np, Kp, g.n, g.walks, g.out_walks, g.out, err,
                               stream);
}

}  // namespace mqw
