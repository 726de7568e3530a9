// Ising diagonal with the reference's arithmetic, in parallel.
//
// The reference (MultiQW.cpp:325-358) walks the 2^n basis states in Gray-code
// order. At Gray rank r >= 1 it flips spin f = ctz(r) and adds the float
// increment
//     d(r) = fl( 4 * fl_seq( sum_k J(f,k) * s_f s_k ) + 2 h_f s_f )
// (the sum over k is a sequential float sum, the k = f term is zero, s are the
// spins after the flip) to a double accumulator E, starting from
// E(0) = double(float(sum J - sum h)). Because every d(r) is a float and the
// running sums stay far below 2^53 ulps of the smallest increment, the double
// accumulation is exact, so a parallel scan over any association reproduces
// the sequential sums bit-for-bit (checked against the oracle). Replicating
// this matters: the float increments drift from exact FP64 energies by ~3e-4
// at n = 20, enough to change the evolution and, for near-degenerate
// instances, the ground-state index.
//
// Layout: Gray ranks are cut into chunks of C = 2^min(n,12) consecutive ranks.
//   diag_chunks  : per chunk, its increment total and running min/max (1 CTA).
//   diag_scan    : per instance, exclusive scan of chunk totals, global
//                  min (first Gray rank wins) / max, E_loc, mid, E_abs.
//   diag_write   : per chunk, the energies; a chunk's ranks map onto one
//                  aligned block of C basis states, so the block is staged in
//                  shared memory and written coalesced.
#include "mqw_internal.h"

namespace mqw {
namespace {

constexpr int kThreads = 256;

struct DiagGeom {
  int n, cl, C, R, active;  // chunk log/size, ranks per thread, threads used
  int chunks;               // chunks per instance
};

__host__ __device__ inline DiagGeom diag_geom(int n) {
  DiagGeom g;
  g.n = n;
  g.cl = n < kDiagChunkLog ? n : kDiagChunkLog;
  g.C = 1 << g.cl;
  g.R = g.cl >= 8 ? (1 << (g.cl - 8)) : 1;
  g.active = g.C / g.R;
  g.chunks = 1 << (n - g.cl);
  return g;
}

// Couplings J(i,j) = float(raw)/2 (symmetric, zero diagonal) and fields,
// MultiQW.cpp:306-323.
__device__ void load_Jh(int n, const double* raw, float* sJ, float* sh) {
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) sJ[idx] = 0.0f;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int base = i * (i - 1) / 2;
    for (int j = 0; j < i; j++) {
      const float v = (float)raw[base + j] * 0.5f;
      sJ[i * n + j] = v;
      sJ[j * n + i] = v;
    }
    sh[i] = (float)raw[n * (n - 1) / 2 + i];
  }
  __syncthreads();
}

// The reference's float increment at Gray rank r >= 1.
__device__ __forceinline__ float gray_increment(int n, const float* sJ,
                                                const float* sh, uint32_t r) {
  const int f = __ffs(r) - 1;
  const uint32_t z = r ^ (r >> 1);
  const uint32_t sf = (z >> f) & 1u;  // spin f after the flip is +1 iff set
  // bit k of y set <=> s_f s_k = -1 (the k = f bit is clear; J(f,f) = 0).
  const uint32_t y = z ^ (sf ? 0xffffffffu : 0u);
  const float* Jf = sJ + f * n;
  float acc = (y & 1u) ? -Jf[0] : Jf[0];
  for (int k = 1; k < n; k++) {
    const float t = ((y >> k) & 1u) ? -Jf[k] : Jf[k];
    acc = __fadd_rn(acc, t);
  }
  // - 2 h_f state(f,f) with state(f,f) = -s_f.
  const float two_h_st = sf ? -2.0f * sh[f] : 2.0f * sh[f];
  return __fsub_rn(4.0f * acc, two_h_st);
}

// Exclusive block scan of one double per thread (exact for exact inputs).
__device__ double block_excl_scan(double v, double* s_tmp, double* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const double y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_tmp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    double w = lane < nw ? s_tmp[lane] : 0.0;
    for (int o = 1; o < 32; o <<= 1) {
      const double y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) s_tmp[lane] = w;
  }
  __syncthreads();
  const double wexcl = warp > 0 ? s_tmp[warp - 1] : 0.0;
  *total = s_tmp[(blockDim.x >> 5) - 1];
  double lane_excl = __shfl_up_sync(0xffffffffu, x, 1);
  if (lane == 0) lane_excl = 0.0;
  const double r = wexcl + lane_excl;
  __syncthreads();
  (void)v;
  return r;
}

__global__ void __launch_bounds__(kThreads)
diag_chunks(int n, const double* raw_all, ChunkPartial* parts) {
  __shared__ float sJ[kMaxN * kMaxN];
  __shared__ float sh[kMaxN];
  __shared__ double s_tmp[32];
  __shared__ double s_min[kThreads], s_max[kThreads];
  __shared__ uint32_t s_rmin[kThreads];
  const DiagGeom g = diag_geom(n);
  const int inst = blockIdx.y;
  const uint32_t chunk = blockIdx.x;
  const double* raw = raw_all + (size_t)inst * (n * (n + 1) / 2);
  load_Jh(n, raw, sJ, sh);

  const int t = threadIdx.x;
  double S = 0.0, vmin = 0.0, vmax = 0.0;
  uint32_t rmin = 0xffffffffu;
  bool have = false;
  if (t < g.active) {
    const uint32_t r0 = (chunk << g.cl) + (uint32_t)t * g.R;
    for (int k = 0; k < g.R; k++) {
      const uint32_t r = r0 + k;
      if (r != 0) S += (double)gray_increment(n, sJ, sh, r);
      if (!have || S < vmin) { vmin = S; rmin = r; }
      if (!have || S > vmax) vmax = S;
      have = true;
    }
  }
  double total;
  const double excl = block_excl_scan(t < g.active ? S : 0.0, s_tmp, &total);
  s_min[t] = have ? excl + vmin : 0.0;
  s_max[t] = have ? excl + vmax : 0.0;
  s_rmin[t] = have ? rmin : 0xffffffffu;
  __syncthreads();
  // Tree reduction: min value, ties to the smallest rank; max value.
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if (t < w) {
      const uint32_t ra = s_rmin[t], rb = s_rmin[t + w];
      if (rb != 0xffffffffu) {
        const double a = s_min[t], b = s_min[t + w];
        if (ra == 0xffffffffu || b < a || (b == a && rb < ra)) {
          s_min[t] = b;
          s_rmin[t] = rb;
        }
        if (ra == 0xffffffffu || s_max[t + w] > s_max[t]) s_max[t] = s_max[t + w];
      }
    }
    __syncthreads();
  }
  if (t == 0) {
    ChunkPartial p;
    p.total = total;
    p.vmin = s_min[0];
    p.vmax = s_max[0];
    p.rmin = s_rmin[0];
    p.pad = 0;
    parts[(size_t)inst * g.chunks + chunk] = p;
  }
}

// One CTA per instance: scan chunk totals, global extrema, spectral data.
__global__ void __launch_bounds__(1024)
diag_scan(int n, const double* raw_all, ChunkPartial* parts, double* chunk_excl,
          DiagOut* out) {
  __shared__ float sJ[kMaxN * kMaxN];
  __shared__ float sh[kMaxN];
  __shared__ double s_tmp[32];
  __shared__ double s_min[1024], s_max[1024];
  __shared__ uint32_t s_rmin[1024];
  __shared__ double s_einit;
  const DiagGeom g = diag_geom(n);
  const int inst = blockIdx.x;
  const double* raw = raw_all + (size_t)inst * (n * (n + 1) / 2);
  load_Jh(n, raw, sJ, sh);
  if (threadIdx.x == 0) {
    // E(all spins -1) = J.sum() - h.sum() in float (MultiQW.cpp:332), summed
    // in storage order.
    float sumJ = 0.0f, sumh = 0.0f;
    for (int i = 0; i < n * n; i++) sumJ = __fadd_rn(sumJ, sJ[i]);
    for (int i = 0; i < n; i++) sumh = __fadd_rn(sumh, sh[i]);
    s_einit = (double)__fsub_rn(sumJ, sumh);
  }
  __syncthreads();
  const ChunkPartial* P = parts + (size_t)inst * g.chunks;
  double* X = chunk_excl + (size_t)inst * g.chunks;
  const int t = threadIdx.x, T = blockDim.x;
  const int per = (g.chunks + T - 1) / T;
  const int c0 = t * per, c1 = min(g.chunks, c0 + per);
  double S = 0.0;
  for (int c = c0; c < c1; c++) S += P[c].total;
  double total;
  const double excl = block_excl_scan(S, s_tmp, &total);
  double run = excl, vmin = 0.0, vmax = 0.0;
  uint32_t rmin = 0xffffffffu;
  bool have = false;
  for (int c = c0; c < c1; c++) {
    X[c] = run;
    const ChunkPartial p = P[c];
    const double a = run + p.vmin, b = run + p.vmax;
    if (!have || a < vmin) { vmin = a; rmin = p.rmin; }
    if (!have || b > vmax) vmax = b;
    have = true;
    run += p.total;
  }
  s_min[t] = vmin;
  s_max[t] = vmax;
  s_rmin[t] = have ? rmin : 0xffffffffu;
  __syncthreads();
  for (int w = T / 2; w > 0; w >>= 1) {
    if (t < w) {
      const uint32_t ra = s_rmin[t], rb = s_rmin[t + w];
      if (rb != 0xffffffffu) {
        const double a = s_min[t], b = s_min[t + w];
        if (ra == 0xffffffffu || b < a || (b == a && rb < ra)) {
          s_min[t] = b;
          s_rmin[t] = rb;
        }
        if (ra == 0xffffffffu || s_max[t + w] > s_max[t]) s_max[t] = s_max[t + w];
      }
    }
    __syncthreads();
  }
  if (t == 0) {
    const double e0 = s_einit + s_min[0];
    const double emax = s_einit + s_max[0];
    DiagOut o;
    o.e0 = e0;
    o.emax = emax;
    o.mid = (emax + e0) / 2;
    o.e_abs = (float)((emax - e0) / 2);
    const uint32_t r = s_rmin[0];
    o.e_loc = r ^ (r >> 1);
    out[inst] = o;
  }
  (void)total;
}

__global__ void __launch_bounds__(kThreads)
diag_write(int n, const double* raw_all, const double* chunk_excl,
           const DiagOut* dout, float* hp_all, double* e_all) {
  __shared__ float sJ[kMaxN * kMaxN];
  __shared__ float sh[kMaxN];
  __shared__ double s_tmp[32];
  __shared__ double s_einit;
  extern __shared__ double s_stage[];  // C doubles (energies of the block)
  const DiagGeom g = diag_geom(n);
  const int inst = blockIdx.y;
  const uint32_t chunk = blockIdx.x;
  const double* raw = raw_all + (size_t)inst * (n * (n + 1) / 2);
  load_Jh(n, raw, sJ, sh);
  if (threadIdx.x == 0) {
    float sumJ = 0.0f, sumh = 0.0f;
    for (int i = 0; i < n * n; i++) sumJ = __fadd_rn(sumJ, sJ[i]);
    for (int i = 0; i < n; i++) sumh = __fadd_rn(sumh, sh[i]);
    s_einit = (double)__fsub_rn(sumJ, sumh);
  }
  const int t = threadIdx.x;
  double S = 0.0;
  if (t < g.active) {
    const uint32_t r0 = (chunk << g.cl) + (uint32_t)t * g.R;
    for (int k = 0; k < g.R; k++) {
      const uint32_t r = r0 + k;
      if (r != 0) S += (double)gray_increment(n, sJ, sh, r);
    }
  }
  double total;
  const double excl = block_excl_scan(t < g.active ? S : 0.0, s_tmp, &total);
  const double base = s_einit + chunk_excl[(size_t)inst * g.chunks + chunk];
  const uint32_t H = chunk;
  const uint32_t hi_flip = (H & 1u) << (g.cl - 1);
  if (t < g.active) {
    const uint32_t r0 = (chunk << g.cl) + (uint32_t)t * g.R;
    double run = excl;
    for (int k = 0; k < g.R; k++) {
      const uint32_t r = r0 + k;
      if (r != 0) run += (double)gray_increment(n, sJ, sh, r);
      const uint32_t L = (uint32_t)t * g.R + k;
      const uint32_t local = (L ^ (L >> 1) ^ (g.cl > 0 ? hi_flip : 0u)) & (g.C - 1);
      s_stage[local] = base + run;
    }
  }
  __syncthreads();
  const size_t N = (size_t)1 << n;
  const size_t zbase = (size_t)(H ^ (H >> 1)) << g.cl;
  const DiagOut o = dout[inst];
  const float midf = (float)o.mid;
  float* hp = hp_all ? hp_all + (size_t)inst * N : nullptr;
  double* e = e_all ? e_all + (size_t)inst * N : nullptr;
  for (int i = t; i < g.C; i += blockDim.x) {
    const double E = s_stage[i];
    if (hp) hp[zbase + i] = __fsub_rn((float)E, midf);
    if (e) e[zbase + i] = E;
  }
  (void)total;
}

// Raw moments of the shifted diagonal, mean(H_P^k) for k = 1..4, in FP64:
// a fixed grid with a grid-stride loop gives each block a fixed set of
// amplitudes, and the block partials are summed in order by one block, so
// the result is run-to-run identical.
constexpr int kMomentBlocks = 1024;
__global__ void moments_partial(const float* __restrict__ hp, size_t N, double* part) {
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (size_t)gridDim.x * blockDim.x) {
    const double x = hp[i], x2 = x * x;
    s[0] += x;
    s[1] += x2;
    s[2] += x2 * x;
    s[3] += x2 * x2;
  }
  __shared__ double red[4][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    double v = s[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[k][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[threadIdx.x][w];
    part[(size_t)blockIdx.x * 4 + threadIdx.x] = v;
  }
}
__global__ void moments_final(const double* part, int blocks, double inv_n, double* out) {
  if (threadIdx.x < 4) {
    double v = 0.0;
    for (int b = 0; b < blocks; b++) v += part[(size_t)b * 4 + threadIdx.x];
    out[threadIdx.x] = v * inv_n;
  }
}

}  // namespace

size_t moments_scratch_bytes() { return (size_t)(kMomentBlocks + 1) * 4 * sizeof(double); }

cudaError_t launch_moments(int n, const float* hp, void* scratch, cudaStream_t stream) {
  if (n < 1 || n > kMaxN || !hp || !scratch) return cudaErrorInvalidValue;
  const size_t N = (size_t)1 << n;
  const size_t want = (N + 255) / 256;
  const int blocks = (int)(want < kMomentBlocks ? want : kMomentBlocks);
  double* part = (double*)scratch;
  double* out = part + (size_t)kMomentBlocks * 4;
  moments_partial<<<blocks, 256, 0, stream>>>(hp, N, part);
  moments_final<<<1, 32, 0, stream>>>(part, blocks, 1.0 / (double)N, out);
  return cudaGetLastError();
}

size_t diag_scratch_bytes(int n, int count) {
  const DiagGeom g = diag_geom(n);
  return (size_t)count * g.chunks * (sizeof(ChunkPartial) + sizeof(double));
}

cudaError_t launch_diag(int n, int count, const double* raw, float* hp,
                        double* energies, DiagOut* out, void* scratch,
                        cudaStream_t stream) {
  if (n < 1 || n > kMaxN || count < 1) return cudaErrorInvalidValue;
  const DiagGeom g = diag_geom(n);
  ChunkPartial* parts = (ChunkPartial*)scratch;
  double* excl = (double*)(parts + (size_t)count * g.chunks);
  for (int i0 = 0; i0 < count; i0 += 65535) {
    const int c = count - i0 < 65535 ? count - i0 : 65535;
    const double* r = raw + (size_t)i0 * (n * (n + 1) / 2);
    dim3 grid(g.chunks, c);
    diag_chunks<<<grid, kThreads, 0, stream>>>(n, r, parts + (size_t)i0 * g.chunks);
    diag_scan<<<c, 1024, 0, stream>>>(n, r, parts + (size_t)i0 * g.chunks,
                                      excl + (size_t)i0 * g.chunks, out + i0);
    const size_t N = (size_t)1 << n;
    diag_write<<<grid, kThreads, (size_t)g.C * sizeof(double), stream>>>(
        n, r, excl + (size_t)i0 * g.chunks, out + i0,
        hp ? hp + (size_t)i0 * N : nullptr,
        energies ? energies + (size_t)i0 * N : nullptr);
  }
  return cudaGetLastError();
}

}  // namespace mqw
