// Stage-2 product basis (FP32).
//
// Every walk of an instance starts stage 2 from its stage-1 output
//   psi_1 = sum_j d1_j w_j,   w_j = U_j(H~_1) psi_0   (the stage-1 basis),
// and applies the instance's stage-2 operator with its own time, i.e.
//   psi_2 = sum_k d2_k U_k(H~_2) psi_1 = sum_{j,k} d1_j d2_k Y_jk,
//   Y_jk = U_k(H~_2) w_j,
// with d the recombination weights of the walk's Chebyshev coefficients
// (d_0 = c_0 - c_2/2, d_j = (c_j - c_{j+2})/2; real for even index, imaginary
// for odd). The Y_jk are real: K_1 x K_2 vectors built by K_1 unit-coefficient
// pass chains (one per stage-1 basis vector) instead of one K_2-pass chain
// per walk. Every walk's psi_2 is then one column of a real GEMM
//   Re psi_2 = sum over (j, k) with j + k even of  s_jk D1_j D2_k Y_jk,
//   Im psi_2 = sum over (j, k) with j + k odd  of       D1_j D2_k Y_jk,
// (D the real magnitudes of d, s_jk = -1 when j and k are both odd), which
// s2_gemm_kernel computes for all walks of the instance at once: the Y
// vectors of one parity class are the GEMM's K dimension, the walks its
// columns, the amplitudes its rows.
#include "mqw_internal.h"

namespace mqw {
namespace {

__global__ void real_to_complex_kernel(float2* __restrict__ dst, const float* __restrict__ src,
                                       size_t N) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (size_t)gridDim.x * blockDim.x)
    dst[i] = make_float2(src[i], 0.0f);
}

// Recombination weight d_j (its real magnitude) of a coefficient list c of
// length K.
__device__ __forceinline__ double recomb_weight(const float* c, int K, int j) {
  const double cj = j < K ? (double)c[j] : 0.0;
  const double cj2 = j + 2 < K ? (double)c[j + 2] : 0.0;
  return j == 0 ? cj - 0.5 * cj2 : 0.5 * (cj - cj2);
}

// C_h[q][col] = s_jk D1_j(col) D2_k(col) for the pair (j, k) = row q of
// parity class h; zero for padding rows and columns.
__global__ void s2_coef_kernel(S2CoefParams p) {
  const size_t rows0 = (size_t)p.rows_pad[0];
  const size_t total = (rows0 + (size_t)p.rows_pad[1]) * p.col_stride;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int h = e >= rows0 * p.col_stride ? 1 : 0;
    const size_t local = e - (h ? rows0 * p.col_stride : 0);
    const int q = (int)(local / p.col_stride);
    const int col = (int)(local % p.col_stride);
    float v = 0.0f;
    if (q < p.lay.rows(h) && col < p.walks) {
      int j, k;
      p.lay.pair(h, q, &j, &k);
      const StageDesc s1 = p.stages[p.job0 + col * p.m + p.sj];
      const StageDesc s2 = p.stages[p.job0 + col * p.m + p.sk];
      const float* c1 = p.coef + s1.coef_off;
      const float* c2 = p.coef + s2.coef_off;
      const double d1 = p.tbasis ? (j < s1.K ? (double)c1[j] : 0.0) : recomb_weight(c1, s1.K, j);
      const double d2 = p.tbasis ? (k < s2.K ? (double)c2[k] : 0.0) : recomb_weight(c2, s2.K, k);
      const double s = (h == 0 && (j & 1) && (k & 1)) ? -1.0 : 1.0;
      v = (float)(s * d1 * d2);
    }
    (h ? p.C1 : p.C0)[local] = v;
  }
}

// out_h (rows: amplitudes, columns: walks) = Y_h (amplitudes x K_h) C_h
// (K_h x walks), FP32. A block of 16 TN threads computes a 128 x 8 TN tile
// over k in steps of 8 with double-buffered shared-memory tiles; a thread
// holds an 8 x 8 sub-tile (rows tm*4 + {0..3} and 64 + tm*4 + {0..3},
// columns tn*4 + {0..3} and 4 TN + tn*4 + {0..3}), so its shared-memory
// reads are float4 and its stores float4 runs of four amplitudes of one
// walk. TN (4, 8 or 16: whole warps) is the smallest that covers the walk
// count in one column tile; a 104-column tile for 100 walks (208 threads)
// measured 7.6 ms against 6.3 ms for the 128-column one at n = 20.
constexpr int kBM = 128, kBK = 8;
__device__ __forceinline__ void fma_row(float (&r)[8], float a, const float4& b0,
                                        const float4& b1) {
  r[0] = fmaf(a, b0.x, r[0]);
  r[1] = fmaf(a, b0.y, r[1]);
  r[2] = fmaf(a, b0.z, r[2]);
  r[3] = fmaf(a, b0.w, r[3]);
  r[4] = fmaf(a, b1.x, r[4]);
  r[5] = fmaf(a, b1.y, r[5]);
  r[6] = fmaf(a, b1.z, r[6]);
  r[7] = fmaf(a, b1.w, r[7]);
}
template <int TN>
__global__ void __launch_bounds__(16 * TN, 2) s2_gemm_kernel(S2GemmParams p) {
  constexpr int T = 16 * TN, BN = 8 * TN;
  constexpr int kALoads = (kBM * kBK / 4 + T - 1) / T;  // float4 of the A tile per thread
  __shared__ __align__(16) float As[2][kBK][kBM];
  __shared__ __align__(16) float Bs[2][kBK][BN];
  const int h = blockIdx.z;
  const size_t N = (size_t)1 << p.n;
  const size_t m0 = (size_t)blockIdx.x * kBM;
  const int c0 = blockIdx.y * BN;
  const int K = h ? p.rows[1] : p.rows[0];
  const int Kp = h ? p.rows_pad[1] : p.rows_pad[0];
  const float* __restrict__ Y = p.Y + (h ? (size_t)p.rows[0] * N : 0);
  const float* __restrict__ C = h ? p.C1 : p.C0;
  float* __restrict__ out = p.out + (size_t)h * p.out_walks * N;
  const int t = threadIdx.x;
  const int br = t / (2 * TN), bc = (t % (2 * TN)) * 4;  // this thread's B-tile float4
  const int tm = t & 15, tn = t >> 4;
  float4 a[kALoads];
  auto load_a = [&](int k0) {
#pragma unroll
    for (int u = 0; u < kALoads; u++) {
      const int e = t + u * T;
      const int q = k0 + (e >> 5);
      a[u] = e < kBM * kBK / 4 && q < K
                 ? __ldcs(reinterpret_cast<const float4*>(Y + (size_t)q * N + m0 + (e & 31) * 4))
                 : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
  };
  auto store_a = [&](int buf) {
#pragma unroll
    for (int u = 0; u < kALoads; u++) {
      const int e = t + u * T;
      if (e < kBM * kBK / 4) *reinterpret_cast<float4*>(&As[buf][e >> 5][(e & 31) * 4]) = a[u];
    }
  };
  auto load_b = [&](int k0) -> float4 {
    return *reinterpret_cast<const float4*>(C + (size_t)(k0 + br) * p.col_stride + c0 + bc);
  };
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) acc[i][j] = 0.0f;
  load_a(0);
  float4 b = load_b(0);
  store_a(0);
  *reinterpret_cast<float4*>(&Bs[0][br][bc]) = b;
  __syncthreads();
  for (int k0 = 0; k0 < Kp; k0 += kBK) {
    const int cur = (k0 / kBK) & 1;
    const bool more = k0 + kBK < Kp;
    if (more) {
      load_a(k0 + kBK);
      b = load_b(k0 + kBK);
    }
#pragma unroll
    for (int kk = 0; kk < kBK; kk++) {
      const float4 a0 = *reinterpret_cast<const float4*>(&As[cur][kk][tm * 4]);
      const float4 a1 = *reinterpret_cast<const float4*>(&As[cur][kk][64 + tm * 4]);
      const float4 b0 = *reinterpret_cast<const float4*>(&Bs[cur][kk][tn * 4]);
      const float4 b1 = *reinterpret_cast<const float4*>(&Bs[cur][kk][4 * TN + tn * 4]);
      fma_row(acc[0], a0.x, b0, b1);
      fma_row(acc[1], a0.y, b0, b1);
      fma_row(acc[2], a0.z, b0, b1);
      fma_row(acc[3], a0.w, b0, b1);
      fma_row(acc[4], a1.x, b0, b1);
      fma_row(acc[5], a1.y, b0, b1);
      fma_row(acc[6], a1.z, b0, b1);
      fma_row(acc[7], a1.w, b0, b1);
    }
    if (more) {
      store_a(cur ^ 1);
      *reinterpret_cast<float4*>(&Bs[cur ^ 1][br][bc]) = b;
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const int col = c0 + (j < 4 ? tn * 4 + j : 4 * TN + tn * 4 + (j - 4));
    if (col >= p.walks) continue;
    float* o = out + (size_t)col * N + m0 + tm * 4;
    *reinterpret_cast<float4*>(o) = make_float4(acc[0][j], acc[1][j], acc[2][j], acc[3][j]);
    *reinterpret_cast<float4*>(o + 64) = make_float4(acc[4][j], acc[5][j], acc[6][j], acc[7][j]);
  }
}

__device__ __forceinline__ double block_sum_d(double v, double* s_red) {
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

// Interleaves a walk's planar psi_2 into its complex state slot and leaves
// the block's |psi_2|^2 in norm_part[b] (fixed order); block b covers
// amplitudes [b 2^L, (b+1) 2^L).
__global__ void __launch_bounds__(256) unpack_kernel(UnpackParams p) {
  __shared__ double s_red[32];
  const size_t chunk = (size_t)1 << p.L;
  const size_t base = (size_t)blockIdx.x * chunk;
  for (int g = 0; g < p.count; g++) {
    const UnpackWalk& W = p.walk[g];
    double nrm = 0.0;
    for (size_t i = base + 4 * threadIdx.x; i < base + chunk; i += 4 * blockDim.x) {
      const float4 re = __ldcs(reinterpret_cast<const float4*>(W.re + i));
      const float4 im = __ldcs(reinterpret_cast<const float4*>(W.im + i));
      float4* o = reinterpret_cast<float4*>(reinterpret_cast<float*>(W.out) + 2 * i);
      o[0] = make_float4(re.x, im.x, re.y, im.y);
      o[1] = make_float4(re.z, im.z, re.w, im.w);
      nrm += (double)re.x * re.x + (double)im.x * im.x + (double)re.y * re.y +
             (double)im.y * im.y + (double)re.z * re.z + (double)im.z * im.z +
             (double)re.w * re.w + (double)im.w * im.w;
    }
    const double sum = block_sum_d(nrm, s_red);
    if (threadIdx.x == 0) W.norm_part[blockIdx.x] = sum;
  }
}

// Projection onto the last two stages (m = 4): per walk w (blockIdx.y) the
// bilinear sum a = sum_i V_i psi_i (complex, no conjugation: psi_4[E_loc] =
// e^T U_4 U_3 psi_2 = sum_i (U_3^T U_4^T e)_i psi_2,i with H~ real symmetric)
// of the walk's recombined vector V and its stage-2 state psi_2, and
// |psi_2|^2; block b covers amplitudes [b 2^L, (b+1) 2^L) and leaves its
// FP64 partials (Re a, Im a, |psi_2|^2) at part[(w nblk + b) 3 + c] (fixed
// order, so the result is reproducible run to run).
__global__ void __launch_bounds__(256) last2_partial_kernel(Last2Params p) {
  __shared__ double s_red[32];
  const size_t N = (size_t)1 << p.n;
  const size_t chunk = (size_t)1 << p.L;
  const size_t base = (size_t)blockIdx.x * chunk;
  const int w = blockIdx.y;
  const float* vr = p.V + (size_t)w * N;
  const float* vi = p.V + (size_t)(p.v_walks + w) * N;
  const float* pr = p.psi + (size_t)w * N;
  const float* pi = p.psi + (size_t)(p.psi_walks + w) * N;
  double are = 0.0, aim = 0.0, nrm = 0.0;
  for (size_t i = base + 4 * threadIdx.x; i < base + chunk; i += 4 * blockDim.x) {
    const float4 a = __ldcs(reinterpret_cast<const float4*>(vr + i));
    const float4 b = __ldcs(reinterpret_cast<const float4*>(vi + i));
    const float4 c = __ldcs(reinterpret_cast<const float4*>(pr + i));
    const float4 d = __ldcs(reinterpret_cast<const float4*>(pi + i));
    are += (double)a.x * c.x - (double)b.x * d.x + (double)a.y * c.y - (double)b.y * d.y +
           (double)a.z * c.z - (double)b.z * d.z + (double)a.w * c.w - (double)b.w * d.w;
    aim += (double)a.x * d.x + (double)b.x * c.x + (double)a.y * d.y + (double)b.y * c.y +
           (double)a.z * d.z + (double)b.z * c.z + (double)a.w * d.w + (double)b.w * c.w;
    nrm += (double)c.x * c.x + (double)d.x * d.x + (double)c.y * c.y + (double)d.y * d.y +
           (double)c.z * c.z + (double)d.z * d.z + (double)c.w * c.w + (double)d.w * d.w;
  }
  const double sa = block_sum_d(are, s_red);
  const double sb = block_sum_d(aim, s_red);
  const double sc = block_sum_d(nrm, s_red);
  if (threadIdx.x == 0) {
    double* o = p.part + ((size_t)w * gridDim.x + blockIdx.x) * 3;
    o[0] = sa;
    o[1] = sb;
    o[2] = sc;
  }
}

// Per walk (one thread each): the partials summed in block order, and
// P = |a|^2 / |psi_2|^2 (the norms of the stage-3 and stage-4 outputs taken
// as their inputs', exact up to the 1e-6 Chebyshev tail).
__global__ void last2_final_kernel(Last2Params p, int nblk) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= p.walks) return;
  double a = 0.0, b = 0.0, c = 0.0;
  const double* q = p.part + (size_t)w * nblk * 3;
  for (int k = 0; k < nblk; k++) {
    a += q[3 * k];
    b += q[3 * k + 1];
    c += q[3 * k + 2];
  }
  p.p_out[w] = (a * a + b * b) / c;
}

}  // namespace

cudaError_t launch_last2(const Last2Params& p, cudaStream_t stream) {
  if (p.n < 8 || p.n > kMaxN || p.L < 8 || p.L > p.n || p.walks < 1 || p.walks > 65535 ||
      p.v_walks < p.walks || p.psi_walks < p.walks || !p.V || !p.psi || !p.part || !p.p_out)
    return cudaErrorInvalidValue;
  const int nblk = 1 << (p.n - p.L);
  last2_partial_kernel<<<dim3((unsigned)nblk, (unsigned)p.walks), 256, 0, stream>>>(p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  last2_final_kernel<<<(p.walks + 127) / 128, 128, 0, stream>>>(p, nblk);
  return cudaGetLastError();
}

size_t last2_part_bytes(int n, int walks) {
  const int L = n < 12 ? n : 12;
  return (size_t)walks * ((size_t)1 << (n - L)) * 3 * sizeof(double);
}

cudaError_t launch_real_to_complex(void* dst, const float* src, int n, cudaStream_t stream) {
  if (n < 1 || n > kMaxN || !dst || !src) return cudaErrorInvalidValue;
  const size_t N = (size_t)1 << n;
  const size_t want = (N + 255) / 256;
  const unsigned blocks = (unsigned)(want < 4096 ? want : 4096);
  real_to_complex_kernel<<<blocks, 256, 0, stream>>>(reinterpret_cast<float2*>(dst), src, N);
  return cudaGetLastError();
}

int s2_tile_cols(int walks) { return walks <= 32 ? 32 : walks <= 64 ? 64 : 128; }

cudaError_t launch_s2_coef(const S2CoefParams& p, cudaStream_t stream) {
  if (!p.stages || !p.coef || !p.C0 || !p.C1 || p.walks < 1 || p.col_stride < p.walks ||
      p.col_stride % 8 != 0 || p.m < 3 || p.lay.Kb < 1 || p.lay.K2 < 1 ||
      p.rows_pad[0] < p.lay.rows(0) || p.rows_pad[1] < p.lay.rows(1))
    return cudaErrorInvalidValue;
  const size_t total = ((size_t)p.rows_pad[0] + p.rows_pad[1]) * p.col_stride;
  const size_t want = (total + 255) / 256;
  const unsigned blocks = (unsigned)(want < 8192 ? want : 8192);
  s2_coef_kernel<<<blocks, 256, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_s2_gemm(const S2GemmParams& p, cudaStream_t stream) {
  const int bn = s2_tile_cols(p.walks);
  if (p.n < 7 || p.n > kMaxN || !p.Y || !p.C0 || !p.C1 || !p.out || p.walks < 1 ||
      p.out_walks < p.walks || p.col_stride % bn != 0 || p.col_stride < p.walks ||
      p.rows[0] < 1 || p.rows[1] < 0)
    return cudaErrorInvalidValue;
  for (int h = 0; h < 2; h++)
    if (p.rows_pad[h] < p.rows[h] || p.rows_pad[h] % kBK != 0) return cudaErrorInvalidValue;
  const size_t N = (size_t)1 << p.n;
  const dim3 grid((unsigned)(N / kBM), (unsigned)(p.col_stride / bn), p.rows[1] > 0 ? 2 : 1);
  switch (bn) {
    case 32: s2_gemm_kernel<4><<<grid, 64, 0, stream>>>(p); break;
    case 64: s2_gemm_kernel<8><<<grid, 128, 0, stream>>>(p); break;
    default: s2_gemm_kernel<16><<<grid, 256, 0, stream>>>(p); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_unpack(const UnpackParams& p, cudaStream_t stream) {
  if (p.n < 6 || p.n > kMaxN || p.L < 6 || p.L > p.n || p.count < 1 || p.count > kMaxGroup)
    return cudaErrorInvalidValue;
  for (int g = 0; g < p.count; g++)
    if (!p.walk[g].re || !p.walk[g].im || !p.walk[g].out || !p.walk[g].norm_part)
      return cudaErrorInvalidValue;
  unpack_kernel<<<(unsigned)((size_t)1 << (p.n - p.L)), 256, 0, stream>>>(p);
  return cudaGetLastError();
}

}  // namespace mqw
