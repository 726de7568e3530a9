// Bandwidth probes of the memory tiers a walk's working set can live in:
// L2 (a buffer that fits in it, read and copied with L1-bypassing loads),
// shared memory (conflict-free 16-byte loads), and HBM (a copy of buffers
// far larger than L2). They give the roofline denominators for workloads
// whose states are L2- or shared-memory-resident; the HBM figure is a
// cross-check of the copy bandwidth measured outside the library.
//
// Every kernel is a bounded loop over buffers the probe owns; times are CUDA
// events on the context's stream around `reps` launches after a warm-up.
#include "mqw_internal.h"

namespace mqw {
namespace {

// Reads n4 float4 of an L2-resident buffer `iters` times (ld.global.cg: L2
// only, so L1 never serves a repeat).
__global__ void l2_read_kernel(const float4* __restrict__ buf, size_t n4, int iters,
                               float* sink) {
  float acc = 0.0f;
  for (int it = 0; it < iters; it++)
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4;
         i += (size_t)gridDim.x * blockDim.x) {
      const float4 v = __ldcg(buf + i);
      acc += v.x + v.y + v.z + v.w;
    }
  if (acc == 1.2345e-30f) *sink = acc;  // keeps the loads; never true for zeros
}

// dst = src over n4 float4 (both L2-resident), `iters` times, through L2.
__global__ void l2_copy_kernel(const float4* __restrict__ src, float4* __restrict__ dst,
                               size_t n4, int iters) {
  for (int it = 0; it < iters; it++)
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4;
         i += (size_t)gridDim.x * blockDim.x)
      __stcg(dst + i, __ldcg(src + i));
}

// Each block reads its 32 KB of shared memory `iters` times with 16-byte
// loads that are consecutive across the warp (no bank conflicts), rotated by
// the iteration so that no load is loop-invariant.
constexpr int kSmemFloat4 = 32 * 1024 / 16;  // a power of two
__global__ void smem_read_kernel(int iters, float* sink) {
  __shared__ float4 s[kSmemFloat4];
  for (int i = threadIdx.x; i < kSmemFloat4; i += blockDim.x)
    s[i] = make_float4((float)i, 0.0f, 0.0f, 0.0f);
  __syncthreads();
  float acc = 0.0f;
  for (int it = 0; it < iters; it++)
#pragma unroll 4
    for (int i = threadIdx.x; i < kSmemFloat4; i += blockDim.x) {
      const float4 v = s[(i + it) & (kSmemFloat4 - 1)];
      acc += v.x + v.y + v.z + v.w;
    }
  if (acc == -1.0f) *sink = acc;  // never true: the values are non-negative
}

// dst = src over n4 float4 of HBM-sized buffers (streaming loads and stores).
__global__ void hbm_copy_kernel(const float4* __restrict__ src, float4* __restrict__ dst,
                                size_t n4) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4;
       i += (size_t)gridDim.x * blockDim.x)
    __stcs(dst + i, __ldcs(src + i));
}

template <typename Launch>
cudaError_t time_ms(cudaStream_t st, int reps, Launch launch, float* ms) {
  cudaEvent_t e0, e1;
  cudaError_t e = cudaEventCreate(&e0);
  if (e != cudaSuccess) return e;
  e = cudaEventCreate(&e1);
  if (e != cudaSuccess) {
    cudaEventDestroy(e0);
    return e;
  }
  launch();  // warm-up
  e = cudaEventRecord(e0, st);
  for (int r = 0; r < reps && e == cudaSuccess; r++) {
    launch();
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(e1, st);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return e;
}

}  // namespace

cudaError_t measure_tiers(cudaStream_t st, int sm_count, double* l2_read_gbs,
                          double* l2_copy_gbs, double* smem_gbs, double* hbm_copy_gbs) {
  const size_t l2_bytes = (size_t)32 << 20;  // well inside the 126 MB L2
  const size_t hbm_bytes = (size_t)1 << 30;  // far beyond it
  float4 *a = nullptr, *b = nullptr;
  float* sink = nullptr;
  cudaError_t e = cudaMalloc(&a, hbm_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&b, hbm_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&sink, sizeof(float));
  if (e == cudaSuccess) e = cudaMemsetAsync(a, 0, hbm_bytes, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(b, 0, hbm_bytes, st);
  const unsigned blocks = (unsigned)(sm_count * 4);
  const int threads = 256;
  float ms = 0.0f;
  if (e == cudaSuccess) {
    const size_t n4 = l2_bytes / 16;
    const int iters = 20, reps = 5;
    e = time_ms(st, reps, [&] { l2_read_kernel<<<blocks, threads, 0, st>>>(a, n4, iters, sink); }, &ms);
    if (e == cudaSuccess) *l2_read_gbs = (double)l2_bytes * iters * reps / (ms * 1e-3) / 1e9;
  }
  if (e == cudaSuccess) {
    const size_t n4 = l2_bytes / 2 / 16;  // 16 MB in, 16 MB out
    const int iters = 20, reps = 5;
    e = time_ms(st, reps, [&] { l2_copy_kernel<<<blocks, threads, 0, st>>>(a, b, n4, iters); }, &ms);
    if (e == cudaSuccess) *l2_copy_gbs = (double)l2_bytes * iters * reps / (ms * 1e-3) / 1e9;
  }
  if (e == cudaSuccess) {
    const int iters = 200, reps = 5;
    const unsigned sblocks = (unsigned)(sm_count * 4);  // 4 x 32 KB per SM
    e = time_ms(st, reps, [&] { smem_read_kernel<<<sblocks, threads, 0, st>>>(iters, sink); }, &ms);
    if (e == cudaSuccess)
      *smem_gbs = (double)sblocks * kSmemFloat4 * 16.0 * iters * reps / (ms * 1e-3) / 1e9;
  }
  if (e == cudaSuccess) {
    const size_t n4 = hbm_bytes / 16;
    const int reps = 5;
    e = time_ms(st, reps, [&] { hbm_copy_kernel<<<blocks * 2, threads, 0, st>>>(a, b, n4); }, &ms);
    if (e == cudaSuccess) *hbm_copy_gbs = 2.0 * (double)hbm_bytes * reps / (ms * 1e-3) / 1e9;
  }
  if (a) cudaFree(a);
  if (b) cudaFree(b);
  if (sink) cudaFree(sink);
  return e;
}

}  // namespace mqw
