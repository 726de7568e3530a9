// Kernels of the learned stage schedule: a small MLP whose weights are stored
// in BF16 and whose products accumulate in FP32.
//
//   forward  : Y = act(X W^T + b)                      (X: B x in, W: out x in)
//   backward : dZ = dY * [Y > 0] (ReLU layers), dX = dZ W, dW = dZ^T X,
//              db = column sums of dZ
//   Adam     : FP32 master weights and moments, refreshed BF16 copy
//
// One tiled GEMM kernel serves all three products. Operands are read through
// strides (so transposes cost nothing), BF16 weights are widened to FP32 as
// they are staged in shared memory, and each thread accumulates a 4 x 4 block
// in FP32. The matrices are at most a few hundred wide: these kernels run in
// microseconds and their job is exactness and checkability, not peak
// throughput.
#include <cuda_bf16.h>

#include "../../include/mqw.h"

namespace {

constexpr int kTile = 64;
constexpr int kK = 16;

struct Operand {
  const void* p;
  long long si, sk;      // element (i, k) at p[i*si + k*sk]
  int bf16;              // 1: BF16 elements, 0: FP32
  const float* mask;     // optional ReLU mask source (same strides): x * [mask > 0]
};

__device__ __forceinline__ float op_load(const Operand& o, long long i, long long k) {
  const long long idx = i * o.si + k * o.sk;
  float v = o.bf16 ? __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(o.p)[idx])
                   : reinterpret_cast<const float*>(o.p)[idx];
  if (o.mask && !(o.mask[idx] > 0.0f)) v = 0.0f;
  return v;
}

// C[M x N] = A[M x K] B[K x N] (+ bias[N]) (ReLU if relu), FP32 accumulate.
// A(i, k) and B(k, j) come from the Operand descriptors.
__global__ void __launch_bounds__(256) gemm_kernel(int M, int N, int K, Operand A,
                                                   Operand B, const float* bias,
                                                   int relu, float* C, long long ldc) {
  __shared__ float sA[kK][kTile + 1];
  __shared__ float sB[kK][kTile + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const long long i0 = (long long)blockIdx.y * kTile, j0 = (long long)blockIdx.x * kTile;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += kK) {
    for (int e = threadIdx.x; e < kK * kTile; e += blockDim.x) {
      const int kk = e / kTile, ii = e % kTile;
      const long long gi = i0 + ii, gj = j0 + ii, gk = k0 + kk;
      sA[kk][ii] = (gi < M && gk < K) ? op_load(A, gi, gk) : 0.0f;
      sB[kk][ii] = (gj < N && gk < K) ? op_load(B, gk, gj) : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kK; kk++) {
      float a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        a[u] = sA[kk][ty * 4 + u];
        b[u] = sB[kk][tx * 4 + u];
      }
#pragma unroll
      for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) acc[u][v] = fmaf(a[u], b[v], acc[u][v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; u++) {
    const long long i = i0 + ty * 4 + u;
    if (i >= M) continue;
#pragma unroll
    for (int v = 0; v < 4; v++) {
      const long long j = j0 + tx * 4 + v;
      if (j >= N) continue;
      float c = acc[u][v];
      if (bias) c += bias[j];
      if (relu && !(c > 0.0f)) c = 0.0f;
      C[i * ldc + j] = c;
    }
  }
}

// db[j] = sum_i dY[i, j] * [Y[i, j] > 0 or !relu], fixed summation order.
__global__ void bias_grad_kernel(int B, int out, const float* dY, const float* Y,
                                 int relu, float* db) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= out) return;
  float s = 0.0f;
  for (int i = 0; i < B; i++) {
    const long long idx = (long long)i * out + j;
    const float g = dY[idx];
    if (!relu || Y[idx] > 0.0f) s += g;
  }
  db[j] = s;
}

__global__ void adam_kernel(int count, float* w, __nv_bfloat16* wb, const float* g,
                            float* m, float* v, float lr, float b1, float b2,
                            float eps, float c1, float c2, float wd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float gi = g[i] + wd * w[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16_rn(wi);
}

__global__ void to_bf16_kernel(int count, const float* w, __nv_bfloat16* wb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) wb[i] = __float2bfloat16_rn(w[i]);
}

mqw_status launch_gemm(int M, int N, int K, const Operand& A, const Operand& B,
                       const float* bias, int relu, float* C, long long ldc,
                       cudaStream_t st) {
  if (M <= 0 || N <= 0 || K <= 0) return MQW_OK;
  dim3 grid((N + kTile - 1) / kTile, (M + kTile - 1) / kTile);
  gemm_kernel<<<grid, 256, 0, st>>>(M, N, K, A, B, bias, relu, C, ldc);
  return cudaGetLastError() == cudaSuccess ? MQW_OK : MQW_ERR_CUDA;
}

}  // namespace

extern "C" {

mqw_status mqw_mlp_linear_forward(int batch, int in, int out,
                                  const uint16_t* W_bf16, const float* b,
                                  const float* X, float* Y, int relu,
                                  void* stream) {
  if (batch < 0 || in < 1 || out < 1 || !W_bf16 || !X || !Y) return MQW_ERR_INVALID;
  Operand A{X, in, 1, 0, nullptr};            // X(i, k) = X[i*in + k]
  Operand B{W_bf16, 1, in, 1, nullptr};       // W^T(k, j) = W[j*in + k]
  return launch_gemm(batch, out, in, A, B, b, relu, Y, out, (cudaStream_t)stream);
}

mqw_status mqw_mlp_linear_backward(int batch, int in, int out,
                                   const uint16_t* W_bf16, const float* X,
                                   const float* Y, const float* dY, float* dX,
                                   float* dW, float* db, int relu,
                                   void* stream) {
  if (batch < 1 || in < 1 || out < 1 || !W_bf16 || !X || !dY || !dW || !db ||
      (relu && !Y))
    return MQW_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  const float* mask = relu ? Y : nullptr;
  // dW[out x in] = dZ^T X: A(i, k) = dZ(k, i), B(k, j) = X(k, j).
  Operand At{dY, 1, out, 0, mask};
  Operand Bx{X, 1, in, 0, nullptr};
  Bx.si = in;  // B(k, j) = X[k*in + j]
  Bx.sk = 1;
  mqw_status s = launch_gemm(out, in, batch, At, Bx, nullptr, 0, dW, in, st);
  if (s != MQW_OK) return s;
  bias_grad_kernel<<<(out + 127) / 128, 128, 0, st>>>(batch, out, dY, Y, relu, db);
  if (cudaGetLastError() != cudaSuccess) return MQW_ERR_CUDA;
  if (dX) {
    // dX[batch x in] = dZ W: A(i, k) = dZ(i, k), B(k, j) = W[k*in + j].
    Operand Ad{dY, out, 1, 0, mask};
    Operand Bw{W_bf16, in, 1, 1, nullptr};
    s = launch_gemm(batch, in, out, Ad, Bw, nullptr, 0, dX, in, st);
  }
  return s;
}

mqw_status mqw_mlp_adam(int count, float* w, uint16_t* w_bf16, const float* g,
                        float* m, float* v, float lr, float beta1, float beta2,
                        float eps, float weight_decay, int step, void* stream) {
  if (count < 0 || !w || !g || !m || !v || step < 1) return MQW_ERR_INVALID;
  if (count == 0) return MQW_OK;
  const float c1 = 1.0f - powf(beta1, (float)step);
  const float c2 = 1.0f - powf(beta2, (float)step);
  adam_kernel<<<(count + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
      count, w, reinterpret_cast<__nv_bfloat16*>(w_bf16), g, m, v, lr, beta1, beta2,
      eps, c1, c2, weight_decay);
  return cudaGetLastError() == cudaSuccess ? MQW_OK : MQW_ERR_CUDA;
}

mqw_status mqw_mlp_to_bf16(int count, const float* w, uint16_t* w_bf16,
                           void* stream) {
  if (count < 0 || !w || !w_bf16) return MQW_ERR_INVALID;
  if (count == 0) return MQW_OK;
  to_bf16_kernel<<<(count + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
      count, w, reinterpret_cast<__nv_bfloat16*>(w_bf16));
  return cudaGetLastError() == cudaSuccess ? MQW_OK : MQW_ERR_CUDA;
}

}  // extern "C"
