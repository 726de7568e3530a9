// Per-(instance, stage, sample) Chebyshev degree and coefficients on the GPU
// in FP64 (one thread per job). The rescaled spectral width is
//   onenorm = fl(E_abs + gamma*n)   (MultiQW.cpp:436, fused multiply-add)
//   s       = double(fl(onenorm * t))  (MultiQW.cpp:438, a float product)
// and the coefficients are those of mqw_cheb.h (MultiQW.cpp:439-440).
#include "mqw_cheb.h"
#include "mqw_internal.h"

namespace mqw {
namespace {

__device__ __forceinline__ void job_s(const CoefJob& j, const DiagOut* diag,
                                      float* onenorm, double* s) {
  const float on = __fmaf_rn(j.gamma, (float)j.n, diag[j.inst].e_abs);
  *onenorm = on;
  *s = (double)__fmul_rn(on, j.t);
}

__global__ void cheb_degree_kernel(const CoefJob* jobs, int count,
                                   const DiagOut* diag, double tol,
                                   int* degree, float* onenorm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  float on;
  double s;
  job_s(jobs[i], diag, &on, &s);
  degree[i] = cheb_coeffs_stream(s, tol, nullptr, 0);
  if (onenorm) onenorm[i] = on;
}

__global__ void cheb_coeffs_kernel(const CoefJob* jobs, int count,
                                   const DiagOut* diag, double tol,
                                   const long long* offset, float* coef) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  float on;
  double s;
  job_s(jobs[i], diag, &on, &s);
  const long long off = offset[i];
  const int room = (int)(offset[i + 1] - off);
  cheb_coeffs_stream(s, tol, coef + off, room);
}

__global__ void cheb_from_s_kernel(const double* s, int count, double tol,
                                   int max_k, float* coef, int* degree) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  degree[i] = cheb_coeffs_stream(s[i], tol, coef + (size_t)i * max_k, max_k);
}

}  // namespace

cudaError_t launch_cheb_degree(const CoefJob* jobs, int count,
                               const DiagOut* diag, double tol, int* degree,
                               float* onenorm, cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  const int T = 128;
  cheb_degree_kernel<<<(count + T - 1) / T, T, 0, stream>>>(jobs, count, diag,
                                                           tol, degree, onenorm);
  return cudaGetLastError();
}

cudaError_t launch_cheb_coeffs(const CoefJob* jobs, int count,
                               const DiagOut* diag, double tol,
                               const long long* offset, float* coef,
                               cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  const int T = 128;
  cheb_coeffs_kernel<<<(count + T - 1) / T, T, 0, stream>>>(jobs, count, diag,
                                                           tol, offset, coef);
  return cudaGetLastError();
}

cudaError_t launch_cheb_from_s(const double* s, int count, double tol,
                               int max_k, float* coef, int* degree,
                               cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  const int T = 128;
  cheb_from_s_kernel<<<(count + T - 1) / T, T, 0, stream>>>(s, count, tol,
                                                           max_k, coef, degree);
  return cudaGetLastError();
}

}  // namespace mqw
