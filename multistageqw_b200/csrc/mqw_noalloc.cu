// mqw_clenshaw_noalloc: the grid-path Clenshaw propagation for callers that
// cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: code that must not synchronise the
// device (cudaMalloc/cudaFree can), and hosts whose own allocator owns all
// device memory (a framework memory pool, an embedded/real-time process with
// a fixed memory budget). For them this entry point takes only caller-owned
// device buffers and keeps its own working space in a fixed file-scope
// device array, so it calls no allocating CUDA or library routine.
//
// The working space is the partial sum P (2^n amplitudes) and one norm
// partial per tile. Its size is fixed at MQW_NOALLOC_MAX_N = 16: 2^16
// complex128 amplitudes plus partials, about 1 MiB, held by every GPU that
// loads the library until the process exits. The caller's output buffer
// doubles as the Clenshaw vector b (it ends holding b_0, the result).
//
// Sharing rules: every call uses the same array and leaves its contents
// behind. Nothing in it has to start at zero — each call writes every element
// it later reads — but two calls that overlap on the GPU (different streams,
// or different host threads without ordering) race on the array; order them
// on one stream.
//
// Set-up: the device address of the array is looked up once per device with
// cudaGetSymbolAddress, with that device current, on the first call made on
// that device. Make that first call before starting any stream capture. The
// address is kept for the life of the process, so a device that has been
// reset (cudaDeviceReset) must not be used with this entry point again.
//
// On any status other than MQW_OK, passes may already be queued: the
// contents of the caller's output buffer are then undefined.
#include <mutex>

#include "../../include/mqw.h"
#include "mqw_internal.h"

namespace mqw {
namespace {

constexpr size_t kNoAllocAmps = (size_t)1 << MQW_NOALLOC_MAX_N;
constexpr size_t kNoAllocPartBytes = kNoAllocAmps * 16;  // complex128 worst case
constexpr size_t kNoAllocNormBytes = 4096 * sizeof(double);

// The working space shared by every call (see the file comment). In host
// code this name is a host-side handle, not a device address: only the
// address returned by cudaGetSymbolAddress may be passed to a kernel.
static __device__ __align__(256) unsigned char
    g_noalloc_scratch[kNoAllocPartBytes + kNoAllocNormBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device, looked up once.
cudaError_t scratch_address(int device, void** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_addr[device] = p;
  }
  *out = g_addr[device];
  return cudaSuccess;
}

}  // namespace
}  // namespace mqw

using namespace mqw;

extern "C" mqw_status mqw_clenshaw_noalloc(int precision, int n, int K,
                                           const float* d_coeffs,
                                           const float* d_hp, float gamma,
                                           float scale, const void* d_psi,
                                           void* d_out, void* stream) {
  if ((precision != MQW_FP32 && precision != MQW_FP64) || K < 1 || !d_coeffs ||
      !d_hp || !d_psi || !d_out || d_psi == d_out || !(scale > 0.0f))
    return MQW_ERR_INVALID;
  if (n < 6) return MQW_ERR_INVALID;
  if (n > MQW_NOALLOC_MAX_N) return MQW_ERR_UNSUPPORTED;  // beyond the fixed scratch
  const PassGeomHost geo = pass_geom(precision, n);
  if (geo.nu != 0) return MQW_ERR_UNSUPPORTED;  // would need a second b buffer
  const size_t tiles = ((size_t)1 << n) >> geo.L;
  if (tiles * sizeof(double) > kNoAllocNormBytes) return MQW_ERR_UNSUPPORTED;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
    return MQW_ERR_NO_DEVICE;
  void* base = nullptr;
  if (scratch_address(device, &base) != cudaSuccess) return MQW_ERR_CUDA;
  unsigned char* scratch = static_cast<unsigned char*>(base);
  void* part = scratch;
  double* norm_part = reinterpret_cast<double*>(scratch + kNoAllocPartBytes);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  for (int r = K - 1; r >= 0; r--) {
    PassParams pp{};
    pp.n = n;
    pp.L = geo.L;
    pp.C = geo.C;
    pp.threads = geo.threads;
    pp.lane_smem = geo.lane_smem;
    pp.tma = geo.tma;
    pp.a = geo.a;
    pp.tiling = (r & 1) ? 2 : 1;
    pp.count = 1;
    PassWalk& W = pp.walk[0];
    W.active = 1;
    W.bin = d_out;  // b is updated in place in the caller's output buffer
    W.bout = d_out;
    W.part = part;
    W.psi = d_psi;
    W.hp = d_hp;
    W.coef = d_coeffs;
    W.kappa = nullptr;
    W.norm_part = norm_part;
    W.gamma = gamma;
    W.scale = scale;
    W.r = r;
    W.K = K;
    W.psi_uniform = 0;
    W.psi0 = 0.0f;
    if (launch_pass(precision, pp, st) != cudaSuccess) return MQW_ERR_CUDA;
  }
  return MQW_OK;
}
