// Host runtime of the C ABI (include/mqw.h): contexts, plans and the launch
// schedule of the propagation.
//
// A plan turns a batch of instances into device work:
//   1. diagonal   : per n-group, launch_diag (reference-exact energies,
//                   E_loc, E_abs) into a pooled hp buffer;
//   2. degrees    : one FP64 thread per (instance, stage, sample) job;
//                   degrees and onenorms are read back (the only host sync
//                   inside execute) to lay out the coefficient pool and the
//                   launch schedule;
//   3. coefficients: written packed into the pool;
//   4. propagation: walks with n <= resident_max_n run in one launch of the
//                   resident kernel (a CTA per walk); larger n run on the
//                   grid path, one launch per Clenshaw term over groups of up
//                   to 8 walks of the same n, instance by instance with the
//                   instance's shared bases: the stage-1 basis (recombined
//                   per basis group), the stage-2 product basis (chains and
//                   one GEMM for all walks, when it pays) and the last-stage
//                   basis (projected per basis group);
//   5. means      : mean ground-state probability per instance.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/mqw.h"
#include "mqw_cheb.h"
#include "mqw_internal.h"

using namespace mqw;

// Owning device allocation.
struct DevMem {
  void* p = nullptr;
  size_t bytes = 0;
  DevMem() = default;
  DevMem(const DevMem&) = delete;
  DevMem& operator=(const DevMem&) = delete;
  ~DevMem() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  cudaError_t ensure(size_t b) {
    if (b <= bytes && p) return cudaSuccess;
    release();
    if (b == 0) b = 16;
    cudaError_t e = cudaMalloc(&p, b);
    if (e == cudaSuccess) bytes = b;
    return e;
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

// Grid-path shape for one (precision, n): tile cap, walks per launch, and
// concurrent launch lanes.
struct GridShape {
  int lmax = 0, group = 1, lanes = 1;
  int threads = 0;  // CTA threads at the widest tile (0: 512)
  int lane_smem = 0;  // lane axes: 1 shared memory, -1 shuffles, 0 (want): any
  int tma = 0;        // staging: 1 bulk copies, 2 a second exchange tile,
                      // -1 cp.async, 0 (want): any
  int cl = 0;         // where the widest tile leaves axes over: 1 a tile
                      // spanning a cluster, -1 single-CTA tiles with those
                      // axes read from global memory, 0 (want): any
  double us = 0.0;  // timed microseconds per walk-pass (0: not timed)
  int bgroup = 1;   // walks per shared-basis group (>= group; set by the plan)
};
constexpr int kMaxLanes = 4;    // walk lanes (the tuner's range)
constexpr int kMaxStreams = 8;  // lane streams: walk lanes and chain lanes
// Chain lanes of the one-chain-per-launch product-basis chains (n >= 19):
// measured at n = 20, m = 4 (26.5 instances/s on 3 lanes, 27.9 on 4).
constexpr int kChainLanes = 4;

// A context owns the reusable device scratch that plans share: the grid-path
// state slots, norm partials, the coefficient pool and its tables, and the
// diagonal's chunk partials. Plans of one context are executed one at a time
// (the ABI's threading rule), so sharing is safe and repeated calls do not
// pay for allocation.
struct mqw_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  int sm_count = 0;
  DevMem state, norm_part, kappa, diag_scratch, tune_coef;
  // Device error word: kernels whose bounded waits give up set bit 0; the
  // host reads and clears it when it collects results.
  DevMem dev_err;
  DevMem basis, basis2;  // shared bases of the instance in flight and of
                         // the next one (+ their slots)
  // The basis stream builds the next instance's bases while the current
  // instance's walks run; events order the two buffers' uses.
  cudaStream_t basis_stream = nullptr;
  cudaEvent_t basis_built[2] = {}, basis_free[2] = {};
  // The basis stream's own lanes (1..): its stage-2 chains run on the basis
  // stream and these, forked and joined like the walk lanes.
  cudaStream_t bld_stream[kMaxStreams] = {};
  cudaEvent_t bld_fork_ev = nullptr;
  cudaEvent_t bld_join_ev[kMaxStreams] = {};
  cudaError_t ensure_basis_stream() {
    cudaError_t e = cudaSuccess;
    if (!basis_stream) e = cudaStreamCreateWithFlags(&basis_stream, cudaStreamNonBlocking);
    for (int k = 0; k < 2 && e == cudaSuccess; k++) {
      if (!basis_built[k]) e = cudaEventCreateWithFlags(&basis_built[k], cudaEventDisableTiming);
      if (e == cudaSuccess && !basis_free[k])
        e = cudaEventCreateWithFlags(&basis_free[k], cudaEventDisableTiming);
    }
    if (e == cudaSuccess && !bld_fork_ev)
      e = cudaEventCreateWithFlags(&bld_fork_ev, cudaEventDisableTiming);
    for (int k = 1; k < kMaxStreams && e == cudaSuccess; k++) {
      if (!bld_stream[k]) e = cudaStreamCreateWithFlags(&bld_stream[k], cudaStreamNonBlocking);
      if (e == cudaSuccess && !bld_join_ev[k])
        e = cudaEventCreateWithFlags(&bld_join_ev[k], cudaEventDisableTiming);
    }
    return e;
  }
  DevMem proj_part;  // last-stage projection partial dots, per lane
  // Stage-2 product basis: the Y vectors, every walk's planar stage-2
  // output, and the coefficient matrices (one instance at a time).
  DevMem s2y, s2psi, s2c;
  DevMem s2chain;  // chain slots of the build-ahead (4 complex vectors)
  DevMem s2part;   // partial P of each batched product-basis chain
  DevMem s3y, s3v, s3part;  // product basis of the last two stages, its
                            // recombined vectors, projection partials
  // Bumped whenever a shared scratch buffer is reallocated: a plan's captured
  // graph holds the old addresses and is re-captured when this changes.
  unsigned long long scratch_gen = 1;
  // Autotuned grid-path geometry per (precision, n).
  std::map<std::pair<int, int>, GridShape> tuned;
  // Concurrent walk-group lanes of the grid path: lane 0 runs on the
  // launching stream, lanes 1.. on these private streams, forked from and
  // joined back into the launching stream with events (which a CUDA graph
  // capture follows, so a captured pipeline keeps its lanes concurrent).
  cudaStream_t lane_stream[kMaxStreams] = {};
  cudaEvent_t fork_ev = nullptr;
  cudaEvent_t join_ev[kMaxStreams] = {};
  cudaError_t ensure_lanes(int lanes) {
    if (!fork_ev) {
      cudaError_t e = cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming);
      if (e != cudaSuccess) return e;
    }
    for (int k = 1; k < lanes && k < kMaxStreams; k++) {
      if (!lane_stream[k]) {
        cudaError_t e = cudaStreamCreateWithFlags(&lane_stream[k], cudaStreamNonBlocking);
        if (e != cudaSuccess) return e;
      }
      if (!join_ev[k]) {
        cudaError_t e = cudaEventCreateWithFlags(&join_ev[k], cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
      }
    }
    return cudaSuccess;
  }
  // Makes lanes 1..lanes-1 wait for the work queued so far on `stream`.
  cudaError_t fork(cudaStream_t stream, int lanes) {
    if (lanes <= 1) return cudaSuccess;
    cudaError_t e = cudaEventRecord(fork_ev, stream);
    for (int k = 1; k < lanes && e == cudaSuccess; k++)
      e = cudaStreamWaitEvent(lane_stream[k], fork_ev, 0);
    return e;
  }
  // Makes `stream` wait for everything queued on lanes 1..lanes-1.
  cudaError_t join(cudaStream_t stream, int lanes) {
    cudaError_t e = cudaSuccess;
    for (int k = 1; k < lanes && e == cudaSuccess; k++) {
      e = cudaEventRecord(join_ev[k], lane_stream[k]);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, join_ev[k], 0);
    }
    return e;
  }
  cudaError_t grow(DevMem& m, size_t bytes) {
    if (bytes <= m.bytes && m.p) return cudaSuccess;
    scratch_gen++;
    return m.ensure(bytes);
  }
};

namespace {

mqw_status fail(mqw_ctx* ctx, mqw_status s, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return s;
}

#define CK(call)                                                            \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess)                                                  \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? MQW_ERR_NOMEM      \
                                                       : MQW_ERR_CUDA,      \
                  "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),   \
                  __FILE__, __LINE__);                                      \
  } while (0)

int params_per(int n) { return n * (n + 1) / 2; }

void default_opts(mqw_options* o) {
  o->precision = MQW_FP32;
  o->samples = MQW_SAMPLES;
  o->cheb_tol = 1e-6;
  o->group = 0;
  o->resident_max_n = 0;
  o->stage_scale = nullptr;
  o->tile_log = 0;
  o->graph = 1;
  o->lanes = 0;
  o->threads = 0;
  o->lane_smem = 0;
  o->tma = 0;
  o->cluster = 0;
  o->stage1_basis = 1;
  o->final_projection = 1;
}

}  // namespace

struct mqw_plan {
  mqw_ctx* ctx = nullptr;
  mqw_options opt{};
  int count = 0;
  int precision = 0;   // storage: 0 FP32, 1 FP64
  int comp = 0;        // MQW_FP32_COMPENSATED: compensated partner sums
  int samples = MQW_SAMPLES;
  std::vector<int> n, m;                 // per instance (caller order)
  std::vector<int> order;                // instances sorted by n (stable)
  std::vector<float> total_t;            // caller order
  // Device inputs (sorted order).
  std::vector<long long> raw_off;        // doubles offset per sorted instance
  std::vector<long long> hp_off;         // hp offset per sorted instance
  std::vector<int> p_off;                // p_sample offset per sorted instance
  DevMem d_raw, d_hp, d_diag;
  // Jobs: one per (walk, stage) in walk-major order.
  std::vector<CoefJob> jobs;
  std::vector<ResidentWalk> walks;       // all walks (resident and grid)
  std::vector<int> walk_is_grid;
  DevMem d_jobs, d_degree, d_onenorm;
  DevMem d_p_sample, d_p_mean, d_p_off, d_p_cnt;
  size_t diag_scratch_bytes = 0;
  // Coefficient pool and launch tables (plan-owned: a captured graph reads them).
  DevMem d_coef, d_coef_off, d_stages, d_walks;
  // Grid-path shape chosen for each n of the plan.
  std::map<int, GridShape> grid_geo;
  // Shared bases per n: vectors of the stage-1 and the last-stage basis
  // (0 = not used for that n), and the unit coefficient list the basis passes
  // read ([0, ..., 0, 1]).
  std::map<int, int> basis_kb1, basis_kb2;
  int basis_buffers = 1;  // 2: the next instance's bases are built ahead
  // Stage-2 product basis per n: the largest stage-2 degree (absent: not
  // used for that n) and the walk capacity of ctx->s2psi.
  std::map<int, int> s2_k2;
  int s2_walks = 0;
  int s2_mode = -1;  // MQW_STAGE2_BASIS: -1 auto, 0 off, 1 whenever it fits
  // Per-buffer sizes (floats) of ctx->s2y / s2psi / s2c: one buffer set, two
  // with the build-ahead.
  size_t s2y_floats = 0, s2psi_floats = 0, s2c_floats = 0;
  size_t s2part_floats = 0;  // ctx->s2part per buffer set (0: no batched chains)
  std::map<int, int> s3_k3;  // n -> largest stage-3 degree: the product basis
                             // of the last two stages is used for this n
  int s3_mode = -1;          // MQW_LAST2_BASIS: -1 auto, 0 off, 1 whenever it fits
  DevMem d_unit;
  int unit_len = 0;
  // CUDA graph of the whole device pipeline, replayed by later executes.
  cudaGraphExec_t gexec = nullptr;
  unsigned long long graph_gen = 0;
  bool counting = true;  // stats are counted while issuing eagerly
  // Host copies of the degree read-back.
  std::vector<int> degree;
  std::vector<float> onenorm;
  std::vector<long long> coef_off;
  mqw_run_stats stats{};
  bool executed = false;
  int eager_runs = 0;  // executions issued eagerly (the second one captures)
  // Propagation-phase timing (recorded on the launching stream).
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool timed = false;
  double create_h2d = 0.0;  // bytes uploaded by plan_create
  ~mqw_plan() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }
};

namespace {

mqw_status check_ctx(mqw_ctx* ctx) {
  if (!ctx) return MQW_ERR_INVALID;
  // A non-sticky error left by the caller's own CUDA calls is not ours to
  // report from the launches below.
  (void)cudaGetLastError();
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess)
    return fail(ctx, MQW_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
  return MQW_OK;
}

// Reads and clears the device error word (after the work that may set it
// has completed): MQW_ERR_TIMEOUT when a kernel's bounded wait gave up.
mqw_status take_device_error(mqw_ctx* ctx) {
  unsigned v = 0;
  CK(cudaMemcpy(&v, ctx->dev_err.p, sizeof v, cudaMemcpyDeviceToHost));
  if (v == 0) return MQW_OK;
  CK(cudaMemset(ctx->dev_err.p, 0, sizeof v));
  return fail(ctx, MQW_ERR_TIMEOUT,
              "a kernel's bounded wait expired (error word %#x: bit 0 a grid-path pass's bulk "
              "copies, bit 1 the tensor-core GEMM's pipeline)", v);
}

int walk_slots(const PassGeomHost& geo) { return geo.nu > 0 ? 4 : 3; }

size_t walk_bytes(int precision, const PassGeomHost& geo, int n) {
  const size_t amp = precision == 0 ? 8 : 16;
  return (walk_slots(geo) * amp + sizeof(float)) * ((size_t)1 << n);
}

// Default group size: keep a launch's working set within ~60 MB (about one
// die's share of the 126 MB L2, which both dies' SMs read from), but give
// every launch at least ~2^20 amplitudes.
int default_group(int precision, const PassGeomHost& geo, int n) {
  size_t g = (60u << 20) / walk_bytes(precision, geo, n);
  if (((size_t)1 << n) * g < ((size_t)1 << 20)) g = ((size_t)1 << 20) >> n;
  if (g < 1) g = 1;
  if (g > (size_t)kMaxGroup) g = kMaxGroup;
  return (int)g;
}

// Times one configuration of the grid path: `reps` full passes (both
// tilings) over G zero-filled walks on each of `lanes` concurrent streams.
// Returns microseconds per walk-pass.
mqw_status time_grid_config(mqw_ctx* ctx, int precision, int n, int lmax,
                            int G, int lanes, int threads, int lane_smem, int tma,
                            double* us_per_walk, int reps = 12, int cluster = 1) {
  const PassGeomHost geo = pass_geom(precision, n, lmax, threads, lane_smem, tma, cluster);
  const size_t N = (size_t)1 << n;
  const size_t amp = precision == 0 ? 8 : 16;
  const int slots = walk_slots(geo);
  const int W = G * lanes;
  CK(ctx->ensure_lanes(lanes));
  CK(ctx->grow(ctx->state, (size_t)W * slots * N * amp + N * sizeof(float)));
  CK(ctx->grow(ctx->norm_part, (size_t)W * (N >> geo.L) * sizeof(double)));
  CK(ctx->tune_coef.ensure(64 * sizeof(float)));
  cudaStream_t st = ctx->stream;
  CK(cudaMemsetAsync(ctx->state.p, 0, (size_t)W * slots * N * amp + N * sizeof(float), st));
  CK(cudaMemsetAsync(ctx->tune_coef.p, 0, 64 * sizeof(float), st));
  char* base = ctx->state.as<char>();
  const float* hp = reinterpret_cast<const float*>(base + (size_t)W * slots * N * amp);
  auto issue = [&](int r, int lane) -> cudaError_t {
    PassParams pp{};
    pp.n = n;
    pp.L = geo.L;
    pp.C = geo.C;
    pp.threads = geo.threads;
    pp.lane_smem = geo.lane_smem;
    pp.tma = geo.tma;
    pp.err = ctx->dev_err.as<unsigned>();
    pp.a = geo.a;
    pp.tiling = (r & 1) ? 2 : 1;
    pp.count = G;
    for (int g = 0; g < G; g++) {
      PassWalk& Wk = pp.walk[g];
      const int wi = lane * G + g;
      char* w = base + (size_t)wi * slots * N * amp;
      Wk.active = 1;
      Wk.bin = w + N * amp;
      Wk.bout = w + (slots == 4 ? 3 : 1) * N * amp;
      Wk.part = w + 2 * N * amp;
      Wk.psi = w;
      Wk.hp = hp;
      Wk.coef = ctx->tune_coef.as<float>();
      Wk.kappa = nullptr;
      Wk.norm_part = ctx->norm_part.as<double>() + (size_t)wi * (N >> geo.L);
      Wk.gamma = 1.0f;
      Wk.scale = 64.0f;
      Wk.r = r;
      Wk.K = 40;
      Wk.psi_uniform = 0;
      Wk.psi0 = 0.0f;
    }
    return launch_pass(precision, pp, lane == 0 ? st : ctx->lane_stream[lane]);
  };
  CK(ctx->fork(st, lanes));
  for (int r = 4; r >= 1; r--)
    for (int l = 0; l < lanes; l++) CK(issue(r, l));
  CK(ctx->join(st, lanes));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, st));
  CK(ctx->fork(st, lanes));
  for (int r = reps; r >= 1; r--)
    for (int l = 0; l < lanes; l++) CK(issue(r, l));
  CK(ctx->join(st, lanes));
  CK(cudaEventRecord(e1, st));
  CK(cudaEventSynchronize(e1));
  float ms = 0.0f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  mqw_status es = take_device_error(ctx);
  if (es != MQW_OK) return es;
  *us_per_walk = 1000.0 * ms / (reps * W);
  return MQW_OK;
}

// Autotuner: picks the grid-path tile cap, group size and lane count for
// (precision, n) by timing the candidates once per context; the result is
// cached. Fixed choices in `want` (non-zero fields) are kept.
mqw_status tune_grid(mqw_ctx* ctx, int precision, int n, GridShape want, GridShape* out) {
  const auto key = std::make_pair(precision, n);
  auto it = ctx->tuned.find(key);
  const bool fixed_none = !want.lmax && !want.group && !want.lanes && !want.threads &&
                          !want.lane_smem && !want.tma && !want.cl;
  if (it != ctx->tuned.end() && fixed_none) {
    *out = it->second;
    return MQW_OK;
  }
  const int def_l = precision == 0 ? 12 : 11;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = (size_t)8 << 30;
  const size_t budget = std::min(free_b / 4, (size_t)16 << 30);
  const bool log = getenv("MQW_TUNE_LOG") != nullptr;
  auto fits = [&](const PassGeomHost& geo, int g, int lanes) {
    return g <= kMaxGroup && (size_t)g * lanes * walk_bytes(precision, geo, n) <= budget;
  };
  auto time = [&](const GridShape& c, double* us) -> mqw_status {
    const PassGeomHost geo = pass_geom(precision, n, c.lmax, c.threads, c.lane_smem > 0, std::max(0, c.tma), c.cl < 0 ? 0 : 1);
    mqw_status s = time_grid_config(ctx, precision, n, c.lmax, c.group, c.lanes, c.threads,
                                    c.lane_smem > 0, std::max(0, c.tma), us, 12, c.cl < 0 ? 0 : 1);
    if (s == MQW_OK && log)
      fprintf(stderr,
              "mqw tune: precision %d n %d tile %d cluster %d global %d threads %d lane_smem %d "
              "tma %d group %d lanes %d: %.3f us/walk-pass\n",
              precision, n, geo.L, geo.C, geo.nu, c.threads ? c.threads : 512, geo.lane_smem,
              geo.tma, c.group, c.lanes, *us);
    return s;
  };
  // Stage 1: the pass shape — tile cap (the default widest tile, one
  // narrower, and in FP32 the 2^13 tile when the default leaves axes to
  // global memory), threads, lane axes, staging — each timed with one walk
  // per launch on two lanes (one if two do not fit).
  std::vector<int> caps = {def_l, def_l - 1};
  if (precision == 0 && n > 2 * def_l - 4) caps.insert(caps.begin() + 1, def_l + 1);
  double best = 1e300;
  GridShape b;
  b.lmax = want.lmax ? want.lmax : def_l;
  b.group = want.group ? want.group : 1;
  b.lanes = want.lanes ? want.lanes : 1;
  b.threads = want.threads == 256 ? 256 : 0;
  b.lane_smem = want.lane_smem;
  b.tma = want.tma;
  // At the widest tile, when axes are left over, both the cluster-spanning
  // tile and the single-CTA tile with global-memory axes are candidates.
  for (int l : caps)
    for (int cl : {1, -1}) {
    if (want.lmax && l != want.lmax) continue;
    if (want.cl && want.cl != cl) continue;
    if (cl < 0 && (l != def_l || n <= 2 * def_l - 4)) continue;
    for (int threads : {0, 256})
      for (int ls : {0, 1})
        for (int tma : {0, 1, 2}) {
          if (want.threads && (want.threads == 256) != (threads == 256)) continue;
          if (want.lane_smem && (want.lane_smem > 0) != (ls == 1)) continue;
          if (want.tma && std::max(0, want.tma) != tma) continue;
          const PassGeomHost geo = pass_geom(precision, n, l, threads, ls, tma, cl < 0 ? 0 : 1);
          if (geo.threads != threads || geo.lane_smem != ls || geo.tma != tma) continue;
          GridShape c;
          c.cl = cl;
          c.lmax = l;
          c.threads = threads;
          c.lane_smem = ls ? 1 : -1;
          c.tma = tma ? tma : -1;
          c.group = want.group ? want.group : 1;
          c.lanes = want.lanes ? want.lanes : (fits(geo, c.group, 2) ? 2 : 1);
          if (!fits(geo, c.group, c.lanes)) continue;
          double us = 0.0;
          mqw_status s = time(c, &us);
          if (s != MQW_OK) return s;
          // Prefer the earlier candidate (larger tile, simpler variant)
          // unless a later one is clearly faster.
          if (us < best * 0.98) {
            best = us;
            c.us = us;
            b = c;
          }
        }
    }
  // Stage 2: walks per launch and lanes for that shape.
  if (best < 1e300 && (!want.group || !want.lanes)) {
    const PassGeomHost geo = pass_geom(precision, n, b.lmax, b.threads, b.lane_smem > 0, std::max(0, b.tma), b.cl < 0 ? 0 : 1);
    const int g0 = default_group(precision, geo, n);
    std::vector<int> groups = {1, 2, 4};
    if (g0 != 1 && g0 != 2 && g0 != 4) groups.push_back(g0);
    const GridShape base = b;
    std::vector<GridShape> cands = {base};
    for (int g : groups) {
      if (want.group && g != want.group) continue;
      for (int lanes = 1; lanes <= kMaxLanes; lanes++) {
        if (want.lanes && lanes != want.lanes) continue;
        if ((g == base.group && lanes == base.lanes) || !fits(geo, g, lanes)) continue;
        GridShape c = base;
        c.group = g;
        c.lanes = lanes;
        mqw_status s = time(c, &c.us);
        if (s != MQW_OK) return s;
        cands.push_back(c);
      }
    }
    // Within 2% of the fastest, take the most walks per launch: the same
    // device time in fewer launches, which is what an eager (not replayed)
    // execution pays for on the host.
    double fastest = 1e300;
    for (const GridShape& c : cands) fastest = std::min(fastest, c.us);
    b = base;
    bool chosen = false;
    for (const GridShape& c : cands) {
      if (c.us > fastest * 1.02) continue;
      if (!chosen || c.group > b.group || (c.group == b.group && c.us < b.us)) {
        b = c;
        chosen = true;
      }
    }
  }
  if (fixed_none) ctx->tuned[key] = b;
  *out = b;
  return MQW_OK;
}

// Runs a group of grid-path walks (all the same n) through all their stages.
// Each walk owns the state slots psi, b and the partial P; when some axes are
// read from global memory (nu > 0) b is double-buffered (b_r in slot x for
// even r and y for odd r), otherwise it is updated in place, which keeps a
// walk at 3 vectors so that two walks of n = 20 stay resident in L2. Pass r
// uses tiling 1 for even r and tiling 2 for odd r.
// `widx` (at most `gmax` walks) is a basis group: its stage-1 recombination
// and its last-stage projection are one launch each, so that every basis
// vector is read once per group; the recurrence stages run in pass groups of
// `G` consecutive walks, each pass group through all of its stages before
// the next starts (its states stay L2-resident meanwhile). Without bases,
// `widx` is one pass group.
// `lane` selects the lane's own slice of the shared scratch (state, norm
// partials, kappa), sized for `gmax` walks.
// With `basis` set (the instance's stage-1 basis of Kb vectors), the first
// stage is recombined from it instead of run as a recurrence per walk; with
// `last` set (the last-stage basis of Kl vectors from e_{E_loc}), the last
// stage is a projection onto it that yields P directly. `proj` is the lane's
// projection scratch.
mqw_status run_grid_group(mqw_plan& P, const std::vector<int>& widx,
                          const PassGeomHost& geo, int lane, int G, int gmax,
                          const float* basis, int Kb, const float* last, int Kl,
                          double* proj, const float* ext_re, const float* ext_im,
                          cudaStream_t stream) {
  mqw_ctx* ctx = P.ctx;
  const int n = P.walks[widx[0]].n;
  const size_t N = (size_t)1 << n;
  const int tiles = (int)(N >> geo.L);
  // The recombination kernels use blocks of 2^rL amplitudes (enough blocks
  // for whole waves at one block per SM); a walk's norm partials are laid
  // out with the larger count of the two.
  const int rL = std::min(geo.L, kRecombineLog);
  const int rtiles = (int)(N >> rL);
  const int W = (int)widx.size();
  const size_t amp = P.precision == 0 ? 8 : 16;
  const int slots = walk_slots(geo);
  char* base = P.ctx->state.as<char>() + (size_t)lane * gmax * slots * N * amp;
  auto buf = [&](int g, int k) -> void* {
    return base + ((size_t)g * slots + k) * N * amp;
  };
  int pi[kMaxGroup], xs[kMaxGroup];
  const int ps = 2;
  const int ys = geo.nu > 0 ? 3 : -1;  // -1: b in place
  for (int g = 0; g < W; g++) {
    pi[g] = 0;
    xs[g] = 1;
  }
  double* norm_part = P.ctx->norm_part.as<double>() + (size_t)lane * gmax * rtiles;
  double* kappa = P.ctx->kappa.as<double>() + (size_t)lane * kMaxGroup;
  double* p_sample = P.d_p_sample.as<double>();
  const float* coef = P.d_coef.as<float>();
  const float* hp = P.d_hp.as<float>();
  const DiagOut* diag = P.d_diag.as<DiagOut>();
  auto degree = [&](int g, int st) {
    const ResidentWalk& w = P.walks[widx[g]];
    return st < w.stages ? P.degree[w.stage_desc_off + st] : 0;
  };
  // Stage-output bookkeeping of walks [g0, g1) after stage st: per-walk
  // norms (and P where recorded), then the output becomes the next psi.
  auto finalize = [&](int g0, int g1, int st, int parts) -> mqw_status {
    FinalParams fp{};
    int fc = 0;
    for (int g = g0; g < g1; g++) {
      const ResidentWalk& w = P.walks[widx[g]];
      if (st >= w.stages) continue;
      FinalTraj& F = fp.traj[fc++];
      F.norm_part = norm_part + (size_t)g * rtiles;
      F.tiles = parts;
      F.kappa = kappa + g;
      F.out = buf(g, xs[g]);
      F.diag = diag + w.inst;
      F.p_out = (w.record_each || st == w.stages - 1)
                    ? p_sample + w.p_off + (w.record_each ? st : 0)
                    : nullptr;
    }
    fp.count = fc;
    CK(launch_finalize(P.precision, fp, stream));
    if (P.counting) P.stats.launches++;
    for (int g = g0; g < g1; g++) {
      if (st >= P.walks[widx[g]].stages) continue;
      std::swap(pi[g], xs[g]);  // the output (slot x) becomes psi
    }
    return MQW_OK;
  };
  int max_stages = 0;
  for (int g = 0; g < W; g++) max_stages = std::max(max_stages, P.walks[widx[g]].stages);
  // The bases are used only by groups of one instance with the same m
  // (>= 2), which issue_rest guarantees.
  const bool combine = basis != nullptr;
  const bool ext = ext_re != nullptr;  // stage-2 outputs given (planar)
  if (ext) {
    UnpackParams up{};
    up.n = n;
    up.L = rL;
    up.count = W;
    for (int g = 0; g < W; g++)
      up.walk[g] = UnpackWalk{ext_re + (size_t)g * N, ext_im + (size_t)g * N, buf(g, xs[g]),
                              norm_part + (size_t)g * rtiles};
    CK(launch_unpack(up, stream));
    if (P.counting) {
      P.stats.launches++;
      P.stats.aux_bytes += (double)W * N * 16.0;
    }
    mqw_status s = finalize(0, W, 1, rtiles);
    if (s != MQW_OK) return s;
  }
  const bool project = last != nullptr && max_stages > 1;
  if (combine) {
    CombineParams cp{};
    cp.basis = basis;
    cp.n = n;
    cp.L = rL;
    cp.Kb = Kb;
    cp.count = W;
    for (int g = 0; g < W; g++) {
      const int job = P.walks[widx[g]].stage_desc_off;
      CombineWalk& C = cp.walk[g];
      C.coef = coef + P.coef_off[job];
      C.K = degree(g, 0);
      C.out = buf(g, xs[g]);
      C.norm_part = norm_part + (size_t)g * rtiles;
    }
    CK(launch_combine(P.precision, cp, stream));
    if (P.counting) {
      P.stats.launches++;
      // the basis once per group, one complex state written per walk
      P.stats.aux_bytes += (double)Kb * N * 4.0 + (double)W * N * 8.0;
    }
    mqw_status s = finalize(0, W, 0, rtiles);
    if (s != MQW_OK) return s;
  }
  // Small n: every term of a walk-stage in one chain launch (a cluster of
  // CTAs per walk) instead of one launch per term.
  const int chain_L = P.comp ? 0 : chain_tile_log(P.precision, n);
  // Recurrence stages [combine, end) of each pass group.
  for (int g0 = 0; g0 < W; g0 += G) {
    const int g1 = std::min(W, g0 + G);
    int end = 0;
    for (int g = g0; g < g1; g++) end = std::max(end, P.walks[widx[g]].stages);
    if (project) end = max_stages - 1;
    for (int st = ext ? 2 : (combine ? 1 : 0); st < end; st++) {
      int K[kMaxGroup], Kmax = 0;
      for (int g = g0; g < g1; g++) {
        K[g - g0] = degree(g, st);
        Kmax = std::max(Kmax, K[g - g0]);
      }
      if (chain_L && Kmax > 0) {
        PassParams pp{};
        pp.n = n;
        pp.L = chain_L;
        pp.a = geo.a;
        pp.tiling = 1;
        pp.err = ctx->dev_err.as<unsigned>();
        pp.count = g1 - g0;
        for (int g = g0; g < g1; g++) {
          PassWalk& Wk = pp.walk[g - g0];
          const ResidentWalk& w = P.walks[widx[g]];
          Wk.active = K[g - g0] > 0;
          if (!Wk.active) continue;
          const int job = w.stage_desc_off + st;
          Wk.bin = Wk.bout = buf(g, xs[g]);  // no axis from global memory: in place
          Wk.part = buf(g, ps);
          Wk.psi = buf(g, pi[g]);
          Wk.hp = hp + w.hp_off;
          Wk.coef = coef + P.coef_off[job];
          Wk.kappa = st == 0 ? nullptr : kappa + g;
          Wk.norm_part = norm_part + (size_t)g * rtiles;
          Wk.gamma = P.jobs[job].gamma;
          Wk.scale = P.onenorm[job];
          Wk.K = K[g - g0];
          Wk.psi_uniform = st == 0;
          Wk.psi0 = (float)(1.0 / std::sqrt((double)N));
          if (P.counting) P.stats.pass_amps += (double)N * K[g - g0];
        }
        CK(launch_pass_chain(P.precision, pp, stream));
        if (P.counting) {
          P.stats.launches++;
          P.stats.term_launches++;
        }
        mqw_status s = finalize(g0, g1, st, (int)(N >> chain_L));
        if (s != MQW_OK) return s;
        continue;
      }
      for (int r = Kmax - 1; r >= 0; r--) {
        PassParams pp{};
        pp.n = n;
        pp.L = geo.L;
        pp.C = geo.C;
        pp.threads = geo.threads;
        pp.lane_smem = geo.lane_smem;
        pp.tma = geo.tma;
        pp.err = ctx->dev_err.as<unsigned>();
        pp.comp = P.comp;
        pp.a = geo.a;
        pp.tiling = (r & 1) ? 2 : 1;
        pp.count = g1 - g0;
        for (int g = g0; g < g1; g++) {
          PassWalk& Wk = pp.walk[g - g0];
          const ResidentWalk& w = P.walks[widx[g]];
          Wk.active = r < K[g - g0];
          if (!Wk.active) continue;
          const int job = w.stage_desc_off + st;
          if (ys < 0) {
            Wk.bin = Wk.bout = buf(g, xs[g]);
          } else {
            Wk.bin = buf(g, (r & 1) ? xs[g] : ys);
            Wk.bout = buf(g, (r & 1) ? ys : xs[g]);
          }
          Wk.part = buf(g, ps);
          Wk.psi = buf(g, pi[g]);
          Wk.hp = hp + w.hp_off;
          Wk.coef = coef + P.coef_off[job];
          Wk.kappa = st == 0 ? nullptr : kappa + g;
          Wk.norm_part = norm_part + (size_t)g * rtiles;
          Wk.gamma = P.jobs[job].gamma;
          Wk.scale = P.onenorm[job];
          Wk.r = r;
          Wk.K = K[g - g0];
          Wk.psi_uniform = st == 0;  // every walk starts from the uniform state
          Wk.psi0 = (float)(1.0 / std::sqrt((double)N));
          if (P.counting) P.stats.pass_amps += (double)N;
        }
        CK(launch_pass(P.precision, pp, stream));
        if (P.counting) {
          P.stats.launches++;
          P.stats.term_launches++;
        }
      }
      mqw_status s = finalize(g0, g1, st, tiles);
      if (s != MQW_OK) return s;
    }
  }
  if (project) {
    const int st = max_stages - 1;
    ProjectParams pr{};
    pr.basis = last;
    pr.n = n;
    pr.L = rL;
    pr.Kb = Kl;
    pr.count = W;
    pr.part = proj;
    for (int g = 0; g < W; g++) {
      const ResidentWalk& w = P.walks[widx[g]];
      ProjectWalk& Q = pr.walk[g];
      Q.coef = coef + P.coef_off[w.stage_desc_off + st];
      Q.K = degree(g, st);
      Q.psi = buf(g, pi[g]);
      Q.kappa = kappa + g;
      Q.p_out = p_sample + w.p_off;
    }
    CK(launch_project(pr, stream));
    if (P.counting) {
      P.stats.launches += 2;
      // the basis once per group, each walk's state once
      P.stats.aux_bytes += (double)Kl * N * 4.0 + (double)W * N * 8.0;
    }
  }
  return MQW_OK;
}

// Layout of ctx->basis for one n (FP32): four complex slots — the basis
// passes' partial P, the recurrence vector b (two when axes are read from
// global memory), the start vector e_{E_loc} — then the real stage-1 basis
// (kb1 vectors) and the real last-stage basis (kb2 vectors).
struct BasisLayout {
  char* base;
  size_t N;
  int kb1, kb2;
  void* slot(int k) const { return base + (size_t)k * N * 8; }
  float* real1() const { return reinterpret_cast<float*>(base + 4 * N * 8); }
  float* real2() const { return real1() + (size_t)kb1 * N; }
  static size_t bytes(int n, int kb1, int kb2) {
    const size_t N = (size_t)1 << n;
    return 4 * N * 8 + (size_t)(kb1 + kb2) * N * 4;
  }
};

// State slots of one unit-coefficient pass chain: the partial P, the
// recurrence vector b (b[1] only when axes are read from global memory) and
// the start vector (not read when `uniform`: the uniform state), complex;
// `start_real` is the same start vector as a real vector, for the real
// chain kernel (nullptr when uniform).
struct ChainSlots {
  void* part;
  void* b[2];
  const void* start;
  bool uniform;
  const float* start_real;
};

// Whether a plan's chains run on the real chain kernel (real_pass_kernel):
// FP32, single-CTA tiles; MQW_REAL_CHAINS=0 keeps them on the complex pass
// kernel (the same results: the real kernel reproduces the real parts bit
// for bit).
bool use_real_chains(const mqw_plan& P, const PassGeomHost& geo) {
  if (P.precision != 0 || geo.C != 0) return false;
  const char* e = getenv("MQW_REAL_CHAINS");
  return !(e && atoi(e) == 0);
}

// One unit-coefficient pass chain: w_j = U_j(H~) v, j < K, for the operator of
// stage `stage` of the instance of walk w0 and the start vector v of `S`,
// Re(w_j) stored at out_of(j) (real FP32, 2^n floats). K single-walk passes
// with c = [0, .., 0, 1] at an even top index R >= K, so that b_R = v and
// every later pass is b_r = 2 H~ b_{r+1} - b_{r+2}; each pass also stores
// Re(b_r). The passes stop at r = R - K + 1 >= 1 (the r = 0 form is never
// used).
// With `tbasis` the chain's vectors are first-kind, w_j = T_j(H~) v (the
// real chain kernel only).
template <typename OutOf>
mqw_status issue_chain(mqw_plan& P, const ResidentWalk& w0, int stage, int K,
                       const ChainSlots& S, const PassGeomHost& geo, OutOf out_of,
                       cudaStream_t stream, bool tbasis = false) {
  mqw_ctx* ctx = P.ctx;
  const size_t N = (size_t)1 << w0.n;
  const int R = K + (K & 1);
  const int job = w0.stage_desc_off + stage;
  if (tbasis && !use_real_chains(P, geo))
    return fail(ctx, MQW_ERR_INVALID, "first-kind chains need the real chain kernel");
  if (use_real_chains(P, geo)) {
    // Every vector of the chain is real: the real chain kernel, writing
    // each b_r straight into its basis slot and reading b_{r+1} back from
    // the previous one (no complex b slot, no separate real copy).
    // Small n: the whole chain in one launch when the outputs are laid out
    // as two interleaved strided sequences (even and odd j), which both the
    // stage-1/last-stage bases and the stage-2 product basis are.
    const int cL = chain_tile_log(0, w0.n);
    if (cL && K > 0) {
      float* base0 = out_of(0);
      float* base1 = K > 1 ? out_of(1) : nullptr;
      const long long stride = K > 2 ? (long long)(out_of(2) - base0) : (long long)(2 * N);
      bool affine = stride >= (long long)N;
      for (int j = 0; j < K && affine; j++)
        affine = out_of(j) == (j & 1 ? base1 : base0) + (size_t)(j >> 1) * (size_t)stride;
      if (affine) {
        RealChainBatch rb{};
        RealChainParams& rp = rb.p;
        rp.n = w0.n;
        rp.L = cL;
        rp.a = geo.a;
        rp.start_uniform = S.uniform ? 1 : 0;
        rp.psi0 = (float)(1.0 / std::sqrt((double)N));
        rp.hp = P.d_hp.as<float>() + w0.hp_off;
        rp.gamma = P.jobs[job].gamma;
        rp.scale = P.onenorm[job];
        rp.K = K;
        rp.R = R;
        rp.out_stride = stride;
        rp.tbasis = tbasis ? 1 : 0;
        rb.chains = 1;
        rb.chain[0] = RealChainDesc{S.start_real, static_cast<float*>(S.part), {base0, base1}};
        CK(launch_real_chain(rb, stream));
        if (P.counting) {
          P.stats.launches++;
          P.stats.term_launches++;
          P.stats.aux_bytes += (double)N * 20.0 * K;
        }
        return MQW_OK;
      }
    }
    for (int j = 0; j < K; j++) {
      RealChainParams rp{};
      rp.n = w0.n;
      rp.L = geo.L;
      rp.a = geo.a;
      rp.tiling = ((R - j) & 1) ? 2 : 1;
      rp.first = j == 0;
      rp.bin = j > 0 ? out_of(j - 1) : nullptr;
      rp.bout = out_of(j);
      rp.part = static_cast<float*>(S.part);
      rp.start = S.start_real;
      rp.start_uniform = S.uniform ? 1 : 0;
      rp.psi0 = (float)(1.0 / std::sqrt((double)N));
      rp.hp = P.d_hp.as<float>() + w0.hp_off;
      rp.gamma = P.jobs[job].gamma;
      rp.scale = P.onenorm[job];
      rp.half_start = tbasis && j == 0;
      rp.half_finish = tbasis && j == 1;
      CK(launch_real_pass(rp, stream));
      if (P.counting) {
        P.stats.launches++;
        P.stats.term_launches++;
        // read b_{r+1}, P, D and write b_r, P: 20 B per amplitude (the
        // first pass reads the start vector instead of b_{r+1} and P)
        P.stats.aux_bytes += (double)N * 20.0;
      }
    }
    return MQW_OK;
  }
  const float* unit = P.d_unit.as<float>() + (P.unit_len - 1 - R);
  for (int j = 0; j < K; j++) {
    PassParams pp{};
    pp.n = w0.n;
    pp.L = geo.L;
    pp.C = geo.C;
    pp.threads = geo.threads;
    pp.lane_smem = geo.lane_smem;
    pp.tma = geo.tma;
    pp.err = ctx->dev_err.as<unsigned>();
    pp.a = geo.a;
    pp.tiling = ((R - j) & 1) ? 2 : 1;
    pp.count = 1;
    PassWalk& W = pp.walk[0];
    W.active = 1;
    if (geo.nu == 0) {
      W.bin = W.bout = S.b[0];  // in place
    } else {
      W.bin = S.b[(j + 1) & 1];  // not read by the first pass
      W.bout = S.b[j & 1];
    }
    W.part = S.part;
    W.psi = S.start;
    W.hp = P.d_hp.as<float>() + w0.hp_off;
    W.coef = unit;
    W.kappa = nullptr;
    W.norm_part = ctx->norm_part.as<double>();  // not written (r >= 1)
    W.gamma = P.jobs[job].gamma;
    W.scale = P.onenorm[job];
    W.r = R - j;
    W.K = R + 1;
    // Only the first pass (b_R = v) uses the start vector: every later
    // coefficient is 0, so those passes take psi as a uniform zero state and
    // do not read it.
    W.psi_uniform = (S.uniform || j > 0) ? 1 : 0;
    W.psi0 = S.uniform ? (float)(1.0 / std::sqrt((double)N)) : 0.0f;
    W.real_out = out_of(j);
    CK(launch_pass(P.precision, pp, stream));
    if (P.counting) {
      P.stats.launches++;
      P.stats.term_launches++;
      P.stats.pass_amps += (double)N;
      P.stats.aux_bytes += (double)N * 4.0;  // the real part stored
    }
  }
  return MQW_OK;
}

// Builds the real basis w_j = U_j(H~) v, j < Kb, of stage `stage` of the
// instance of walk w0 into `real` (Kb vectors of 2^n floats): v is the
// uniform state for the first stage and e_{E_loc} for the last.
mqw_status issue_basis(mqw_plan& P, const ResidentWalk& w0, int stage, int Kb,
                       const BasisLayout& B, const PassGeomHost& geo, float* real,
                       cudaStream_t stream, bool tbasis = false) {
  const size_t N = (size_t)1 << w0.n;
  const bool from_eloc = stage > 0;
  const bool real_chain = use_real_chains(P, geo);
  if (from_eloc) {
    mqw_ctx* ctx = P.ctx;
    if (real_chain)
      CK(launch_unit_eloc_real(static_cast<float*>(B.slot(3)), w0.n,
                               P.d_diag.as<DiagOut>() + w0.inst, stream));
    else
      CK(launch_unit_eloc(B.slot(3), w0.n, P.d_diag.as<DiagOut>() + w0.inst, stream));
    if (P.counting) P.stats.launches++;
  }
  const ChainSlots S{B.slot(0), {B.slot(1), B.slot(2)}, B.slot(3), !from_eloc,
                     from_eloc ? static_cast<const float*>(B.slot(3)) : nullptr};
  return issue_chain(P, w0, stage, Kb, S, geo, [&](int j) { return real + (size_t)j * N; },
                     stream, tbasis);
}

// The stage-2 product basis of one instance (FP32): Y_jk = U_k(H~_2) w_j for
// the Kb stage-1 basis vectors w_j (in `basis`) and k < K2, one chain of K2
// passes per w_j, dealt round-robin to `lanes` lanes (each on its own walk
// slots of the shared state), then the coefficient matrices and the GEMM
// that leave every walk's stage-2 output, planar, in ctx->s2psi. `extra`
// (if set) is issued beside the chains on one more lane (the last lane when
// all four are in use): the instance's last-stage basis build.
// `buf` selects one of the plan's stage-2 buffer sets (two with the
// build-ahead, which calls this on the basis stream with `builder` set: the
// chains then run on the basis stream's own lanes and on the context's chain
// slots, one set per lane, instead of the walk lanes and their slots).
// With `last2` set the same machinery builds the product basis of the last
// two stages instead (m = 4): Y'_jk = U_k(H~_3) w'_j from the last-stage
// basis w'_j = U_j(H~_4) e_{E_loc} (`basis`, Kb vectors) with chains of
// stage 3 (K2 passes), into ctx->s3y, and the GEMM leaves every walk's
// V = sum_jk d4_j d3_k Y'_jk, planar, in ctx->s3v (see issue_last2).
mqw_status issue_stage2(mqw_plan& P, const std::vector<int>& ws, size_t b0, size_t b1,
                        const float* basis, int Kb, int K2, const PassGeomHost& geo,
                        int lanes,
                        const std::function<mqw_status(cudaStream_t)>& extra,
                        cudaStream_t stream, int buf = 0, bool builder = false,
                        bool last2 = false) {
  mqw_ctx* ctx = P.ctx;
  const ResidentWalk& w0 = P.walks[ws[b0]];
  const int n = w0.n;
  const size_t N = (size_t)1 << n;
  const int nw = (int)(b1 - b0);
  const S2Layout lay{Kb, K2};
  // the chains' stage and the coefficient stages of the basis index j and
  // the chain index k
  const int chain_stage = last2 ? w0.stages - 2 : 1;
  const int sj = last2 ? w0.stages - 1 : 0;
  float* Y = last2 ? ctx->s3y.as<float>()
                   : ctx->s2y.as<float>() + (size_t)buf * P.s2y_floats;
  const int slots = walk_slots(geo);
  // Small n: all Kb chains in chain launches of up to kMaxChainBatch chains
  // each (a cluster per chain, each with its own partial P) on the launching
  // stream, instead of one chain after another on each lane.
  const int cL = use_real_chains(P, geo) && P.s2part_floats >= (size_t)Kb * N
                     ? chain_tile_log(0, n) : 0;
  auto chain_out = [&](int j, int k) {
    const int h = (j + k) & 1;
    return Y + ((size_t)(h ? lay.rows(0) : 0) + lay.index(j, k)) * N;
  };
  bool batched = cL > 0 && K2 > 0;
  for (int j = 0; j < Kb && batched; j++)
    for (int k = 2; k < K2 && batched; k++)
      batched = chain_out(j, k) == chain_out(j, k - 2) + N;
  // Larger n: the chains in per-term launches of up to B chains each (the
  // batches dealt round-robin to the lanes, each chain with its own partial
  // P), instead of one single-chain launch per term. B = 8 up to n = 18
  // (measured at n = 18, m = 4: 84.2 -> 88.5 instances/s); from n = 20 the
  // batched chains' vectors no longer fit in L2 beside each other and one
  // chain per launch is faster (measured at n = 20, m = 4: 26.5 instances/s
  // with one chain per launch on 3 lanes, 26.1-26.3 with 2 chains per launch
  // on 2-3 lanes, 23.6 with 8 on one lane), B = 1. MQW_CHAIN_BATCH sets B.
  int B = 1;
  if (!batched && use_real_chains(P, geo) && P.s2part_floats >= (size_t)Kb * N && K2 > 0) {
    const char* e = getenv("MQW_CHAIN_BATCH");
    B = std::min(kMaxChainBatch, std::max(1, e ? atoi(e) : (n <= 18 ? 8 : 1)));
    for (int j = 0; j < Kb && B > 1; j++)
      for (int k = 2; k < K2 && B > 1; k++)
        if (chain_out(j, k) != chain_out(j, k - 2) + N) B = 1;
  }
  // One chain per launch (the walks' lanes' state slots, packed): from
  // n = 19 on kChainLanes lanes (MQW_CHAIN_LANES sets it), as far as the
  // state buffer holds their slots.
  const size_t chain_slot_bytes = (size_t)slots * N * 8;
  if (!builder && !batched && B == 1 && Kb > 0 && K2 > 0) {
    const char* e = getenv("MQW_CHAIN_LANES");
    int cl = e ? atoi(e) : (use_real_chains(P, geo) && n >= 19 ? kChainLanes : lanes);
    cl = std::min(cl, (int)std::min<size_t>(kMaxStreams - 1, ctx->state.bytes / chain_slot_bytes));
    lanes = std::max(1, std::min(std::max(cl, 1), Kb));
  }
  const int all = extra ? std::min(lanes + 1, builder ? kMaxLanes : kMaxStreams) : lanes;
  cudaStream_t* lane_st = builder ? ctx->bld_stream : ctx->lane_stream;
  if (builder) {  // fork the basis stream's lanes
    CK(cudaEventRecord(ctx->bld_fork_ev, stream));
    for (int k = 1; k < all; k++) CK(cudaStreamWaitEvent(ctx->bld_stream[k], ctx->bld_fork_ev, 0));
  } else {
    CK(ctx->fork(stream, all));
  }
  if (extra) {
    const int xl = all - 1;
    mqw_status s = extra(xl == 0 ? stream : lane_st[xl]);
    if (s != MQW_OK) return s;
  }
  if (batched) {
    const int job = w0.stage_desc_off + chain_stage;
    float* part = ctx->s2part.as<float>() + (size_t)buf * P.s2part_floats;
    for (int c0 = 0; c0 < Kb; c0 += kMaxChainBatch) {
      RealChainBatch rb{};
      RealChainParams& rp = rb.p;
      rp.n = n;
      rp.L = cL;
      rp.a = geo.a;
      rp.psi0 = (float)(1.0 / std::sqrt((double)N));
      rp.hp = P.d_hp.as<float>() + w0.hp_off;
      rp.gamma = P.jobs[job].gamma;
      rp.scale = P.onenorm[job];
      rp.K = K2;
      rp.R = K2 + (K2 & 1);
      rp.out_stride = (long long)N;
      rp.tbasis = last2 ? 1 : 0;
      rb.chains = std::min(kMaxChainBatch, Kb - c0);
      for (int c = 0; c < rb.chains; c++) {
        const int j = c0 + c;
        rb.chain[c] = RealChainDesc{basis + (size_t)j * N, part + (size_t)j * N,
                                    {chain_out(j, 0), K2 > 1 ? chain_out(j, 1) : nullptr}};
      }
      CK(launch_real_chain(rb, stream));
      if (P.counting) {
        P.stats.launches++;
        P.stats.term_launches++;
        P.stats.aux_bytes += (double)N * 20.0 * K2 * rb.chains;
      }
    }
  }
  if (B > 1) {
    const int job = w0.stage_desc_off + chain_stage;
    float* part = ctx->s2part.as<float>() + (size_t)buf * P.s2part_floats;
    const int nbatch = (Kb + B - 1) / B;
    for (int i = 0; i < nbatch; i++) {
      const int lane = i % lanes;
      cudaStream_t st = lane == 0 ? stream : lane_st[lane];
      RealChainBatch rb{};
      RealChainParams& rp = rb.p;
      rp.n = n;
      rp.L = geo.L;
      rp.a = geo.a;
      rp.psi0 = (float)(1.0 / std::sqrt((double)N));
      rp.hp = P.d_hp.as<float>() + w0.hp_off;
      rp.gamma = P.jobs[job].gamma;
      rp.scale = P.onenorm[job];
      rp.K = K2;
      rp.R = K2 + (K2 & 1);
      rp.out_stride = (long long)N;
      rp.tbasis = last2 ? 1 : 0;
      rb.chains = std::min(B, Kb - i * B);
      for (int c = 0; c < rb.chains; c++) {
        const int j = i * B + c;
        rb.chain[c] = RealChainDesc{basis + (size_t)j * N, part + (size_t)j * N,
                                    {chain_out(j, 0), K2 > 1 ? chain_out(j, 1) : nullptr}};
      }
      for (int k = 0; k < K2; k++) {
        CK(launch_real_batch(rb, k, st));
        if (P.counting) {
          P.stats.launches++;
          P.stats.term_launches++;
          P.stats.aux_bytes += (double)N * 20.0 * rb.chains;
        }
      }
    }
  }
  for (int j = 0; j < Kb && !batched && B == 1; j++) {
    const int lane = j % lanes;
    cudaStream_t st = lane == 0 ? stream : lane_st[lane];
    char* base = builder ? ctx->s2chain.as<char>() + (size_t)lane * 4 * N * 8
                         : ctx->state.as<char>() + (size_t)lane * chain_slot_bytes;
    auto slot = [&](int k) -> void* { return base + (size_t)k * N * 8; };
    const ChainSlots S{slot(0), {slot(1), slot(2)}, slot(slots - 1), false, basis + (size_t)j * N};
    if (!use_real_chains(P, geo)) {  // the complex kernel starts from a complex copy
      CK(launch_real_to_complex(slot(slots - 1), basis + (size_t)j * N, n, st));
      if (P.counting) {
        P.stats.launches++;
        P.stats.aux_bytes += (double)N * 12.0;
      }
    }
    auto out_of = [&](int k) {
      const int h = (j + k) & 1;
      return Y + ((size_t)(h ? lay.rows(0) : 0) + lay.index(j, k)) * N;
    };
    mqw_status s = issue_chain(P, w0, chain_stage, K2, S, geo, out_of, st, last2);
    if (s != MQW_OK) return s;
  }
  if (builder) {
    for (int k = 1; k < all; k++) {
      CK(cudaEventRecord(ctx->bld_join_ev[k], ctx->bld_stream[k]));
      CK(cudaStreamWaitEvent(stream, ctx->bld_join_ev[k], 0));
    }
  } else {
    CK(ctx->join(stream, all));
  }
  const int bn = s2_tile_cols(nw);
  const int col_stride = (nw + bn - 1) / bn * bn;
  S2CoefParams cp{};
  cp.stages = P.d_stages.as<StageDesc>();
  cp.coef = P.d_coef.as<float>();
  cp.job0 = w0.stage_desc_off;
  cp.m = w0.stages;
  cp.sj = sj;
  cp.sk = chain_stage;
  cp.tbasis = last2 ? 1 : 0;
  cp.walks = nw;
  cp.col_stride = col_stride;
  cp.lay = lay;
  cp.rows_pad[0] = (lay.rows(0) + 7) / 8 * 8;
  cp.rows_pad[1] = (lay.rows(1) + 7) / 8 * 8;
  cp.C0 = ctx->s2c.as<float>() + (size_t)buf * P.s2c_floats;
  cp.C1 = cp.C0 + (size_t)cp.rows_pad[0] * col_stride;
  S2GemmParams gp{};
  gp.Y = Y;
  gp.C0 = cp.C0;
  gp.C1 = cp.C1;
  for (int h = 0; h < 2; h++) {
    gp.rows[h] = lay.rows(h);
    gp.rows_pad[h] = cp.rows_pad[h];
  }
  gp.col_stride = col_stride;
  gp.n = n;
  gp.walks = nw;
  gp.out_walks = P.s2_walks;
  gp.out = last2 ? ctx->s3v.as<float>() : ctx->s2psi.as<float>() + (size_t)buf * P.s2psi_floats;
  // The GEMM on the tensor cores (tcgen05, three-product TF32 split) unless
  // MQW_S2_GEMM=simt selects the FP32 SIMT kernel.
  const char* gemm_env = getenv("MQW_S2_GEMM");
  const bool simt_env = gemm_env && std::string(gemm_env) == "simt";
  if (!simt_env && s2_tc_np(nw) <= 128 && n >= 8 && lay.rows(1) >= 1) {
    CK(launch_s2_gemm_tc(cp, cp.C0, gp, ctx->dev_err.as<unsigned>(), stream));
  } else {
    CK(launch_s2_coef(cp, stream));
    CK(launch_s2_gemm(gp, stream));
  }
  if (P.counting) {
    P.stats.launches += 2;
    // the product basis once, every walk's planar state written
    P.stats.aux_bytes += (double)Kb * K2 * N * 4.0 + (double)nw * N * 8.0;
  }
  return MQW_OK;
}


// Diagonals (per group of equal n; instances are sorted by n) and the degree
// pass.
mqw_status issue_diag_degree(mqw_plan& P, cudaStream_t stream) {
  mqw_ctx* ctx = P.ctx;
  DiagOut* d_diag = P.d_diag.as<DiagOut>();
  for (int s = 0; s < P.count;) {
    const int n = P.n[P.order[s]];
    int e = s;
    while (e < P.count && P.n[P.order[e]] == n) e++;
    CK(launch_diag(n, e - s, P.d_raw.as<double>() + P.raw_off[s],
                   P.d_hp.as<float>() + P.hp_off[s], nullptr, d_diag + s,
                   P.ctx->diag_scratch.p, stream));
    if (P.counting) P.stats.launches += 3;
    s = e;
  }
  CK(launch_cheb_degree(P.d_jobs.as<CoefJob>(), (int)P.jobs.size(), d_diag,
                        P.opt.cheb_tol, P.d_degree.as<int>(),
                        P.d_onenorm.as<float>(), stream));
  if (P.counting) P.stats.launches++;
  return MQW_OK;
}

// Coefficients, propagation (resident and grid walks) and the means.
mqw_status issue_rest(mqw_plan& P, cudaStream_t stream) {
  mqw_ctx* ctx = P.ctx;
  const int nj = (int)P.jobs.size();
  DiagOut* d_diag = P.d_diag.as<DiagOut>();
  CK(launch_cheb_coeffs(P.d_jobs.as<CoefJob>(), nj, d_diag, P.opt.cheb_tol,
                        P.d_coef_off.as<long long>(), P.d_coef.as<float>(),
                        stream));
  if (P.counting) P.stats.launches++;
  if (P.counting) CK(cudaEventRecord(P.ev0, stream));
  int res_count = 0, res_max_n = 0;
  std::map<int, std::vector<int>> grid_by_n;
  for (size_t w = 0; w < P.walks.size(); w++) {
    if (P.walk_is_grid[w]) {
      grid_by_n[P.walks[w].n].push_back((int)w);
    } else {
      res_count++;
      res_max_n = std::max(res_max_n, P.walks[w].n);
    }
  }
  if (res_count > 0) {
    CK(launch_resident(P.precision, P.d_walks.as<ResidentWalk>(), res_count,
                       res_max_n, P.d_stages.as<StageDesc>(),
                       P.d_coef.as<float>(), P.d_hp.as<float>(), d_diag,
                       P.d_p_sample.as<double>(), stream));
    if (P.counting) P.stats.launches++;
  }
  for (auto& kv : grid_by_n) {
    const int n = kv.first;
    const GridShape gs = P.grid_geo.at(n);
    const PassGeomHost geo = pass_geom(P.precision, n, gs.lmax, gs.threads, gs.lane_smem > 0, std::max(0, gs.tma), gs.cl < 0 ? 0 : 1);
    const int G = gs.group;
    const std::vector<int>& ws = kv.second;
    const int kb1 = P.basis_kb1.count(n) ? P.basis_kb1.at(n) : 0;
    const int kb2 = P.basis_kb2.count(n) ? P.basis_kb2.at(n) : 0;
    // Blocks of walks: one block per instance when a shared basis is used
    // (the bases are built before, and read during, the block), else all.
    struct Block {
      size_t b0, b1;
      int Kb, Kl;  // basis sizes (0: none)
    };
    std::vector<Block> blocks;
    for (size_t b0 = 0; b0 < ws.size();) {
      Block bk{b0, ws.size(), 0, 0};
      if (kb1 > 0 || kb2 > 0) {
        size_t b1 = b0;
        while (b1 < ws.size() && P.walks[ws[b1]].inst == P.walks[ws[b0]].inst) b1++;
        bk.b1 = b1;
        const ResidentWalk& w0 = P.walks[ws[b0]];
        if (!w0.record_each && w0.stages >= 2) {
          int Kb = 0, Kl = 0;
          for (size_t k = b0; k < b1; k++) {
            Kb = std::max(Kb, P.degree[P.walks[ws[k]].stage_desc_off]);
            Kl = std::max(Kl, P.degree[P.walks[ws[k]].stage_desc_off + w0.stages - 1]);
          }
          bk.Kb = kb1 > 0 && Kb <= kb1 ? Kb : 0;
          bk.Kl = kb2 > 0 && Kl <= kb2 ? Kl : 0;
        }
      }
      blocks.push_back(bk);
      b0 = bk.b1;
    }
    // The bases of block i+1 are built on the context's basis stream into
    // the other of two buffers while block i's walks run (one buffer and no
    // overlap when two do not fit): block i waits for its build, the build
    // into a buffer waits until the block that last read it has joined.
    const int nbuf = P.basis_buffers;
    const BasisLayout Bs[2] = {{ctx->basis.as<char>(), (size_t)1 << n, kb1, kb2},
                               {ctx->basis2.as<char>(), (size_t)1 << n, kb1, kb2}};
    // The stage-2 product basis of a block (instance), and its largest
    // stage-2 degree.
    auto use_s2 = [&](const Block& bk) {
      const ResidentWalk& wb = P.walks[ws[bk.b0]];
      const int nwb = (int)(bk.b1 - bk.b0);
      return bk.Kb > 0 && P.s2_k2.count(n) && wb.stages >= 3 && nwb <= P.s2_walks &&
             (P.s2_mode > 0 || 2 * bk.Kb <= nwb);
    };
    // The product basis of the last two stages of a block (m = 4, stage-2
    // product basis, last-stage basis, one instance per block in order; the
    // walks' sample offsets consecutive).
    auto use_last2 = [&](const Block& bk) {
      const ResidentWalk& wb = P.walks[ws[bk.b0]];
      if (!P.s3_k3.count(n) || wb.stages != 4 || !bk.Kl || !use_s2(bk) || nbuf == 2 ||
          !use_real_chains(P, geo))
        return false;
      int K3b = 0;
      long long sum3 = 0;  // the per-walk recurrences' passes
      for (size_t k = bk.b0; k < bk.b1; k++) {
        const ResidentWalk& w = P.walks[ws[k]];
        if (w.stages != 4 || w.record_each || w.p_off != wb.p_off + (int)(k - bk.b0)) return false;
        K3b = std::max(K3b, P.degree[w.stage_desc_off + 2]);
        sum3 += P.degree[w.stage_desc_off + 2];
      }
      // real chain passes at 0.6 of a complex pass (see the layout)
      return K3b > 0 && K3b <= P.s3_k3.at(n) &&
             (P.s3_mode > 0 || 3LL * bk.Kl * K3b <= 5 * sum3);
    };
    auto s2_degree = [&](const Block& bk) {
      int K2b = 0;
      for (size_t k = bk.b0; k < bk.b1; k++)
        K2b = std::max(K2b, P.degree[P.walks[ws[k]].stage_desc_off + 1]);
      return K2b;
    };
    // A block's bases on one stream (the build-ahead's side stream): stage 1,
    // last stage, then the stage-2 product basis and its GEMM.
    auto build = [&](const Block& bk, int buf, cudaStream_t st) -> mqw_status {
      const ResidentWalk& w0 = P.walks[ws[bk.b0]];
      const BasisLayout& B = Bs[buf];
      if (bk.Kb) {
        mqw_status s = issue_basis(P, w0, 0, bk.Kb, B, geo, B.real1(), st);
        if (s != MQW_OK) return s;
      }
      if (use_s2(bk)) {  // the last-stage basis beside the chains
        std::function<mqw_status(cudaStream_t)> last_build;
        if (bk.Kl)
          last_build = [&](cudaStream_t ls) {
            return issue_basis(P, w0, w0.stages - 1, bk.Kl, B, geo, B.real2(), ls);
          };
        return issue_stage2(P, ws, bk.b0, bk.b1, B.real1(), bk.Kb, s2_degree(bk), geo,
                            std::min(gs.lanes, bk.Kb), last_build, st, buf, true);
      }
      if (bk.Kl) {
        mqw_status s = issue_basis(P, w0, w0.stages - 1, bk.Kl, B, geo, B.real2(), st);
        if (s != MQW_OK) return s;
      }
      return MQW_OK;
    };
    const bool overlap = nbuf == 2;
    cudaStream_t bst = ctx->basis_stream;
    if (overlap) {
      // Buffers free and inputs ready: everything queued so far.
      CK(cudaEventRecord(ctx->basis_free[0], stream));
      CK(cudaEventRecord(ctx->basis_free[1], stream));
    }
    bool built_next = false;  // block i's bases already issued on bst
    for (size_t bi = 0; bi < blocks.size(); bi++) {
      const Block& bk = blocks[bi];
      const int buf = overlap ? (int)(bi & 1) : 0;
      const bool has = bk.Kb || bk.Kl;
      // The stage-2 product basis of this instance (then no stage-1
      // recombination: the walks start from their stage-2 outputs). In order
      // (no build-ahead) its chains run on the lanes with the last-stage
      // basis beside them.
      const ResidentWalk& wb = P.walks[ws[bk.b0]];
      const bool s2 = use_s2(bk);
      if (s2 && !overlap) {
        mqw_status s = issue_basis(P, wb, 0, bk.Kb, Bs[0], geo, Bs[0].real1(), stream);
        if (s != MQW_OK) return s;
      } else if (has) {
        if (overlap) {
          if (!built_next) {
            CK(cudaStreamWaitEvent(bst, ctx->basis_free[buf], 0));
            mqw_status s = build(bk, buf, bst);
            if (s != MQW_OK) return s;
            CK(cudaEventRecord(ctx->basis_built[buf], bst));
          }
          CK(cudaStreamWaitEvent(stream, ctx->basis_built[buf], 0));
        } else {
          mqw_status s = build(bk, 0, stream);
          if (s != MQW_OK) return s;
        }
      }
      built_next = false;
      const BasisLayout& B = Bs[buf];
      const float* basis = bk.Kb ? B.real1() : nullptr;
      const float* lastb = bk.Kl ? B.real2() : nullptr;
      if (s2 && !overlap) {
        const int K2b = s2_degree(bk);
        std::function<mqw_status(cudaStream_t)> last_build;
        if (bk.Kl)
          last_build = [&](cudaStream_t st) {
            // first-kind vectors when they seed the last two stages' basis
            return issue_basis(P, wb, wb.stages - 1, bk.Kl, B, geo, B.real2(), st,
                               use_last2(bk));
          };
        mqw_status s = issue_stage2(P, ws, bk.b0, bk.b1, basis, bk.Kb, K2b, geo,
                                    std::min(gs.lanes, bk.Kb), last_build, stream);
        if (s != MQW_OK) return s;
        if (use_last2(bk)) {
          // m = 4: the last two stages by projection onto their product
          // basis; no walk runs a recurrence.
          int K3b = 0;
          for (size_t k = bk.b0; k < bk.b1; k++)
            K3b = std::max(K3b, P.degree[P.walks[ws[k]].stage_desc_off + 2]);
          s = issue_stage2(P, ws, bk.b0, bk.b1, lastb, bk.Kl, K3b, geo,
                           std::min(gs.lanes, bk.Kl), nullptr, stream, 0, false, true);
          if (s != MQW_OK) return s;
          Last2Params lp{};
          lp.V = ctx->s3v.as<float>();
          lp.psi = ctx->s2psi.as<float>();
          lp.n = n;
          lp.L = std::min(n, 12);
          lp.walks = (int)(bk.b1 - bk.b0);
          lp.v_walks = lp.psi_walks = P.s2_walks;
          lp.part = ctx->s3part.as<double>();
          lp.p_out = P.d_p_sample.as<double>() + wb.p_off;
          CK(launch_last2(lp, stream));
          if (P.counting) {
            P.stats.launches += 2;
            P.stats.aux_bytes += (double)lp.walks * ((size_t)1 << n) * 16.0;
          }
          continue;
        }
      }
      // Groups are dealt round-robin to the lanes, which run concurrently.
      // With shared bases a group is a basis group of up to gs.bgroup walks
      // (pass groups of G inside it), and the block's walks are split into
      // lanes x k groups of near-equal size so that the lanes finish
      // together; otherwise a group is one pass group of G walks.
      const int nw = (int)(bk.b1 - bk.b0);
      const bool shared = bk.Kb || bk.Kl;
      const int lanes = std::min(gs.lanes, (nw + G - 1) / G);
      const int per = shared ? std::max(G, gs.bgroup) : G;
      const int ngroups = shared ? lanes * ((nw + lanes * per - 1) / (lanes * per))
                                 : (nw + G - 1) / G;
      CK(ctx->fork(stream, lanes));
      // The next block's bases, overlapping this block's walks.
      if (overlap && bi + 1 < blocks.size() && (blocks[bi + 1].Kb || blocks[bi + 1].Kl)) {
        const int nb = (int)((bi + 1) & 1);
        CK(cudaStreamWaitEvent(bst, ctx->basis_free[nb], 0));
        mqw_status s = build(blocks[bi + 1], nb, bst);
        if (s != MQW_OK) return s;
        CK(cudaEventRecord(ctx->basis_built[nb], bst));
        built_next = true;
      }
      size_t a = bk.b0;
      for (int i = 0; i < ngroups && a < bk.b1; i++) {
        const size_t size = shared ? (size_t)(nw / ngroups + (i < nw % ngroups ? 1 : 0))
                                   : std::min((size_t)G, bk.b1 - a);
        std::vector<int> grp(ws.begin() + a, ws.begin() + a + size);
        const float* ext_re = nullptr;
        const float* ext_im = nullptr;
        if (s2) {
          const size_t N = (size_t)1 << n;
          const float* set = ctx->s2psi.as<float>() + (size_t)buf * P.s2psi_floats;
          ext_re = set + (a - bk.b0) * N;
          ext_im = set + (P.s2_walks + (a - bk.b0)) * N;
        }
        a += size;
        if (grp.empty()) continue;
        const int lane = i % lanes;
        double* proj = ctx->proj_part.as<double>() +
                       (size_t)lane * gs.bgroup *
                           (((size_t)1 << n) >> std::min(geo.L, kRecombineLog)) * 2;
        mqw_status s = run_grid_group(P, grp, geo, lane, G, gs.bgroup, s2 ? nullptr : basis,
                                      bk.Kb, lastb, bk.Kl, proj, ext_re, ext_im,
                                      lane == 0 ? stream : ctx->lane_stream[lane]);
        if (s != MQW_OK) return s;
      }
      CK(ctx->join(stream, lanes));
      if (overlap) CK(cudaEventRecord(ctx->basis_free[buf], stream));
    }
    // The basis stream must be joined back before the end of a capture.
    if (overlap) {
      CK(cudaEventRecord(ctx->basis_built[0], bst));
      CK(cudaStreamWaitEvent(stream, ctx->basis_built[0], 0));
    }
  }
  if (P.counting) CK(cudaEventRecord(P.ev1, stream));
  CK(launch_mean(P.d_p_sample.as<double>(), P.d_p_off.as<int>(),
                 P.d_p_cnt.as<int>(), P.count, P.d_p_mean.as<double>(), stream));
  if (P.counting) P.stats.launches++;
  return MQW_OK;
}

mqw_status plan_execute(mqw_plan& P, cudaStream_t stream) {
  mqw_ctx* ctx = P.ctx;
  if (!P.ev0) CK(cudaEventCreate(&P.ev0));
  if (!P.ev1) CK(cudaEventCreate(&P.ev1));
  // Replay the captured pipeline when the shared scratch it was captured
  // with is still in place.
  // (Its timing events bracket the whole graph: the diagonal and coefficient
  // kernels add < 0.3% to the propagation they time in an eager run.)
  if (P.gexec && P.graph_gen == ctx->scratch_gen) {
    CK(cudaEventRecord(P.ev0, stream));
    CK(cudaGraphLaunch(P.gexec, stream));
    CK(cudaEventRecord(P.ev1, stream));
    P.timed = true;
    P.executed = true;
    return MQW_OK;
  }
  P.counting = true;
  P.stats.launches = P.stats.term_launches = 0;
  P.stats.pass_amps = 0;
  P.stats.aux_bytes = 0;
  P.stats.h2d_bytes = P.stats.d2h_bytes = 0;
  // Geometry and shared scratch for every n of the plan, sized up front so
  // that nothing is allocated while the pipeline is issued or captured.
  std::map<int, int> grid_count;
  for (size_t w = 0; w < P.walks.size(); w++)
    if (P.walk_is_grid[w]) grid_count[P.walks[w].n]++;
  size_t state_b = 0, norm_b = 0;
  int lanes_max = 1;
  for (auto& kv : grid_count) {
    const int n = kv.first;
    GridShape gs;
    gs.lmax = std::max(0, P.opt.tile_log);
    gs.group = std::max(0, P.opt.group);
    gs.lanes = std::min(std::max(0, P.opt.lanes), kMaxLanes);
    gs.threads = P.opt.threads == 256 ? 256 : 0;
    gs.lane_smem = P.opt.lane_smem;
    gs.tma = P.opt.tma;
    gs.cl = P.opt.cluster;  // fixed (1 / -1) or tuned (0; clusters when not tuned)
    if (!gs.lmax || !gs.group || !gs.lanes || !P.opt.threads || !P.opt.lane_smem ||
        !P.opt.tma) {
      GridShape want = gs;
      want.threads = P.opt.threads;  // 0: tuned, else fixed
      GridShape t;
      mqw_status s = tune_grid(ctx, P.precision, n, want, &t);
      if (s != MQW_OK) return s;
      gs = t;
    }
    if (P.comp) {  // the compensated kernel exists in the default shape only
      gs.threads = 0;
      gs.lane_smem = -1;
      gs.tma = -1;
      gs.lmax = std::min(gs.lmax, 12);
      if (pass_geom(P.precision, n, gs.lmax, 0, 0, 0, gs.cl < 0 ? 0 : 1).C > 0)
        gs.lmax = 11;  // single-CTA tiles
    }
    gs.group = std::min(std::min(gs.group, kMaxGroup), kv.second);
    const int ngroups = (kv.second + gs.group - 1) / gs.group;
    gs.lanes = std::max(1, std::min(gs.lanes, ngroups));
    const PassGeomHost geo = pass_geom(P.precision, n, gs.lmax, gs.threads, gs.lane_smem > 0, std::max(0, gs.tma), gs.cl < 0 ? 0 : 1);
    // Walks per shared-basis group: the stage-1 recombination and the
    // last-stage projection read each basis vector once per group, so the
    // group is as large as the launch structures allow (kMaxGroup) within a
    // state budget of a quarter of the free memory (16 GB at most).
    // MQW_BASIS_GROUP caps it (1: one basis read per pass group).
    gs.bgroup = gs.group;
    if ((P.opt.stage1_basis || P.opt.final_projection) && P.precision == 0 && !P.comp) {
      size_t free_b = 0, total_b = 0;
      if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = (size_t)8 << 30;
      const size_t budget = std::min(free_b / 4, (size_t)16 << 30);
      int bg = std::min(kMaxGroup, kv.second);
      if (const char* e = getenv("MQW_BASIS_GROUP")) bg = std::min(bg, std::max(1, atoi(e)));
      while (bg > gs.group && (size_t)gs.lanes * bg * walk_bytes(P.precision, geo, n) > budget)
        bg--;
      gs.bgroup = std::max(gs.group, bg);
    }
    P.grid_geo[n] = gs;
    lanes_max = std::max(lanes_max, gs.lanes);
    const size_t N = (size_t)1 << n;
    const size_t amp = P.precision == 0 ? 8 : 16;
    const size_t walks = (size_t)gs.lanes * gs.bgroup;
    state_b = std::max(state_b, walks * walk_slots(geo) * N * amp);
    norm_b = std::max(norm_b, walks * (N >> std::min(geo.L, kRecombineLog)) * sizeof(double));
  }
  CK(ctx->ensure_lanes(lanes_max));
  CK(ctx->grow(ctx->diag_scratch, P.diag_scratch_bytes));
  if (state_b) CK(ctx->grow(ctx->state, state_b));
  if (norm_b) CK(ctx->grow(ctx->norm_part, norm_b));
  CK(ctx->grow(ctx->kappa, kMaxLanes * kMaxGroup * sizeof(double)));

  // 1-2. Diagonals and degrees; degrees and onenorms are read back to lay
  // out the coefficient pool and the launch schedule.
  mqw_status s = issue_diag_degree(P, stream);
  if (s != MQW_OK) return s;
  const int nj = (int)P.jobs.size();
  P.degree.resize(nj);
  P.onenorm.resize(nj);
  CK(cudaMemcpyAsync(P.degree.data(), P.d_degree.p, nj * sizeof(int),
                     cudaMemcpyDeviceToHost, stream));
  CK(cudaMemcpyAsync(P.onenorm.data(), P.d_onenorm.p, nj * sizeof(float),
                     cudaMemcpyDeviceToHost, stream));
  P.stats.d2h_bytes += (double)nj * (sizeof(int) + sizeof(float));
  CK(cudaStreamSynchronize(stream));
  P.coef_off.assign(nj + 1, 0);
  P.stats.terms = 0;
  for (int j = 0; j < nj; j++) {
    if (P.degree[j] < 1)
      return fail(ctx, MQW_ERR_INVALID,
                  "Chebyshev degree failed for job %d (non-finite time?)", j);
    P.coef_off[j + 1] = P.coef_off[j] + P.degree[j];
    P.stats.terms += P.degree[j];
  }
  std::vector<StageDesc> sdesc(nj);
  for (int j = 0; j < nj; j++) {
    sdesc[j].coef_off = P.coef_off[j];
    sdesc[j].K = P.degree[j];
    sdesc[j].gamma = P.jobs[j].gamma;
    sdesc[j].onenorm = P.onenorm[j];
  }
  std::vector<ResidentWalk> res;
  P.stats.term_amps = 0;
  for (size_t w = 0; w < P.walks.size(); w++) {
    for (int st = 0; st < P.walks[w].stages; st++)
      P.stats.term_amps += (double)P.degree[P.walks[w].stage_desc_off + st] *
                           (double)(1u << P.walks[w].n);
    if (!P.walk_is_grid[w]) res.push_back(P.walks[w]);
  }
  // Shared bases (FP32): the largest first- and last-stage degrees per n
  // decide the buffers; an n whose bases would not fit the budget drops the
  // last-stage basis first, then the stage-1 basis.
  P.basis_kb1.clear();
  P.basis_kb2.clear();
  const bool want1 = P.opt.stage1_basis && P.precision == 0 && !P.comp;
  const bool want2 = P.opt.final_projection && P.precision == 0 && !P.comp;
  if (want1 || want2) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = (size_t)8 << 30;
    // Up to half the free memory (64 GB at most): at n = 28 the stage-1
    // basis alone is ~K_1 GB.
    const size_t budget = std::min(free_b / 2, (size_t)64 << 30);
    std::map<int, std::pair<int, int>> kb;
    std::map<int, int> s2k;             // largest stage-2 degree (m >= 3 walks)
    std::map<int, int> s3k;             // largest stage-3 degree (m == 4 walks)
    std::map<int, int> inst_walks;      // walks of one instance (largest)
    std::map<std::pair<int, int>, int> per_inst;
    for (size_t w = 0; w < P.walks.size(); w++) {
      const ResidentWalk& wk = P.walks[w];
      if (!P.walk_is_grid[w] || wk.record_each || wk.stages < 2) continue;
      auto& k = kb[wk.n];
      k.first = std::max(k.first, P.degree[wk.stage_desc_off]);
      k.second = std::max(k.second, P.degree[wk.stage_desc_off + wk.stages - 1]);
      if (wk.stages >= 3) {
        s2k[wk.n] = std::max(s2k[wk.n], P.degree[wk.stage_desc_off + 1]);
        if (wk.stages == 4)
          s3k[wk.n] = std::max(s3k[wk.n], P.degree[wk.stage_desc_off + 2]);
        const int c = ++per_inst[std::make_pair(wk.n, wk.inst)];
        inst_walks[wk.n] = std::max(inst_walks[wk.n], c);
      }
    }
    size_t basis_b = 0, proj_b = 0;
    int rmax = 0;
    for (auto& e : kb) {
      const int n = e.first;
      const GridShape& gs = P.grid_geo.at(n);
      const PassGeomHost geo = pass_geom(P.precision, n, gs.lmax, gs.threads,
                                         gs.lane_smem > 0, std::max(0, gs.tma), gs.cl < 0 ? 0 : 1);
      int k1 = want1 && e.second.first <= kMaxBasis ? e.second.first : 0;
      int k2 = want2 && e.second.second <= kMaxBasis ? e.second.second : 0;
      if (BasisLayout::bytes(n, k1, k2) > budget) k2 = 0;
      if (BasisLayout::bytes(n, k1, k2) > budget) k1 = 0;
      if (!k1 && !k2) continue;
      P.basis_kb1[n] = k1;
      P.basis_kb2[n] = k2;
      basis_b = std::max(basis_b, BasisLayout::bytes(n, k1, k2));
      // projection partials: per lane, per walk, per recombination block
      proj_b = std::max(proj_b, (size_t)gs.lanes * gs.bgroup *
                                    (((size_t)1 << n) >> std::min(geo.L, kRecombineLog)) *
                                    2 * sizeof(double));
      rmax = std::max(rmax, std::max(k1 + (k1 & 1), k2 + (k2 & 1)));
    }
    P.basis_buffers = 1;
    // Building the next instance's bases ahead measured within 1% (the walks
    // already keep the GPU busy), so it is opt-in: MQW_BASIS_AHEAD=1.
    static const bool ahead_env =
        getenv("MQW_BASIS_AHEAD") && atoi(getenv("MQW_BASIS_AHEAD")) != 0;
    const bool ahead = ahead_env && basis_b && 2 * basis_b <= budget;
    // Stage-2 product basis (walks of m >= 3 with the stage-1 basis): worth
    // it when its chains (one per stage-1 basis vector) are fewer than half
    // of the instance's walks (MQW_STAGE2_BASIS=0 turns it off, =1 uses it
    // whenever it fits). With the build-ahead its buffers are doubled.
    P.s2_k2.clear();
    P.s2_walks = 0;
    size_t s2y_b = 0, s2psi_n = 0, s2c_b = 0, s2part_n = 0;
    {
      const char* env = getenv("MQW_STAGE2_BASIS");
      const int mode = env ? atoi(env) : -1;
      P.s2_mode = mode;
      for (auto& e : s2k) {
        const int n = e.first, K2 = e.second;
        if (mode == 0 || !P.basis_kb1.count(n) || P.basis_kb1.at(n) == 0) continue;
        const int k1 = P.basis_kb1.at(n), wpi = inst_walks[n];
        if (mode < 0 && 2 * k1 > wpi) continue;
        const size_t N = (size_t)1 << n;
        const size_t yb = std::max(s2y_b, (size_t)k1 * K2 * N * 4);
        const size_t pb = 2 * (size_t)std::max(P.s2_walks, wpi) * std::max(s2psi_n, N) * 4;
        // one partial P per chain for the batched chain launches
        const size_t cb = std::max(s2part_n, (size_t)k1 * N) * 4;
        if ((ahead ? 2 : 1) * (basis_b + yb + pb + cb) > budget) continue;
        P.s2_k2[n] = K2;
        P.s2_walks = std::max(P.s2_walks, wpi);
        s2y_b = yb;
        s2psi_n = std::max(s2psi_n, N);
        // coefficient matrices: the SIMT GEMM's row-major pair, or the
        // tensor-core GEMM's K-major hi/lo copies, whichever is larger
        s2c_b = std::max(s2c_b, ((size_t)k1 * K2 + 16) * (size_t)((wpi + 127) / 128 * 128) * 4);
        s2c_b = std::max(s2c_b, s2_tc_coef_floats(wpi, S2Layout{k1, K2}) * 4);
        rmax = std::max(rmax, K2 + (K2 & 1));
        // the product basis's chains run batched, one partial P each
        s2part_n = cb / 4;
      }
    }
    // The product basis of the last two stages (m = 4 instances with the
    // stage-2 product basis and a last-stage basis): Y'_jk = U_k(H~_3) w'_j,
    // its walks' recombined vectors and the projection partials, one
    // instance at a time, without the build-ahead. Its cost is one real
    // chain of K_3 passes per last-stage basis vector against one complex
    // recurrence per walk; a real pass costs about 0.6 of a complex one
    // (measured at n = 20: 4.5 against 7.8 us). Laid out when the basis
    // vectors are at most 5/3 of an instance's walks and chosen per instance
    // (use_last2 in issue_rest) by that cost, or always with
    // MQW_LAST2_BASIS=1; MQW_LAST2_BASIS=0 turns it off.
    P.s3_k3.clear();
    size_t s3y_b = 0, s3v_b = 0, s3p_b = 0;
    {
      const char* env = getenv("MQW_LAST2_BASIS");
      const int mode = env ? atoi(env) : -1;
      P.s3_mode = mode;
      for (auto& e : s3k) {
        const int n = e.first, K3 = e.second;
        if (mode == 0 || ahead || !P.s2_k2.count(n) || !P.basis_kb2.count(n)) continue;
        const int k4 = P.basis_kb2.at(n), wpi = inst_walks[n];
        if (k4 == 0 || K3 == 0 || (mode < 0 && 3 * k4 > 5 * wpi)) continue;
        const size_t N = (size_t)1 << n;
        const size_t yb = std::max(s3y_b, (size_t)k4 * K3 * N * 4);
        // V has the stage-2 outputs' walk stride (the GEMM writes both alike)
        const size_t vb = std::max(s3v_b, 2 * (size_t)P.s2_walks * N * 4);
        const size_t qb = std::max(s3p_b, last2_part_bytes(n, wpi));
        const size_t cb = std::max(s2part_n, (size_t)k4 * N) * 4;
        if (basis_b + s2y_b + 2 * (size_t)P.s2_walks * s2psi_n * 4 + cb + yb + vb > budget)
          continue;
        P.s3_k3[n] = K3;
        s3y_b = yb;
        s3v_b = vb;
        s3p_b = qb;
        s2part_n = cb / 4;
        s2c_b = std::max(s2c_b, ((size_t)k4 * K3 + 16) * (size_t)((wpi + 127) / 128 * 128) * 4);
        s2c_b = std::max(s2c_b, s2_tc_coef_floats(wpi, S2Layout{k4, K3}) * 4);
        rmax = std::max(rmax, K3 + (K3 & 1));
      }
    }
    if (!P.s3_k3.empty()) {
      CK(ctx->grow(ctx->s3y, s3y_b));
      CK(ctx->grow(ctx->s3v, s3v_b));
      CK(ctx->grow(ctx->s3part, s3p_b));
    }
    if (!P.s2_k2.empty()) {
      const size_t nb = ahead ? 2 : 1;
      CK(ctx->ensure_lanes(kMaxStreams));  // chain lanes and the last-stage basis beside them
      P.s2y_floats = s2y_b / 4;
      P.s2psi_floats = 2 * (size_t)P.s2_walks * s2psi_n;
      P.s2c_floats = s2c_b / 4;
      CK(ctx->grow(ctx->s2y, nb * s2y_b));
      CK(ctx->grow(ctx->s2psi, nb * P.s2psi_floats * 4));
      CK(ctx->grow(ctx->s2c, nb * s2c_b));
      if (ahead) CK(ctx->grow(ctx->s2chain, (size_t)kMaxLanes * 4 * s2psi_n * 8));
      P.s2part_floats = s2part_n;
      if (s2part_n) CK(ctx->grow(ctx->s2part, nb * s2part_n * 4));
    }
    if (basis_b) {
      CK(ctx->grow(ctx->basis, basis_b));
      if (ahead) {  // a second buffer to build ahead into
        CK(ctx->grow(ctx->basis2, basis_b));
        CK(ctx->ensure_basis_stream());
        P.basis_buffers = 2;
      }
      CK(ctx->grow(ctx->proj_part, proj_b));
      if (P.unit_len < rmax + 1) {
        std::vector<float> unit(rmax + 1, 0.0f);
        unit[rmax] = 1.0f;
        CK(P.d_unit.ensure(unit.size() * sizeof(float)));
        CK(cudaMemcpyAsync(P.d_unit.p, unit.data(), unit.size() * sizeof(float),
                           cudaMemcpyHostToDevice, stream));
        CK(cudaStreamSynchronize(stream));  // `unit` is a local buffer
        P.unit_len = rmax + 1;
        P.stats.h2d_bytes += (double)unit.size() * sizeof(float);
      }
    }
  }
  // A re-layout drops any captured graph (its addresses may change).
  if (P.gexec) {
    cudaGraphExecDestroy(P.gexec);
    P.gexec = nullptr;
  }
  CK(P.d_coef_off.ensure((nj + 1) * sizeof(long long)));
  CK(P.d_coef.ensure(P.coef_off[nj] * sizeof(float)));
  CK(P.d_stages.ensure(nj * sizeof(StageDesc)));
  CK(P.d_walks.ensure(std::max<size_t>(1, res.size()) * sizeof(ResidentWalk)));
  CK(cudaMemcpyAsync(P.d_coef_off.p, P.coef_off.data(), (nj + 1) * sizeof(long long),
                     cudaMemcpyHostToDevice, stream));
  CK(cudaMemcpyAsync(P.d_stages.p, sdesc.data(), nj * sizeof(StageDesc),
                     cudaMemcpyHostToDevice, stream));
  if (!res.empty())
    CK(cudaMemcpyAsync(P.d_walks.p, res.data(), res.size() * sizeof(ResidentWalk),
                       cudaMemcpyHostToDevice, stream));
  P.stats.h2d_bytes += (double)(nj + 1) * sizeof(long long) +
                       (double)nj * sizeof(StageDesc) +
                       (double)res.size() * sizeof(ResidentWalk);
  // 3-5. Coefficients, propagation, means.
  s = issue_rest(P, stream);
  if (s != MQW_OK) return s;
  P.timed = true;
  P.executed = true;
  P.eager_runs++;
  // Capture the whole device pipeline for later executes, once the plan is
  // executed a second time (a plan run once pays no capture). The capture
  // runs on the context's private stream (nothing executes while
  // capturing); the graph is later launched on whatever stream the caller
  // passes. Very large pipelines (over kMaxGraphLaunches kernels) stay
  // eager: their launch overhead is already negligible and a graph of
  // millions of nodes costs host memory and instantiation time.
  constexpr long long kMaxGraphLaunches = 200000;
  if (P.opt.graph && P.eager_runs >= 2 && P.stats.launches <= kMaxGraphLaunches) {
    CK(cudaStreamSynchronize(stream));
    cudaStream_t cs = ctx->stream;
    P.counting = false;
    CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    mqw_status s1 = issue_diag_degree(P, cs);
    mqw_status s2 = s1 == MQW_OK ? issue_rest(P, cs) : s1;
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(cs, &graph);
    P.counting = true;
    if (s2 != MQW_OK) {
      if (graph) cudaGraphDestroy(graph);
      return s2;
    }
    CK(ec);
    const cudaError_t ei = cudaGraphInstantiate(&P.gexec, graph, 0);
    cudaGraphDestroy(graph);
    CK(ei);
    P.graph_gen = ctx->scratch_gen;
  }
  return MQW_OK;
}

}  // namespace

extern "C" {

int mqw_abi_version(void) { return MQW_ABI_VERSION; }

const char* mqw_status_string(mqw_status s) {
  switch (s) {
    case MQW_OK: return "ok";
    case MQW_ERR_INVALID: return "invalid argument";
    case MQW_ERR_CUDA: return "CUDA error";
    case MQW_ERR_NOMEM: return "out of memory";
    case MQW_ERR_IO: return "I/O error";
    case MQW_ERR_TIMEOUT: return "device wait timed out";
    case MQW_ERR_UNSUPPORTED: return "unsupported";
    case MQW_ERR_NO_DEVICE: return "no sm_100 CUDA device";
  }
  return "unknown status";
}

void mqw_default_options(mqw_options* opt) {
  if (opt) default_opts(opt);
}

mqw_status mqw_create(mqw_ctx** out, int device) {
  if (!out) return MQW_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return MQW_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return MQW_ERR_NO_DEVICE;
  if (prop.major != 10) return MQW_ERR_NO_DEVICE;  // built for sm_100a only
  if (cudaSetDevice(device) != cudaSuccess) return MQW_ERR_NO_DEVICE;
  std::unique_ptr<mqw_ctx> ctx(new mqw_ctx);
  ctx->device = device;
  ctx->sm_count = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess)
    return MQW_ERR_CUDA;
  if (ctx->dev_err.ensure(sizeof(unsigned)) != cudaSuccess ||
      cudaMemset(ctx->dev_err.p, 0, sizeof(unsigned)) != cudaSuccess)
    return MQW_ERR_CUDA;
  *out = ctx.release();
  return MQW_OK;
}

void mqw_destroy(mqw_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  for (int k = 1; k < kMaxStreams; k++) {
    if (ctx->lane_stream[k]) cudaStreamDestroy(ctx->lane_stream[k]);
    if (ctx->join_ev[k]) cudaEventDestroy(ctx->join_ev[k]);
  }
  if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
  if (ctx->basis_stream) cudaStreamDestroy(ctx->basis_stream);
  for (int k = 1; k < kMaxStreams; k++) {
    if (ctx->bld_stream[k]) cudaStreamDestroy(ctx->bld_stream[k]);
    if (ctx->bld_join_ev[k]) cudaEventDestroy(ctx->bld_join_ev[k]);
  }
  if (ctx->bld_fork_ev) cudaEventDestroy(ctx->bld_fork_ev);
  for (int k = 0; k < 2; k++) {
    if (ctx->basis_built[k]) cudaEventDestroy(ctx->basis_built[k]);
    if (ctx->basis_free[k]) cudaEventDestroy(ctx->basis_free[k]);
  }
  delete ctx;
}

const char* mqw_last_error(const mqw_ctx* ctx) {
  if (!ctx) return "null context";
  return ctx->err.c_str();
}

mqw_status mqw_read_instances(const char* filename, int n, long long start,
                              long long problems, double* raw_out) {
  if (!filename || n < 1 || n > MQW_MAX_N || start < 0 || problems < 0 ||
      (problems > 0 && !raw_out))
    return MQW_ERR_INVALID;
  FILE* f = fopen(filename, "rb");
  if (!f) return MQW_ERR_IO;
  const long long per = params_per(n);
  if (fseeko(f, (off_t)(start * per * 8), SEEK_SET) != 0) {
    fclose(f);
    return MQW_ERR_IO;
  }
  const size_t want = (size_t)(problems * per);
  const size_t got = fread(raw_out, sizeof(double), want, f);
  fclose(f);
  return got == want ? MQW_OK : MQW_ERR_IO;
}

mqw_status mqw_plan_create(mqw_ctx* ctx, int count, const int* n, const int* m,
                           const double* raw, const mqw_options* opt_in,
                           mqw_plan** out) {
  mqw_status s = check_ctx(ctx);
  if (s != MQW_OK) return s;
  if (!out || count < 1 || !n || !m || !raw)
    return fail(ctx, MQW_ERR_INVALID, "plan_create: bad arguments");
  mqw_options opt;
  default_opts(&opt);
  if (opt_in) opt = *opt_in;
  if (opt.precision != MQW_FP32 && opt.precision != MQW_FP64 &&
      opt.precision != MQW_FP32_COMPENSATED)
    return fail(ctx, MQW_ERR_INVALID,
                "precision must be MQW_FP32, MQW_FP64 or MQW_FP32_COMPENSATED");
  if (opt.samples < 1 || opt.samples > MQW_SAMPLES)
    return fail(ctx, MQW_ERR_INVALID, "samples must be in 1..100");
  if (!(opt.cheb_tol > 0.0) || opt.cheb_tol >= 1.0)
    return fail(ctx, MQW_ERR_INVALID, "cheb_tol must be in (0, 1)");
  for (int i = 0; i < count; i++) {
    if (n[i] < 1 || n[i] > MQW_MAX_N)
      return fail(ctx, MQW_ERR_INVALID, "instance %d: n=%d outside 1..%d", i, n[i], MQW_MAX_N);
    if (m[i] < 1 || m[i] > MQW_MAX_M)
      return fail(ctx, MQW_ERR_INVALID, "instance %d: m=%d outside 1..%d", i, m[i], MQW_MAX_M);
  }
  std::unique_ptr<mqw_plan> P(new mqw_plan);
  P->ctx = ctx;
  P->opt = opt;
  P->count = count;
  P->comp = opt.precision == MQW_FP32_COMPENSATED;
  P->precision = P->comp ? MQW_FP32 : opt.precision;
  P->opt.precision = P->precision;
  P->samples = opt.samples;
  P->n.assign(n, n + count);
  P->m.assign(m, m + count);
  P->total_t.assign(count, 0.0f);
  std::vector<long long> caller_off(count + 1, 0), stage_off(count + 1, 0);
  for (int i = 0; i < count; i++) {
    caller_off[i + 1] = caller_off[i] + params_per(n[i]);
    stage_off[i + 1] = stage_off[i] + m[i];
  }
  P->order.resize(count);
  std::iota(P->order.begin(), P->order.end(), 0);
  std::stable_sort(P->order.begin(), P->order.end(),
                   [&](int a, int b) { return n[a] < n[b]; });
  // Raw inputs in sorted order; hp pool offsets; schedules on the host.
  std::vector<double> raw_sorted;
  raw_sorted.reserve(caller_off[count]);
  P->raw_off.resize(count);
  P->hp_off.resize(count);
  P->p_off.resize(count);
  long long hp_total = 0;
  std::vector<int> p_cnt(count);
  const int res_max =
      opt.resident_max_n < 0 ? 0
      : P->comp ? 5  // compensated sums live in the grid path (n >= 6)
      : opt.resident_max_n == 0 ? resident_max_n(P->precision)
      : std::min(opt.resident_max_n, resident_max_n(P->precision));
  int p_total = 0;
  std::vector<float> gam(MQW_MAX_M), st(MQW_MAX_M), times(MQW_MAX_M * MQW_SAMPLES);
  for (int k = 0; k < count; k++) {
    const int i = P->order[k];
    const int ni = n[i], mi = m[i];
    P->raw_off[k] = (long long)raw_sorted.size();
    raw_sorted.insert(raw_sorted.end(), raw + caller_off[i], raw + caller_off[i + 1]);
    P->hp_off[k] = hp_total;
    hp_total += 1ll << ni;
    float tot = 0.0f;
    mqw_schedule(ni, mi, raw + caller_off[i], gam.data(), st.data(), times.data(), &tot);
    P->total_t[i] = tot;
    if (opt.stage_scale) {
      for (int s2 = 0; s2 < mi; s2++) {
        const float fg = opt.stage_scale[(size_t)(stage_off[i] + s2) * 2 + 0];
        const float ft = opt.stage_scale[(size_t)(stage_off[i] + s2) * 2 + 1];
        if (!(fg > 0.0f) || !(ft > 0.0f) || !std::isfinite(fg) || !std::isfinite(ft))
          return fail(ctx, MQW_ERR_INVALID, "stage_scale must be positive and finite");
        gam[s2] *= fg;
        for (int j = 0; j < MQW_SAMPLES; j++) times[s2 * MQW_SAMPLES + j] *= ft;
      }
    }
    P->p_off[k] = p_total;
    p_cnt[k] = opt.samples;
    p_total += opt.samples;
    const bool grid = ni > res_max && ni >= 6;  // the grid path needs n >= 6
    auto add_walk = [&](int stages, int record_each, int p_at) {
      ResidentWalk w;
      w.inst = k;
      w.n = ni;
      w.stages = stages;
      w.record_each = record_each;
      w.stage_desc_off = (int)P->jobs.size();
      w.p_off = p_at;
      w.hp_off = P->hp_off[k];
      P->walks.push_back(w);
      P->walk_is_grid.push_back(grid ? 1 : 0);
    };
    if (mi == 1) {
      // One cumulative walk over the sorted, differenced times.
      add_walk(opt.samples, 1, P->p_off[k]);
      for (int j = 0; j < opt.samples; j++)
        P->jobs.push_back(CoefJob{k, ni, gam[0], times[j]});
    } else {
      for (int j = 0; j < opt.samples; j++) {
        add_walk(mi, 0, P->p_off[k] + j);
        for (int s2 = 0; s2 < mi; s2++)
          P->jobs.push_back(CoefJob{k, ni, gam[s2], times[s2 * MQW_SAMPLES + j]});
      }
    }
  }
  P->stats.instances = count;
  P->create_h2d = (double)raw_sorted.size() * sizeof(double) + (double)P->jobs.size() * sizeof(CoefJob) +
                  2.0 * count * sizeof(int);
  P->stats.trajectories = (long long)p_total;
  // Uploads.
  cudaStream_t stream = ctx->stream;
  CK(P->d_raw.ensure(raw_sorted.size() * sizeof(double)));
  CK(cudaMemcpyAsync(P->d_raw.p, raw_sorted.data(), raw_sorted.size() * sizeof(double),
                     cudaMemcpyHostToDevice, stream));
  CK(P->d_hp.ensure((size_t)hp_total * sizeof(float)));
  CK(P->d_diag.ensure(count * sizeof(DiagOut)));
  size_t scratch = 0;
  for (int k = 0; k < count;) {
    const int ni = n[P->order[k]];
    int e = k;
    while (e < count && n[P->order[e]] == ni) e++;
    scratch = std::max(scratch, diag_scratch_bytes(ni, e - k));
    k = e;
  }
  P->diag_scratch_bytes = scratch;
  const size_t nj = P->jobs.size();
  CK(P->d_jobs.ensure(nj * sizeof(CoefJob)));
  CK(cudaMemcpyAsync(P->d_jobs.p, P->jobs.data(), nj * sizeof(CoefJob),
                     cudaMemcpyHostToDevice, stream));
  CK(P->d_degree.ensure(nj * sizeof(int)));
  CK(P->d_onenorm.ensure(nj * sizeof(float)));
  CK(P->d_p_sample.ensure((size_t)p_total * sizeof(double)));
  CK(P->d_p_mean.ensure(count * sizeof(double)));
  CK(P->d_p_off.ensure(count * sizeof(int)));
  CK(P->d_p_cnt.ensure(count * sizeof(int)));
  CK(cudaMemcpyAsync(P->d_p_off.p, P->p_off.data(), count * sizeof(int),
                     cudaMemcpyHostToDevice, stream));
  CK(cudaMemcpyAsync(P->d_p_cnt.p, p_cnt.data(), count * sizeof(int),
                     cudaMemcpyHostToDevice, stream));
  CK(cudaStreamSynchronize(stream));
  *out = P.release();
  return MQW_OK;
}

mqw_status mqw_plan_execute(mqw_plan* plan, void* stream) {
  if (!plan) return MQW_ERR_INVALID;
  mqw_ctx* ctx = plan->ctx;
  mqw_status s = check_ctx(ctx);
  if (s != MQW_OK) return s;
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  plan->timed = false;
  return plan_execute(*plan, st);
}

mqw_status mqw_plan_results(mqw_plan* plan, double* p_out, float* total_t,
                            uint32_t* e_loc, double* p_sample) {
  if (!plan) return MQW_ERR_INVALID;
  mqw_ctx* ctx = plan->ctx;
  mqw_status s = check_ctx(ctx);
  if (s != MQW_OK) return s;
  if (!plan->executed) return fail(ctx, MQW_ERR_INVALID, "plan not executed");
  CK(cudaDeviceSynchronize());
  s = take_device_error(ctx);
  if (s != MQW_OK) return s;
  const int count = plan->count;
  std::vector<double> pm(count);
  std::vector<DiagOut> dg(count);
  CK(cudaMemcpy(pm.data(), plan->d_p_mean.p, count * sizeof(double), cudaMemcpyDeviceToHost));
  plan->stats.d2h_bytes += (double)count * (sizeof(double) + sizeof(DiagOut));
  CK(cudaMemcpy(dg.data(), plan->d_diag.p, count * sizeof(DiagOut), cudaMemcpyDeviceToHost));
  std::vector<double> ps;
  if (p_sample) {
    ps.resize((size_t)count * plan->samples);
    CK(cudaMemcpy(ps.data(), plan->d_p_sample.p, ps.size() * sizeof(double),
                  cudaMemcpyDeviceToHost));
    plan->stats.d2h_bytes += (double)ps.size() * sizeof(double);
  }
  for (int k = 0; k < count; k++) {
    const int i = plan->order[k];
    if (p_out) p_out[i] = pm[k];
    if (e_loc) e_loc[i] = dg[k].e_loc;
    if (p_sample)
      std::copy(ps.begin() + plan->p_off[k], ps.begin() + plan->p_off[k] + plan->samples,
                p_sample + (size_t)i * plan->samples);
  }
  if (total_t)
    for (int i = 0; i < count; i++) total_t[i] = plan->total_t[i];
  return MQW_OK;
}

mqw_status mqw_measure_peaks(mqw_ctx* ctx, mqw_tier_peaks* out) {
  mqw_status st = check_ctx(ctx);
  if (st != MQW_OK) return st;
  if (!out) return fail(ctx, MQW_ERR_INVALID, "mqw_measure_peaks: null output");
  CK(measure_tiers(ctx->stream, ctx->sm_count, &out->l2_read_gbs, &out->l2_copy_gbs,
                   &out->smem_gbs, &out->hbm_copy_gbs));
  return MQW_OK;
}

mqw_status mqw_selftest_wait_timeout(mqw_ctx* ctx) {
  mqw_status st = check_ctx(ctx);
  if (st != MQW_OK) return st;
  // One FP32 n = 14 pass with bulk-copy staging whose mbarrier expects 16
  // bytes that no copy delivers: every CTA's bounded wait (5 ms) runs out,
  // sets the error word and returns. Nothing else is in flight.
  const int n = 14;
  const size_t N = (size_t)1 << n;
  const PassGeomHost geo = pass_geom(0, n, 0, 0, 0, 1);
  CK(ctx->grow(ctx->state, 3 * N * 8 + N * sizeof(float)));
  CK(ctx->grow(ctx->norm_part, (N >> geo.L) * sizeof(double)));
  CK(ctx->tune_coef.ensure(64 * sizeof(float)));
  CK(cudaMemsetAsync(ctx->state.p, 0, 3 * N * 8 + N * sizeof(float), ctx->stream));
  CK(cudaMemsetAsync(ctx->tune_coef.p, 0, 64 * sizeof(float), ctx->stream));
  char* base = ctx->state.as<char>();
  PassParams pp{};
  pp.n = n;
  pp.L = geo.L;
  pp.C = 0;
  pp.a = geo.a;
  pp.tma = 1;
  pp.tiling = 1;
  pp.count = 1;
  pp.err = ctx->dev_err.as<unsigned>();
  pp.wait_ns = 5000000ull;
  pp.test_stall = 1;
  PassWalk& W = pp.walk[0];
  W.active = 1;
  W.psi = base;
  W.bin = W.bout = base + N * 8;
  W.part = base + 2 * N * 8;
  W.hp = reinterpret_cast<const float*>(base + 3 * N * 8);
  W.coef = ctx->tune_coef.as<float>();
  W.norm_part = ctx->norm_part.as<double>();
  W.gamma = 1.0f;
  W.scale = 64.0f;
  W.r = 4;
  W.K = 40;
  CK(launch_pass(0, pp, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return take_device_error(ctx);
}

mqw_status mqw_grid_shape_for(mqw_ctx* ctx, int precision, int n,
                              mqw_grid_shape* out) {
  mqw_status st = check_ctx(ctx);
  if (st != MQW_OK) return st;
  if (!out || (precision != MQW_FP32 && precision != MQW_FP64) || n < 6 || n > kMaxN)
    return fail(ctx, MQW_ERR_INVALID, "mqw_grid_shape_for: bad arguments");
  GridShape want, gs;
  want.group = want.lanes = 0;  // nothing fixed
  st = tune_grid(ctx, precision, n, want, &gs);
  if (st != MQW_OK) return st;
  const PassGeomHost geo = pass_geom(precision, n, gs.lmax, gs.threads, gs.lane_smem > 0, std::max(0, gs.tma), gs.cl < 0 ? 0 : 1);
  out->tile_log = geo.L;
  out->threads = geo.threads ? geo.threads : 512;
  out->lane_smem = geo.lane_smem;
  out->tma = geo.tma;
  out->cluster_log = geo.C;
  out->global_axes = geo.nu;
  out->group = gs.group;
  out->lanes = gs.lanes;
  out->us_per_walk_pass = gs.us;
  return MQW_OK;
}

mqw_status mqw_pass_timing(mqw_ctx* ctx, int precision, int n, int reps,
                           double* us_per_launch, double* us_per_walk_pass,
                           int* walks_per_launch, int* lanes) {
  mqw_status st = check_ctx(ctx);
  if (st != MQW_OK) return st;
  if ((precision != MQW_FP32 && precision != MQW_FP64) || n < 6 || n > kMaxN || reps < 1 ||
      reps > 100000)
    return fail(ctx, MQW_ERR_INVALID, "mqw_pass_timing: bad arguments");
  GridShape want, gs;
  want.group = want.lanes = 0;
  st = tune_grid(ctx, precision, n, want, &gs);
  if (st != MQW_OK) return st;
  double us = 0.0;
  st = time_grid_config(ctx, precision, n, gs.lmax, gs.group, gs.lanes, gs.threads,
                        gs.lane_smem > 0, std::max(0, gs.tma), &us, reps, gs.cl < 0 ? 0 : 1);
  if (st != MQW_OK) return st;
  // time_grid_config returns the elapsed time per walk-pass: launches carry
  // `group` walks and `lanes` launches are in flight at a time.
  if (us_per_walk_pass) *us_per_walk_pass = us;
  if (us_per_launch) *us_per_launch = us * gs.group;
  if (walks_per_launch) *walks_per_launch = gs.group;
  if (lanes) *lanes = gs.lanes;
  return MQW_OK;
}

mqw_status mqw_chain_pass_timing(mqw_ctx* ctx, int n, int reps, double* us_per_launch,
                                 int* lanes_out, int* tile_log, int* chains_per_launch) {
  mqw_status st = check_ctx(ctx);
  if (st != MQW_OK) return st;
  if (n < 6 || n > kMaxN || reps < 1 || reps > 100000)
    return fail(ctx, MQW_ERR_INVALID, "mqw_chain_pass_timing: bad arguments");
  // The plan's shape for this n: its tuned tile; the product-basis chains'
  // launches (B chains per per-term launch where the plan batches them:
  // 8 at n = 17-18, MQW_CHAIN_BATCH if set; one elsewhere) and their lanes
  // (batches: the tuned walk lanes; one chain per launch: kChainLanes from
  // n = 19, MQW_CHAIN_LANES if set, else the tuned walk lanes).
  GridShape want, gs;
  want.group = want.lanes = 0;
  st = tune_grid(ctx, MQW_FP32, n, want, &gs);
  if (st != MQW_OK) return st;
  const PassGeomHost geo = pass_geom(0, n, gs.lmax, gs.threads, gs.lane_smem > 0,
                                     std::max(0, gs.tma), gs.cl < 0 ? 0 : 1);
  if (geo.C != 0)
    return fail(ctx, MQW_ERR_UNSUPPORTED, "mqw_chain_pass_timing: cluster-spanning tiles");
  const char* be = getenv("MQW_CHAIN_BATCH");
  const int B = chain_tile_log(0, n) > 0
                    ? 1
                    : std::min(kMaxChainBatch, std::max(1, be ? atoi(be) : (n <= 18 ? 8 : 1)));
  const char* env = getenv("MQW_CHAIN_LANES");
  int lanes = B > 1 ? gs.lanes : env ? atoi(env) : (n >= 19 ? kChainLanes : gs.lanes);
  lanes = std::max(1, std::min(lanes, kMaxStreams - 1));
  const size_t N = (size_t)1 << n;
  // per chain: its two output slots (each 2N: pass j writes b_r at
  // out_base[j & 1] + (j >> 1) N) and P, or for a single-chain launch two
  // vectors (alternating b_{r+1} / b_r) and P; then D
  const size_t per_chain = B > 1 ? 5 * N : 3 * N;
  CK(ctx->ensure_lanes(lanes));
  const size_t bytes = ((size_t)lanes * B * per_chain + N) * sizeof(float);
  CK(ctx->grow(ctx->state, bytes));
  cudaStream_t s0 = ctx->stream;
  CK(cudaMemsetAsync(ctx->state.p, 0, bytes, s0));
  float* base = ctx->state.as<float>();
  const float* hp = base + (size_t)lanes * B * per_chain;
  auto issue = [&](int j, int lane) -> cudaError_t {
    cudaStream_t st = lane == 0 ? s0 : ctx->lane_stream[lane];
    if (B > 1) {
      // passes j = 2, 3, 2, 3, ... of a batch (both tilings, b_{r+1} read
      // from the other slot), as the plan's per-term batch launches
      RealChainBatch rb{};
      RealChainParams& rp = rb.p;
      rp.n = n;
      rp.L = geo.L;
      rp.a = geo.a;
      rp.start_uniform = 1;
      rp.psi0 = 1.0f;
      rp.hp = hp;
      rp.gamma = 1.0f;
      rp.scale = 64.0f;
      rp.K = 4;
      rp.R = 4;
      rp.out_stride = (long long)N;
      rb.chains = B;
      for (int c = 0; c < B; c++) {
        float* v = base + ((size_t)lane * B + c) * per_chain;
        rb.chain[c] = RealChainDesc{nullptr, v + 4 * N, {v, v + 2 * N}};
      }
      return launch_real_batch(rb, 2 + (j & 1), st);
    }
    float* v = base + (size_t)lane * 3 * N;
    RealChainParams rp{};
    rp.n = n;
    rp.L = geo.L;
    rp.a = geo.a;
    rp.tiling = (j & 1) ? 2 : 1;
    rp.first = 0;
    rp.bin = v + (size_t)((j + 1) & 1) * N;
    rp.bout = v + (size_t)(j & 1) * N;
    rp.part = v + 2 * N;
    rp.start_uniform = 1;
    rp.hp = hp;
    rp.gamma = 1.0f;
    rp.scale = 64.0f;
    return launch_real_pass(rp, st);
  };
  CK(ctx->fork(s0, lanes));
  for (int j = 0; j < 4; j++)
    for (int l = 0; l < lanes; l++) CK(issue(j, l));
  CK(ctx->join(s0, lanes));
  // The passes as the plan runs them: a CUDA graph of `reps` passes per
  // lane (forked from and joined into the stream like the plan's lanes),
  // replayed once untimed and once between the events.
  CK(cudaStreamSynchronize(s0));
  cudaGraph_t graph = nullptr;
  CK(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
  cudaError_t ce = ctx->fork(s0, lanes);
  for (int j = 0; j < reps && ce == cudaSuccess; j++)
    for (int l = 0; l < lanes && ce == cudaSuccess; l++) ce = issue(j, l);
  if (ce == cudaSuccess) ce = ctx->join(s0, lanes);
  const cudaError_t ee = cudaStreamEndCapture(s0, &graph);
  if (ce != cudaSuccess || ee != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    CK(ce != cudaSuccess ? ce : ee);
  }
  cudaGraphExec_t gexec = nullptr;
  const cudaError_t ie = cudaGraphInstantiate(&gexec, graph, 0);
  cudaGraphDestroy(graph);
  CK(ie);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaGraphLaunch(gexec, s0);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  if (e == cudaSuccess) e = cudaEventRecord(e0, s0);
  if (e == cudaSuccess) e = cudaGraphLaunch(gexec, s0);
  if (e == cudaSuccess) e = cudaEventRecord(e1, s0);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  float ms = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaGraphExecDestroy(gexec);
  CK(e);
  st = take_device_error(ctx);
  if (st != MQW_OK) return st;
  if (us_per_launch) *us_per_launch = 1000.0 * ms / ((double)reps * lanes);
  if (lanes_out) *lanes_out = lanes;
  if (tile_log) *tile_log = geo.L;
  if (chains_per_launch) *chains_per_launch = B;
  return MQW_OK;
}

mqw_status mqw_plan_stats(const mqw_plan* plan, mqw_run_stats* stats) {
  if (!plan || !stats) return MQW_ERR_INVALID;
  *stats = plan->stats;
  stats->h2d_bytes += plan->create_h2d;
  if (plan->timed) {
    float ms = 0.0f;
    if (cudaEventSynchronize(plan->ev1) == cudaSuccess &&
        cudaEventElapsedTime(&ms, plan->ev0, plan->ev1) == cudaSuccess)
      stats->kernel_ms = ms;
    else
      (void)cudaGetLastError();  // leave no pending error behind
  }
  return MQW_OK;
}

void mqw_plan_destroy(mqw_plan* plan) {
  if (!plan) return;
  if (plan->ctx) cudaSetDevice(plan->ctx->device);
  delete plan;
}

mqw_status mqw_run_problems(mqw_ctx* ctx, int n, int m, const double* raw,
                            int count, const mqw_options* opt, double* p_out,
                            float* total_t_out, uint32_t* e_loc_out,
                            mqw_run_stats* stats) {
  mqw_status s = check_ctx(ctx);
  if (s != MQW_OK) return s;
  if (count < 0 || !raw || (count > 0 && !p_out))
    return fail(ctx, MQW_ERR_INVALID, "run_problems: bad arguments");
  if (count == 0) return MQW_OK;
  std::vector<int> nv(count, n), mv(count, m);
  mqw_plan* plan = nullptr;
  s = mqw_plan_create(ctx, count, nv.data(), mv.data(), raw, opt, &plan);
  if (s != MQW_OK) return s;
  s = mqw_plan_execute(plan, nullptr);
  if (s == MQW_OK) s = mqw_plan_results(plan, p_out, total_t_out, e_loc_out, nullptr);
  if (s == MQW_OK && stats) mqw_plan_stats(plan, stats);
  mqw_plan_destroy(plan);
  return s;
}

mqw_status mqw_build_diag(mqw_ctx* ctx, int n, const double* raw, float* hp,
                          double* energies, mqw_diag_info* info) {
  mqw_status s = check_ctx(ctx);
  if (s != MQW_OK) return s;
  if (n < 1 || n > MQW_MAX_N || !raw)
    return fail(ctx, MQW_ERR_INVALID, "build_diag: bad arguments");
  const size_t N = (size_t)1 << n;
  DevMem d_raw, d_hp, d_e, d_out, d_scr;
  CK(d_raw.ensure(params_per(n) * sizeof(double)));
  CK(d_hp.ensure(N * sizeof(float)));
  if (energies) CK(d_e.ensure(N * sizeof(double)));
  CK(d_out.ensure(sizeof(DiagOut)));
  CK(d_scr.ensure(diag_scratch_bytes(n, 1)));
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(d_raw.p, raw, params_per(n) * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(launch_diag(n, 1, d_raw.as<double>(), d_hp.as<float>(),
                 energies ? d_e.as<double>() : nullptr, d_out.as<DiagOut>(), d_scr.p, st));
  DiagOut o;
  CK(cudaMemcpyAsync(&o, d_out.p, sizeof o, cudaMemcpyDeviceToHost, st));
  if (hp) CK(cudaMemcpyAsync(hp, d_hp.p, N * sizeof(float), cudaMemcpyDeviceToHost, st));
  if (energies) CK(cudaMemcpyAsync(energies, d_e.p, N * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (info) {
    info->e0 = o.e0;
    info->emax = o.emax;
    info->mid = o.mid;
    info->e_abs = o.e_abs;
    info->e_loc = o.e_loc;
  }
  return MQW_OK;
}

mqw_status mqw_diag_moments(mqw_ctx* ctx, int n, const double* raw, double* moments,
                            mqw_diag_info* info) {
  mqw_status s = check_ctx(ctx);
  if (s != MQW_OK) return s;
  if (n < 1 || n > MQW_MAX_N || !raw || !moments)
    return fail(ctx, MQW_ERR_INVALID, "diag_moments: bad arguments");
  const size_t N = (size_t)1 << n;
  DevMem d_raw, d_hp, d_out, d_scr, d_mom;
  CK(d_raw.ensure(params_per(n) * sizeof(double)));
  CK(d_hp.ensure(N * sizeof(float)));
  CK(d_out.ensure(sizeof(DiagOut)));
  CK(d_scr.ensure(diag_scratch_bytes(n, 1)));
  CK(d_mom.ensure(moments_scratch_bytes()));
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(d_raw.p, raw, params_per(n) * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(launch_diag(n, 1, d_raw.as<double>(), d_hp.as<float>(), nullptr, d_out.as<DiagOut>(),
                 d_scr.p, st));
  CK(launch_moments(n, d_hp.as<float>(), d_mom.p, st));
  DiagOut o;
  CK(cudaMemcpyAsync(&o, d_out.p, sizeof o, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(moments, d_mom.as<char>() + moments_scratch_bytes() - 4 * sizeof(double),
                     4 * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (info) {
    info->e0 = o.e0;
    info->emax = o.emax;
    info->mid = o.mid;
    info->e_abs = o.e_abs;
    info->e_loc = o.e_loc;
  }
  return MQW_OK;
}

mqw_status mqw_cheb_coeffs(mqw_ctx* ctx, int count, const double* s_in,
                           double tol, int max_k, float* coeffs, int* degrees) {
  mqw_status s = check_ctx(ctx);
  if (s != MQW_OK) return s;
  if (count < 0 || max_k < 1 || (count > 0 && (!s_in || !coeffs || !degrees)))
    return fail(ctx, MQW_ERR_INVALID, "cheb_coeffs: bad arguments");
  if (count == 0) return MQW_OK;
  DevMem d_s, d_c, d_k;
  CK(d_s.ensure(count * sizeof(double)));
  CK(d_c.ensure((size_t)count * max_k * sizeof(float)));
  CK(d_k.ensure(count * sizeof(int)));
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(d_s.p, s_in, count * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(d_c.p, 0, (size_t)count * max_k * sizeof(float), st));
  CK(launch_cheb_from_s(d_s.as<double>(), count, tol, max_k, d_c.as<float>(),
                        d_k.as<int>(), st));
  CK(cudaMemcpyAsync(coeffs, d_c.p, (size_t)count * max_k * sizeof(float),
                     cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(degrees, d_k.p, count * sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return MQW_OK;
}

mqw_status mqw_clenshaw(mqw_ctx* ctx, int precision, int n, int K,
                        const float* coeffs, const float* hp, float gamma,
                        float scale, const void* psi, void* out) {
  mqw_status s = check_ctx(ctx);
  if (s != MQW_OK) return s;
  if ((precision != MQW_FP32 && precision != MQW_FP64 && precision != MQW_FP32_COMPENSATED) ||
      n < 6 || n > MQW_MAX_N || K < 1 || !coeffs || !hp || !psi || !out)
    return fail(ctx, MQW_ERR_INVALID, "clenshaw: bad arguments (n must be in 6..30)");
  const int comp = precision == MQW_FP32_COMPENSATED;
  if (comp) precision = MQW_FP32;  // FP32 storage, compensated partner sums
  const size_t N = (size_t)1 << n;
  const size_t amp = precision == 0 ? 8 : 16;
  // Single-CTA tiles: where the widest tile leaves axes to neither tiling
  // they are read from global memory (tiles spread over a cluster measured
  // slower).
  const PassGeomHost geo = pass_geom(precision, n, 0, 0, 0, 0, 0);
  const int tiles = (int)(N >> geo.L);
  // Small n: all K terms in one chain launch (in place, nothing read from
  // global memory).
  const int chain_L = comp ? 0 : chain_tile_log(precision, n);
  DevMem d_st, d_hp, d_c, d_np;
  CK(d_st.ensure(4 * N * amp));
  CK(d_hp.ensure(N * sizeof(float)));
  CK(d_c.ensure(K * sizeof(float)));
  CK(d_np.ensure(tiles * sizeof(double)));
  cudaStream_t st = ctx->stream;
  char* b = d_st.as<char>();
  void* P0 = b;
  void* X = b + N * amp;
  void* Y = b + 2 * N * amp;
  void* Pt = b + 3 * N * amp;
  CK(cudaMemcpyAsync(P0, psi, N * amp, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_hp.p, hp, N * sizeof(float), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_c.p, coeffs, K * sizeof(float), cudaMemcpyHostToDevice, st));
  if (chain_L) {
    PassParams pp{};
    pp.n = n;
    pp.L = chain_L;
    pp.a = geo.a;
    pp.tiling = 1;
    pp.err = ctx->dev_err.as<unsigned>();
    pp.count = 1;
    PassWalk& W = pp.walk[0];
    W.active = 1;
    W.bin = W.bout = X;  // b_0 ends in X, as with one launch per term
    W.part = Pt;
    W.psi = P0;
    W.hp = d_hp.as<float>();
    W.coef = d_c.as<float>();
    W.norm_part = d_np.as<double>();  // N >> chain_L <= tiles partials
    W.gamma = gamma;
    W.scale = scale;
    W.K = K;
    CK(launch_pass_chain(precision, pp, st));
  }
  for (int r = chain_L ? -1 : K - 1; r >= 0; r--) {
    PassParams pp{};
    pp.n = n;
    pp.L = geo.L;
    pp.C = geo.C;
    pp.threads = geo.threads;
    pp.lane_smem = geo.lane_smem;
    pp.tma = geo.tma;
    pp.err = ctx->dev_err.as<unsigned>();
    pp.a = geo.a;
    pp.tiling = (r & 1) ? 2 : 1;
    pp.count = 1;
    PassWalk& W = pp.walk[0];
    W.active = 1;
    W.bin = (r & 1) ? X : Y;
    W.bout = (r & 1) ? Y : X;
    W.part = Pt;
    W.psi = P0;
    W.hp = d_hp.as<float>();
    W.coef = d_c.as<float>();
    W.kappa = nullptr;
    W.norm_part = d_np.as<double>();
    W.gamma = gamma;
    W.scale = scale;
    W.r = r;
    W.K = K;
    W.psi_uniform = 0;
    pp.comp = comp;
    CK(launch_pass(precision, pp, st));
  }
  CK(cudaMemcpyAsync(out, X, N * amp, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return MQW_OK;
}

mqw_status mqw_multiqw(mqw_ctx* ctx, int n, int m, const char* filename,
                       long long start, long long problems,
                       const char* out_dir, int print) {
  mqw_status s = check_ctx(ctx);
  if (s != MQW_OK) return s;
  if (!filename || n < 1 || n > MQW_MAX_N || m < 1 || m > MQW_MAX_M || start < 0 ||
      problems < 0 || problems > 0x7fffffffll)  // run_problems takes an int count
    return fail(ctx, MQW_ERR_INVALID, "multiqw: bad arguments");
  std::vector<double> raw((size_t)problems * params_per(n));
  s = mqw_read_instances(filename, n, start, problems, raw.data());
  if (s != MQW_OK)
    return fail(ctx, s, "cannot read %lld instances of n=%d from '%s' at instance %lld",
                problems, n, filename, start);
  std::vector<double> p(problems);
  std::vector<float> tt(problems);
  if (problems > 0) {
    s = mqw_run_problems(ctx, n, m, raw.data(), (int)problems, nullptr, p.data(),
                         tt.data(), nullptr, nullptr);
    if (s != MQW_OK) return s;
  }
  std::vector<float> res(problems);
  for (long long i = 0; i < problems; i++) {
    res[i] = (float)p[i];
    if (print) printf("%g %g\n", tt[i], res[i]);  // MultiQW.cpp:423, 455
  }
  if (print) fflush(stdout);
  char name[64];
  snprintf(name, sizeof name, "output_%d_%d", n, m);  // MultiQW.cpp:265
  std::string path = out_dir && *out_dir ? std::string(out_dir) + "/" + name : name;
  FILE* f = fopen(path.c_str(), "ab");  // ios::app, MultiQW.cpp:266
  if (!f) return fail(ctx, MQW_ERR_IO, "cannot open '%s' for append", path.c_str());
  const size_t w = problems ? fwrite(res.data(), sizeof(float), problems, f) : 0;
  fclose(f);
  if (w != (size_t)problems) return fail(ctx, MQW_ERR_IO, "short write to '%s'", path.c_str());
  return MQW_OK;
}

}  // extern "C"
