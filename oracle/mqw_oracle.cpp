// ORACLE — test infrastructure only.
//
// A CPU restatement of the reference program MultiQW.cpp (Asa-Hopkins/
// MultiStageQW), used as the checker for the CUDA path. Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg may load this
// library; the product (multistageqw_b200, include/mqw.h, the MultiQW binary)
// never links, loads or calls it.
//
// Parity status: PARTLY PINNED.
//  * Pinned against the reference's own code: the partial build in
//    oracle/_ref (MultiQW.cpp:16-173 compiled from the reference source with a
//    project-written VCL2 shim) supplies the reference's inverse-normal helper
//    my_normcdfinvf and its FP32 Clenshaw_step; tests compare this file's
//    restatements with them.
//  * Pinned against mathematics: brute-force energies, dense matrix
//    exponentials (scipy.linalg.expm) and Bessel values (scipy.special.jv).
//  * Unpinned: the Chebyshev coefficient routine (ApproxTools
//    Chebyshev<double>::RCF_odd_even, MultiQW.cpp:440) is an empty submodule
//    in the reference snapshot. This oracle (and the CUDA path) use the
//    Jacobi–Anger coefficients of exp(i s x) with the tail-sum degree rule
//    below. Eigen's vectorised reduction orders (J.sum(), norms) are restated
//    as sequential sums; they move results at the 1e-7 level only.
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=fast, the same contraction
// policy g++ applies to the reference by default).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

namespace {

constexpr double kPi = 3.1415926535897932384626;  // MultiQW.cpp:11
constexpr int kSamples = 100;                     // MultiQW.cpp:257
constexpr unsigned long kSeed = 29552825458725UL; // MultiQW.cpp:387
constexpr double kChebTol = 1e-6;                 // MultiQW.cpp:440

// Instance layout, MultiQW.cpp:306-323: the first n(n-1)/2 doubles are J(i,j)
// for i = 1..n-1, j = 0..i-1 (in that loop order); then n doubles of h.
// J is cast to float, symmetrised and halved: Jsym(i,j) = Jsym(j,i) =
// float(raw)/2 (an exact halving).
void load_instance(int n, const double* raw, float* J, float* h) {
  std::fill(J, J + n * n, 0.0f);
  int k = 0;
  for (int i = 1; i < n; i++)
    for (int j = 0; j < i; j++) {
      float v = (float)raw[k++];
      J[i * n + j] = v / 2;
      J[j * n + i] = v / 2;
    }
  for (int i = 0; i < n; i++) h[i] = (float)raw[n * (n - 1) / 2 + i];
}

// Upper-tail standard-normal quantile Q^{-1}(p) = Phi^{-1}(1 - p), returned
// as float. The reference evaluates this as my_normcdfinvf (MultiQW.cpp:39-86,
// a float polynomial approximation with <= 4.1 ulp error, which returns
// +Phi^{-1}(1-p)). Here it is solved to double accuracy by Halley iteration on
// 0.5*erfc(x/sqrt(2)) = p, then rounded once.
float inv_norm_upper(float pf) {
  double p = pf;
  if (!(p > 0.0) || !(p < 1.0)) return p <= 0.0 ? INFINITY : -INFINITY;
  if (p == 0.5) return 0.0f;
  double x;
  if (p < 0.5) {
    double t = std::sqrt(-2.0 * std::log(p));
    x = t - (2.515517 + t * (0.802853 + t * 0.010328)) /
                (1.0 + t * (1.432788 + t * (0.189269 + t * 0.001308)));
  } else {
    double t = std::sqrt(-2.0 * std::log(1.0 - p));
    x = -(t - (2.515517 + t * (0.802853 + t * 0.010328)) /
                  (1.0 + t * (1.432788 + t * (0.189269 + t * 0.001308))));
  }
  const double isq2 = 0.70710678118654752440;
  const double isq2pi = 0.39894228040143267794;
  for (int it = 0; it < 60; it++) {
    double q = 0.5 * std::erfc(x * isq2);
    double phi = isq2pi * std::exp(-0.5 * x * x);
    double f = q - p;               // f(x) = Q(x) - p, f' = -phi, f'' = x*phi
    double d = f / phi;             // Newton step is +d
    double step = d / (1.0 - 0.5 * x * d);  // Halley
    x += step;
    if (std::fabs(step) <= 1e-16 * std::max(1.0, std::fabs(x))) break;
  }
  return (float)x;
}

// The inverse normal the schedule uses: this restatement's (default) or an
// external one with the reference's my_normcdfinvf signature (float ->
// float) — the reference's own, from the partial build in oracle/_ref — so
// that a whole run can be driven by the reference's schedule arithmetic.
typedef float (*InvNormFn)(float);
InvNormFn g_inv_norm = nullptr;
// Not inlined: the schedule then sees an opaque call either way, as the
// CUDA path's host code does (its inverse normal lives in another
// translation unit), so the compiler fuses the same multiply-add around it.
__attribute__((noinline)) float sched_inv_norm(float p) {
  return g_inv_norm ? g_inv_norm(p) : inv_norm_upper(p);
}

struct DiagInfo {
  double e0, emax, mid;
  float e_abs;
  uint32_t e_loc;
};

// Ising energies with the reference's arithmetic, MultiQW.cpp:325-362.
// Starting from all spins -1 (state 0), a Gray-code sweep flips one spin per
// step. Each increment 4*sum_k J(f,k)*state(f,k) - 2*h(f)*state(f,f) is a
// float (the inner sum is sequential in k), accumulated into a double E.
// state(f,k) = s_f*s_k for k != f and state(f,f) = -s_f, exactly as the
// reference's row/column/diagonal sign flips leave it. E_0 / E_loc / E_max
// use strict comparisons in Gray order (the first minimum wins).
void energies_ref(int n, const float* J, const float* h, double* E_out,
                  DiagInfo* info) {
  const uint32_t N = 1u << n;
  float sumJ = 0.0f, sumh = 0.0f;
  for (int i = 0; i < n * n; i++) sumJ += J[i];
  for (int i = 0; i < n; i++) sumh += h[i];
  double E = (double)(float)(sumJ - sumh);
  E_out[0] = E;
  double e0 = E, emax = E;
  uint32_t eloc = 0;
  std::vector<float> st(n * n, 1.0f);
  for (uint32_t i = 1; i < N; i++) {
    int f = __builtin_ctz(i);
    for (int k = 0; k < n; k++) st[f * n + k] *= -1.0f;
    for (int k = 0; k < n; k++) st[k * n + f] *= -1.0f;
    st[f * n + f] *= -1.0f;
    float s = J[f * n + 0] * st[f * n + 0];
    for (int k = 1; k < n; k++) s += J[f * n + k] * st[f * n + k];
    float d = 4 * s - 2 * h[f] * st[f * n + f];
    E += d;
    uint32_t z = i ^ (i >> 1);
    E_out[z] = E;
    if (E < e0) { e0 = E; eloc = z; }
    if (E > emax) emax = E;
  }
  info->e0 = e0;
  info->emax = emax;
  info->mid = (emax + e0) / 2;
  info->e_abs = (float)((emax - e0) / 2);
  info->e_loc = eloc;
}

// H_P as the reference stores it: float(E) minus float((E_max+E_0)/2)
// (MultiQW.cpp:346, 361; Eigen converts the double scalar to float first).
void shifted_diag(int n, const double* E, const DiagInfo& info, float* hp) {
  const uint32_t N = 1u << n;
  const float midf = (float)info.mid;
  for (uint32_t z = 0; z < N; z++) hp[z] = (float)E[z] - midf;
}

// Per-stage hopping rates and time samples, MultiQW.cpp:365-422.
// Expression shapes follow the reference so that g++ applies the same
// float/double promotions (and, with its default -ffp-contract=fast, the same
// multiply-add fusions).
void schedule(int n, int m, const float* J, const float* h, float* gammas,
              float* short_ts, float* times /* m * kSamples */,
              float* total_t_out) {
  const unsigned N = 1u << n;
  float e_m = 0.577215664901532860;
  float e = 2.718281828459045;
  float b = sched_inv_norm(1 / (float)N);
  float a = (1 - e_m) * b + e_m * sched_inv_norm(1 / (e * N));
  float JJ = 0.0f, hh = 0.0f;
  for (int i = 0; i < n * n; i++) JJ += J[i] * J[i];
  for (int i = 0; i < n; i++) hh += h[i] * h[i];
  float HP2 = 2 * JJ + hh;
  std::mt19937 gen(kSeed);
  for (int i = 0; i < m; i++)
    gammas[i] = a * std::sqrt(HP2) / std::tan(kPi * (i + 1) / (2 * m + 2)) / n;
  float total_t = 0;
  float delta2 = 16 * JJ + 4 * hh;
  for (int i = 0; i < m; i++) {
    float last_denom = std::sqrt(2 / kPi) * gammas[i] * std::sqrt(n * delta2);
    float gamma_last =
        (i == 0) ? 1 : gammas[i - 1] / std::sqrt(1 + gammas[i - 1] * gammas[i - 1]);
    float gamma_next =
        (i + 1 == m) ? 0 : gammas[i + 1] / std::sqrt(1 + gammas[i + 1] * gammas[i + 1]);
    float dH = gamma_last - gamma_next;
    float first_t = std::sqrt(4 * (unsigned)n * dH / delta2);
    float last_t = std::sqrt(2 * (unsigned)n * dH / last_denom);
    float short_t = (i == 0) ? first_t : std::max(first_t, last_t);
    std::uniform_real_distribution<float> rand_t(short_t, 2 * short_t);
    total_t += short_t;
    short_ts[i] = short_t;
    for (int j = 0; j < kSamples; j++) times[i * kSamples + j] = rand_t(gen);
  }
  // Single stage: sorted times become successive differences and the walk is
  // evolved cumulatively (MultiQW.cpp:426-430).
  if (m == 1) {
    std::sort(times, times + kSamples);
    for (int j = kSamples - 1; j >= 1; j--) times[j] -= times[j - 1];
  }
  *total_t_out = total_t;
}

// Chebyshev coefficients of exp(i s x) on [-1, 1] (Jacobi–Anger):
// c_0 = J_0(s), c_k = 2 (-1)^floor(k/2) J_k(s); even-k terms are the real
// (cos) part and odd-k terms the imaginary (sin) part, which is how the
// reference applies the coefficients of sin(sx)+cos(sx) (MultiQW.cpp:206-221).
// Degree rule: the smallest K >= 1 with sum_{k>=K} |c_k| <= tol, so the
// truncation error is at most tol on [-1, 1].
// Bessel values: Miller's backward recurrence f_{k-1} = (2k/s) f_k - f_{k+1}
// from f_{top+1} = 0, f_top = 1e-300, top = ceil(s) + 40 + 4*isqrt(ceil(s))
// (made even), normalised by J_0 + 2 sum_{k>=1} J_2k = 1 with the sum taken
// from the top down. For s >= 1e-8 the growth from f_top to the peak stays
// below 1e600, so no rescaling is needed; below 1e-8, c = {1}.
int cheb_coeffs(double s, double tol, double* c, int max_k) {
  s = std::fabs(s);
  if (s < 1e-8) {
    c[0] = 1.0;
    return 1;
  }
  const int cs = (int)std::ceil(s);
  int r = 0;
  while ((r + 1) * (r + 1) <= cs) r++;
  int top = cs + 40 + 4 * r;
  top += top & 1;
  std::vector<double> f(top + 2, 0.0);
  f[top + 1] = 0.0;
  f[top] = 1e-300;
  for (int k = top; k >= 1; k--) f[k - 1] = std::fma(2.0 * k / s, f[k], -f[k + 1]);
  double norm = 0.0;
  for (int k = top; k >= 2; k -= 2) norm += 2.0 * f[k];
  norm += f[0];
  double tail = 0.0;
  int K = 1;
  for (int k = top; k >= 1; k--) {
    tail += 2.0 * std::fabs(f[k] / norm);
    if (tail > tol) {
      K = k + 1;
      break;
    }
  }
  if (K > max_k) return -K;
  for (int k = 0; k < K; k++) {
    double v = f[k] / norm;
    if (k > 0) v *= ((k / 2) & 1) ? -2.0 : 2.0;
    c[k] = v;
  }
  return K;
}

// One FP32 Clenshaw step on one real half, in the reference's operation
// order (MultiQW.cpp:88-173): b2 <- coef*psi + 2*((hp - gamma*sum_q X_q)/scale)
// b1 - b2, computed as new_scale*(b2/(-new_scale) - b1*hp/gamma + X-sums)
// + psi*coef with new_scale = -2*gamma/scale. Axis order: 0..3, then
// 15..n-1 (pass 1), then 4..14 (pass 2). Valid for any n >= 1 (the reference
// itself needs n >= 4). The two multiply-adds are fused exactly where g++
// -O3 fuses them in the reference's Vec16f code (checked bit-for-bit against
// the partial build in oracle/_ref): b2*(-1/new_scale) - b1*hp/gamma in pass 1
// and b*new_scale + psi*coef in pass 2.
void clenshaw_step_f32(const float* b1, float* b2, const float* hp,
                       const float* psi, int n, float scale, float gamma,
                       float coef) {
  const uint32_t N = 1u << n;
  const int max_cache = 15;
  float new_scale = -2.0f * gamma / scale;
  float new_scale_inv = 1.0f / new_scale;
  for (uint32_t i = 0; i < N; i++) {
    const float x = b1[i] * hp[i] / gamma;
    float b = std::fma(b2[i], -new_scale_inv, -x);
    for (int q = 0; q < std::min(n, 4); q++) b += b1[i ^ (1u << q)];
    if (n > max_cache)
      for (int q = max_cache; q < n; q++) b += b1[i ^ (1u << q)];
    b2[i] = b;
  }
  int end = std::min(n, max_cache);
  for (uint32_t i = 0; i < N; i++) {
    float b = b2[i];
    for (int q = 4; q < end; q++) b += b1[i ^ (1u << q)];
    if (coef != 0)
      b = std::fma(b, new_scale, psi[i] * coef);
    else
      b *= new_scale;
    b2[i] = b;
  }
}

// One FP64 Clenshaw step (same inputs, double arithmetic):
// b2 <- coef*psi + (2/scale)*(hp*b1 - gamma*sum_q b1[i^2^q]) - b2.
void clenshaw_step_f64(const double* b1, double* b2, const double* hp,
                       const double* psi, int n, double scale, double gamma,
                       double coef) {
  const uint32_t N = 1u << n;
  const double alpha = 2.0 / scale;
  for (uint32_t i = 0; i < N; i++) {
    double acc = 0.0;
    for (int q = 0; q < n; q++) acc += b1[i ^ (1u << q)];
    b2[i] = coef * psi[i] + alpha * (hp[i] * b1[i] - gamma * acc) - b2[i];
  }
}

// Clenshaw evaluation of sum_k c_k T_k(H~) psi, H~ = (hp - gamma*sum X)/scale,
// with c_k real for even k and imaginary for odd k (MultiQW.cpp:177-236).
// State vectors are planar: [Re(0..N-1) | Im(0..N-1)].
template <typename T, typename StepFn>
void clenshaw(int n, int K, const float* coeffs, const T* hp, float gamma,
              float scale, const T* psi, T* out, bool psi_real, StepFn step) {
  const size_t N = size_t(1) << n;
  std::vector<T> b1(2 * N, T(0)), b2(2 * N, T(0));
  const T im_coef = psi_real ? T(0) : T(1);
  bool first = true;
  for (int r = K - 1; r > 0; --r) {
    T c = (T)coeffs[r];
    if (!first) {
      if (r & 1) {
        step(b1.data(), b2.data(), hp, psi + N, n, (T)scale, (T)gamma, -im_coef * c);
        step(b1.data() + N, b2.data() + N, hp, psi, n, (T)scale, (T)gamma, c);
      } else {
        step(b1.data(), b2.data(), hp, psi, n, (T)scale, (T)gamma, c);
        step(b1.data() + N, b2.data() + N, hp, psi + N, n, (T)scale, (T)gamma, im_coef * c);
      }
    } else {
      if (r & 1) {
        if (!psi_real)
          for (size_t i = 0; i < N; i++) b2[i] -= psi[N + i] * c;
        for (size_t i = 0; i < N; i++) b2[N + i] += psi[i] * c;
      } else {
        if (!psi_real)
          for (size_t i = 0; i < N; i++) b2[N + i] += psi[N + i] * c;
        for (size_t i = 0; i < N; i++) b2[i] += psi[i] * c;
      }
    }
    first = false;
    std::swap(b1, b2);
  }
  T c0 = (T)coeffs[0];
  step(b1.data(), b2.data(), hp, psi, n, (T)(2.0 * scale), (T)gamma, c0);
  step(b1.data() + N, b2.data() + N, hp, psi + N, n, (T)(2.0 * scale), (T)gamma, im_coef * c0);
  std::copy(b2.begin(), b2.end(), out);
}

// An external FP32 step with the reference's Clenshaw_step signature
// (MultiQW.cpp:88); used to drive the reference's own hot loop from the
// partial build in oracle/_ref.
typedef void (*ext_step_fn)(float*, float*, float*, float*, unsigned, float,
                            float, float);

struct StepF32 {
  ext_step_fn ext = nullptr;
  void operator()(const float* b1, float* b2, const float* hp, const float* psi,
                  int n, float scale, float gamma, float coef) const {
    if (ext)
      ext(const_cast<float*>(b1), b2, const_cast<float*>(hp),
          const_cast<float*>(psi), (unsigned)n, scale, gamma, coef);
    else
      clenshaw_step_f32(b1, b2, hp, psi, n, scale, gamma, coef);
  }
};
struct StepF64 {
  void operator()(const double* b1, double* b2, const double* hp,
                  const double* psi, int n, double scale, double gamma,
                  double coef) const {
    clenshaw_step_f64(b1, b2, hp, psi, n, scale, gamma, coef);
  }
};

}  // namespace

extern "C" {

struct orc_diag_info {
  double e0, emax, mid;
  float e_abs;
  uint32_t e_loc;
};

int orc_version() { return 1; }

float orc_inv_norm_upper(float p) { return inv_norm_upper(p); }

// Selects the schedule's inverse normal: fn (float -> float, the
// reference's my_normcdfinvf signature), or this restatement's when null.
void orc_set_inv_norm(void* fn) { g_inv_norm = reinterpret_cast<InvNormFn>(fn); }

void orc_load_instance(int n, const double* raw, float* J, float* h) {
  load_instance(n, raw, J, h);
}

// Reference-arithmetic energies (indexed by basis state) and the shifted
// float diagonal H_P. Either output pointer may be null.
int orc_energies_ref(int n, const double* raw, double* E, float* hp,
                     orc_diag_info* info) {
  if (n < 1 || n > 30) return -1;
  std::vector<float> J(n * n), h(n);
  load_instance(n, raw, J.data(), h.data());
  std::vector<double> Ebuf;
  if (!E) {
    Ebuf.resize(size_t(1) << n);
    E = Ebuf.data();
  }
  DiagInfo d;
  energies_ref(n, J.data(), h.data(), E, &d);
  if (hp) shifted_diag(n, E, d, hp);
  if (info) {
    info->e0 = d.e0;
    info->emax = d.emax;
    info->mid = d.mid;
    info->e_abs = d.e_abs;
    info->e_loc = d.e_loc;
  }
  return 0;
}

// Exact FP64 energies of the float-cast couplings and fields:
// E(z) = sum_{i>j} float(raw_ij) s_i s_j + sum_i float(h_i) s_i, s_i = +1 iff
// bit i of z is set.
void orc_energies_exact(int n, const double* raw, double* E) {
  std::vector<float> J(n * n), h(n);
  load_instance(n, raw, J.data(), h.data());
  const uint32_t N = 1u << n;
  for (uint32_t z = 0; z < N; z++) {
    double e = 0.0;
    for (int i = 0; i < n; i++) {
      double si = (z >> i) & 1 ? 1.0 : -1.0;
      e += (double)h[i] * si;
      for (int j = 0; j < i; j++) {
        double sj = (z >> j) & 1 ? 1.0 : -1.0;
        e += 2.0 * (double)J[i * n + j] * si * sj;
      }
    }
    E[z] = e;
  }
}

void orc_schedule(int n, int m, const double* raw, float* gammas,
                  float* short_ts, float* times, float* total_t) {
  std::vector<float> J(n * n), h(n);
  load_instance(n, raw, J.data(), h.data());
  schedule(n, m, J.data(), h.data(), gammas, short_ts, times, total_t);
}

int orc_cheb_coeffs(double s, double tol, double* c, int max_k) {
  return cheb_coeffs(s, tol, c, max_k);
}

void orc_clenshaw_step_f32(const float* b1, float* b2, const float* hp,
                           const float* psi, int n, float scale, float gamma,
                           float coef) {
  clenshaw_step_f32(b1, b2, hp, psi, n, scale, gamma, coef);
}

// One Clenshaw propagation of a planar state. mode 0: FP32 (reference op
// order); mode 1: FP64 with the same float inputs.
void orc_clenshaw_f32_ext(int n, int K, const float* coeffs, const float* hp,
                          float gamma, float scale, const float* psi,
                          float* out, int psi_real, void* ext_step) {
  StepF32 st;
  st.ext = (ext_step_fn)ext_step;
  clenshaw<float>(n, K, coeffs, hp, gamma, scale, psi, out, psi_real != 0, st);
}
void orc_clenshaw_f32(int n, int K, const float* coeffs, const float* hp,
                      float gamma, float scale, const float* psi, float* out,
                      int psi_real) {
  orc_clenshaw_f32_ext(n, K, coeffs, hp, gamma, scale, psi, out, psi_real, nullptr);
}
void orc_clenshaw_f64(int n, int K, const float* coeffs, const double* hp,
                      float gamma, float scale, const double* psi, double* out,
                      int psi_real) {
  clenshaw<double>(n, K, coeffs, hp, gamma, scale, psi, out, psi_real != 0, StepF64());
}

// The whole per-instance pipeline of MultiQW.cpp:296-455 for `count`
// consecutive instances. samples_used <= 100 evaluates the first samples of
// the reference's 100 (the time draws are always the reference's 100 per
// stage). mode 0 = FP32 (reference arithmetic), 1 = FP64 propagation.
// ext_step (mode 0 only, nullable) replaces the FP32 step by an external one
// with the reference's Clenshaw_step signature.
// Outputs per instance: mean ground-state probability, total_t, E_loc and
// the summed Chebyshev degree (work accounting).
// Samples [s_begin, s_end) of each instance; p_out receives the mean over
// them, and psum_out (nullable) their sum. With m == 1 the samples are
// cumulative steps of one walk (MultiQW.cpp:426-430), so s_begin must be 0.
static int run_samples(int n, int m, const double* raw, int count, int s_begin,
                       int samples_used, int mode, double* p_out, double* psum_out,
                       float* total_t_out, uint32_t* e_loc_out, long long* terms_out,
                       void* ext_step) {
  if (n < 1 || n > 30 || m < 1 || count < 0) return -1;
  if (samples_used < 1 || samples_used > kSamples) return -1;
  if (s_begin < 0 || s_begin >= samples_used || (m == 1 && s_begin != 0)) return -1;
  const size_t N = size_t(1) << n;
  const int per = n * (n + 1) / 2;
  std::vector<float> J(n * n), h(n), hp(N), psi(2 * N), out(2 * N);
  std::vector<double> E(N), hpd, psid, outd;
  if (mode == 1) {
    hpd.resize(N);
    psid.resize(2 * N);
    outd.resize(2 * N);
  }
  std::vector<float> gammas(m), short_ts(m), times(m * kSamples);
  std::vector<double> cd(4096);
  std::vector<float> cf(4096);
  const float psi0 = (float)(1 / std::sqrt((double)N));
  for (int p = 0; p < count; p++) {
    const double* r = raw + (size_t)p * per;
    load_instance(n, r, J.data(), h.data());
    DiagInfo d;
    energies_ref(n, J.data(), h.data(), E.data(), &d);
    shifted_diag(n, E.data(), d, hp.data());
    float total_t;
    schedule(n, m, J.data(), h.data(), gammas.data(), short_ts.data(),
             times.data(), &total_t);
    if (mode == 1)
      for (size_t z = 0; z < N; z++) hpd[z] = hp[z];
    long long terms = 0;
    // Reset to the uniform superposition (MultiQW.cpp:326-328, 447-451).
    auto reset = [&]() {
      std::fill(psi.begin(), psi.begin() + N, psi0);
      std::fill(psi.begin() + N, psi.end(), 0.0f);
      if (mode == 1) {
        std::fill(psid.begin(), psid.begin() + N, (double)psi0);
        std::fill(psid.begin() + N, psid.end(), 0.0);
      }
    };
    reset();
    bool psi_real = true;
    double psum = 0.0;
    for (int j = s_begin; j < samples_used; j++) {
      for (int i = 0; i < m; i++) {
        float gamma = gammas[i];
        // E_abs + gamma*n (MultiQW.cpp:436), with the multiply-add fused as
        // g++ -O3 -march=native fuses it; the CUDA path fuses it the same way.
        float onenorm = std::fma(gamma, (float)n, d.e_abs);
        double scale = onenorm * times[i * kSamples + j];
        int K = cheb_coeffs(scale, kChebTol, cd.data(), (int)cd.size());
        if (K < 0) return -2;
        for (int k = 0; k < K; k++) cf[k] = (float)cd[k];
        terms += K;
        if (mode == 0) {
          orc_clenshaw_f32_ext(n, K, cf.data(), hp.data(), gamma, onenorm,
                               psi.data(), out.data(), psi_real, ext_step);
          // psi /= ||psi|| (MultiQW.cpp:443) with a float norm and float
          // division. The reference's norm is Eigen's vectorised float
          // reduction; its order is a library detail that is not restated.
          // The sum of squares is accumulated in double here (as the CUDA
          // path does): a sequential float sum over 2^17 terms alone moves
          // P by ~1e-5, far more than the FP32 recurrence does.
          double ss = 0.0;
          for (size_t z = 0; z < 2 * N; z++) ss += (double)out[z] * out[z];
          float nrm = std::sqrt((float)ss);
          for (size_t z = 0; z < 2 * N; z++) psi[z] = out[z] / nrm;
        } else {
          orc_clenshaw_f64(n, K, cf.data(), hpd.data(), gamma, onenorm,
                           psid.data(), outd.data(), psi_real);
          double ss = 0.0;
          for (size_t z = 0; z < 2 * N; z++) ss += outd[z] * outd[z];
          double nrm = std::sqrt(ss);
          for (size_t z = 0; z < 2 * N; z++) psid[z] = outd[z] / nrm;
        }
        psi_real = false;
      }
      if (mode == 0) {
        float pj = psi[d.e_loc] * psi[d.e_loc] + psi[d.e_loc + N] * psi[d.e_loc + N];
        psum += pj;
      } else {
        double pj = psid[d.e_loc] * psid[d.e_loc] + psid[d.e_loc + N] * psid[d.e_loc + N];
        psum += pj;
      }
      if (m != 1) {
        reset();
        psi_real = true;
      }
    }
    // Mean over samples (MultiQW.cpp:454), accumulated in double.
    p_out[p] = psum / (samples_used - s_begin);
    if (psum_out) psum_out[p] = psum;
    if (total_t_out) total_t_out[p] = total_t;
    if (e_loc_out) e_loc_out[p] = d.e_loc;
    if (terms_out) terms_out[p] = terms;
  }
  return 0;
}

int orc_run_problems_ext(int n, int m, const double* raw, int count,
                         int samples_used, int mode, double* p_out,
                         float* total_t_out, uint32_t* e_loc_out,
                         long long* terms_out, void* ext_step) {
  return run_samples(n, m, raw, count, 0, samples_used, mode, p_out, nullptr, total_t_out,
                     e_loc_out, terms_out, ext_step);
}

// Samples [s_begin, s_end) of one instance: the sum of their ground-state
// probabilities (so that ranges run in separate processes add up to the
// reference's per-instance sum, MultiQW.cpp:432-454) and their summed degree.
int orc_run_sample_range_ext(int n, int m, const double* raw, int s_begin, int s_end,
                             int mode, double* psum_out, long long* terms_out,
                             void* ext_step) {
  double p = 0.0;
  return run_samples(n, m, raw, 1, s_begin, s_end, mode, &p, psum_out, nullptr, nullptr,
                     terms_out, ext_step);
}

int orc_run_problems(int n, int m, const double* raw, int count,
                     int samples_used, int mode, double* p_out,
                     float* total_t_out, uint32_t* e_loc_out,
                     long long* terms_out) {
  return orc_run_problems_ext(n, m, raw, count, samples_used, mode, p_out,
                              total_t_out, e_loc_out, terms_out, nullptr);
}

}  // extern "C"
