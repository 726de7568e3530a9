// Host-side instance unpacking and stage schedule (no GPU involved).
//
// Compiled with g++ -O2 -march=x86-64-v3 -ffp-contract=fast: the same
// multiply-add fusion policy g++ applies to the reference's own
// `g++ -O3 -march=native` build, and the expressions below keep the
// reference's float/double promotions, so gamma and the time samples match
// the reference to the last bit wherever its inputs do (the inverse normal is
// correctly rounded here and within 1 ulp of the reference's approximation).
#include <algorithm>
#include <cmath>
#include <random>

#include "../../include/mqw.h"
#include "mqw_cheb.h"

namespace {

constexpr double kPi = 3.1415926535897932384626;  // MultiQW.cpp:11
constexpr unsigned long kSeed = 29552825458725UL; // MultiQW.cpp:387

// Initial guess for the upper-tail quantile: Abramowitz & Stegun 26.2.23.
double quantile_guess(double p) {
  const double q = p < 0.5 ? p : 1.0 - p;
  const double t = std::sqrt(-2.0 * std::log(q));
  const double x = t - (2.515517 + t * (0.802853 + t * 0.010328)) /
                           (1.0 + t * (1.432788 + t * (0.189269 + t * 0.001308)));
  return p < 0.5 ? x : -x;
}

}  // namespace

extern "C" {

// Phi^{-1}(1 - p): Halley's iteration on Q(x) = erfc(x/sqrt2)/2 = p in double,
// rounded once to float. Replaces my_normcdfinvf (MultiQW.cpp:80-86), which
// returns the same quantity as a float approximation (<= 4.1 ulp).
float mqw_inv_norm_upper(float pf) {
  const double p = pf;
  if (!(p > 0.0)) return INFINITY;
  if (!(p < 1.0)) return -INFINITY;
  if (p == 0.5) return 0.0f;
  double x = quantile_guess(p);
  const double inv_sqrt2 = 0.70710678118654752440;
  const double inv_sqrt2pi = 0.39894228040143267794;
  for (int it = 0; it < 60; it++) {
    const double q = 0.5 * std::erfc(x * inv_sqrt2);
    const double phi = inv_sqrt2pi * std::exp(-0.5 * x * x);
    const double d = (q - p) / phi;
    const double step = d / (1.0 - 0.5 * x * d);
    x += step;
    if (std::fabs(step) <= 1e-16 * std::max(1.0, std::fabs(x))) break;
  }
  return (float)x;
}

mqw_status mqw_load_instance(int n, const double* raw, float* J, float* h) {
  if (n < 1 || n > MQW_MAX_N || !raw || !J || !h) return MQW_ERR_INVALID;
  std::fill(J, J + n * n, 0.0f);
  int k = 0;
  for (int i = 1; i < n; i++)
    for (int j = 0; j < i; j++) {
      const float v = (float)raw[k++] / 2;  // (J + J^T)/2, MultiQW.cpp:318-319
      J[i * n + j] = v;
      J[j * n + i] = v;
    }
  for (int i = 0; i < n; i++) h[i] = (float)raw[n * (n - 1) / 2 + i];
  return MQW_OK;
}

mqw_status mqw_schedule(int n, int m, const double* raw, float* gammas,
                        float* short_ts, float* times, float* total_t_out) {
  if (n < 1 || n > MQW_MAX_N || m < 1 || m > MQW_MAX_M || !raw || !gammas ||
      !times)
    return MQW_ERR_INVALID;
  float J[MQW_MAX_N * MQW_MAX_N], h[MQW_MAX_N];
  mqw_load_instance(n, raw, J, h);
  const unsigned N = 1u << n;
  // Expected maximum of N Gaussians (MultiQW.cpp:365-370).
  const float b = mqw_inv_norm_upper(1 / (float)N);
  const float e_m = 0.577215664901532860;
  const float e = 2.718281828459045;
  const float a = (1 - e_m) * b + e_m * mqw_inv_norm_upper(1 / (e * N));
  // Second moments of the couplings (MultiQW.cpp:375, 395), storage order.
  float JJ = 0.0f, hh = 0.0f;
  for (int i = 0; i < n * n; i++) JJ += J[i] * J[i];
  for (int i = 0; i < n; i++) hh += h[i] * h[i];
  const float HP2 = 2 * JJ + hh;
  std::mt19937 gen(kSeed);  // re-seeded per instance (MultiQW.cpp:387)
  for (int i = 0; i < m; i++)
    gammas[i] = a * std::sqrt(HP2) / std::tan(kPi * (i + 1) / (2 * m + 2)) / n;
  float total_t = 0;
  const float delta2 = 16 * JJ + 4 * hh;
  for (int i = 0; i < m; i++) {
    // Stage-time lower bounds (MultiQW.cpp:397-416).
    const float last_denom = std::sqrt(2 / kPi) * gammas[i] * std::sqrt(n * delta2);
    const float g_last =
        (i == 0) ? 1 : gammas[i - 1] / std::sqrt(1 + gammas[i - 1] * gammas[i - 1]);
    const float g_next =
        (i + 1 == m) ? 0 : gammas[i + 1] / std::sqrt(1 + gammas[i + 1] * gammas[i + 1]);
    const float dH = g_last - g_next;
    const float first_t = std::sqrt(4 * (unsigned)n * dH / delta2);
    const float last_t = std::sqrt(2 * (unsigned)n * dH / last_denom);
    const float short_t = (i == 0) ? first_t : std::max(first_t, last_t);
    std::uniform_real_distribution<float> rand_t(short_t, 2 * short_t);
    total_t += short_t;
    if (short_ts) short_ts[i] = short_t;
    for (int j = 0; j < MQW_SAMPLES; j++) times[i * MQW_SAMPLES + j] = rand_t(gen);
  }
  // One stage: sorted times, differenced, evolved cumulatively
  // (MultiQW.cpp:426-430).
  if (m == 1) {
    std::sort(times, times + MQW_SAMPLES);
    for (int j = MQW_SAMPLES - 1; j >= 1; j--) times[j] -= times[j - 1];
  }
  if (total_t_out) *total_t_out = total_t;
  return MQW_OK;
}

mqw_status mqw_cheb_coeffs_host(int count, const double* s, double tol,
                                int max_k, float* coeffs, int* degrees) {
  if (count < 0 || max_k < 1 || (count > 0 && (!s || !coeffs || !degrees)) ||
      !(tol > 0.0))
    return MQW_ERR_INVALID;
  for (int i = 0; i < count; i++) {
    float* out = coeffs + (size_t)i * max_k;
    std::fill(out, out + max_k, 0.0f);
    degrees[i] = mqw::cheb_coeffs_stream(s[i], tol, out, max_k);
    if (degrees[i] < 1) return MQW_ERR_INVALID;
  }
  return MQW_OK;
}

}  // extern "C"
