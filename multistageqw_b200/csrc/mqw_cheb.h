// Chebyshev coefficients of exp(i s x) on [-1, 1], streamed in FP64.
//
// The reference obtains these from Chebyshev<double>::RCF_odd_even(f, 1e-6)
// with f(x) = sin(sx) + cos(sx) (MultiQW.cpp:436-440; the ApproxTools
// submodule that defines it is empty in the reference snapshot). This is the
// closed form of the same expansion (Jacobi–Anger):
//   c_0 = J_0(s),  c_k = 2 (-1)^floor(k/2) J_k(s)  (k >= 1),
// even k applied as real, odd k as imaginary coefficients. Truncation: the
// smallest K >= 1 with sum_{k>=K} |c_k| <= tol.
//
// Bessel values come from Miller's backward recurrence
//   f_{k-1} = (2k/s) f_k - f_{k+1},  f_{top+1} = 0, f_top = 1e-300,
//   top = ceil(s) + 40 + 4*isqrt(ceil(s)), made even,
// normalised by J_0 + 2 sum J_2k = 1 (sum from the top down). For s >= 1e-8
// the values never overflow, so the recurrence is run twice instead of being
// stored: pass 1 for the normalisation, pass 2 for the tail sums and the
// coefficients. Every operation is an IEEE double op with explicit fma, so
// host and device produce identical bits.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define MQW_HD __host__ __device__
#else
#define MQW_HD
#endif

namespace mqw {

MQW_HD inline int cheb_top(double s) {
  const int cs = (int)ceil(s);
  int r = (int)sqrt((double)cs);
  while (r * r > cs) r--;
  while ((r + 1) * (r + 1) <= cs) r++;
  int top = cs + 40 + 4 * r;
  return top + (top & 1);
}

// Returns the degree K; writes float(c_k) for k < min(K, max_k) into out when
// out != nullptr. Returns -1 for non-finite s.
MQW_HD inline int cheb_coeffs_stream(double s, double tol, float* out,
                                     int max_k) {
  s = fabs(s);
  if (!(s == s) || s > 1e7) return -1;
  if (s < 1e-8) {
    if (out && max_k > 0) out[0] = 1.0f;
    return 1;
  }
  const int top = cheb_top(s);
  // Pass 1: normalisation.
  double fk1 = 0.0, fk = 1e-300, norm = 2.0 * fk;  // top is even
  for (int k = top; k >= 1; k--) {
    const double fm = fma(2.0 * k / s, fk, -fk1);
    fk1 = fk;
    fk = fm;
    const int km = k - 1;
    if (km >= 2 && !(km & 1)) norm += 2.0 * fk;
  }
  norm += fk;  // f_0
  // Pass 2: tail sums from the top, then the kept coefficients.
  fk1 = 0.0;
  fk = 1e-300;
  double tail = 2.0 * fabs(fk / norm);
  int K = (tail > tol) ? top + 1 : 1;
  bool found = tail > tol;
  if (found && out && top < max_k) {
    double v = fk / norm;
    v *= ((top / 2) & 1) ? -2.0 : 2.0;
    out[top] = (float)v;
  }
  for (int k = top; k >= 1; k--) {
    const double fm = fma(2.0 * k / s, fk, -fk1);
    fk1 = fk;
    fk = fm;
    const int km = k - 1;  // index of fm
    if (!found && km >= 1) {
      tail += 2.0 * fabs(fm / norm);
      if (tail > tol) {
        K = km + 1;
        found = true;
      }
    }
    if (!found && km == 0) found = true;  // K = 1: only c_0 is kept
    if (found && out && km < max_k) {
      double v = fm / norm;
      if (km > 0) v *= ((km / 2) & 1) ? -2.0 : 2.0;
      out[km] = (float)v;
    }
  }
  return K;
}

}  // namespace mqw
