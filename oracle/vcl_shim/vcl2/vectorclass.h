// Project-written stand-in for the subset of Agner Fog's Vector Class Library
// (VCL2) that the reference's Clenshaw_step uses (MultiQW.cpp:88-173):
// Vec16f (16 packed floats) with load/store, arithmetic with vectors and
// broadcast scalars, compound assignment, and permute16<i0..i15>, whose lane k
// takes a[i_k]. Written from the library's documented semantics, not from its
// source. Test infrastructure only (oracle/_ref partial build).
#pragma once
#include <cstdint>

#if defined(__AVX512F__)
#include <immintrin.h>

class Vec16f {
 public:
  Vec16f() = default;
  Vec16f(float f) : v_(_mm512_set1_ps(f)) {}
  Vec16f(__m512 x) : v_(x) {}
  operator __m512() const { return v_; }
  Vec16f& load(const float* p) {
    v_ = _mm512_loadu_ps(p);
    return *this;
  }
  void store(float* p) const { _mm512_storeu_ps(p, v_); }

 private:
  __m512 v_;
};

static inline Vec16f operator+(Vec16f a, Vec16f b) { return _mm512_add_ps(a, b); }
static inline Vec16f operator-(Vec16f a, Vec16f b) { return _mm512_sub_ps(a, b); }
static inline Vec16f operator*(Vec16f a, Vec16f b) { return _mm512_mul_ps(a, b); }
static inline Vec16f operator/(Vec16f a, Vec16f b) { return _mm512_div_ps(a, b); }

template <int i0, int i1, int i2, int i3, int i4, int i5, int i6, int i7,
          int i8, int i9, int i10, int i11, int i12, int i13, int i14, int i15>
static inline Vec16f permute16(Vec16f a) {
  const __m512i idx = _mm512_setr_epi32(i0, i1, i2, i3, i4, i5, i6, i7, i8, i9,
                                        i10, i11, i12, i13, i14, i15);
  return _mm512_permutexvar_ps(idx, a);
}

#else  // portable fallback: 16 floats, element-wise loops

class Vec16f {
 public:
  Vec16f() = default;
  Vec16f(float f) {
    for (int k = 0; k < 16; k++) v_[k] = f;
  }
  Vec16f& load(const float* p) {
    for (int k = 0; k < 16; k++) v_[k] = p[k];
    return *this;
  }
  void store(float* p) const {
    for (int k = 0; k < 16; k++) p[k] = v_[k];
  }
  float operator[](int k) const { return v_[k]; }
  float& operator[](int k) { return v_[k]; }

 private:
  float v_[16];
};

#define MQW_VCL_BINOP(OP)                                   \
  static inline Vec16f operator OP(Vec16f a, Vec16f b) {    \
    Vec16f r;                                               \
    for (int k = 0; k < 16; k++) r[k] = a[k] OP b[k];       \
    return r;                                               \
  }
MQW_VCL_BINOP(+)
MQW_VCL_BINOP(-)
MQW_VCL_BINOP(*)
MQW_VCL_BINOP(/)
#undef MQW_VCL_BINOP

template <int i0, int i1, int i2, int i3, int i4, int i5, int i6, int i7,
          int i8, int i9, int i10, int i11, int i12, int i13, int i14, int i15>
static inline Vec16f permute16(Vec16f a) {
  const int idx[16] = {i0, i1, i2,  i3,  i4,  i5,  i6,  i7,
                       i8, i9, i10, i11, i12, i13, i14, i15};
  Vec16f r;
  for (int k = 0; k < 16; k++) r[k] = a[idx[k]];
  return r;
}

#endif

static inline Vec16f& operator+=(Vec16f& a, Vec16f b) { return a = a + b; }
static inline Vec16f& operator-=(Vec16f& a, Vec16f b) { return a = a - b; }
static inline Vec16f& operator*=(Vec16f& a, Vec16f b) { return a = a * b; }
static inline Vec16f& operator/=(Vec16f& a, Vec16f b) { return a = a / b; }
static inline Vec16f operator-(Vec16f a) { return Vec16f(0.0f) - a; }
