// Small complex and math helpers shared by the kernels.
//
// Everything here is __host__ __device__ so that the same arithmetic can be
// compiled for the CPU test harness (tests/cpu_harness), which checks the
// kernels' own math against the FP64 oracle without a GPU.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define LMB_HD __host__ __device__ __forceinline__
#else
#define LMB_HD inline
#endif

namespace lmb {

template <typename T>
struct cplx {
  T re, im;
};

template <typename T>
LMB_HD cplx<T> mk(T re, T im) {
  cplx<T> z;
  z.re = re;
  z.im = im;
  return z;
}
template <typename T>
LMB_HD cplx<T> operator+(cplx<T> a, cplx<T> b) { return mk(a.re + b.re, a.im + b.im); }
template <typename T>
LMB_HD cplx<T> operator-(cplx<T> a, cplx<T> b) { return mk(a.re - b.re, a.im - b.im); }
template <typename T>
LMB_HD cplx<T> operator-(cplx<T> a) { return mk(-a.re, -a.im); }
template <typename T>
LMB_HD cplx<T> operator*(cplx<T> a, cplx<T> b) {
  return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <typename T>
LMB_HD cplx<T> operator*(T s, cplx<T> a) { return mk(s * a.re, s * a.im); }
template <typename T>
LMB_HD cplx<T> operator*(cplx<T> a, T s) { return mk(s * a.re, s * a.im); }
template <typename T>
LMB_HD cplx<T> operator+(cplx<T> a, T s) { return mk(a.re + s, a.im); }
template <typename T>
LMB_HD cplx<T> operator+(T s, cplx<T> a) { return mk(a.re + s, a.im); }
template <typename T>
LMB_HD cplx<T> operator-(T s, cplx<T> a) { return mk(s - a.re, -a.im); }
template <typename T>
LMB_HD cplx<T> operator-(cplx<T> a, T s) { return mk(a.re - s, a.im); }
template <typename T>
LMB_HD cplx<T> conj(cplx<T> a) { return mk(a.re, -a.im); }
// multiply by i
template <typename T>
LMB_HD cplx<T> mul_i(cplx<T> a) { return mk(-a.im, a.re); }
template <typename T>
LMB_HD T norm2(cplx<T> a) { return a.re * a.re + a.im * a.im; }

// Complex division by Smith's method (R. L. Smith, CACM 5, 435 (1962)),
// the scaling numpy applies to complex128 division.
template <typename T>
LMB_HD cplx<T> operator/(cplx<T> a, cplx<T> b) {
  T ar = b.re < T(0) ? -b.re : b.re;
  T ai = b.im < T(0) ? -b.im : b.im;
  if (ar >= ai) {
    T rat = b.im / b.re;
    T scl = T(1) / (b.re + b.im * rat);
    return mk((a.re + a.im * rat) * scl, (a.im - a.re * rat) * scl);
  } else {
    T rat = b.re / b.im;
    T scl = T(1) / (b.im + b.re * rat);
    return mk((a.re * rat + a.im) * scl, (a.im * rat - a.re) * scl);
  }
}
template <typename T>
LMB_HD cplx<T> operator/(T s, cplx<T> b) { return mk(s, T(0)) / b; }

// 1/x with one correctly rounded reciprocal on the device (the instruction
// rcp.rn.f64), 1/x on the host.  In a dependent chain this is about half
// the latency of an IEEE division.
LMB_HD double rcp_d(double x) {
#if defined(__CUDA_ARCH__)
  return __drcp_rn(x);
#else
  return 1. / x;
#endif
}

// 1/b.  Where |re| + |im| lies in 1e-150..1e150, so that |b|^2 neither
// overflows nor underflows, as conj(b) / |b|^2 with one reciprocal; else
// (and for NaN or infinite b) by Smith's scaled division, above, which costs
// two dependent divisions.  The recurrences' denominators are almost always
// in the fast range.
LMB_HD cplx<double> recip(cplx<double> b) {
  const double a = fabs(b.re) + fabs(b.im);
  if (a > 1e-150 && a < 1e150) {
    const double r = rcp_d(b.re * b.re + b.im * b.im);
    return mk(b.re * r, -b.im * r);
  }
  return mk(1., 0.) / b;
}
template <typename T>
LMB_HD cplx<T> operator/(cplx<T> a, T s) { return mk(a.re / s, a.im / s); }

// e^{i t}
LMB_HD cplx<double> cis(double t) {
  double s, c;
#if defined(__CUDA_ARCH__)
  sincos(t, &s, &c);
#else
  s = sin(t);
  c = cos(t);
#endif
  return mk(c, s);
}
LMB_HD cplx<float> cis(float t) {
  float s, c;
#if defined(__CUDA_ARCH__)
  sincosf(t, &s, &c);
#else
  s = sinf(t);
  c = cosf(t);
#endif
  return mk(c, s);
}

// Two FP32 lanes in one register pair, operated on by the packed sm_100
// instructions (fma/mul/add .rn.f32x2: each lane rounds exactly like its
// scalar counterpart, so the host emulation below is bit-identical).
#if defined(__CUDACC__)
typedef float2 f2;
#else
struct f2 {
  float x, y;
};
#endif
LMB_HD f2 pk(float x, float y) {
  f2 r;
  r.x = x;
  r.y = y;
  return r;
}
LMB_HD f2 pfma(f2 a, f2 b, f2 c) {
#if defined(__CUDA_ARCH__)
  return __ffma2_rn(a, b, c);
#else
  return pk(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y));
#endif
}
LMB_HD f2 pmul(f2 a, f2 b) {
#if defined(__CUDA_ARCH__)
  return __fmul2_rn(a, b);
#else
  return pk(a.x * b.x, a.y * b.y);
#endif
}
LMB_HD f2 padd(f2 a, f2 b) {
#if defined(__CUDA_ARCH__)
  return __fadd2_rn(a, b);
#else
  return pk(a.x + b.x, a.y + b.y);
#endif
}

// Approximate FP32 reciprocal square root (a few ulp): the starting value
// of the FP64 Newton-Raphson step of phase_turns64.
LMB_HD float rsqrt_seed(float x) {
#if defined(__CUDA_ARCH__)
  return rsqrtf(x);
#else
  return 1.f / sqrtf(x);
#endif
}

// sqrt(x) to a few ulp (x >= 0), for error estimates.
LMB_HD float approx_sqrt(float x) {
  return x > 1e-30f ? x * rsqrt_seed(x) : 0.f;
}

// e^{2 pi i t}
LMB_HD cplx<float> cis_turns(float t) {
  float s, c;
#if defined(__CUDA_ARCH__)
  sincospif(2.f * t, &s, &c);
#else
  const double a = 6.283185307179586 * double(t);
  s = float(sin(a));
  c = float(cos(a));
#endif
  return mk(c, s);
}

LMB_HD float lsqrt(float x) { return sqrtf(x); }
LMB_HD double lsqrt(double x) { return sqrt(x); }
LMB_HD float labs_(float x) { return fabsf(x); }
LMB_HD double labs_(double x) { return fabs(x); }

}  // namespace lmb
