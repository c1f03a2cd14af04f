// Per-pixel Lorenz-Mie partial-wave sum, its Jacobian, and the hologram.
//
// Follows theory/LorenzMie.py:183-342 (LorenzMie.lorenzmie):
//   geometry from kdr with kz flipped (:221-237); Riccati-Bessel starting
//   values with the sign(kz) convention (:249-251); for n = 1..nmax the
//   Wiscombe pi_n/tau_n, xi_n = (2n-1) xi_{n-1}/kr - xi_{n-2},
//   D_n = n xi_n/kr - xi_{n-1} and the vector-spherical-harmonic sums
//   (:272-317); geometric factors restored at the end (:322-325); Cartesian
//   projection (:331-340); phase exp(-i k z_p) (:157-158); hologram
//   |E + x|^2 (:131-133).
//
// Two reformulations keep FP32 accurate without changing the result:
//  * xi_n = e^{i sigma kr} h_n, where h_n obeys the same real-coefficient
//    recurrence from h_{-1} = 1, h_0 = -i sigma.  The pure phase
//    e^{i(sigma kr - k z_p)} is applied once per pixel.  For the default
//    convention (sigma = sign(kz)) its argument equals
//    sign(kz) krho^2 / (kr + |kz|) - k z, which is free of the cancellation
//    between kr and k z_p (both ~10^2 rad) that FP32 cannot resolve.
//  * The order-n coefficients are pre-multiplied by the prefactor:
//    alpha_n = i E_n a_n, beta_n = E_n b_n, E_n = i^n (2n+1)/(n(n+1)), and
//    the sums are regrouped as
//      S0 = sum pi (n(n+1) alpha h),
//      S1 = sum tau (alpha Dh) - pi (beta h),
//      S2 = sum pi (alpha Dh) - tau (beta h).
//
//  * The Wiscombe recurrence is carried in s = 1 - |cos(theta)| and
//    Delta_n = pi_n - pi_{n-1}:
//      tau_n = pi_{n-1} - n Delta_n + n s pi_n,
//      Delta_{n+1} = c_n Delta_n - (1 + c_n) s pi_n,  c_n = 1 + 1/n,
//      pi_{n+1} = pi_n + Delta_{n+1},
//    which is the reference's swisc/twisc update with mu = 1 - s.  s is
//    formed as krho^2 / (kr (kr + |kz|)), so the angle near the optical
//    axis keeps its relative precision (FP32 cos(theta) near 1 does not,
//    and pi_n is very sensitive there).  For cos(theta) < 0 the parities
//    pi_n(-mu) = (-1)^{n-1} pi_n(mu), tau_n(-mu) = (-1)^n tau_n(mu) are
//    folded into h_n (h~_n = (-1)^{n-1} h_n obeys the recurrence with kr
//    negated), which leaves a sign on some of the summed components.
//
// The Jacobian is forward mode.  In the order loop it carries tangents in kr
// of the phase-reduced h_n (the differentiated recurrence, which starts
// from zero because h_{-1}, h_0 are constants: this keeps the small
// derivative of the slowly varying h_n at full relative precision), in
// cos(theta) (differentiated Wiscombe recurrence), and in the particle's
// a_p and n_p (through d alpha_n, d beta_n from the FP64 coefficient kernel).
// The per-pixel epilogue is evaluated in dual numbers over (kx, ky, kz).
// d/dk_p = i d/dn_p because a_n, b_n are holomorphic in the relative index.
// On the optical axis (krho = 0) phi is taken as 0 with zero derivative,
// the safe branch of theory/jaxLorenzMie.py:170-175.
#pragma once

#include "lmb_math.cuh"

namespace lmb {

// Per-order record staged in shared memory by the kernels.
//   c0 = (alpha.re, alpha.im, beta.re, beta.im)
//   c1 = (n(n+1) alpha.re, n(n+1) alpha.im, 1 + 1/n, n)
// and, for the Jacobian, the a_p and n_p derivatives of alpha and beta:
//   c2 = d/da_p (alpha, beta), c3 = d/dn_p (alpha, beta),
//   c4 = n(n+1) d/da_p alpha, n(n+1) d/dn_p alpha.
// JAC_QUADS records per order for the Jacobian, 2 for the value.
template <typename R>
struct Quad {
  R x, y, z, w;
};

enum { JAC_QUADS = 5 };

template <typename R>
struct Geometry {
  R kr, ikr, mu, sint, cosp, sinp, krho;
  R s1mu;           // 1 - |cos(theta)|, to full relative precision
  R smu;            // sign of cos(theta) (+1 when cos(theta) == 0)
  R ikrs;           // smu / kr: the recurrence coefficient's scale
  R sigma;          // +1, -1, or 0 (pixel in the particle's plane)
  cplx<R> phase;    // e^{i(sigma kr - k z_p)}
  cplx<R> hm1, h0;  // h_{-1}, h_0
};

// Geometry of one pixel relative to one particle.
//   dx, dy, dzc: coordinate minus particle position (pixels, FP64)
//   z: the pixel's own z coordinate; zp: the particle's z
LMB_HD double reduce_2pi(double t) { return remainder(t, 6.283185307179586); }

// The phase sign(kz) k (r - |dzc|) - k z of a pixel, in turns (units of
// 2 pi) and reduced to [-1/2, 1/2], in FP64: r = sqrt(rho^2 + dzc^2) from
// an FP32 starting value of 1/sqrt refined by one Newton-Raphson step
// (y <- y (3 - x y^2) / 2, which squares its relative error of ~2^-22 to
// ~1e-13), then w = (k / 2 pi) (r - |dzc|) and w - rint(w).  The error is
// ~1e-10 turns at the largest distances of a frame, against ~1e-5 for the
// same argument in FP32.  Outside 1e-30 < r^2 < 1e30 (the FP32 range of
// the starting value) r is the FP64 square root.
LMB_HD double phase_turns64(double k, double dx, double dy, double dzc,
                            double s, double z) {
  const double kt = k * 0.15915494309189535;  // k / (2 pi)
  const double r2 = fma(dzc, dzc, fma(dx, dx, dy * dy));
  double r;
  if (r2 > 1e-30 && r2 < 1e30) {
    const double y = rsqrt_seed(float(r2));
    const double t = r2 * y;
    r = t * fma(-0.5 * t, y, 1.5);
  } else {
    r = sqrt(r2);
  }
  double w = s * fma(kt, r, -kt * fabs(dzc));
  if (z != 0.) w = fma(-kt, z, w);
  return w - rint(w);
}

// kPhase64: form the phase sign(kz) (kr - |kz|) - k z in FP64 from the FP64
// offsets (phase_turns64; R = float only).  Far from the particle (kr ~
// 10^3 rad) the FP32 argument, and even the FP32 roundings of kx, ky and kz
// that it is formed from, are off by ~1e-4 rad; in FP64 the phase is exact
// to FP32 rounding.  The fits' crops (kr ~ 10^2) do not need it.
template <typename R, bool kPhase64 = false>
LMB_HD Geometry<R> geometry(double k, double dx, double dy, double dzc,
                            double z, double zp, bool bohren) {
  Geometry<R> g;
  const R kx = R(k * dx);
  const R ky = R(k * dy);
  const R kz = R(-k * dzc);
  const R krho2 = kx * kx + ky * ky;
  const R krho = lsqrt(krho2);
  const R kr = lsqrt(krho2 + kz * kz);
  const R ikr = R(1) / kr;
  g.kr = kr;
  g.ikr = ikr;
  g.krho = krho;
  g.mu = kz * ikr;
  g.sint = krho * ikr;
  g.s1mu = krho2 / (kr * (kr + labs_(kz)));
  g.smu = kz < R(0) ? R(-1) : R(1);
  g.ikrs = g.smu * ikr;
  if (krho > R(0)) {
    const R ikrho = R(1) / krho;
    g.cosp = kx * ikrho;
    g.sinp = ky * ikrho;
  } else {
    g.cosp = R(1);
    g.sinp = R(0);
  }
  const R s = kz > R(0) ? R(1) : (kz < R(0) ? R(-1) : R(0));
  const R sigma = bohren ? s : -s;
  g.sigma = sigma;
  if (sigma != R(0)) {
    g.hm1 = mk(R(1), R(0));
    g.h0 = mk(R(0), -sigma);
    if (sigma == s) {
      // sign(kz) (kr - |kz|) - k z, with kr - |kz| = krho^2/(kr + |kz|)
      if constexpr (kPhase64) {
        static_assert(sizeof(R) == sizeof(float), "FP32 geometry only");
        g.phase = cis_turns(float(phase_turns64(k, dx, dy, dzc, double(s), z)));
      } else {
        R arg = s * krho2 / (kr + labs_(kz));
        if (z != 0.) arg += R(reduce_2pi(-k * z));
        g.phase = cis(arg);
      }
    } else {
      const double kr64 = k * sqrt(dx * dx + dy * dy + dzc * dzc);
      g.phase = cis(R(reduce_2pi(double(sigma) * kr64 - k * zp)));
    }
  } else {
    // kz == 0: real standing-wave start, xi_{-1} = cos kr, xi_0 = sin kr
    const double kr64 = k * sqrt(dx * dx + dy * dy + dzc * dzc);
    const cplx<R> e = cis(R(reduce_2pi(kr64)));
    g.hm1 = mk(e.re, R(0));
    g.h0 = mk(e.im, R(0));
    g.phase = cis(R(reduce_2pi(-k * zp)));
  }
  g.h0 = g.smu * g.h0;  // h~_0 = sign(mu) h_0
  return g;
}

template <typename R>
struct Sums {
  cplx<R> s0, s1, s2;
};

// The partial-wave sum for the field value only.
// coef: per-order records (2 Quads per order, index n*2 + {0,1}).
template <typename R>
LMB_HD Sums<R> order_sum(const Geometry<R>& g, const Quad<R>* coef,
                         int nmax) {
  Sums<R> acc;
  acc.s0 = mk(R(0), R(0));
  acc.s1 = acc.s0;
  acc.s2 = acc.s0;
  R pim1 = R(0), pi = R(1), del = R(1);
  cplx<R> h2 = g.hm1, h1 = g.h0;
  const R sv = g.s1mu, ikr = g.ikrs;
#pragma unroll 2
  for (int n = 1; n <= nmax; ++n) {
    const Quad<R> c0 = coef[2 * n];
    const Quad<R> c1 = coef[2 * n + 1];
    const R fn = c1.w;
    const R spi = sv * pi;
    const R tau = pim1 - fn * del + fn * spi;
    const R a2 = (fn + fn - R(1)) * ikr;
    const cplx<R> h = mk(a2 * h1.re - h2.re, a2 * h1.im - h2.im);
    const R a1 = fn * ikr;
    const cplx<R> dh = mk(a1 * h.re - h1.re, a1 * h.im - h1.im);
    // X = alpha dh, Y = beta h, Z = n(n+1) alpha h
    const cplx<R> X = mk(c0.x * dh.re - c0.y * dh.im, c0.x * dh.im + c0.y * dh.re);
    const cplx<R> Y = mk(c0.z * h.re - c0.w * h.im, c0.z * h.im + c0.w * h.re);
    const cplx<R> Z = mk(c1.x * h.re - c1.y * h.im, c1.x * h.im + c1.y * h.re);
    acc.s0.re += pi * Z.re;
    acc.s0.im += pi * Z.im;
    acc.s1.re += tau * X.re - pi * Y.re;
    acc.s1.im += tau * X.im - pi * Y.im;
    acc.s2.re += pi * X.re - tau * Y.re;
    acc.s2.im += pi * X.im - tau * Y.im;
    del = c1.z * del - (c1.z + R(1)) * spi;
    pim1 = pi;
    pi = pi + del;
    h2 = h1;
    h1 = h;
  }
  acc.s2 = g.smu * acc.s2;
  return acc;
}

// Restore the geometric factors and (optionally) project onto Cartesian
// axes; multiply by the phase.  Returns the field of one particle.
template <typename R>
LMB_HD void epilogue(const Geometry<R>& g, const Sums<R>& s, bool cartesian,
                     cplx<R>* e) {
  const R ikr = g.ikr;
  const cplx<R> es0 = (g.cosp * g.sint * ikr * ikr) * s.s0;
  const cplx<R> es1 = (g.cosp * ikr) * s.s1;
  const cplx<R> es2 = (g.sinp * ikr) * s.s2;
  cplx<R> c0, c1, c2;
  if (cartesian) {
    c0 = (g.sint * g.cosp) * es0 + (g.mu * g.cosp) * es1 - g.sinp * es2;
    c1 = (g.sint * g.sinp) * es0 + (g.mu * g.sinp) * es1 + g.cosp * es2;
    c2 = g.mu * es0 - g.sint * es1;
  } else {
    c0 = es0;
    c1 = es1;
    c2 = es2;
  }
  e[0] = g.phase * c0;
  e[1] = g.phase * c1;
  e[2] = g.phase * c2;
}

// ---------------------------------------------------------------------------
// Jacobian

template <typename R>
struct JacSums {
  cplx<R> s[3];   // value
  cplx<R> t[3];   // d/dkr of the phase-reduced sums
  cplx<R> u[3];   // d/dmu
  cplx<R> a[3];   // d/da_p
  cplx<R> p[3];   // d/dn_p
};

// coef: JAC_QUADS Quads per order (index n*JAC_QUADS + j), see Quad above.
template <typename R>
LMB_HD JacSums<R> order_sum_jac(const Geometry<R>& g, const Quad<R>* coef,
                                int nmax) {
  JacSums<R> A;
  const cplx<R> zero = mk(R(0), R(0));
  for (int c = 0; c < 3; ++c) {
    A.s[c] = zero;
    A.t[c] = zero;
    A.u[c] = zero;
    A.a[c] = zero;
    A.p[c] = zero;
  }
  // pi, Delta and their derivatives with respect to s = 1 - |mu|
  R pim1 = R(0), pi = R(1), del = R(1);
  R dpim1 = R(0), dpi = R(0), ddel = R(0);
  cplx<R> h2 = g.hm1, h1 = g.h0;
  cplx<R> hp2 = mk(R(0), R(0)), hp1 = hp2;  // d h~/dkr
  const R sv = g.s1mu, ikr = g.ikrs, ikr2 = g.ikrs * g.ikr;
#pragma unroll 2
  for (int n = 1; n <= nmax; ++n) {
    const Quad<R> c0 = coef[JAC_QUADS * n];
    const Quad<R> c1 = coef[JAC_QUADS * n + 1];
    const Quad<R> c2 = coef[JAC_QUADS * n + 2];
    const Quad<R> c3 = coef[JAC_QUADS * n + 3];
    const Quad<R> c4 = coef[JAC_QUADS * n + 4];
    const R fn = c1.w;
    const R cn = c1.z;
    const R spi = sv * pi;
    const R tau = pim1 - fn * del + fn * spi;
    const R dspi = pi + sv * dpi;
    const R dtau = dpim1 - fn * ddel + fn * dspi;
    const R tn1 = fn + fn - R(1);
    const R a2 = tn1 * ikr;
    const cplx<R> h = mk(a2 * h1.re - h2.re, a2 * h1.im - h2.im);
    const R a1 = fn * ikr;
    const cplx<R> dh = mk(a1 * h.re - h1.re, a1 * h.im - h1.im);
    // d/dkr of h~_n = (2n-1) ikr h~_{n-1} - h~_{n-2} and of dh
    const R b2 = tn1 * ikr2, b1 = fn * ikr2;
    const cplx<R> hp = mk(a2 * hp1.re - b2 * h1.re - hp2.re,
                          a2 * hp1.im - b2 * h1.im - hp2.im);
    const cplx<R> dhp = mk(a1 * hp.re - b1 * h.re - hp1.re,
                           a1 * hp.im - b1 * h.im - hp1.im);
    const cplx<R> al = mk(c0.x, c0.y), be = mk(c0.z, c0.w);
    const cplx<R> al1 = mk(c1.x, c1.y);
    const cplx<R> ala = mk(c2.x, c2.y), bea = mk(c2.z, c2.w);
    const cplx<R> aln = mk(c3.x, c3.y), ben = mk(c3.z, c3.w);
    // value: X = alpha dh, Y = beta h, Z = n(n+1) alpha h
    const cplx<R> X = al * dh, Y = be * h, Z = al1 * h;
    A.s[0] = A.s[0] + pi * Z;
    A.s[1] = A.s[1] + tau * X - pi * Y;
    A.s[2] = A.s[2] + pi * X - tau * Y;
    // s tangent: same X, Y, Z with dpi/ds, dtau/ds
    A.u[0] = A.u[0] + dpi * Z;
    A.u[1] = A.u[1] + dtau * X - dpi * Y;
    A.u[2] = A.u[2] + dpi * X - dtau * Y;
    // kr tangent: h -> hp, dh -> dhp
    const cplx<R> Xk = al * dhp, Yk = be * hp, Zk = al1 * hp;
    A.t[0] = A.t[0] + pi * Zk;
    A.t[1] = A.t[1] + tau * Xk - pi * Yk;
    A.t[2] = A.t[2] + pi * Xk - tau * Yk;
    // a_p (c4 holds n(n+1) d alpha)
    const cplx<R> ala1 = mk(c4.x, c4.y), aln1 = mk(c4.z, c4.w);
    const cplx<R> Xa = ala * dh, Ya = bea * h, Za = ala1 * h;
    A.a[0] = A.a[0] + pi * Za;
    A.a[1] = A.a[1] + tau * Xa - pi * Ya;
    A.a[2] = A.a[2] + pi * Xa - tau * Ya;
    const cplx<R> Xn = aln * dh, Yn = ben * h, Zn = aln1 * h;
    A.p[0] = A.p[0] + pi * Zn;
    A.p[1] = A.p[1] + tau * Xn - pi * Yn;
    A.p[2] = A.p[2] + pi * Xn - tau * Yn;
    const R deln = cn * del - (cn + R(1)) * spi;
    const R ddeln = cn * ddel - (cn + R(1)) * dspi;
    pim1 = pi;
    pi = pi + deln;
    del = deln;
    dpim1 = dpi;
    dpi = dpi + ddeln;
    ddel = ddeln;
    h2 = h1;
    h1 = h;
    hp2 = hp1;
    hp1 = hp;
  }
  // Undo the parity folding (identity when cos(theta) >= 0) and turn the
  // s tangent into d/dmu: d/dmu = -sign(mu) d/ds on pi~, tau~.
  const R sg = g.smu;
  A.s[2] = sg * A.s[2];
  A.a[2] = sg * A.a[2];
  A.p[2] = sg * A.p[2];
  A.t[2] = sg * A.t[2];
  A.u[0] = (-sg) * A.u[0];
  A.u[1] = (-sg) * A.u[1];
  A.u[2] = -A.u[2];
  return A;
}

// ---------------------------------------------------------------------------
// The Jacobian order loop for two pixels of one particle at once, in packed
// two-lane FP32 (one pfma does the work of two scalar FMAs in one issue
// slot).  Same recurrences and sums as order_sum_jac; the differences are
// signs chosen so that every update is a plain fused multiply-add:
//  * h'_n = s_n h~_n with s_n = +1, -1, -1, +1 for n = 0, 1, 2, 3 (mod 4):
//      h'_n = [(-1)^n (2n-1) ikr] h'_{n-1} + h'_{n-2}
//    and the same sign on the kr tangent hp'_n;
//  * dh''_n = sig_n dh_n with sig_n = (-1)^{n+1} s_n:
//      dh''_n = [(-1)^{n+1} n ikr] h'_n + h'_{n-1}
//    (and the same for the tangent, with -ikr2 terms from the chain rule);
//  * the Wiscombe state keeps -Delta_n, so that tau_n = pi_{n-1} +
//    n (s pi_n - Delta_n) and Delta_{n+1} follow from one shared sum;
//  * the signs s_n, sig_n and the minus of the beta terms are folded into
//    the per-order coefficients, which also carry -Im of every complex
//    coefficient (a complex product is then two multiplies and two fmas).
// Per order: PAIR_VALUES values, each duplicated into both lanes (float2):
//   0 n, 1 c_n = 1 + 1/n, 2 (-1)^n (2n-1), 3 (-1)^{n+1} n,
//   then nine complex coefficients as (re, im, -im):
//   4 sig alpha, 7 -s beta, 10 s n(n+1) alpha, 13..21 the same for
//   d/da_p, 22..30 for d/dn_p; 31 unused.
enum { PAIR_VALUES = 32, PAIR_QUADS = PAIR_VALUES / 2 };

struct PairIn {
  f2 sv;              // s = 1 - |cos(theta)|
  f2 ikr;             // sign(mu) / kr
  f2 mkr;             // -1 / kr
  cplx<f2> hm1, h0;   // h_{-1}, h~_0
};

struct PairSums {
  cplx<f2> s[3], t[3], u[3], a[3], p[3];
};

// c * v for a coefficient stored as (re, im, -im)
LMB_HD cplx<f2> pcmul(f2 re, f2 im, f2 nim, cplx<f2> v) {
  return mk(pfma(re, v.re, pmul(nim, v.im)), pfma(re, v.im, pmul(im, v.re)));
}
// acc + w v
LMB_HD cplx<f2> pacc(cplx<f2> acc, f2 w, cplx<f2> v) {
  return mk(pfma(w, v.re, acc.re), pfma(w, v.im, acc.im));
}

// rec: PAIR_QUADS float4 per order (index n * PAIR_QUADS + j); the two
// values of a float4 are (x, y) and (z, w).  U: the order loop's unroll
// factor (the fit's evaluation kernels pick it by their pixels per thread).
template <int U = 2, typename Q4>
LMB_HD void order_sum_jac_pair(const PairIn& in, const Q4* rec, int nmax,
                               PairSums& A) {
  const f2 z2 = pk(0.f, 0.f), m1 = pk(-1.f, -1.f);
  const cplx<f2> zero = mk(z2, z2);
  for (int c = 0; c < 3; ++c) {
    A.s[c] = zero;
    A.t[c] = zero;
    A.u[c] = zero;
    A.a[c] = zero;
    A.p[c] = zero;
  }
  f2 pim1 = z2, pi = pk(1.f, 1.f), nd = m1;  // nd = -Delta
  f2 dpim1 = z2, dpi = z2, ndd = z2;         // d/ds
  cplx<f2> h2 = in.hm1, h1 = in.h0, hp2 = zero, hp1 = zero;
  const f2 sv = in.sv, ikr = in.ikr, mkr = in.mkr;
#pragma unroll U
  for (int n = 1; n <= nmax; ++n) {
    const Q4* r = rec + PAIR_QUADS * n;
    f2 v[PAIR_VALUES];
#pragma unroll
    for (int j = 0; j < PAIR_QUADS; ++j) {
      const Q4 q = r[j];
      v[2 * j] = pk(q.x, q.y);
      v[2 * j + 1] = pk(q.z, q.w);
    }
    const f2 fn = v[0], cn = v[1], tns = v[2], fns = v[3];
    // Wiscombe pi, tau and their s tangents
    const f2 spi = pmul(sv, pi);
    const f2 w = padd(nd, spi);
    const f2 tau = pfma(fn, w, pim1);
    const f2 ndn = pfma(cn, w, spi);
    const f2 dspi = pfma(sv, dpi, pi);
    const f2 wd = padd(ndd, dspi);
    const f2 dtau = pfma(fn, wd, dpim1);
    const f2 nddn = pfma(cn, wd, dspi);
    // Riccati-Bessel recurrences (signed as described above)
    const f2 a2 = pmul(tns, ikr), a1 = pmul(fns, ikr);
    const cplx<f2> h = mk(pfma(a2, h1.re, h2.re), pfma(a2, h1.im, h2.im));
    const cplx<f2> dh = mk(pfma(a1, h.re, h1.re), pfma(a1, h.im, h1.im));
    // kr tangents: the chain-rule terms -a2 h'/kr and -a1 h/kr are folded
    // into the recurrence coefficients' arguments (a (hp - h/kr))
    const cplx<f2> hp = mk(pfma(a2, pfma(mkr, h1.re, hp1.re), hp2.re),
                           pfma(a2, pfma(mkr, h1.im, hp1.im), hp2.im));
    const cplx<f2> dhp = mk(pfma(a1, pfma(mkr, h.re, hp.re), hp1.re),
                            pfma(a1, pfma(mkr, h.im, hp.im), hp1.im));
    // value and the s tangent
    {
      const cplx<f2> X = pcmul(v[4], v[5], v[6], dh);
      const cplx<f2> Y = pcmul(v[7], v[8], v[9], h);
      const cplx<f2> Z = pcmul(v[10], v[11], v[12], h);
      A.s[0] = pacc(A.s[0], pi, Z);
      A.s[1] = pacc(pacc(A.s[1], tau, X), pi, Y);
      A.s[2] = pacc(pacc(A.s[2], pi, X), tau, Y);
      A.u[0] = pacc(A.u[0], dpi, Z);
      A.u[1] = pacc(pacc(A.u[1], dtau, X), dpi, Y);
      A.u[2] = pacc(pacc(A.u[2], dpi, X), dtau, Y);
    }
    // kr tangent
    {
      const cplx<f2> X = pcmul(v[4], v[5], v[6], dhp);
      const cplx<f2> Y = pcmul(v[7], v[8], v[9], hp);
      const cplx<f2> Z = pcmul(v[10], v[11], v[12], hp);
      A.t[0] = pacc(A.t[0], pi, Z);
      A.t[1] = pacc(pacc(A.t[1], tau, X), pi, Y);
      A.t[2] = pacc(pacc(A.t[2], pi, X), tau, Y);
    }
    // a_p
    {
      const cplx<f2> X = pcmul(v[13], v[14], v[15], dh);
      const cplx<f2> Y = pcmul(v[16], v[17], v[18], h);
      const cplx<f2> Z = pcmul(v[19], v[20], v[21], h);
      A.a[0] = pacc(A.a[0], pi, Z);
      A.a[1] = pacc(pacc(A.a[1], tau, X), pi, Y);
      A.a[2] = pacc(pacc(A.a[2], pi, X), tau, Y);
    }
    // n_p
    {
      const cplx<f2> X = pcmul(v[22], v[23], v[24], dh);
      const cplx<f2> Y = pcmul(v[25], v[26], v[27], h);
      const cplx<f2> Z = pcmul(v[28], v[29], v[30], h);
      A.p[0] = pacc(A.p[0], pi, Z);
      A.p[1] = pacc(pacc(A.p[1], tau, X), pi, Y);
      A.p[2] = pacc(pacc(A.p[2], pi, X), tau, Y);
    }
    pim1 = pi;
    pi = pfma(m1, ndn, pi);
    nd = ndn;
    dpim1 = dpi;
    dpi = pfma(m1, nddn, dpi);
    ndd = nddn;
    h2 = h1;
    h1 = h;
    hp2 = hp1;
    hp1 = hp;
  }
}

// The value-only loop (field and hologram) for two pixels at once, with
// the signs and records of order_sum_jac_pair restricted to the value:
// per order PAIRV_VALUES values, each duplicated into both lanes:
//   0 n, 1 c_n, 2 (-1)^n (2n-1), 3 (-1)^{n+1} n,
//   4 sig alpha, 7 -s beta, 10 s n(n+1) alpha (each re, im, -im); 13 unused.
enum { PAIRV_VALUES = 14, PAIRV_QUADS = PAIRV_VALUES / 2 };

struct PairSumsV {
  cplx<f2> s[3];
};

template <typename Q4>
LMB_HD void order_sum_pair(const PairIn& in, const Q4* rec, int nmax,
                           PairSumsV& A) {
  const f2 z2 = pk(0.f, 0.f), m1 = pk(-1.f, -1.f);
  const cplx<f2> zero = mk(z2, z2);
  for (int c = 0; c < 3; ++c) A.s[c] = zero;
  f2 pim1 = z2, pi = pk(1.f, 1.f), nd = m1;
  cplx<f2> h2 = in.hm1, h1 = in.h0;
  const f2 sv = in.sv, ikr = in.ikr;
#pragma unroll 2
  for (int n = 1; n <= nmax; ++n) {
    const Q4* r = rec + PAIRV_QUADS * n;
    f2 v[PAIRV_VALUES];
#pragma unroll
    for (int j = 0; j < PAIRV_QUADS; ++j) {
      const Q4 q = r[j];
      v[2 * j] = pk(q.x, q.y);
      v[2 * j + 1] = pk(q.z, q.w);
    }
    const f2 fn = v[0], cn = v[1], tns = v[2], fns = v[3];
    const f2 spi = pmul(sv, pi);
    const f2 w = padd(nd, spi);
    const f2 tau = pfma(fn, w, pim1);
    const f2 ndn = pfma(cn, w, spi);
    const f2 a2 = pmul(tns, ikr), a1 = pmul(fns, ikr);
    const cplx<f2> h = mk(pfma(a2, h1.re, h2.re), pfma(a2, h1.im, h2.im));
    const cplx<f2> dh = mk(pfma(a1, h.re, h1.re), pfma(a1, h.im, h1.im));
    const cplx<f2> X = pcmul(v[4], v[5], v[6], dh);
    const cplx<f2> Y = pcmul(v[7], v[8], v[9], h);
    const cplx<f2> Z = pcmul(v[10], v[11], v[12], h);
    A.s[0] = pacc(A.s[0], pi, Z);
    A.s[1] = pacc(pacc(A.s[1], tau, X), pi, Y);
    A.s[2] = pacc(pacc(A.s[2], pi, X), tau, Y);
    pim1 = pi;
    pi = pfma(m1, ndn, pi);
    nd = ndn;
    h2 = h1;
    h1 = h;
  }
}

// One lane of the value sums, with order_sum's parity unfolding.
LMB_HD Sums<float> pair_lane_value(const PairSumsV& P, int lane, float sg) {
  Sums<float> S;
  cplx<float> t[3];
  for (int c = 0; c < 3; ++c)
    t[c] = lane ? mk(P.s[c].re.y, P.s[c].im.y) : mk(P.s[c].re.x, P.s[c].im.x);
  S.s0 = t[0];
  S.s1 = t[1];
  S.s2 = sg * t[2];
  return S;
}

// One lane of the packed sums as the scalar loop's JacSums, with the same
// parity unfolding and s -> mu conversion at the end of order_sum_jac.
LMB_HD JacSums<float> pair_lane(const PairSums& P, int lane, float sg) {
  JacSums<float> A;
  for (int c = 0; c < 3; ++c) {
#define LMB_LANE(dst, src)                                   \
  dst[c] = lane ? mk(src[c].re.y, src[c].im.y) : mk(src[c].re.x, src[c].im.x)
    LMB_LANE(A.s, P.s);
    LMB_LANE(A.t, P.t);
    LMB_LANE(A.u, P.u);
    LMB_LANE(A.a, P.a);
    LMB_LANE(A.p, P.p);
#undef LMB_LANE
  }
  A.s[2] = sg * A.s[2];
  A.a[2] = sg * A.a[2];
  A.p[2] = sg * A.p[2];
  A.t[2] = sg * A.t[2];
  A.u[0] = (-sg) * A.u[0];
  A.u[1] = (-sg) * A.u[1];
  A.u[2] = -A.u[2];
  return A;
}

LMB_HD PairIn pair_in(const Geometry<float>& g0, const Geometry<float>& g1) {
  PairIn in;
  in.sv = pk(g0.s1mu, g1.s1mu);
  in.ikr = pk(g0.ikrs, g1.ikrs);
  in.mkr = pk(-g0.ikr, -g1.ikr);
  in.hm1 = mk(pk(g0.hm1.re, g1.hm1.re), pk(g0.hm1.im, g1.hm1.im));
  in.h0 = mk(pk(g0.h0.re, g1.h0.re), pk(g0.h0.im, g1.h0.im));
  return in;
}

// Dual numbers over the three displacement coordinates (kx, ky, kz).
template <typename R>
struct dr3 {
  R v, g[3];
};
template <typename R>
struct dc3 {
  cplx<R> v, g[3];
};
template <typename R>
LMB_HD dr3<R> dmul(dr3<R> a, dr3<R> b) {
  dr3<R> r;
  r.v = a.v * b.v;
  for (int i = 0; i < 3; ++i) r.g[i] = a.g[i] * b.v + a.v * b.g[i];
  return r;
}
template <typename R>
LMB_HD dc3<R> dmul(dc3<R> a, dr3<R> b) {
  dc3<R> r;
  r.v = b.v * a.v;
  for (int i = 0; i < 3; ++i) r.g[i] = b.v * a.g[i] + b.g[i] * a.v;
  return r;
}
template <typename R>
LMB_HD dc3<R> dmul(dc3<R> a, dc3<R> b) {
  dc3<R> r;
  r.v = a.v * b.v;
  for (int i = 0; i < 3; ++i) r.g[i] = a.g[i] * b.v + a.v * b.g[i];
  return r;
}
template <typename R>
LMB_HD dc3<R> dadd(dc3<R> a, dc3<R> b) {
  dc3<R> r;
  r.v = a.v + b.v;
  for (int i = 0; i < 3; ++i) r.g[i] = a.g[i] + b.g[i];
  return r;
}
template <typename R>
LMB_HD dc3<R> dsub(dc3<R> a, dc3<R> b) {
  dc3<R> r;
  r.v = a.v - b.v;
  for (int i = 0; i < 3; ++i) r.g[i] = a.g[i] - b.g[i];
  return r;
}

// Field of one particle and its derivatives with respect to the particle
// parameters, in the order x_p, y_p, z_p, a_p, n_p, k_p:
//   e[c]        field component c (Cartesian)
//   de[j][c]    d e[c] / d param_j
// Forward mode (dual numbers).  The kernels need only the hologram's
// derivatives and use holo_jac_reverse; this form gives the field's own
// derivatives and is the reference the reverse form is checked against.
template <typename R>
LMB_HD void epilogue_jac(const Geometry<R>& g, const JacSums<R>& A, R k,
                         cplx<R>* e, cplx<R> (*de)[3]) {
  const R ikr = g.ikr, mu = g.mu, st = g.sint, cp = g.cosp, sp = g.sinp;
  // d kr / d(kx, ky, kz)
  const R krg[3] = {st * cp, st * sp, mu};
  dr3<R> IKR, MU, ST, CP, SP;
  IKR.v = ikr;
  MU.v = mu;
  ST.v = st;
  CP.v = cp;
  SP.v = sp;
  for (int i = 0; i < 3; ++i) IKR.g[i] = -ikr * ikr * krg[i];
  MU.g[0] = -mu * krg[0] * ikr;
  MU.g[1] = -mu * krg[1] * ikr;
  MU.g[2] = st * st * ikr;
  ST.g[0] = cp * mu * mu * ikr;
  ST.g[1] = sp * mu * mu * ikr;
  ST.g[2] = -st * mu * ikr;
  if (g.krho > R(0)) {
    const R ik = R(1) / g.krho;
    CP.g[0] = sp * sp * ik;
    CP.g[1] = -cp * sp * ik;
    SP.g[0] = -cp * sp * ik;
    SP.g[1] = cp * cp * ik;
  } else {
    CP.g[0] = CP.g[1] = SP.g[0] = SP.g[1] = R(0);
  }
  CP.g[2] = SP.g[2] = R(0);
  // phase-reduced sums as duals: S' = t dkr + u dmu
  dc3<R> S[3];
  for (int c = 0; c < 3; ++c) {
    S[c].v = A.s[c];
    for (int i = 0; i < 3; ++i) S[c].g[i] = krg[i] * A.t[c] + MU.g[i] * A.u[c];
  }
  // The phase e^{i(sigma kr - k z_p)}: its kz tangent also carries the
  // explicit -k z_p (kz = k (z_p - z)), so that d/dz_p = k d/dkz.  The
  // combined rate sigma mu - 1 equals -(1 - |mu|) when sigma = sign(mu),
  // which is formed without cancellation.
  dc3<R> PH;
  PH.v = g.phase;
  {
    const cplx<R> ip = g.sigma * mul_i(g.phase);
    PH.g[0] = krg[0] * ip;
    PH.g[1] = krg[1] * ip;
    const R rate = (g.sigma != R(0) && g.sigma == g.smu) ? -g.s1mu
                                                          : g.sigma * mu - R(1);
    PH.g[2] = rate * mul_i(g.phase);
  }
  // geometric factors
  const dr3<R> G0 = dmul(dmul(CP, ST), dmul(IKR, IKR));
  const dr3<R> G1 = dmul(CP, IKR);
  const dr3<R> G2 = dmul(SP, IKR);
  const dc3<R> es0 = dmul(S[0], G0), es1 = dmul(S[1], G1), es2 = dmul(S[2], G2);
  const dc3<R> c0 = dsub(dadd(dmul(es0, dmul(ST, CP)), dmul(es1, dmul(MU, CP))),
                         dmul(es2, SP));
  const dc3<R> c1 = dadd(dadd(dmul(es0, dmul(ST, SP)), dmul(es1, dmul(MU, SP))),
                         dmul(es2, CP));
  const dc3<R> c2 = dsub(dmul(es0, MU), dmul(es1, ST));
  const dc3<R> E[3] = {dmul(c0, PH), dmul(c1, PH), dmul(c2, PH)};
  // material sums share the value geometry
  const R g0 = G0.v, g1 = G1.v, g2 = G2.v;
  for (int c = 0; c < 3; ++c) {
    e[c] = E[c].v;
    // kx = k (x - x_p), ky = k (y - y_p), kz = k (z_p - z)
    de[0][c] = (-k) * E[c].g[0];
    de[1][c] = (-k) * E[c].g[1];
    de[2][c] = k * E[c].g[2];
  }
  cplx<R> ma[3], mn[3];
  {
    const cplx<R> a0 = g0 * A.a[0], a1 = g1 * A.a[1], a2 = g2 * A.a[2];
    const cplx<R> n0 = g0 * A.p[0], n1 = g1 * A.p[1], n2 = g2 * A.p[2];
    ma[0] = (st * cp) * a0 + (mu * cp) * a1 - sp * a2;
    ma[1] = (st * sp) * a0 + (mu * sp) * a1 + cp * a2;
    ma[2] = mu * a0 - st * a1;
    mn[0] = (st * cp) * n0 + (mu * cp) * n1 - sp * n2;
    mn[1] = (st * sp) * n0 + (mu * sp) * n1 + cp * n2;
    mn[2] = mu * n0 - st * n1;
  }
  for (int c = 0; c < 3; ++c) {
    de[3][c] = g.phase * ma[c];
    de[4][c] = g.phase * mn[c];
    de[5][c] = mul_i(de[4][c]);
  }
}

// Hologram and its six parameter derivatives in reverse mode: the same
// quantities as epilogue_jac followed by dH_j = 2 Re(conj(E + x) dE_j), at a
// third of the arithmetic.  Forward: E_c = phase * sum_k q_ck G_k S_k with
// the geometric factors G = (cos(phi) sin(theta)/kr^2, cos(phi)/kr,
// sin(phi)/kr) and the Cartesian projection q_ck(theta, phi).  Reverse:
// from Ebar = 2 (E + x) the adjoints of the projected sums, of the sums
// S_k (which carry the a_p, n_p, k_p columns, since the material sums enter
// where S_k does) and of the real geometric variables, which the chain rule
// then maps onto (kx, ky, kz).  The phase's kz rate and the on-axis branch
// are those of epilogue_jac.  For a complex z, zbar = dH/dRe z + i dH/dIm z.
// With kAberr the particle's field carries a phase e^{i Phi} (spherical
// aberration, theory/Aberrated.py:62-85): |E e^{i Phi} + x|^2 = |E + w x|^2
// with w = e^{-i Phi}, so w replaces the unit reference wave, and
// *hphi = dH/dPhi = 2 Im(conj(E_x + w) w) for the caller's chain rule.
template <typename R, bool kAberr = false>
LMB_HD void holo_jac_reverse(const Geometry<R>& g, const JacSums<R>& A, R k,
                             R* H, R* dH, cplx<R> w = mk(R(1), R(0)),
                             R* hphi = nullptr) {
  const R ikr = g.ikr, mu = g.mu, st = g.sint, cp = g.cosp, sp = g.sinp;
  const R ikr2 = ikr * ikr;
  // forward
  const R G[3] = {cp * st * ikr2, cp * ikr, sp * ikr};
  cplx<R> es[3];
  for (int j = 0; j < 3; ++j) es[j] = G[j] * A.s[j];
  const R q00 = st * cp, q01 = mu * cp, q10 = st * sp, q11 = mu * sp;
  cplx<R> c[3];
  c[0] = q00 * es[0] + q01 * es[1] - sp * es[2];
  c[1] = q10 * es[0] + q11 * es[1] + cp * es[2];
  c[2] = mu * es[0] - st * es[1];
  cplx<R> et[3];
  for (int j = 0; j < 3; ++j) et[j] = g.phase * c[j];
  if constexpr (kAberr) {
    et[0] = et[0] + w;
    *hphi = R(2) * (conj(et[0]) * w).im;
  } else {
    et[0].re += R(1);
  }
  *H = norm2(et[0]) + norm2(et[1]) + norm2(et[2]);
  // reverse: E = phase c
  cplx<R> cb[3], phb = mk(R(0), R(0));
  const cplx<R> cph = conj(g.phase);
  for (int j = 0; j < 3; ++j) {
    const cplx<R> eb = R(2) * et[j];
    cb[j] = cph * eb;
    phb = phb + eb * conj(c[j]);
  }
  const cplx<R> zp = conj(phb) * g.phase;
  const R thb = -zp.im;  // d/dtheta of phase = i phase
  // c = q es
  cplx<R> esb[3];
  esb[0] = q00 * cb[0] + q10 * cb[1] + mu * cb[2];
  esb[1] = q01 * cb[0] + q11 * cb[1] - st * cb[2];
  esb[2] = cp * cb[1] - sp * cb[0];
  auto re_dot = [](cplx<R> a, cplx<R> b) { return a.re * b.re + a.im * b.im; };
  const R q00b = re_dot(cb[0], es[0]), q01b = re_dot(cb[0], es[1]);
  const R q02b = re_dot(cb[0], es[2]);  // coefficient -sp
  const R q10b = re_dot(cb[1], es[0]), q11b = re_dot(cb[1], es[1]);
  const R q12b = re_dot(cb[1], es[2]);  // coefficient cp
  const R q20b = re_dot(cb[2], es[0]), q21b = re_dot(cb[2], es[1]);  // mu, -st
  // es = G S
  cplx<R> sb[3];
  R Gb[3];
  for (int j = 0; j < 3; ++j) {
    sb[j] = G[j] * esb[j];
    Gb[j] = re_dot(esb[j], A.s[j]);
  }
  R krb = 0, mub = 0, da = 0, dn = 0, dk = 0;
  for (int j = 0; j < 3; ++j) {
    krb += re_dot(sb[j], A.t[j]);
    mub += re_dot(sb[j], A.u[j]);
    da += re_dot(sb[j], A.a[j]);
    dn += re_dot(sb[j], A.p[j]);
    dk += sb[j].im * A.p[j].re - sb[j].re * A.p[j].im;  // Re(conj(sb) i p)
  }
  // real geometric variables
  R stb = q00b * cp + q10b * sp - q21b + Gb[0] * cp * ikr2;
  R cpb = q00b * st + q01b * mu + q12b + Gb[0] * st * ikr2 + Gb[1] * ikr;
  R spb = q10b * st + q11b * mu - q02b + Gb[2] * ikr;
  mub += q01b * cp + q11b * sp + q20b;
  const R ikrb = Gb[0] * R(2) * cp * st * ikr + Gb[1] * cp + Gb[2] * sp;
  // chain to (kx, ky, kz)
  const R krg[3] = {st * cp, st * sp, mu};
  const R dmu[3] = {-mu * krg[0] * ikr, -mu * krg[1] * ikr, st * st * ikr};
  const R dst[3] = {cp * mu * mu * ikr, sp * mu * mu * ikr, -st * mu * ikr};
  R dcp[3] = {R(0), R(0), R(0)}, dsp[3] = {R(0), R(0), R(0)};
  if (g.krho > R(0)) {
    const R ik = R(1) / g.krho;
    dcp[0] = sp * sp * ik;
    dcp[1] = -cp * sp * ik;
    dsp[0] = -cp * sp * ik;
    dsp[1] = cp * cp * ik;
  }
  const R rate = (g.sigma != R(0) && g.sigma == g.smu) ? -g.s1mu
                                                       : g.sigma * mu - R(1);
  const R dth[3] = {g.sigma * krg[0], g.sigma * krg[1], rate};
  R dk3[3];
  for (int i = 0; i < 3; ++i)
    dk3[i] = (krb - ikrb * ikr2) * krg[i] + mub * dmu[i] + stb * dst[i] +
             cpb * dcp[i] + spb * dsp[i] + thb * dth[i];
  dH[0] = (-k) * dk3[0];
  dH[1] = (-k) * dk3[1];
  dH[2] = k * dk3[2];
  dH[3] = da;
  dH[4] = dn;
  dH[5] = dk;
}

// Spherical aberration in the fits (theory/Aberrated.py:62-79): the phase
// Phi = c r^4 / (r^2 + z_p^2)^2 of a particle's field at a pixel, returned
// as w = e^{-i Phi} (the reference wave as the aberrated field sees it),
// with dPhi/d(x_p, y_p, z_p) in dphi; (dx, dy) is the pixel minus the
// particle, zp the particle's height:
//   dPhi/dx_p = -4 c r^2 z_p^2 dx / (r^2 + z_p^2)^3 (and y alike),
//   dPhi/dz_p = -4 c r^4 z_p / (r^2 + z_p^2)^3.
template <typename R>
LMB_HD cplx<R> aberration_wave(double c, double dx, double dy, double zp,
                               R* dphi) {
  const double rsq = dx * dx + dy * dy;
  const double z2 = zp * zp;
  const double den = rsq + z2;
  if (!(den > 0.)) {
    dphi[0] = dphi[1] = dphi[2] = R(0);
    return mk(R(1), R(0));
  }
  const double q = rsq / den;
  const double phi = c * q * q;
  const double t = 4. * c * q / (den * den);  // 4 c r^2 / (r^2 + z_p^2)^3
  dphi[0] = R(-t * z2 * dx);
  dphi[1] = R(-t * z2 * dy);
  dphi[2] = R(-t * rsq * zp);
  return conj(cis(R(reduce_2pi(phi))));
}

// Hologram from the total scattered field: |E + x|^2 = |E|^2 + 2 Re(E_x) + 1
template <typename R>
LMB_HD R intensity(const cplx<R>* e) {
  return norm2(e[0]) + norm2(e[1]) + norm2(e[2]) + R(2) * e[0].re + R(1);
}

// ---------------------------------------------------------------------------
// Error bound of an FP32 hologram pixel, for the FP64 re-summation of the
// pixels where FP32 cannot reach HOLO_TOL.
//
// The FP32 field of one particle at a pixel (phase in FP64, as the field
// kernels form it) differs from its FP64 value by at most about
//   HOLO_FIELD_REL |E_p| + HOLO_FIELD_FLOOR A_p / kr,
// where A_p = sum_n (n + 1/2)(|a_n| + |b_n|) is the particle's partial-wave
// amplitude and A_p / kr the size of the terms of its sums at the pixel.
// The first term is the relative error of the coefficient records and the
// recurrences (a few ulp of the field where it is large, e.g. on the axis
// of a big sphere that focuses the light), the second the rounding left
// where the sums cancel.  Measured on the CPU build of the packed loop over
// 21 frames of 1280x1024 px with 3-16 spheres each (a_p 0.4-3 um, n_p
// 1.38-1.70, z_p 50-600 px and at least 10 px above the sphere's top): the
// actual hologram error is at most 0.59 of the bound below, the bound
// exceeds HOLO_TOL on 0.06-1.1 % of the pixels, and the largest error left
// on the others is 8.5e-6.  Since dH = 2 Re(conj(E + x) dE), the hologram
// is off by at most
//   2 sqrt(H) sum_p (HOLO_FIELD_REL |E_p| + HOLO_FIELD_FLOOR A_p / kr),
// and pixels where that exceeds HOLO_TOL are summed again in FP64.
#define HOLO_FIELD_REL 3e-6f
#define HOLO_FIELD_FLOOR 1e-7f
#define HOLO_TOL 2e-5f

// (n + 1/2)(|a_n| + |b_n|): order n's share of A_p (FP32: the bound needs
// no more).
LMB_HD float order_amplitude(const cplx<double>* ab, int n) {
  const float a2 = norm2(mk(float(ab[0].re), float(ab[0].im)));
  const float b2 = norm2(mk(float(ab[1].re), float(ab[1].im)));
  return (float(n) + 0.5f) * (approx_sqrt(a2) + approx_sqrt(b2));
}

// Per-pixel accumulation of the bound over the particles: m1 += |E_p|,
// m0 += A_p / kr.
LMB_HD void holo_bound_add(const cplx<float>* ep, float amp, float ikr,
                           float& m1, float& m0) {
  m1 += approx_sqrt(norm2(ep[0]) + norm2(ep[1]) + norm2(ep[2]));
  m0 += amp * ikr;
}

// True when the FP32 value h may be off by more than HOLO_TOL.
LMB_HD bool holo_needs_fp64(float h, float m1, float m0) {
  const float bound =
      2.f * sqrtf(fmaxf(h, 0.f)) * (HOLO_FIELD_REL * m1 + HOLO_FIELD_FLOOR * m0);
  return bound > HOLO_TOL;
}

}  // namespace lmb
