// FP64 Mie coefficients a_n, b_n of a homogeneous sphere, with forward-mode
// tangents with respect to the sphere radius a_p and index n_p.
//
// Algorithm of theory/Sphere.py:147-226 (Sphere.mie_coefficients): zero-start
// downward recurrence of the logarithmic derivative D1 inside the sphere
// (z = m x, :190-198) and in the medium (z = x, :201-204), upward recurrence of
// psi, zeta, psi*zeta and D3 (:207-214), then Eqs. (5) and (6) of Pena & Pal
// (2009) (:217-224).  n_max follows Sphere.wiscombe_yang (:91-123).
//
// The tangents propagate d/dz through the inside recurrence and d/dx through
// the medium recurrences.  a_n(x, m) is holomorphic in m, so
//   d/da_p = k d/dx,  d/dn_p = (1/n_m) d/dm,  d/dk_p = (i/n_m) d/dm = i d/dn_p.
// n_max is treated as locally constant, as the reference's JAX Jacobian does
// (theory/jaxLorenzMie.py:354-361).
//
// The phases are split so that a warp forms the per-order quotients n/z,
// n/z^2, n/x, n/x^2 on all lanes, runs the two downward recurrences on two
// lanes and then computes a_n, b_n for all n in parallel.  On the
// recurrences' dependent chains each complex reciprocal is conj(w)/|w|^2
// with one reciprocal (recip).
#pragma once

#include "lmb_math.cuh"

namespace lmb {

typedef cplx<double> zd;

// Number of partial waves, theory/Sphere.py:110-123.  For a scalar size
// parameter np.roll(x, -1) is x itself, so n_stop = max(n_s, |x m|).
LMB_HD int wiscombe_yang(double x, zd m) {
  double xl = fabs(x);
  double ns;
  if (xl <= 8.)
    ns = floor(xl + 4. * cbrt(xl) + 1.);
  else if (xl <= 4200.)
    ns = floor(xl + 4.05 * cbrt(xl) + 2.);
  else
    ns = floor(xl + 4. * cbrt(xl) + 2.);
  double xm = hypot(x * m.re, x * m.im);
  double nstop = ns > xm ? ns : xm;
  return (int)nstop;
}

struct MieScalars {
  double k;    // wave number in the medium, rad/um (Sphere.py:174-175)
  double x;    // size parameter k a_p
  double n_m;  // medium index (real part)
  zd m;        // relative index (n_p + i k_p)/n_m
  int nmax;
};

LMB_HD MieScalars mie_setup(double a_p, double n_p, double k_p, double n_m,
                            double wavelength) {
  MieScalars s;
  double k = 2. * 3.141592653589793 / wavelength;
  k *= n_m;
  s.k = k;
  s.x = k * a_p;
  s.n_m = n_m;
  s.m = mk(n_p / n_m, k_p / n_m);
  s.nmax = wiscombe_yang(s.x, s.m);
  return s;
}


// Per-order quotients of the recurrences for order n (1 <= n <= nmax), off
// the recurrences' chains, so that a warp forms them in parallel: inside,
// nz = n/z and nz2 = n/z^2 with z = m x.
LMB_HD void mie_orders_inside(const MieScalars& s, int n, zd* nz, zd* nz2) {
  const zd z = s.x * s.m;
  const zd z2 = z * z;
  nz[n] = double(n) / z;
  nz2[n] = double(n) / z2;
}

// The medium's: nx = n/x, nx2 = n/x^2.
LMB_HD void mie_orders_medium(const MieScalars& s, int n, double* nx,
                              double* nx2) {
  nx[n] = double(n) / s.x;
  nx2[n] = nx[n] / s.x;
}

// D1(x) in the medium (real because x is real), with dD1/dx.
LMB_HD void mie_d1_medium(const MieScalars& s, const double* nx,
                          const double* nx2, double* d1, double* d1x) {
  double d = 0., dx = 0.;
  d1[s.nmax] = d;
  d1x[s.nmax] = dx;
  for (int n = s.nmax; n > 0; --n) {
    const double inv = rcp_d(d + nx[n]);
    const double dw = dx - nx2[n];
    d = nx[n] - inv;
    dx = inv * inv * dw - nx2[n];
    d1[n - 1] = d;
    d1x[n - 1] = dx;
  }
}

// D1(m x) inside the sphere, with dD1/dz at z = m x: the zero-start
// downward recurrence from n_max (Sphere.py), complex.
LMB_HD void mie_d1_inside(const MieScalars& s, const zd* nz, const zd* nz2,
                          zd* d1in, zd* d1inz) {
  zd d = mk(0., 0.), dz = mk(0., 0.);
  d1in[s.nmax] = d;
  d1inz[s.nmax] = dz;
  for (int n = s.nmax; n > 0; --n) {
    const zd inv = recip(d + nz[n]);
    const zd dw = dz - nz2[n];
    d = nz[n] - inv;
    dz = (inv * inv) * dw - nz2[n];
    d1in[n - 1] = d;
    d1inz[n - 1] = dz;
  }
}

// Upward psi (real), zeta, with d/dx; needs the medium D1.
LMB_HD void mie_upward(const MieScalars& s, const double* nxs,
                       const double* nx2s, const double* d1, const double* d1x,
                       double* psi, double* psix, zd* zeta, zd* zetax) {
  const double x = s.x;
  double sx, cx;
#if defined(__CUDA_ARCH__)
  sincos(x, &sx, &cx);
#else
  sx = sin(x);
  cx = cos(x);
#endif
  const zd e1 = mk(cx, sx);           // e^{ix}
  const zd e2 = e1 * e1;              // e^{2ix}
  double p = sx, px = cx;             // psi_0, d/dx
  zd zt = mk(sx, -cx), ztx = e1;      // zeta_0 = -i e^{ix}, d/dx = e^{ix}
  zd pz = 0.5 * (1. - e2);            // psi*zeta, Eq. (18a)
  zd pzx = mk(e2.im, -e2.re);         // d/dx = -i e^{2ix}
  zd d3 = mk(0., 1.), d3x = mk(0., 0.);
  psi[0] = p;
  psix[0] = px;
  zeta[0] = zt;
  zetax[0] = ztx;
  for (int n = 1; n <= s.nmax; ++n) {
    const double nx = nxs[n];
    const double nx2 = nx2s[n];
    const double t1 = nx - d1[n - 1];
    const double t1x = -nx2 - d1x[n - 1];
    const zd t3 = nx - d3;
    const zd t3x = (-nx2) - d3x;
    const double pn = p * t1;
    const double pnx = px * t1 + p * t1x;
    const zd zn = zt * t3;
    const zd znx = ztx * t3 + zt * t3x;
    const zd t13 = t1 * t3;
    const zd t13x = t1x * t3 + t1 * t3x;
    const zd pzn = pz * t13;
    const zd pznx = pzx * t13 + pz * t13x;
    const zd ipz = recip(pzn);
    d3 = d1[n] + mul_i(ipz);
    d3x = d1x[n] - mul_i(pznx * (ipz * ipz));
    p = pn;
    px = pnx;
    zt = zn;
    ztx = znx;
    pz = pzn;
    pzx = pznx;
    psi[n] = p;
    psix[n] = px;
    zeta[n] = zt;
    zetax[n] = ztx;
  }
}

// a_n, b_n (out[0], out[1]) and, if dout != 0, their derivatives
// dout = {da/da_p, db/da_p, da/dn_p, db/dn_p}, for 1 <= n <= nmax.
LMB_HD void mie_coefficient(const MieScalars& s, int n, const zd* d1in,
                            const zd* d1inz, const double* psi,
                            const double* psix, const zd* zeta,
                            const zd* zetax, zd* out, zd* dout) {
  const double x = s.x;
  const zd m = s.m;
  const double nx = double(n) / x;
  const double nx2 = nx / x;
  const zd ha = d1in[n];
  const zd hz = d1inz[n];
  const zd ha_x = m * hz;           // d/dx of D1(m x)
  const zd ha_m = x * hz;           // d/dm of D1(m x)
  const double ps = psi[n], ps1 = psi[n - 1];
  const double psx = psix[n], ps1x = psix[n - 1];
  const zd ze = zeta[n], ze1 = zeta[n - 1];
  const zd zex = zetax[n], ze1x = zetax[n - 1];

  // a_n, Eq. (5): fac = Ha/m + n/x
  const zd im = recip(m);
  const zd fa = ha * im + nx;
  const zd numa = fa * ps - ps1;
  const zd dena = fa * ze - ze1;
  const zd ida = recip(dena);
  const zd a = numa * ida;
  // b_n, Eq. (6): fac = Hb m + n/x
  const zd fb = ha * m + nx;
  const zd numb = fb * ps - ps1;
  const zd denb = fb * ze - ze1;
  const zd idb = recip(denb);
  const zd b = numb * idb;
  out[0] = a;
  out[1] = b;
  if (dout == 0) return;

  const zd fa_x = ha_x * im - nx2;
  const zd fa_m = ha_m * im - ha * (im * im);
  const zd fb_x = ha_x * m - nx2;
  const zd fb_m = ha_m * m + ha;
  const zd a_x = ((fa_x * ps + fa * psx - ps1x) - a * (fa_x * ze + fa * zex - ze1x)) * ida;
  const zd a_m = (fa_m * ps - a * (fa_m * ze)) * ida;
  const zd b_x = ((fb_x * ps + fb * psx - ps1x) - b * (fb_x * ze + fb * zex - ze1x)) * idb;
  const zd b_m = (fb_m * ps - b * (fb_m * ze)) * idb;
  const double inm = 1. / s.n_m;
  dout[0] = s.k * a_x;
  dout[1] = s.k * b_x;
  dout[2] = inm * a_m;
  dout[3] = inm * b_m;
}

}  // namespace lmb
