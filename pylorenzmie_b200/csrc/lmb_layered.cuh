// FP64 Mie coefficients of a multilayer (core-shell) sphere, with
// forward-mode tangents.
//
// Algorithm of lib/obsolete/sphere_coefficients.py:65-215 (Yang, Appl. Opt.
// 42, 1710 (2003); equation numbers of Pena & Pal (2009)): per layer the
// zero-start downward recurrence of D1 at z1 = m_l x_l and z2 = m_l x_{l-1}
// from n_max+1 (:129-131, :151-153), the upward psi*zeta / D3 recurrences
// (:133-138, :156-166), the Q ratios (:169-173) and the Ha/Hb recurrences
// across layers (:176-189); the medium's psi, zeta, D3 (:192-207) and
// Eqs. (5)/(6) (:209-215).  n_max follows wiscombe_yang over all layers
// (:40-62, its list handling repaired as in the oracle).
//
// Tangents: d/ds with every radius scaled by s (radius fractions fixed), and
// d/dm_L for the outer layer's relative index (a_n, b_n are holomorphic in
// it).  Then d/da_p = (1/a_p) d/ds and d/dn_p = (1/n_m) d/dm_L, the same
// layout as the homogeneous sphere's derivatives, so every field and fit
// kernel consumes layered spheres unchanged.
#pragma once

#include "lmb_mie.cuh"

namespace lmb {

enum { LMB_MAX_LAYERS = 8 };

// complex value with two complex tangents
struct dz {
  zd v, s, m;
};

LMB_HD dz dconst(zd v) {
  dz r;
  r.v = v;
  r.s = mk(0., 0.);
  r.m = mk(0., 0.);
  return r;
}
LMB_HD dz operator+(dz a, dz b) { return dz{a.v + b.v, a.s + b.s, a.m + b.m}; }
LMB_HD dz operator-(dz a, dz b) { return dz{a.v - b.v, a.s - b.s, a.m - b.m}; }
LMB_HD dz operator*(dz a, dz b) {
  return dz{a.v * b.v, a.s * b.v + a.v * b.s, a.m * b.v + a.v * b.m};
}
LMB_HD dz operator*(zd c, dz a) { return dz{c * a.v, c * a.s, c * a.m}; }
LMB_HD dz operator*(double c, dz a) { return dz{c * a.v, c * a.s, c * a.m}; }
LMB_HD dz operator+(dz a, double c) { return dz{a.v + c, a.s, a.m}; }
LMB_HD dz dinv(dz a) {
  const zd i = recip(a.v);
  const zd i2 = -(i * i);
  return dz{i, i2 * a.s, i2 * a.m};
}
LMB_HD dz operator/(dz a, dz b) { return a * dinv(b); }
LMB_HD dz operator/(double c, dz b) { return c * dinv(b); }
LMB_HD dz operator-(double c, dz a) { return dz{c - a.v, -a.s, -a.m}; }
// e^{i c z}
LMB_HD dz dexpi(double c, dz z) {
  const double e = exp(-c * z.v.im);
  const zd w = e * cis(c * z.v.re);
  const zd d = mk(0., c) * w;
  return dz{w, d * z.s, d * z.m};
}

// n_max over the layers, lib/obsolete/sphere_coefficients.py:40-62 with
// scalar max over the per-layer |x_l m_l| and |x_{l+1} m_l| (roll by -1).
LMB_HD int wiscombe_yang_layers(const double* x, const zd* m, int L) {
  const double xl = fabs(x[L - 1]);
  double ns;
  if (xl <= 8.)
    ns = floor(xl + 4. * cbrt(xl) + 1.);
  else if (xl <= 4200.)
    ns = floor(xl + 4.05 * cbrt(xl) + 2.);
  else
    ns = floor(xl + 4. * cbrt(xl) + 2.);
  double best = ns;
  for (int l = 0; l < L; ++l) {
    const double a = hypot(x[l] * m[l].re, x[l] * m[l].im);
    const int r = (l + 1) % L;
    const double b = hypot(x[r] * m[l].re, x[r] * m[l].im);
    if (a > best) best = a;
    if (b > best) best = b;
  }
  return (int)best;
}

struct LayeredScalars {
  int L, nmax;
  double k, n_m, a_out;
  double x[LMB_MAX_LAYERS];
  zd m[LMB_MAX_LAYERS];
};

LMB_HD LayeredScalars layered_setup(const double* radii, const double* idx,
                                    int L, double n_m, double wavelength) {
  LayeredScalars s;
  s.L = L;
  s.n_m = n_m;
  s.k = 2. * 3.141592653589793 * n_m / wavelength;
  for (int l = 0; l < L; ++l) {
    s.x[l] = s.k * radii[l];
    s.m[l] = mk(idx[2 * l] / n_m, idx[2 * l + 1] / n_m);
  }
  s.a_out = radii[L - 1];
  s.nmax = wiscombe_yang_layers(s.x, s.m, L);
  return s;
}

// zero-start downward D1 at z from n_max+1 into d[0..nmax] (dual)
LMB_HD void layered_d1_down(dz z, int nmax, dz* d) {
  dz cur = dconst(mk(0., 0.));
  const dz iz = dinv(z);  // n / z = n * (1/z), the loop's invariant
  for (int n = nmax + 1; n > 0; --n) {
    const dz nz = double(n) * iz;
    cur = nz - dinv(cur + nz);
    if (n - 1 <= nmax) d[n - 1] = cur;
  }
}

// Ha, Hb of the outermost layer after the core and all shells.
//   d1a, d1b: scratch of nmax+1 duals each; ha, hb: nmax+1 duals (output)
// Runs on one thread; with two lanes available the caller may split the
// two downward recurrences (see block_layered_ab).
LMB_HD void layered_core(const LayeredScalars& s, dz* d1a, dz* ha, dz* hb) {
  const int L = s.L;
  dz z1;
  z1.v = s.x[0] * s.m[0];
  z1.s = z1.v;
  z1.m = (L == 1) ? mk(s.x[0], 0.) : mk(0., 0.);
  layered_d1_down(z1, s.nmax, d1a);
  for (int n = 0; n <= s.nmax; ++n) {
    ha[n] = d1a[n];
    hb[n] = d1a[n];
  }
}

// Constants of shell ii >= 1: the layer's arguments z1 = m_ii x_ii,
// z2 = m_ii x_{ii-1}, its index and its inner neighbour's (with the outer
// layer's index tangent), and the starting values of the upward
// recurrences.
struct ShellSetup {
  dz z1, z2, mi, mo;
  double xr2;
};

LMB_HD ShellSetup layered_shell_setup(const LayeredScalars& s, int ii) {
  const int L = s.L;
  const bool outer = (ii == L - 1);
  ShellSetup h;
  h.z1.v = s.x[ii] * s.m[ii];
  h.z1.s = h.z1.v;
  h.z1.m = outer ? mk(s.x[ii], 0.) : mk(0., 0.);
  h.z2.v = s.x[ii - 1] * s.m[ii];
  h.z2.s = h.z2.v;
  h.z2.m = outer ? mk(s.x[ii - 1], 0.) : mk(0., 0.);
  h.mi = dconst(s.m[ii]);
  if (outer) h.mi.m = mk(1., 0.);
  h.mo = dconst(s.m[ii - 1]);  // the inner neighbour is never the outer layer
  const double xr = s.x[ii - 1] / s.x[ii];
  h.xr2 = xr * xr;  // independent of the radius scale
  return h;
}

// The upward recurrence of one argument z of a shell (z1 or z2) for
// n = 1..nmax: psi*zeta (Eq. (13)) and D3 (Eq. (14)), given D1 at z;
// stores D3 in d3[0..nmax].  The only serial chain of a shell: the ratio
// Q (Eq. (15)) follows from the stored D1, D3 order by order
// (layered_q_ratio, layered_q_product).
LMB_HD void layered_d3_up(dz z, int nmax, const dz* d1, dz* d3) {
  const zd ii1 = mk(0., 1.);
  dz pz = 0.5 * (1. - dexpi(2., z));
  dz cur = dconst(ii1);
  d3[0] = cur;
  const dz iz = dinv(z);
  for (int n = 1; n <= nmax; ++n) {
    const dz nz = double(n) * iz;
    pz = pz * ((nz - d1[n - 1]) * (nz - cur));
    cur = d1[n] + ii1 * dinv(pz);
    d3[n] = cur;
  }
}

// The factor of order n >= 1 in Q_n = Q_{n-1} * r_n (Eq. (15)):
//   r_n = (x_{l-1}/x_l)^2 (z1 D1_n(z1) + n)(n - z1 D3_{n-1}(z1))
//                       / ((z2 D1_n(z2) + n)(n - z2 D3_{n-1}(z2))).
// Orders are independent.
LMB_HD dz layered_q_ratio(const ShellSetup& h, int n, const dz* d1a,
                          const dz* d1b, const dz* d3a, const dz* d3b) {
  const double fn = double(n);
  const dz num = (h.z1 * d1a[n] + fn) * (fn - h.z1 * d3a[n - 1]);
  const dz den = (h.z2 * d1b[n] + fn) * (fn - h.z2 * d3b[n - 1]);
  return h.xr2 * (num / den);
}

// Q_n for n = 1..nmax, in place over the factors r_n that q[1..nmax] holds
// on entry, from Q_0 = (e^{-2i z2} - 1) / (e^{-2i z1} - 1).
LMB_HD void layered_q_product(const ShellSetup& h, int nmax, dz* q) {
  dz cur = (dexpi(-2., h.z2) + (-1.)) / (dexpi(-2., h.z1) + (-1.));
  for (int n = 1; n <= nmax; ++n) {
    cur = cur * q[n];
    q[n] = cur;
  }
}

// Ha, Hb of order n >= 1 carried through shell ii (Eqs. (7b), (8b),
// (12)-(15)), in place.  Orders are independent here.
LMB_HD void layered_shell_update(const ShellSetup& h, int n, const dz* d1a,
                                 const dz* d1b, const dz* d3a, const dz* d3b,
                                 const dz* q, dz* ha, dz* hb) {
  {
    const dz g1 = h.mi * ha[n] - h.mo * d1b[n];
    const dz g2 = h.mi * ha[n] - h.mo * d3b[n];
    const dz t = q[n] * g1;
    ha[n] = (g2 * d1a[n] - t * d3a[n]) / (g2 - t);
  }
  {
    const dz g1 = h.mo * hb[n] - h.mi * d1b[n];
    const dz g2 = h.mo * hb[n] - h.mi * d3b[n];
    const dz t = q[n] * g1;
    hb[n] = (g2 * d1a[n] - t * d3a[n]) / (g2 - t);
  }
}

// One shell ii >= 1 given the downward D1 at z1 (d1a) and z2 (d1b):
// upward psi*zeta, D3, Q, and Ha/Hb updated in place for n = 1..nmax, in
// one serial pass (no scratch).  The same recurrences as layered_d3_up,
// layered_q_ratio, layered_q_product and layered_shell_update, which the
// warp-parallel form uses; Q's factors are grouped differently there, so
// the two forms agree to rounding.
LMB_HD void layered_shell_up(const LayeredScalars& s, int ii, const dz* d1a,
                             const dz* d1b, dz* ha, dz* hb) {
  const ShellSetup h = layered_shell_setup(s, ii);
  const zd ii1 = mk(0., 1.);
  dz pza = 0.5 * (1. - dexpi(2., h.z1));
  dz pzb = 0.5 * (1. - dexpi(2., h.z2));
  dz d3a = dconst(ii1), d3b = dconst(ii1);
  dz q = (dexpi(-2., h.z2) + (-1.)) / (dexpi(-2., h.z1) + (-1.));
  ha[0] = dconst(mk(0., 0.));
  hb[0] = dconst(mk(0., 0.));
  const dz iz1 = dinv(h.z1), iz2 = dinv(h.z2);
  for (int n = 1; n <= s.nmax; ++n) {
    const double fn = double(n);
    const dz nz1 = fn * iz1, nz2 = fn * iz2;
    const dz d3a_prev = d3a, d3b_prev = d3b;
    pza = pza * ((nz1 - d1a[n - 1]) * (nz1 - d3a_prev));
    pzb = pzb * ((nz2 - d1b[n - 1]) * (nz2 - d3b_prev));
    d3a = d1a[n] + ii1 * dinv(pza);
    d3b = d1b[n] + ii1 * dinv(pzb);
    const dz num = (h.z1 * d1a[n] + fn) * (fn - h.z1 * d3a_prev);
    const dz den = (h.z2 * d1b[n] + fn) * (fn - h.z2 * d3b_prev);
    q = h.xr2 * (q * num / den);
    {
      const dz g1 = h.mi * ha[n] - h.mo * d1b[n];
      const dz g2 = h.mi * ha[n] - h.mo * d3b;
      const dz t = q * g1;
      ha[n] = (g2 * d1a[n] - t * d3a) / (g2 - t);
    }
    {
      const dz g1 = h.mo * hb[n] - h.mi * d1b[n];
      const dz g2 = h.mo * hb[n] - h.mi * d3b;
      const dz t = q * g1;
      hb[n] = (g2 * d1a[n] - t * d3a) / (g2 - t);
    }
  }
}

// a_n, b_n and their (a_p, n_p) derivatives from the outer Ha, Hb and the
// medium's psi, zeta (with d/dx); same output layout as mie_coefficient.
LMB_HD void layered_coefficient(const LayeredScalars& s, int n, const dz& ha,
                                const dz& hb, const double* psi,
                                const double* psix, const zd* zeta,
                                const zd* zetax, zd* out, zd* dout) {
  const int L = s.L;
  const double x = s.x[L - 1];
  const zd m = s.m[L - 1];
  const double nx = double(n) / x;
  const double ps = psi[n], ps1 = psi[n - 1];
  // d/ds of psi(x(s)) = psi'(x) x
  const double pss = psix[n] * x, ps1s = psix[n - 1] * x;
  const zd ze = zeta[n], ze1 = zeta[n - 1];
  const zd zes = x * zetax[n], ze1s = x * zetax[n - 1];
  const zd im = recip(m);
  // a_n: fac = Ha/m + n/x
  const zd fa = ha.v * im + nx;
  const zd fa_s = ha.s * im - nx;          // d(n/x)/ds = -n/x
  const zd fa_m = ha.m * im - ha.v * (im * im);
  const zd numa = fa * ps - ps1, dena = fa * ze - ze1;
  const zd ida = recip(dena);
  const zd a = numa * ida;
  // b_n: fac = Hb m + n/x
  const zd fb = hb.v * m + nx;
  const zd fb_s = hb.s * m - nx;
  const zd fb_m = hb.m * m + hb.v;
  const zd numb = fb * ps - ps1, denb = fb * ze - ze1;
  const zd idb = recip(denb);
  const zd b = numb * idb;
  out[0] = a;
  out[1] = b;
  if (dout == 0) return;
  const zd a_s = ((fa_s * ps + fa * pss - ps1s) - a * (fa_s * ze + fa * zes - ze1s)) * ida;
  const zd a_m = (fa_m * ps - a * (fa_m * ze)) * ida;
  const zd b_s = ((fb_s * ps + fb * pss - ps1s) - b * (fb_s * ze + fb * zes - ze1s)) * idb;
  const zd b_m = (fb_m * ps - b * (fb_m * ze)) * idb;
  const double ia = 1. / s.a_out, inm = 1. / s.n_m;
  dout[0] = ia * a_s;
  dout[1] = ia * b_s;
  dout[2] = inm * a_m;
  dout[3] = inm * b_m;
}

}  // namespace lmb
