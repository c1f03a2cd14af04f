// Per-order coefficient records read by the per-pixel loops (lmb_pixel.cuh),
// built from the FP64 Mie coefficients a_n, b_n and their tangents.
//
// The prefactor E_n = i^n (2n+1)/(n(n+1)) of theory/LorenzMie.py:279-281 is
// folded in: alpha_n = i E_n a_n, beta_n = E_n b_n.  Shared by the kernels
// and the CPU test harness so that both stage exactly the same numbers.
#pragma once

#include "lmb_mie.cuh"
#include "lmb_pixel.cuh"

namespace lmb {

LMB_HD zd rot_i(zd z, int k) {  // z * i^k
  switch (k & 3) {
    case 0: return z;
    case 1: return mk(-z.im, z.re);
    case 2: return mk(-z.re, -z.im);
    default: return mk(z.im, -z.re);
  }
}

// Scalar records of order n (2 Quads for the value, JAC_QUADS with the
// tangents).  ab: [2] (a_n, b_n); dab: [4] (da/da_p, db/da_p, da/dn_p,
// db/dn_p) or null.
template <typename R>
LMB_HD void order_record(const zd* ab, const zd* dab, int n, int w, Quad<R>* q) {
  for (int j = 0; j < w; ++j) q[j].x = q[j].y = q[j].z = q[j].w = R(0);
  if (n == 0) return;
  const double fn = double(n);
  const double nn1 = fn * (fn + 1.);
  const double en = (2. * fn + 1.) / nn1;
  const zd al = en * rot_i(ab[0], n + 1);
  const zd be = en * rot_i(ab[1], n);
  q[0].x = R(al.re); q[0].y = R(al.im); q[0].z = R(be.re); q[0].w = R(be.im);
  q[1].x = R(nn1 * al.re); q[1].y = R(nn1 * al.im);
  q[1].z = R(1. + 1. / fn); q[1].w = R(fn);
  if (w == JAC_QUADS) {
    const zd ala = en * rot_i(dab[0], n + 1);
    const zd bea = en * rot_i(dab[1], n);
    const zd aln = en * rot_i(dab[2], n + 1);
    const zd ben = en * rot_i(dab[3], n);
    q[2].x = R(ala.re); q[2].y = R(ala.im); q[2].z = R(bea.re); q[2].w = R(bea.im);
    q[3].x = R(aln.re); q[3].y = R(aln.im); q[3].z = R(ben.re); q[3].w = R(ben.im);
    q[4].x = R(nn1 * ala.re); q[4].y = R(nn1 * ala.im);
    q[4].z = R(nn1 * aln.re); q[4].w = R(nn1 * aln.im);
  }
}

// The PAIR_VALUES values of order n for order_sum_jac_pair (one lane's
// worth; the stager duplicates each into both lanes).
LMB_HD void pair_record(const zd* ab, const zd* dab, int n, float* v) {
  for (int j = 0; j < PAIR_VALUES; ++j) v[j] = 0.f;
  if (n == 0) return;
  const double fn = double(n);
  const double nn1 = fn * (fn + 1.);
  const double en = (2. * fn + 1.) / nn1;
  // s_n = +1, -1, -1, +1 for n = 0, 1, 2, 3 (mod 4); sig_n = (-1)^{n+1} s_n
  const double s = ((n & 3) == 1 || (n & 3) == 2) ? -1. : 1.;
  const double odd = (n & 1) ? 1. : -1.;  // (-1)^{n+1}
  const double sig = odd * s;
  v[0] = float(fn);
  v[1] = float(1. + 1. / fn);
  v[2] = float(-odd * (2. * fn - 1.));
  v[3] = float(odd * fn);
  zd c[9];
  c[0] = sig * (en * rot_i(ab[0], n + 1));
  c[1] = (-s) * (en * rot_i(ab[1], n));
  c[2] = (s * nn1) * (en * rot_i(ab[0], n + 1));
  c[3] = sig * (en * rot_i(dab[0], n + 1));
  c[4] = (-s) * (en * rot_i(dab[1], n));
  c[5] = (s * nn1) * (en * rot_i(dab[0], n + 1));
  c[6] = sig * (en * rot_i(dab[2], n + 1));
  c[7] = (-s) * (en * rot_i(dab[3], n));
  c[8] = (s * nn1) * (en * rot_i(dab[2], n + 1));
  for (int j = 0; j < 9; ++j) {
    v[4 + 3 * j] = float(c[j].re);
    v[5 + 3 * j] = float(c[j].im);
    v[6 + 3 * j] = -float(c[j].im);
  }
}

// Part `part` (0, 1, 2) of the PAIRV_VALUES values of order n for
// order_sum_pair (value only; the first 13 values of pair_record): part 0
// writes v[0..6] (n, c_n, the signed recurrence factors and sig alpha),
// part 1 v[7..9] (-s beta), part 2 v[10..13] (s n(n+1) alpha, and the
// unused v[13] = 0).  The parts let a block stage an order on 3 threads.
LMB_HD void pair_value_part(const zd* ab, int n, int part, float* v) {
  const int lo = part == 0 ? 0 : (part == 1 ? 7 : 10);
  const int hi = part == 0 ? 7 : (part == 1 ? 10 : PAIRV_VALUES);
  for (int j = lo; j < hi; ++j) v[j] = 0.f;
  if (n == 0) return;
  const double fn = double(n);
  const double nn1 = fn * (fn + 1.);
  const double en = (2. * fn + 1.) / nn1;
  const double s = ((n & 3) == 1 || (n & 3) == 2) ? -1. : 1.;
  const double odd = (n & 1) ? 1. : -1.;  // (-1)^{n+1}
  const double sig = odd * s;
  zd c;
  if (part == 0) {
    v[0] = float(fn);
    v[1] = float(1. + 1. / fn);
    v[2] = float(-odd * (2. * fn - 1.));
    v[3] = float(odd * fn);
    c = sig * (en * rot_i(ab[0], n + 1));
  } else if (part == 1) {
    c = (-s) * (en * rot_i(ab[1], n));
  } else {
    c = (s * nn1) * (en * rot_i(ab[0], n + 1));
  }
  const int k = 4 + 3 * part;
  v[k] = float(c.re);
  v[k + 1] = float(c.im);
  v[k + 2] = -float(c.im);
}

// All PAIRV_VALUES values of order n.
LMB_HD void pair_value_record(const zd* ab, int n, float* v) {
  for (int part = 0; part < 3; ++part) pair_value_part(ab, n, part, v);
}

}  // namespace lmb
