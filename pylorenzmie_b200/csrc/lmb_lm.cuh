// Levenberg-Marquardt step logic for one feature, in FP64.
//
// The reference fits with scipy.optimize.least_squares(method='lm')
// (analysis/Optimizer.py:104-113, 221), which runs MINPACK lmder: Moré's
// trust-region Levenberg-Marquardt (J. J. Moré, "The Levenberg-Marquardt
// algorithm: implementation and theory", Lecture Notes in Mathematics 630
// (1978); MINPACK-1 user guide, ANL-80-74 (1980)).  This file restates that
// published algorithm -- the outer/inner loops of lmder, the step-bound
// update, the convergence tests and the lmpar search for the damping
// parameter -- for a problem with at most six unknowns, written against
// the normal equations J^T J, J^T f instead of the QR factors of J:
//   * qrfac with column pivoting  -> pivoted Cholesky of J^T J (R^T R = P^T J^T J P,
//                                    the same pivot rule: largest remaining
//                                    column norm = largest Schur diagonal);
//   * Q^T f (first n)              -> R^{-T} P^T J^T f;
//   * qrsolv                        -> Cholesky of R^T R + P^T D^2 P;
//   * ||R P^T p||                   -> sqrt(p^T R^T R p) in pivoted order.
// These give the same iterates in exact arithmetic.  The per-pixel sums
// J^T J, J^T f and f^T f come from the evaluation kernel.
//
// Settings follow scipy's call of lmder (scipy/optimize/_lsq/least_squares.py,
// call_minpack): factor = 100, mode 1 (x_scale='jac': diag from the column
// norms of J, never decreasing), maxfev = max_nfev.
#pragma once

#include "lmb_math.cuh"

namespace lmb {

enum { LM_NV = 6 };  // x_p, y_p, z_p, a_p, n_p, k_p

// Packed upper-triangular index of (i, j), i <= j, for a 6x6 symmetric matrix.
LMB_HD int sym6(int i, int j) {
  if (i > j) {
    int t = i;
    i = j;
    j = t;
  }
  return i * LM_NV - (i * (i - 1)) / 2 + (j - i);
}

struct LMSettings {
  double ftol, xtol, gtol, factor;
  int maxfev;
};

// Phases of the per-feature state machine.
enum {
  LM_PHASE_INIT = 0,       // ab of the start point not yet computed
  LM_PHASE_FIRST = 1,      // evaluation of the start point pending
  LM_PHASE_TRIAL = 2,      // evaluation of a trial point pending
  LM_PHASE_DONE = 3
};

struct LMState {
  int n;              // number of free variables
  int slot[LM_NV];    // parameter slot (0..5) of each free variable
  int phase, info, iter, nfev, njev, nsing;
  double x[LM_NV];    // current free-variable values
  double p[LM_NV];    // step under trial
  double diag[LM_NV];
  double acnorm[LM_NV];
  double jtf[LM_NV];              // J^T f at x (free variables)
  double jtj[LM_NV * LM_NV];      // J^T J at x (free variables)
  double r[LM_NV * LM_NV];        // pivoted Cholesky factor, row-major
  int ipvt[LM_NV];
  double qtf[LM_NV];
  double delta, par, fnorm, xnorm, gnorm, pnorm, prered, dirder;
  double f2_final;
};

// Sums over the pixels of one feature for one parameter vector.
struct LMEval {
  double f2;
  double jtj[21];  // packed upper over the 6 slots
  double jtf[6];
};

// 1/sqrt(d) for d > 0: the device's reciprocal square root (a few ulp),
// so that a Cholesky pivot's square root and its reciprocal come from one
// operation and the divisions by the pivot become multiplications.
LMB_HD double lm_rsqrt(double d) {
#if defined(__CUDA_ARCH__)
  return rsqrt(d);
#else
  return 1. / sqrt(d);
#endif
}

LMB_HD double enorm(const double* v, int n) {
  double s = 0.;
  for (int i = 0; i < n; ++i) s += v[i] * v[i];
  return sqrt(s);
}

// Extract the free-variable normal equations of an evaluation.
LMB_HD void lm_take(LMState& s, const LMEval& ev) {
  const int n = s.n;
  for (int a = 0; a < n; ++a) {
    s.jtf[a] = ev.jtf[s.slot[a]];
    for (int b = 0; b < n; ++b) s.jtj[a * LM_NV + b] = ev.jtj[sym6(s.slot[a], s.slot[b])];
  }
}

// base[k * stride] for a runtime k with lo <= k < N, and its store, by
// compare-selects over the unrolled indices (see lm_get).
template <int N>
LMB_HD double lm_gets(const double* base, int stride, int k, int lo) {
  double r = base[lo * stride];
#pragma unroll
  for (int l = 0; l < N; ++l)
    if (l > lo) r = k == l ? base[l * stride] : r;
  return r;
}
template <int N>
LMB_HD void lm_puts(double* base, int stride, int k, int lo, double val) {
#pragma unroll
  for (int l = 0; l < N; ++l)
    if (l >= lo && k == l) base[l * stride] = val;
}

// Pivoted Cholesky of J^T J (the qrfac equivalent), column norms, Q^T f,
// for N free variables: MINPACK's qrfac pivot rule (largest remaining
// column norm = largest Schur diagonal), written with N a compile-time
// constant so that the work arrays are indexed by constants (the pivot
// swaps by compare-selects).  The arithmetic, comparisons and swaps are
// those of the loops to n, in the same order.
template <int N>
LMB_HD void lm_factor_n(LMState& s) {
  double w[N * N], r[N * N], rinv[N], jf[N], qt[N];
  int piv[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    jf[i] = s.jtf[i];
#pragma unroll
    for (int j = 0; j < N; ++j) w[i * N + j] = s.jtj[i * LM_NV + j];
  }
#pragma unroll
  for (int j = 0; j < N; ++j) {
    piv[j] = j;
    const double c = w[j * N + j];
    s.acnorm[j] = sqrt(c > 0. ? c : 0.);
  }
#pragma unroll
  for (int i = 0; i < N * N; ++i) r[i] = 0.;
  int nsing = N;
  bool stop = false;
#pragma unroll
  for (int j = 0; j < N; ++j) {
    if (stop) break;
    int kmax = j;
    double best = w[j * N + j];
#pragma unroll
    for (int k = j + 1; k < N; ++k)
      if (w[k * N + k] > best) {
        best = w[k * N + k];
        kmax = k;
      }
    if (kmax != j) {
#pragma unroll
      for (int i = 0; i < N; ++i) {  // columns j and kmax
        const double t = w[i * N + j];
        w[i * N + j] = lm_gets<N>(w + i * N, 1, kmax, j + 1);
        lm_puts<N>(w + i * N, 1, kmax, j + 1, t);
      }
#pragma unroll
      for (int i = 0; i < N; ++i) {  // rows j and kmax
        const double t = w[j * N + i];
        w[j * N + i] = lm_gets<N>(w + i, N, kmax, j + 1);
        lm_puts<N>(w + i, N, kmax, j + 1, t);
      }
#pragma unroll
      for (int i = 0; i < j; ++i) {  // rows of R already formed
        const double t = r[i * N + j];
        r[i * N + j] = lm_gets<N>(r + i * N, 1, kmax, j + 1);
        lm_puts<N>(r + i * N, 1, kmax, j + 1, t);
      }
      int pk = piv[j];
#pragma unroll
      for (int l = 0; l < N; ++l)
        if (l > j && l == kmax) pk = piv[l];
#pragma unroll
      for (int l = 0; l < N; ++l)
        if (l > j && l == kmax) piv[l] = piv[j];
      piv[j] = pk;
    }
    const double d = w[j * N + j];
    if (!(d > 0.)) {
      nsing = j;
      stop = true;
      break;
    }
    const double inv = lm_rsqrt(d);
    rinv[j] = inv;
    r[j * N + j] = d * inv;
#pragma unroll
    for (int k = j + 1; k < N; ++k) r[j * N + k] = w[j * N + k] * inv;
#pragma unroll
    for (int i = j + 1; i < N; ++i)
#pragma unroll
      for (int k = j + 1; k < N; ++k) w[i * N + k] -= r[j * N + i] * r[j * N + k];
  }
  // R^T qtf = P^T J^T f on the nonsingular block; zero beyond it
#pragma unroll
  for (int j = 0; j < N; ++j) {
    if (j >= nsing) {
      qt[j] = 0.;
      continue;
    }
    double sum = lm_gets<N>(jf, 1, piv[j], 0);
#pragma unroll
    for (int i = 0; i < j; ++i) sum -= r[i * N + j] * qt[i];
    qt[j] = sum * rinv[j];
  }
  s.nsing = nsing;
#pragma unroll
  for (int i = 0; i < LM_NV * LM_NV; ++i) s.r[i] = 0.;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    s.ipvt[i] = piv[i];
    s.qtf[i] = qt[i];
#pragma unroll
    for (int j = 0; j < N; ++j) s.r[i * LM_NV + j] = r[i * N + j];
  }
}

LMB_HD void lm_factor(LMState& s) {
  switch (s.n) {
    case 1: lm_factor_n<1>(s); break;
    case 2: lm_factor_n<2>(s); break;
    case 3: lm_factor_n<3>(s); break;
    case 4: lm_factor_n<4>(s); break;
    case 5: lm_factor_n<5>(s); break;
    default: lm_factor_n<6>(s); break;
  }
}

// v[k] and v[k] = val for a runtime k < N, by compare-selects over the
// unrolled indices, so that v can stay in registers.
template <int N>
LMB_HD double lm_get(const double* v, int k) {
  double r = v[0];
#pragma unroll
  for (int l = 1; l < N; ++l) r = k == l ? v[l] : r;
  return r;
}
template <int N>
LMB_HD void lm_put(double* v, int k, double val) {
#pragma unroll
  for (int l = 0; l < N; ++l)
    if (k == l) v[l] = val;
}

// lmpar and its qrsolv for N free variables (the loops of MINPACK's lmpar
// and qrsolv, restated on the normal equations as described above), with
// N a compile-time constant: the loops unroll, and R, the pivots and the
// work arrays are indexed by constants (pivot-indexed accesses by
// compare-selects), so that they can live in registers.  The arithmetic
// and its order are those of the loops to n.
template <int N>
struct LMPar {
  double R[N * N];   // R (upper triangle used), row-major N x N
  double rinv[N];    // 1 / R[j][j] for j < nsing
  double qtf[N], diag[N];
  int piv[N];
  int nsing;
};

// qrsolv equivalent: S = chol(R^T R + D_p^2) (pivoted order, D_p[j] =
// dg[ipvt[j]]), solve S^T S z = R^T qtb, x[ipvt[j]] = z[j].
template <int N>
LMB_HD void lm_qrsolv_n(const LMPar<N>& q, const double* dg, double* x,
                        double* sm, double* sdiag, double* sinv) {
  double m[N * N];
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = i; j < N; ++j) {
      double sum = 0.;
#pragma unroll
      for (int k = 0; k <= i; ++k) sum += q.R[k * N + i] * q.R[k * N + j];
      m[i * N + j] = sum;
    }
#pragma unroll
  for (int j = 0; j < N; ++j) {
    const double d = lm_get<N>(dg, q.piv[j]);
    m[j * N + j] += d * d;
  }
#pragma unroll
  for (int i = 0; i < N * N; ++i) sm[i] = 0.;
  int nsing = N;
  bool stop = false;
#pragma unroll
  for (int j = 0; j < N; ++j) {
    if (stop) break;
    double d = m[j * N + j];
#pragma unroll
    for (int k = 0; k < j; ++k) d -= sm[k * N + j] * sm[k * N + j];
    if (!(d > 0.)) {
      nsing = j;
      stop = true;
      break;
    }
    const double inv = lm_rsqrt(d);
    sinv[j] = inv;
    sm[j * N + j] = d * inv;
#pragma unroll
    for (int i = j + 1; i < N; ++i) {
      double e = m[j * N + i];
#pragma unroll
      for (int k = 0; k < j; ++k) e -= sm[k * N + j] * sm[k * N + i];
      sm[j * N + i] = e * inv;
    }
  }
#pragma unroll
  for (int j = 0; j < N; ++j) {
    sdiag[j] = j < nsing ? sm[j * N + j] : 0.;
    if (j >= nsing) sinv[j] = 0.;
  }
  // rhs = R^T qtb
  double z[N];
#pragma unroll
  for (int j = 0; j < N; ++j) {
    double sum = 0.;
#pragma unroll
    for (int i = 0; i <= j; ++i) sum += q.R[i * N + j] * q.qtf[i];
    z[j] = sum;
  }
#pragma unroll
  for (int j = 0; j < N; ++j) {  // S^T y = rhs
    if (j >= nsing) {
      z[j] = 0.;
      continue;
    }
    double sum = z[j];
#pragma unroll
    for (int i = 0; i < j; ++i) sum -= sm[i * N + j] * z[i];
    z[j] = sum * sinv[j];
  }
#pragma unroll
  for (int j = N - 1; j >= 0; --j) {  // S z = y
    if (j >= nsing) continue;
    double sum = z[j];
#pragma unroll
    for (int i = j + 1; i < N; ++i)
      if (i < nsing) sum -= sm[j * N + i] * z[i];
    z[j] = sum * sinv[j];
  }
#pragma unroll
  for (int j = 0; j < N; ++j) lm_put<N>(x, q.piv[j], z[j]);
}

// lmpar: damping parameter and the step x (the step is p = -x).
template <int N>
LMB_HD void lm_par_n(LMState& s, double* x) {
  const double dwarf = 2.2250738585072014e-308;
  const double p1 = 0.1, p001 = 0.001;
  LMPar<N> q;
  q.nsing = s.nsing;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    q.piv[i] = s.ipvt[i];
    q.qtf[i] = s.qtf[i];
    q.diag[i] = s.diag[i];
#pragma unroll
    for (int j = 0; j < N; ++j) q.R[i * N + j] = s.r[i * LM_NV + j];
  }
  double wa1[N], wa2[N], sm[N * N], sdiag[N], sinv[N];
  // reciprocals of R's diagonal, independent of one another, so that the
  // dependent chains of the triangular solves below only multiply
#pragma unroll
  for (int j = 0; j < N; ++j) q.rinv[j] = j < q.nsing ? 1. / q.R[j * N + j] : 0.;
  // Gauss-Newton direction
#pragma unroll
  for (int j = 0; j < N; ++j) wa1[j] = j < q.nsing ? q.qtf[j] : 0.;
#pragma unroll
  for (int j = N - 1; j >= 0; --j) {
    if (j >= q.nsing) continue;
    wa1[j] *= q.rinv[j];
    const double t = wa1[j];
#pragma unroll
    for (int i = 0; i < j; ++i) wa1[i] -= q.R[i * N + j] * t;
  }
#pragma unroll
  for (int j = 0; j < N; ++j) lm_put<N>(x, q.piv[j], wa1[j]);
  int iter = 0;
#pragma unroll
  for (int j = 0; j < N; ++j) wa2[j] = q.diag[j] * x[j];
  double dxnorm = enorm(wa2, N);
  double fp = dxnorm - s.delta;
  if (fp <= p1 * s.delta) {
    s.par = 0.;
    return;
  }
  // lower bound
  double parl = 0.;
  if (q.nsing >= N) {
    const double idx = 1. / dxnorm;
#pragma unroll
    for (int j = 0; j < N; ++j) {
      const int l = q.piv[j];
      wa1[j] = lm_get<N>(q.diag, l) * (lm_get<N>(wa2, l) * idx);
    }
#pragma unroll
    for (int j = 0; j < N; ++j) {
      double sum = 0.;
#pragma unroll
      for (int i = 0; i < j; ++i) sum += q.R[i * N + j] * wa1[i];
      wa1[j] = (wa1[j] - sum) * q.rinv[j];
    }
    const double t = enorm(wa1, N);
    parl = ((fp / s.delta) / t) / t;
  }
  // upper bound
#pragma unroll
  for (int j = 0; j < N; ++j) {
    double sum = 0.;
#pragma unroll
    for (int i = 0; i <= j; ++i) sum += q.R[i * N + j] * q.qtf[i];
    wa1[j] = sum / lm_get<N>(q.diag, q.piv[j]);
  }
  const double gnorm = enorm(wa1, N);
  double paru = gnorm / s.delta;
  if (paru == 0.) paru = dwarf / (s.delta < p1 ? s.delta : p1);
  double par = s.par;
  if (par < parl) par = parl;
  if (par > paru) par = paru;
  if (par == 0.) par = gnorm / dxnorm;
  for (;;) {
    ++iter;
    if (par == 0.) par = dwarf > p001 * paru ? dwarf : p001 * paru;
    const double t = sqrt(par);
    double dg[N];
#pragma unroll
    for (int j = 0; j < N; ++j) dg[j] = t * q.diag[j];
    lm_qrsolv_n<N>(q, dg, x, sm, sdiag, sinv);
#pragma unroll
    for (int j = 0; j < N; ++j) wa2[j] = q.diag[j] * x[j];
    dxnorm = enorm(wa2, N);
    const double temp = fp;
    fp = dxnorm - s.delta;
    if (fabs(fp) <= p1 * s.delta || (parl == 0. && fp <= temp && temp < 0.) ||
        iter == 10)
      break;
    // Newton correction: solve S^T w = D P^T x / ||D x||
    const double idx = 1. / dxnorm;
#pragma unroll
    for (int j = 0; j < N; ++j) {
      const int l = q.piv[j];
      wa1[j] = lm_get<N>(q.diag, l) * (lm_get<N>(wa2, l) * idx);
    }
#pragma unroll
    for (int j = 0; j < N; ++j) {
      wa1[j] *= sinv[j];
      const double tj = wa1[j];
#pragma unroll
      for (int i = j + 1; i < N; ++i) wa1[i] -= sm[j * N + i] * tj;
    }
    const double tn = enorm(wa1, N);
    const double parc = ((fp / s.delta) / tn) / tn;
    if (fp > 0.) parl = parl > par ? parl : par;
    if (fp < 0.) paru = paru < par ? paru : par;
    par = parl > par + parc ? parl : par + parc;
  }
  s.par = par;
}

LMB_HD void lm_par(LMState& s, double* x) {
  switch (s.n) {
    case 1: lm_par_n<1>(s, x); break;
    case 2: lm_par_n<2>(s, x); break;
    case 3: lm_par_n<3>(s, x); break;
    case 4: lm_par_n<4>(s, x); break;
    case 5: lm_par_n<5>(s, x); break;
    default: lm_par_n<6>(s, x); break;
  }
}

// Inner loop head: choose the next trial step.  Writes s.p.
template <int N>
LMB_HD void lm_trial_n(LMState& s) {
  double x[LM_NV];
  lm_par_n<N>(s, x);
  double p[N], wa3[N];
#pragma unroll
  for (int j = 0; j < N; ++j) {
    p[j] = -x[j];
    s.p[j] = p[j];
    wa3[j] = s.diag[j] * p[j];
  }
  s.pnorm = enorm(wa3, N);
  if (s.iter == 1 && s.pnorm < s.delta) s.delta = s.pnorm;
  // predicted reduction from ||R P^T p||
#pragma unroll
  for (int j = 0; j < N; ++j) wa3[j] = 0.;
#pragma unroll
  for (int j = 0; j < N; ++j) {
    const double t = lm_get<N>(p, s.ipvt[j]);
#pragma unroll
    for (int i = 0; i <= j; ++i) wa3[i] += s.r[i * LM_NV + j] * t;
  }
  const double temp1 = enorm(wa3, N) / s.fnorm;
  const double temp2 = (sqrt(s.par) * s.pnorm) / s.fnorm;
  s.prered = temp1 * temp1 + temp2 * temp2 / 0.5;
  s.dirder = -(temp1 * temp1 + temp2 * temp2);
}

LMB_HD void lm_trial(LMState& s) {
  switch (s.n) {
    case 1: lm_trial_n<1>(s); break;
    case 2: lm_trial_n<2>(s); break;
    case 3: lm_trial_n<3>(s); break;
    case 4: lm_trial_n<4>(s); break;
    case 5: lm_trial_n<5>(s); break;
    default: lm_trial_n<6>(s); break;
  }
}

// Outer loop body after a new Jacobian at x: scaling, gradient test, trial.
// Returns nonzero when the fit has terminated.
LMB_HD int lm_outer(LMState& s, const LMSettings& set) {
  const int n = s.n;
  s.njev += 1;
  lm_factor(s);
  if (s.iter == 1) {
    for (int j = 0; j < n; ++j) s.diag[j] = s.acnorm[j] == 0. ? 1. : s.acnorm[j];
    double wa3[LM_NV];
    for (int j = 0; j < n; ++j) wa3[j] = s.diag[j] * s.x[j];
    s.xnorm = enorm(wa3, n);
    s.delta = set.factor * s.xnorm;
    if (s.delta == 0.) s.delta = set.factor;
  }
  s.gnorm = 0.;
  if (s.fnorm != 0.) {
    const double ifn = 1. / s.fnorm;
    double acn[LM_NV];
#pragma unroll
    for (int l = 0; l < LM_NV; ++l) acn[l] = s.acnorm[l];
#pragma unroll
    for (int j = 0; j < LM_NV; ++j) {
      if (j >= n) break;
      const double a = lm_get<LM_NV>(acn, s.ipvt[j]);
      if (a == 0.) continue;
      double sum = 0.;
#pragma unroll
      for (int i = 0; i <= j; ++i) sum += s.r[i * LM_NV + j] * (s.qtf[i] * ifn);
      const double g = fabs(sum / a);
      if (g > s.gnorm) s.gnorm = g;
    }
  }
  if (s.gnorm <= set.gtol) {
    s.info = 4;
    return 1;
  }
  for (int j = 0; j < n; ++j)
    if (s.acnorm[j] > s.diag[j]) s.diag[j] = s.acnorm[j];
  lm_trial(s);
  return 0;
}

// First evaluation (start point with its Jacobian).  Returns nonzero when
// the fit has terminated.
LMB_HD int lm_start(LMState& s, const LMEval& ev, const LMSettings& set) {
  s.nfev = 1;
  s.njev = 0;
  s.info = 0;
  s.f2_final = ev.f2;
  if (!(ev.f2 <= 1.7976931348623157e308)) {  // non-finite residuals
    s.info = -2;
    return 1;
  }
  s.fnorm = sqrt(ev.f2);
  s.par = 0.;
  s.iter = 1;
  lm_take(s, ev);
  return lm_outer(s, set);
}

// Evaluation of the trial point x + p (value and Jacobian there).
// Returns nonzero when the fit has terminated.
LMB_HD int lm_after_trial(LMState& s, const LMEval& ev, const LMSettings& set) {
  const int n = s.n;
  const double epsmch = 2.220446049250313e-16;
  s.nfev += 1;
  const double fnorm1 = sqrt(ev.f2);
  double actred = -1.;
  if (0.1 * fnorm1 < s.fnorm) actred = 1. - (fnorm1 / s.fnorm) * (fnorm1 / s.fnorm);
  double ratio = 0.;
  if (s.prered != 0.) ratio = actred / s.prered;
  if (ratio <= 0.25) {
    double temp;
    if (actred >= 0.)
      temp = 0.5;
    else
      temp = 0.5 * s.dirder / (s.dirder + 0.5 * actred);
    if (0.1 * fnorm1 >= s.fnorm || temp < 0.1) temp = 0.1;
    const double pn = s.pnorm / 0.1;
    s.delta = temp * (s.delta < pn ? s.delta : pn);
    s.par = s.par / temp;
  } else if (s.par == 0. || ratio >= 0.75) {
    s.delta = s.pnorm / 0.5;
    s.par = 0.5 * s.par;
  }
  const bool success = ratio >= 1e-4;
  if (success) {
    double wa2[LM_NV];
    for (int j = 0; j < n; ++j) {
      s.x[j] = s.x[j] + s.p[j];
      wa2[j] = s.diag[j] * s.x[j];
    }
    s.xnorm = enorm(wa2, n);
    s.fnorm = fnorm1;
    s.f2_final = ev.f2;
    s.iter += 1;
    lm_take(s, ev);
  }
  const bool fconv = fabs(actred) <= set.ftol && s.prered <= set.ftol && 0.5 * ratio <= 1.;
  if (fconv) s.info = 1;
  if (s.delta <= set.xtol * s.xnorm) s.info = fconv ? 3 : 2;
  if (s.info != 0) return 1;
  if (s.nfev >= set.maxfev) s.info = 5;
  if (fabs(actred) <= epsmch && s.prered <= epsmch && 0.5 * ratio <= 1.) s.info = 6;
  if (s.delta <= epsmch * s.xnorm) s.info = 7;
  if (s.gnorm <= epsmch) s.info = 8;
  if (s.info != 0) return 1;
  if (success) return lm_outer(s, set);
  lm_trial(s);
  return 0;
}

// scipy's status for a MINPACK info (FROM_MINPACK_TO_COMMON); the stringent
// tolerance exits 6/7/8 are reported as the ftol/xtol/gtol successes they
// refine.  Negative values are this library's own failures.
LMB_HD int lm_scipy_status(int info) {
  switch (info) {
    case 1: return 2;
    case 2: return 3;
    case 3: return 4;
    case 4: return 1;
    case 5: return 0;
    case 6: return 2;
    case 7: return 3;
    case 8: return 1;
    default: return info < 0 ? info : -1;
  }
}

// Symmetric eigen-decomposition by cyclic Jacobi rotations (n <= 6).
// a is overwritten; w gets eigenvalues, v (row-major) eigenvectors in columns.
// The loops run to LM_NV with the entries past n skipped, so that every
// index is a compile-time constant once unrolled and a, v stay in registers;
// the arithmetic and its order are those of the loops to n.
LMB_HD void jacobi_eigh(double* a, int n, double* w, double* v) {
#pragma unroll
  for (int i = 0; i < LM_NV; ++i)
#pragma unroll
    for (int j = 0; j < LM_NV; ++j)
      if (i < n && j < n) v[i * LM_NV + j] = i == j ? 1. : 0.;
  for (int sweep = 0; sweep < 30; ++sweep) {
    double off = 0., tot = 0.;
#pragma unroll
    for (int i = 0; i < LM_NV; ++i)
#pragma unroll
      for (int j = 0; j < LM_NV; ++j) {
        if (i >= n || j >= n) continue;
        const double t = a[i * LM_NV + j] * a[i * LM_NV + j];
        tot += t;
        if (i != j) off += t;
      }
    if (off <= 1e-30 * tot || off == 0.) break;
#pragma unroll
    for (int p = 0; p < LM_NV - 1; ++p)
#pragma unroll
      for (int q = p + 1; q < LM_NV; ++q) {
        if (q >= n) continue;
        const double apq = a[p * LM_NV + q];
        if (apq == 0.) continue;
        const double app = a[p * LM_NV + p], aqq = a[q * LM_NV + q];
        const double theta = (aqq - app) / (2. * apq);
        const double t = (theta >= 0. ? 1. : -1.) /
                         (fabs(theta) + sqrt(theta * theta + 1.));
        const double c = 1. / sqrt(t * t + 1.), sn = t * c;
#pragma unroll
        for (int k = 0; k < LM_NV; ++k) {
          if (k >= n) continue;
          const double akp = a[k * LM_NV + p], akq = a[k * LM_NV + q];
          a[k * LM_NV + p] = c * akp - sn * akq;
          a[k * LM_NV + q] = sn * akp + c * akq;
        }
#pragma unroll
        for (int k = 0; k < LM_NV; ++k) {
          if (k >= n) continue;
          const double apk = a[p * LM_NV + k], aqk = a[q * LM_NV + k];
          a[p * LM_NV + k] = c * apk - sn * aqk;
          a[q * LM_NV + k] = sn * apk + c * aqk;
        }
#pragma unroll
        for (int k = 0; k < LM_NV; ++k) {
          if (k >= n) continue;
          const double vkp = v[k * LM_NV + p], vkq = v[k * LM_NV + q];
          v[k * LM_NV + p] = c * vkp - sn * vkq;
          v[k * LM_NV + q] = sn * vkp + c * vkq;
        }
      }
  }
#pragma unroll
  for (int i = 0; i < LM_NV; ++i)
    if (i < n) w[i] = a[i * LM_NV + i];
}

// redchi and uncertainties of Optimizer._statistics (analysis/Optimizer.py:
// 262-278): pcov = pinv(J^T J) keeping singular values of J above
// eps * max(npix, n) * s_max; d = sqrt(redchi * diag(pcov)).
LMB_HD void lm_statistics(const LMState& s, long long npix, double* redchi,
                          double* dp) {
  const int n = s.n;
  const double ndeg = double(npix - n);
  *redchi = s.f2_final / ndeg;
  double a[LM_NV * LM_NV], v[LM_NV * LM_NV], w[LM_NV];
  for (int i = 0; i < LM_NV * LM_NV; ++i) a[i] = s.jtj[i];
  jacobi_eigh(a, n, w, v);
  double wmax = 0.;
#pragma unroll
  for (int i = 0; i < LM_NV; ++i)
    if (i < n && w[i] > wmax) wmax = w[i];
  const double big = double(npix > n ? npix : n);
  const double thr = 2.220446049250313e-16 * big;
  const double thr2 = thr * thr * wmax;
#pragma unroll
  for (int i = 0; i < LM_NV; ++i) {
    if (i >= n) continue;
    double c = 0.;
#pragma unroll
    for (int k = 0; k < LM_NV; ++k)
      if (k < n && w[k] > thr2 && w[k] > 0.)
        c += v[i * LM_NV + k] * v[i * LM_NV + k] / w[k];
    dp[i] = sqrt(*redchi * c);
  }
}

}  // namespace lmb
