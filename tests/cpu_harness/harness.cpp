// CPU build of the kernels' own arithmetic, for tests without a GPU.
//
// Compiles the __host__ __device__ headers of pylorenzmie_b200/csrc with g++
// so that tests/test_cpu_harness.py can check, on the CPU, the Mie
// recurrences, the per-pixel sums (FP32 and FP64), the forward-mode
// Jacobian and the Levenberg-Marquardt state machine against the FP64
// oracle and scipy.  Test infrastructure only: the library never calls it.
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "lmb_layered.cuh"
#include "lmb_lm.cuh"
#include "lmb_mie.cuh"
#include "lmb_pixel.cuh"
#include "lmb_records.cuh"

using namespace lmb;

#define API extern "C"

// ab: [cap+1][2] complex (4 doubles per n), dab: [cap+1][4] complex.
API int h_sphere_ab(double a_p, double n_p, double k_p, double n_m, double lam,
                int cap, double* ab, double* dab, int* nmax) {
  MieScalars s = mie_setup(a_p, n_p, k_p, n_m, lam);
  *nmax = s.nmax;
  if (s.nmax > cap) return 3;
  std::vector<zd> d1in(s.nmax + 1), d1inz(s.nmax + 1), zeta(s.nmax + 1),
      zetax(s.nmax + 1);
  std::vector<double> d1m(s.nmax + 1), d1mx(s.nmax + 1), psi(s.nmax + 1),
      psix(s.nmax + 1);
  std::vector<zd> nz(s.nmax + 1), nz2(s.nmax + 1);
  std::vector<double> nx(s.nmax + 1), nx2(s.nmax + 1);
  for (int n = 1; n <= s.nmax; ++n) {  // as the kernel's two warps
    mie_orders_inside(s, n, nz.data(), nz2.data());
    mie_orders_medium(s, n, nx.data(), nx2.data());
  }
  mie_d1_inside(s, nz.data(), nz2.data(), d1in.data(), d1inz.data());
  mie_d1_medium(s, nx.data(), nx2.data(), d1m.data(), d1mx.data());
  mie_upward(s, nx.data(), nx2.data(), d1m.data(), d1mx.data(), psi.data(),
             psix.data(), zeta.data(), zetax.data());
  memset(ab, 0, sizeof(double) * 4 * (cap + 1));
  if (dab) memset(dab, 0, sizeof(double) * 8 * (cap + 1));
  for (int n = 1; n <= s.nmax; ++n) {
    zd out[2], dout[4];
    mie_coefficient(s, n, d1in.data(), d1inz.data(), psi.data(), psix.data(),
                    zeta.data(), zetax.data(), out, dab ? dout : 0);
    ab[4 * n + 0] = out[0].re;
    ab[4 * n + 1] = out[0].im;
    ab[4 * n + 2] = out[1].re;
    ab[4 * n + 3] = out[1].im;
    if (dab)
      for (int j = 0; j < 4; ++j) {
        dab[8 * n + 2 * j] = dout[j].re;
        dab[8 * n + 2 * j + 1] = dout[j].im;
      }
  }
  return 0;
}

// Multilayer coefficients: radii [L], idx [L][2]; outputs as h_sphere_ab.
static int layered_ab_impl(const double* radii, const double* idx, int L,
                           double n_m, double lam, int cap, double* ab,
                           double* dab, int* nmax, bool split);

API int h_layered_ab(const double* radii, const double* idx, int L, double n_m,
                     double lam, int cap, double* ab, double* dab, int* nmax) {
  return layered_ab_impl(radii, idx, L, n_m, lam, cap, ab, dab, nmax, false);
}

// The same through the split shell functions that the warp-parallel
// kernel path uses (upward recurrences stored, then per-order updates).
API int h_layered_ab_split(const double* radii, const double* idx, int L,
                           double n_m, double lam, int cap, double* ab,
                           double* dab, int* nmax) {
  return layered_ab_impl(radii, idx, L, n_m, lam, cap, ab, dab, nmax, true);
}

static int layered_ab_impl(const double* radii, const double* idx, int L,
                           double n_m, double lam, int cap, double* ab,
                           double* dab, int* nmax, bool split) {
  LayeredScalars s = layered_setup(radii, idx, L, n_m, lam);
  *nmax = s.nmax;
  if (s.nmax > cap) return 3;
  const int nm = s.nmax;
  std::vector<dz> d1a(nm + 2), d1b(nm + 2), ha(nm + 2), hb(nm + 2);
  layered_core(s, d1a.data(), ha.data(), hb.data());
  for (int ii = 1; ii < L; ++ii) {
    const bool outer = ii == L - 1;
    dz z1, z2;
    z1.v = s.x[ii] * s.m[ii];
    z1.s = z1.v;
    z1.m = outer ? mk(s.x[ii], 0.) : mk(0., 0.);
    z2.v = s.x[ii - 1] * s.m[ii];
    z2.s = z2.v;
    z2.m = outer ? mk(s.x[ii - 1], 0.) : mk(0., 0.);
    layered_d1_down(z1, nm, d1a.data());
    layered_d1_down(z2, nm, d1b.data());
    if (split) {
      std::vector<dz> d3a(nm + 2), d3b(nm + 2), q(nm + 2);
      const ShellSetup h = layered_shell_setup(s, ii);
      layered_d3_up(h.z1, nm, d1a.data(), d3a.data());
      layered_d3_up(h.z2, nm, d1b.data(), d3b.data());
      for (int n = 1; n <= nm; ++n)
        q[n] = layered_q_ratio(h, n, d1a.data(), d1b.data(), d3a.data(),
                               d3b.data());
      layered_q_product(h, nm, q.data());
      ha[0] = dconst(mk(0., 0.));
      hb[0] = dconst(mk(0., 0.));
      for (int n = 1; n <= nm; ++n)
        layered_shell_update(h, n, d1a.data(), d1b.data(), d3a.data(),
                             d3b.data(), q.data(), ha.data(), hb.data());
    } else {
      layered_shell_up(s, ii, d1a.data(), d1b.data(), ha.data(), hb.data());
    }
  }
  MieScalars med;
  med.k = s.k;
  med.x = s.x[L - 1];
  med.n_m = n_m;
  med.m = s.m[L - 1];
  med.nmax = nm;
  std::vector<double> d1m(nm + 1), d1mx(nm + 1), psi(nm + 1), psix(nm + 1);
  std::vector<zd> zeta(nm + 1), zetax(nm + 1);
  std::vector<double> nx(nm + 1), nx2(nm + 1);
  for (int n = 1; n <= nm; ++n) mie_orders_medium(med, n, nx.data(), nx2.data());
  mie_d1_medium(med, nx.data(), nx2.data(), d1m.data(), d1mx.data());
  mie_upward(med, nx.data(), nx2.data(), d1m.data(), d1mx.data(), psi.data(),
             psix.data(), zeta.data(), zetax.data());
  memset(ab, 0, sizeof(double) * 4 * (cap + 1));
  if (dab) memset(dab, 0, sizeof(double) * 8 * (cap + 1));
  for (int n = 1; n <= nm; ++n) {
    zd out[2], dout[4];
    layered_coefficient(s, n, ha[n], hb[n], psi.data(), psix.data(), zeta.data(),
                        zetax.data(), out, dab ? dout : 0);
    ab[4 * n + 0] = out[0].re;
    ab[4 * n + 1] = out[0].im;
    ab[4 * n + 2] = out[1].re;
    ab[4 * n + 3] = out[1].im;
    if (dab)
      for (int j = 0; j < 4; ++j) {
        dab[8 * n + 2 * j] = dout[j].re;
        dab[8 * n + 2 * j + 1] = dout[j].im;
      }
  }
  return 0;
}

// Records staged exactly as the kernels stage them (lmb_records.cuh).
template <typename R>
static void stage(const double* ab, const double* dab, int nmax, Quad<R>* q,
                  int w) {
  for (int n = 0; n <= nmax; ++n) {
    zd a[2], d[4];
    for (int j = 0; j < 2; ++j) a[j] = mk(ab[4 * n + 2 * j], ab[4 * n + 2 * j + 1]);
    if (w == JAC_QUADS)
      for (int j = 0; j < 4; ++j) d[j] = mk(dab[8 * n + 2 * j], dab[8 * n + 2 * j + 1]);
    order_record<R>(a, d, n, w, q + w * n);
  }
}

static void stage_pair_host(const double* ab, const double* dab, int nmax,
                            Quad<float>* q) {
  for (int n = 0; n <= nmax; ++n) {
    zd a[2], d[4];
    for (int j = 0; j < 2; ++j) a[j] = mk(ab[4 * n + 2 * j], ab[4 * n + 2 * j + 1]);
    for (int j = 0; j < 4; ++j) d[j] = mk(dab[8 * n + 2 * j], dab[8 * n + 2 * j + 1]);
    float v[PAIR_VALUES];
    pair_record(a, d, n, v);
    for (int j = 0; j < PAIR_QUADS; ++j)
      q[PAIR_QUADS * n + j] = Quad<float>{v[2 * j], v[2 * j], v[2 * j + 1], v[2 * j + 1]};
  }
}

// Field of one sphere at coords [3][npts]; out: [3][npts] complex (re, im).
template <typename R>
static void field_one(const double* coords, long long npts, const double* p,
                      const double* ab, int nmax, double k, int flags,
                      double* out) {
  std::vector<Quad<R>> q(2 * (nmax + 1));
  stage<R>(ab, 0, nmax, q.data(), 2);
  for (long long i = 0; i < npts; ++i) {
    const double x = coords[i], y = coords[npts + i], z = coords[2 * npts + i];
    Geometry<R> g = geometry<R>(k, x - p[0], y - p[1], z - p[2], z, p[2], flags & 2);
    Sums<R> s = order_sum<R>(g, q.data(), nmax);
    cplx<R> e[3];
    epilogue<R>(g, s, flags & 1, e);
    for (int c = 0; c < 3; ++c) {
      out[2 * (c * npts + i)] = e[c].re;
      out[2 * (c * npts + i) + 1] = e[c].im;
    }
  }
}

API void h_field(const double* coords, long long npts, const double* p,
             const double* ab, int nmax, double k, int flags, int fp64,
             double* out) {
  if (fp64)
    field_one<double>(coords, npts, p, ab, nmax, k, flags, out);
  else
    field_one<float>(coords, npts, p, ab, nmax, k, flags, out);
}

// Field of one sphere through the packed two-pixel value loop (pixels i and
// i + 1 share one pass; an odd last pixel is paired with itself), FP32 with
// the phase argument in FP64, as k_field_pair computes it.
API void h_field_pair(const double* coords, long long npts, const double* p,
                  const double* ab, int nmax, double k, int flags,
                  double* out) {
  std::vector<Quad<float>> q(PAIRV_QUADS * (nmax + 1));
  for (int n = 0; n <= nmax; ++n) {
    zd a[2];
    for (int j = 0; j < 2; ++j) a[j] = mk(ab[4 * n + 2 * j], ab[4 * n + 2 * j + 1]);
    float v[PAIRV_VALUES];
    pair_value_record(a, n, v);
    for (int j = 0; j < PAIRV_QUADS; ++j)
      q[PAIRV_QUADS * n + j] = Quad<float>{v[2 * j], v[2 * j], v[2 * j + 1], v[2 * j + 1]};
  }
  for (long long i = 0; i < npts; i += 2) {
    const long long i1 = i + 1 < npts ? i + 1 : i;
    Geometry<float> g[2];
    for (int l = 0; l < 2; ++l) {
      const long long ii = l ? i1 : i;
      const double x = coords[ii], y = coords[npts + ii], z = coords[2 * npts + ii];
      g[l] = geometry<float, true>(k, x - p[0], y - p[1], z - p[2], z, p[2], flags & 2);
    }
    PairSumsV S;
    order_sum_pair(pair_in(g[0], g[1]), q.data(), nmax, S);
    for (int l = 0; l < 2; ++l) {
      const long long ii = l ? i1 : i;
      cplx<float> e[3];
      epilogue<float>(g[l], pair_lane_value(S, l, g[l].smu), flags & 1, e);
      for (int c = 0; c < 3; ++c) {
        out[2 * (c * npts + ii)] = e[c].re;
        out[2 * (c * npts + ii) + 1] = e[c].im;
      }
    }
  }
}

// FP32 hologram of np spheres p [np][6] through the packed two-pixel value
// loop with the FP64 phase and the per-pixel error bound, as
// k_field_pair<true> computes it: holo[i] = H, or -1 where the bound asks
// for the FP64 sum (flags & 8: the FP32 value everywhere).  ab:
// [np][cap+1][2] complex, nmax: [np].  terms (optional, [2][npts]):
// 2 sqrt(H) sum |E_p| and 2 sqrt(H) sum A_p / kr.
API void h_hologram_pair(const double* coords, long long npts, const double* p,
                         int np, const double* ab, const int* nmax, int cap,
                         double k, int flags, float* holo, float* terms) {
  std::vector<std::vector<Quad<float>>> q(np);
  std::vector<float> amp(np);
  for (int j = 0; j < np; ++j) {
    const double* abj = ab + size_t(j) * (cap + 1) * 4;
    q[j].resize(PAIRV_QUADS * (nmax[j] + 1));
    float a = 0.f;
    for (int n = 0; n <= nmax[j]; ++n) {
      zd c[2];
      for (int i = 0; i < 2; ++i) c[i] = mk(abj[4 * n + 2 * i], abj[4 * n + 2 * i + 1]);
      float v[PAIRV_VALUES];
      pair_value_record(c, n, v);
      for (int i = 0; i < PAIRV_QUADS; ++i)
        q[j][PAIRV_QUADS * n + i] = Quad<float>{v[2 * i], v[2 * i], v[2 * i + 1], v[2 * i + 1]};
      if (n > 0) a += order_amplitude(c, n);
    }
    amp[j] = a;
  }
  for (long long i = 0; i < npts; i += 2) {
    const long long i1 = i + 1 < npts ? i + 1 : i;
    cplx<float> e[2][3];
    float m1[2] = {0.f, 0.f}, m0[2] = {0.f, 0.f};
    for (int l = 0; l < 2; ++l)
      for (int c = 0; c < 3; ++c) e[l][c] = mk(0.f, 0.f);
    for (int j = 0; j < np; ++j) {
      const double* pj = p + 6 * j;
      Geometry<float> g[2];
      for (int l = 0; l < 2; ++l) {
        const long long ii = l ? i1 : i;
        const double x = coords[ii], y = coords[npts + ii], z = coords[2 * npts + ii];
        g[l] = geometry<float, true>(k, x - pj[0], y - pj[1], z - pj[2], z, pj[2], flags & 2);
      }
      PairSumsV S;
      order_sum_pair(pair_in(g[0], g[1]), q[j].data(), nmax[j], S);
      for (int l = 0; l < 2; ++l) {
        cplx<float> ep[3];
        epilogue<float>(g[l], pair_lane_value(S, l, g[l].smu), flags & 1, ep);
        for (int c = 0; c < 3; ++c) e[l][c] = e[l][c] + ep[c];
        holo_bound_add(ep, amp[j], g[l].ikr, m1[l], m0[l]);
      }
    }
    for (int l = 0; l < 2; ++l) {
      const float h = intensity<float>(e[l]);
      holo[l ? i1 : i] = (flags & 8) == 0 && holo_needs_fp64(h, m1[l], m0[l]) ? -1.f : h;
      if (terms) {  // the bound's two terms before their constants
        terms[l ? i1 : i] = 2.f * sqrtf(fmaxf(h, 0.f)) * m1[l];
        terms[npts + (l ? i1 : i)] = 2.f * sqrtf(fmaxf(h, 0.f)) * m0[l];
      }
    }
  }
}

// Hologram and Jacobian of one sphere: holo [npts], jac [6][npts].
template <typename R>
static void jac_one(const double* coords, long long npts, const double* p,
                    const double* ab, const double* dab, int nmax, double k,
                    int flags, double* holo, double* jac) {
  std::vector<Quad<R>> q(JAC_QUADS * (nmax + 1));
  stage<R>(ab, dab, nmax, q.data(), JAC_QUADS);
  for (long long i = 0; i < npts; ++i) {
    const double x = coords[i], y = coords[npts + i], z = coords[2 * npts + i];
    Geometry<R> g = geometry<R>(k, x - p[0], y - p[1], z - p[2], z, p[2], flags & 2);
    JacSums<R> A = order_sum_jac<R>(g, q.data(), nmax);
    cplx<R> e[3], de[6][3];
    epilogue_jac<R>(g, A, R(k), e, de);
    holo[i] = intensity<R>(e);
    const cplx<R> et0 = mk(e[0].re + R(1), e[0].im);
    for (int j = 0; j < 6; ++j)
      jac[j * npts + i] = 2 * (et0.re * de[j][0].re + et0.im * de[j][0].im +
                               e[1].re * de[j][1].re + e[1].im * de[j][1].im +
                               e[2].re * de[j][2].re + e[2].im * de[j][2].im);
  }
}

API void h_jacobian(const double* coords, long long npts, const double* p,
                const double* ab, const double* dab, int nmax, double k,
                int flags, int fp64, double* holo, double* jac) {
  if (fp64)
    jac_one<double>(coords, npts, p, ab, dab, nmax, k, flags, holo, jac);
  else
    jac_one<float>(coords, npts, p, ab, dab, nmax, k, flags, holo, jac);
}

// Hologram and Jacobian of one sphere through the packed two-pixel loop
// (pixels i and i + 1 share one pass; an odd last pixel is paired with
// itself), FP32 only.
API void h_jacobian_pair(const double* coords, long long npts, const double* p,
                     const double* ab, const double* dab, int nmax, double k,
                     int flags, double* holo, double* jac) {
  std::vector<Quad<float>> q(PAIR_QUADS * (nmax + 1));
  stage_pair_host(ab, dab, nmax, q.data());
  for (long long i = 0; i < npts; i += 2) {
    const long long i1 = i + 1 < npts ? i + 1 : i;
    Geometry<float> g[2];
    for (int l = 0; l < 2; ++l) {
      const long long ii = l ? i1 : i;
      const double x = coords[ii], y = coords[npts + ii], z = coords[2 * npts + ii];
      g[l] = geometry<float>(k, x - p[0], y - p[1], z - p[2], z, p[2], flags & 2);
    }
    PairSums P;
    order_sum_jac_pair(pair_in(g[0], g[1]), q.data(), nmax, P);
    for (int l = 0; l < 2; ++l) {
      const long long ii = l ? i1 : i;
      const JacSums<float> A = pair_lane(P, l, g[l].smu);
      float H, dH[6];
      holo_jac_reverse<float>(g[l], A, float(k), &H, dH);
      holo[ii] = H;
      for (int j = 0; j < 6; ++j) jac[j * npts + ii] = dH[j];
    }
  }
}

// Hologram and Jacobian of one sphere with the reverse-mode epilogue
// (holo_jac_reverse) after the scalar order loop.
// aberr != 0: the spherical-aberration phase of the device fits
// (aberration_wave) in the epilogue and the x_p, y_p, z_p columns.
template <typename R>
static void jac_rev_one(const double* coords, long long npts, const double* p,
                        const double* ab, const double* dab, int nmax, double k,
                        int flags, double* holo, double* jac, double aberr = 0.) {
  std::vector<Quad<R>> q(JAC_QUADS * (nmax + 1));
  stage<R>(ab, dab, nmax, q.data(), JAC_QUADS);
  for (long long i = 0; i < npts; ++i) {
    const double x = coords[i], y = coords[npts + i], z = coords[2 * npts + i];
    Geometry<R> g = geometry<R>(k, x - p[0], y - p[1], z - p[2], z, p[2], flags & 2);
    JacSums<R> A = order_sum_jac<R>(g, q.data(), nmax);
    R H, dH[6];
    if (aberr != 0.) {
      R dphi[3], hphi;
      const cplx<R> w = aberration_wave<R>(aberr, x - p[0], y - p[1], p[2], dphi);
      holo_jac_reverse<R, true>(g, A, R(k), &H, dH, w, &hphi);
      for (int j = 0; j < 3; ++j) dH[j] += hphi * dphi[j];
    } else {
      holo_jac_reverse<R>(g, A, R(k), &H, dH);
    }
    holo[i] = H;
    for (int j = 0; j < 6; ++j) jac[j * npts + i] = dH[j];
  }
}

API void h_jacobian_aberrated(const double* coords, long long npts,
                              const double* p, const double* ab,
                              const double* dab, int nmax, double k, int flags,
                              int fp64, double aberr, double* holo,
                              double* jac) {
  if (fp64)
    jac_rev_one<double>(coords, npts, p, ab, dab, nmax, k, flags, holo, jac, aberr);
  else
    jac_rev_one<float>(coords, npts, p, ab, dab, nmax, k, flags, holo, jac, aberr);
}

API void h_jacobian_rev(const double* coords, long long npts, const double* p,
                    const double* ab, const double* dab, int nmax, double k,
                    int flags, int fp64, double* holo, double* jac) {
  if (fp64)
    jac_rev_one<double>(coords, npts, p, ab, dab, nmax, k, flags, holo, jac);
  else
    jac_rev_one<float>(coords, npts, p, ab, dab, nmax, k, flags, holo, jac);
}

// Levenberg-Marquardt state machine driven from Python.
struct HLM {
  LMState s;
  LMSettings set;
  int started;
  int done;
};

API void* h_lm_new(int n, const int* slots, const double* x0, double ftol,
               double xtol, double gtol, double factor, int maxfev) {
  HLM* h = (HLM*)calloc(1, sizeof(HLM));
  h->s.n = n;
  for (int a = 0; a < n; ++a) {
    h->s.slot[a] = slots[a];
    h->s.x[a] = x0[a];
  }
  h->set.ftol = ftol;
  h->set.xtol = xtol;
  h->set.gtol = gtol;
  h->set.factor = factor;
  h->set.maxfev = maxfev;
  return h;
}

API void h_lm_free(void* p) { free(p); }

// Feed the evaluation of the point last requested.  Returns 1 when done;
// otherwise writes the next point (free variables) to xnext.
API int h_lm_feed(void* p, double f2, const double* jtj21, const double* jtf6,
              double* xnext) {
  HLM* h = (HLM*)p;
  LMEval ev;
  ev.f2 = f2;
  for (int j = 0; j < 21; ++j) ev.jtj[j] = jtj21[j];
  for (int j = 0; j < 6; ++j) ev.jtf[j] = jtf6[j];
  int done = h->started ? lm_after_trial(h->s, ev, h->set) : lm_start(h->s, ev, h->set);
  h->started = 1;
  h->done = done;
  if (!done)
    for (int a = 0; a < h->s.n; ++a) xnext[a] = h->s.x[a] + h->s.p[a];
  return done;
}

API void h_lm_result(void* p, long long npix, double* x, int* info, int* nfev,
                 int* njev, double* redchi, double* dp) {
  HLM* h = (HLM*)p;
  for (int a = 0; a < h->s.n; ++a) x[a] = h->s.x[a];
  *info = h->s.info;
  *nfev = h->s.nfev;
  *njev = h->s.njev;
  lm_statistics(h->s, npix, redchi, dp);
}

API int h_sym6(int i, int j) { return sym6(i, j); }

