// Device kernels of lmb200 (sm_100a).  Included by lmb200.cu only.
//
// Data layout in HBM (all row-major, struct-of-arrays where it is read by
// pixel):
//   coordinates        [3][npts] FP64
//   ab                 [nparticles][nmax_cap+1][2] complex128 (a_n, b_n)
//   dab                [nparticles][nmax_cap+1][4] complex128
//   field / hologram   [items][3][npts] complex, [items][npts] real
//   fit data           packed float32 crops, one contiguous run per feature
//   fit tiles          int2 (feature, first pixel); partial sums [tile][28]
// The per-order coefficients of the particle being summed are staged once
// per CTA into shared memory as FP32 (or FP64) records with the order
// prefactor folded in; every pixel of the CTA reads them as broadcasts.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "lmb200.h"
#include "lmb_layered.cuh"
#include "lmb_lm.cuh"
#include "lmb_mie.cuh"
#include "lmb_pixel.cuh"
#include "lmb_records.cuh"

namespace lmb {

// ---------------------------------------------------------------------------
// Mie coefficients: one two-warp block per sphere.

struct AbScratch {
  zd *d1in, *d1inz, *zeta, *zetax, *nz, *nz2;
  double *d1m, *d1mx, *psi, *psix, *nx, *nx2;
};

__host__ __device__ inline size_t ab_scratch_bytes(int nmaxp) {
  return size_t(nmaxp) * (6 * sizeof(zd) + 6 * sizeof(double));
}

__device__ inline AbScratch carve_ab_scratch(char* base, int nmaxp) {
  AbScratch s;
  s.d1in = reinterpret_cast<zd*>(base);
  s.d1inz = s.d1in + nmaxp;
  s.zeta = s.d1inz + nmaxp;
  s.zetax = s.zeta + nmaxp;
  s.nz = s.zetax + nmaxp;
  s.nz2 = s.nz + nmaxp;
  s.d1m = reinterpret_cast<double*>(s.nz2 + nmaxp);
  s.d1mx = s.d1m + nmaxp;
  s.psi = s.d1mx + nmaxp;
  s.psix = s.psi + nmaxp;
  s.nx = s.psix + nmaxp;
  s.nx2 = s.nx + nmaxp;
  return s;
}

// Called by all 64 threads of a two-warp block.  ab: [nmaxp][2] zd, dab:
// [nmaxp][4] zd (may be null).  The serial recurrences are FP64 chains of
// dependent operations, so their time is latency: warp 0 runs the inside
// D1 while warp 1 runs the medium's D1 and then its upward psi/zeta, and
// the two warps interleave (two branches of one warp would run one after
// the other).  Then warp 0 forms a_n, b_n over the orders.  Both warps pass
// the one __syncthreads whatever the inputs.  Returns the status on warp 0
// (uniform over it); warp 1's return value means nothing.
__device__ int block_sphere_ab(double a_p, double n_p, double k_p, double n_m,
                               double wavelength, int nmax_cap, AbScratch w,
                               zd* ab, zd* dab, int* nmax_out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nmaxp = nmax_cap + 1;
  const MieScalars s = mie_setup(a_p, n_p, k_p, n_m, wavelength);
  const bool ok = (s.x > 0.) && (s.x < 1e7) && s.nmax >= 1 &&
                  s.nmax <= nmax_cap && isfinite(s.m.re) && isfinite(s.m.im);
  if (ok) {
    if (warp == 0) {
      for (int n = 1 + lane; n <= s.nmax; n += 32) mie_orders_inside(s, n, w.nz, w.nz2);
      __syncwarp();
      if (lane == 0) mie_d1_inside(s, w.nz, w.nz2, w.d1in, w.d1inz);
    } else {
      for (int n = 1 + lane; n <= s.nmax; n += 32) mie_orders_medium(s, n, w.nx, w.nx2);
      __syncwarp();
      if (lane == 0) {
        mie_d1_medium(s, w.nx, w.nx2, w.d1m, w.d1mx);
        mie_upward(s, w.nx, w.nx2, w.d1m, w.d1mx, w.psi, w.psix, w.zeta, w.zetax);
      }
    }
  }
  __syncthreads();
  if (warp != 0) return LMB_OK;
  if (!ok) {
    for (int n = lane; n < nmaxp; n += 32) {
      ab[2 * n] = ab[2 * n + 1] = mk(0., 0.);
      if (dab)
        for (int j = 0; j < 4; ++j) dab[4 * n + j] = mk(0., 0.);
    }
    if (lane == 0) *nmax_out = (s.nmax >= 0 && s.nmax < (1 << 30)) ? s.nmax : 0;
    __syncwarp();
    return LMB_ERR_NMAX;
  }
  for (int n = lane; n < nmaxp; n += 32) {
    if (n == 0 || n > s.nmax) {
      ab[2 * n] = ab[2 * n + 1] = mk(0., 0.);
      if (dab)
        for (int j = 0; j < 4; ++j) dab[4 * n + j] = mk(0., 0.);
      continue;
    }
    zd out[2], dout[4];
    mie_coefficient(s, n, w.d1in, w.d1inz, w.psi, w.psix, w.zeta, w.zetax, out,
                    dab ? dout : (zd*)0);
    ab[2 * n] = out[0];
    ab[2 * n + 1] = out[1];
    if (dab)
      for (int j = 0; j < 4; ++j) dab[4 * n + j] = dout[j];
  }
  if (lane == 0) *nmax_out = s.nmax;
  __syncwarp();
  return LMB_OK;
}

// One two-warp block (64 threads) per sphere.
__global__ void k_sphere_ab(const lmb_sphere* spheres, int n, double n_m,
                            double wavelength, int nmax_cap, zd* ab, zd* dab,
                            int* nmax, int* status) {
  extern __shared__ __align__(16) char smem[];
  const int i = blockIdx.x;
  if (i >= n) return;
  const int nmaxp = nmax_cap + 1;
  AbScratch w = carve_ab_scratch(smem, nmaxp);
  const lmb_sphere sp = spheres[i];
  const int st = block_sphere_ab(sp.a_p, sp.n_p, sp.k_p, n_m, wavelength,
                                 nmax_cap, w, ab + size_t(i) * nmaxp * 2,
                                 dab ? dab + size_t(i) * nmaxp * 4 : (zd*)0,
                                 nmax + i);
  if (threadIdx.x == 0) status[i] = st;
}

// ---------------------------------------------------------------------------
// Multilayer spheres: one two-warp block per sphere (block_layered_ab).

__host__ __device__ inline size_t layered_scratch_serial_bytes(int nmaxp) {
  return 4 * size_t(nmaxp + 1) * sizeof(dz) + ab_scratch_bytes(nmaxp);
}

// The warp-parallel form keeps every shell's downward D1 at both of its
// arguments and its upward recurrences (5 arrays a shell), the core's D1,
// and Ha, Hb.
__host__ __device__ inline size_t layered_scratch_parallel_bytes(int nmaxp, int L) {
  return size_t(3 + 5 * (L - 1)) * size_t(nmaxp + 1) * sizeof(dz) +
         ab_scratch_bytes(nmaxp);
}

// The parallel form is used when its scratch fits in shared memory.
__host__ __device__ inline bool layered_parallel(int nmaxp, int L) {
  return layered_scratch_parallel_bytes(nmaxp, L) <= size_t(200) * 1024;
}

__host__ __device__ inline size_t layered_scratch_bytes(int nmaxp, int L) {
  return layered_parallel(nmaxp, L) ? layered_scratch_parallel_bytes(nmaxp, L)
                                    : layered_scratch_serial_bytes(nmaxp);
}

// radii [L] ascending (um), idx [L][2] (re, im), core first.  Called by all
// 64 threads of a two-warp block.  Warp 1 runs the medium's recurrences
// (D1, then upward psi/zeta) while warp 0 runs the layers' and their Ha/Hb;
// the two warps interleave.  Then warp 0 forms a_n, b_n over the orders.
// Both warps pass the one __syncthreads whatever the inputs.  Returns the
// status on warp 0 (uniform over it); warp 1's return value means nothing.
__device__ int block_layered_ab(const double* radii, const double* idx, int L,
                                double n_m, double wavelength, int nmax_cap,
                                char* scratch, zd* ab, zd* dab, int* nmax_out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nmaxp = nmax_cap + 1;
  bool ok = L >= 1 && L <= LMB_MAX_LAYERS;
  for (int l = 0; ok && l < L; ++l)
    ok = radii[l] > 0. && (l == 0 || radii[l] > radii[l - 1]) &&
         isfinite(idx[2 * l]) && isfinite(idx[2 * l + 1]);
  LayeredScalars s;
  if (ok) {
    s = layered_setup(radii, idx, L, n_m, wavelength);
    ok = s.nmax >= 1 && s.nmax <= nmax_cap && s.x[L - 1] < 1e7;
  }
  const size_t na = size_t(nmaxp + 1);
  const bool par = layered_parallel(nmaxp, L);
  // parallel form: the core's D1, then shell ii's d1a, d1b, d3a, d3b, q at
  // sh + 5 (ii-1) na; serial form: d1a, d1b.  Then Ha, Hb, the medium's.
  dz* d1c = reinterpret_cast<dz*>(scratch);
  dz* sh = d1c + na;
  dz* ha = par ? sh + 5 * (L - 1) * na : d1c + 2 * na;
  dz* hb = ha + na;
  const AbScratch w = carve_ab_scratch(reinterpret_cast<char*>(hb + na), nmaxp);
  if (ok && warp == 1) {
    MieScalars med;
    med.k = s.k;
    med.x = s.x[L - 1];
    med.n_m = n_m;
    med.m = s.m[L - 1];
    med.nmax = s.nmax;
    for (int n = 1 + lane; n <= s.nmax; n += 32) mie_orders_medium(med, n, w.nx, w.nx2);
    __syncwarp();
    if (lane == 0) {
      mie_d1_medium(med, w.nx, w.nx2, w.d1m, w.d1mx);
      mie_upward(med, w.nx, w.nx2, w.d1m, w.d1mx, w.psi, w.psix, w.zeta, w.zetax);
    }
  } else if (ok && par) {
    // Each phase on one code path across the lanes: the downward D1 chains
    // of the core (lane 0) and of both arguments of each shell (lanes
    // 1..2L-2); each shell argument's upward D3 chain (lanes 0..2L-3); Q's
    // factors over (shell, order) pairs and their running products one lane
    // per shell; the shells in order, their Ha/Hb updates over the orders.
    if (lane < 2 * L - 1) {
      dz z;
      dz* out;
      if (lane == 0) {
        z.v = s.x[0] * s.m[0];
        z.s = z.v;
        z.m = (L == 1) ? mk(s.x[0], 0.) : mk(0., 0.);
        out = d1c;
      } else {
        const int ii = (lane - 1) / 2 + 1, which = (lane - 1) & 1;
        const bool outer = ii == L - 1;
        const double xx = which == 0 ? s.x[ii] : s.x[ii - 1];
        z.v = xx * s.m[ii];
        z.s = z.v;
        z.m = outer ? mk(xx, 0.) : mk(0., 0.);
        out = sh + (5 * (ii - 1) + which) * na;
      }
      layered_d1_down(z, s.nmax, out);
    }
    __syncwarp();
    if (lane < 2 * (L - 1)) {
      const int ii = lane / 2 + 1, which = lane & 1;
      const ShellSetup h = layered_shell_setup(s, ii);
      dz* b = sh + 5 * (ii - 1) * na;
      layered_d3_up(which == 0 ? h.z1 : h.z2, s.nmax, b + which * na,
                    b + (2 + which) * na);
    }
    for (int n = lane; n <= s.nmax; n += 32) {
      ha[n] = d1c[n];
      hb[n] = d1c[n];
    }
    __syncwarp();
    for (int j = lane; j < (L - 1) * s.nmax; j += 32) {
      const int ii = j / s.nmax + 1, n = j - (ii - 1) * s.nmax + 1;
      dz* b = sh + 5 * (ii - 1) * na;
      b[4 * na + n] = layered_q_ratio(layered_shell_setup(s, ii), n, b, b + na,
                                      b + 2 * na, b + 3 * na);
    }
    __syncwarp();
    if (lane < L - 1)
      layered_q_product(layered_shell_setup(s, lane + 1), s.nmax,
                        sh + (5 * lane + 4) * na);
    __syncwarp();
    for (int ii = 1; ii < L; ++ii) {
      const ShellSetup h = layered_shell_setup(s, ii);
      const dz* b = sh + 5 * (ii - 1) * na;
      if (lane == 0) {
        ha[0] = dconst(mk(0., 0.));
        hb[0] = dconst(mk(0., 0.));
      }
      for (int n = 1 + lane; n <= s.nmax; n += 32)
        layered_shell_update(h, n, b, b + na, b + 2 * na, b + 3 * na, b + 4 * na,
                             ha, hb);
      __syncwarp();
    }
  } else if (ok) {
    // serial form, for scratch too large for the parallel one
    dz* d1a = d1c;
    dz* d1b = d1c + na;
    if (lane == 0) layered_core(s, d1a, ha, hb);
    __syncwarp();
    for (int ii = 1; ii < L; ++ii) {
      const bool outer = ii == L - 1;
      if (lane < 2) {
        dz z;
        const double xx = lane == 0 ? s.x[ii] : s.x[ii - 1];
        z.v = xx * s.m[ii];
        z.s = z.v;
        z.m = outer ? mk(xx, 0.) : mk(0., 0.);
        layered_d1_down(z, s.nmax, lane == 0 ? d1a : d1b);
      }
      __syncwarp();
      if (lane == 0) layered_shell_up(s, ii, d1a, d1b, ha, hb);
      __syncwarp();
    }
  }
  __syncthreads();
  if (warp != 0) return LMB_OK;
  for (int n = lane; n < nmaxp; n += 32) {
    if (!ok || n == 0 || n > s.nmax) {
      ab[2 * n] = ab[2 * n + 1] = mk(0., 0.);
      if (dab)
        for (int j = 0; j < 4; ++j) dab[4 * n + j] = mk(0., 0.);
      continue;
    }
    zd out[2], dout[4];
    layered_coefficient(s, n, ha[n], hb[n], w.psi, w.psix, w.zeta, w.zetax, out,
                        dab ? dout : (zd*)0);
    ab[2 * n] = out[0];
    ab[2 * n + 1] = out[1];
    if (dab)
      for (int j = 0; j < 4; ++j) dab[4 * n + j] = dout[j];
  }
  if (lane == 0) *nmax_out = ok ? s.nmax : 0;
  __syncwarp();
  return ok ? LMB_OK : LMB_ERR_NMAX;
}

// One two-warp block (64 threads) per sphere.
__global__ void k_layered_ab(const double* radii, const double* indices, int L,
                             int n, double n_m, double wavelength, int nmax_cap,
                             zd* ab, zd* dab, int* nmax, int* status) {
  extern __shared__ __align__(16) char smem[];
  const int i = blockIdx.x;
  if (i >= n) return;
  const int nmaxp = nmax_cap + 1;
  const int st = block_layered_ab(radii + size_t(i) * L, indices + size_t(i) * L * 2,
                                  L, n_m, wavelength, nmax_cap, smem,
                                  ab + size_t(i) * nmaxp * 2,
                                  dab ? dab + size_t(i) * nmaxp * 4 : (zd*)0,
                                  nmax + i);
  if (threadIdx.x == 0) status[i] = st;
}

// ---------------------------------------------------------------------------
// Staging of per-order records (see lmb_pixel.cuh, struct Quad).

// Shared-memory layout of the FP64 re-summation in k_field_pair<true>
// (256 threads, 512 pixels a block): the marked-pixel list, the FP64 field
// accumulators of up to 512 pixels, then the particles' FP64 records.
enum { RESUM_LIST_BYTES = 512 * 4, RESUM_ACC_BYTES = 512 * 6 * 8 };

template <typename R, bool kJac>
__device__ void stage_coef(const zd* ab, const zd* dab, int nmax,
                           Quad<R>* sm) {
  constexpr int W = kJac ? int(JAC_QUADS) : 2;
  for (int n = threadIdx.x; n <= nmax; n += blockDim.x) {
    Quad<R> q[JAC_QUADS];
    order_record<R>(ab + 2 * n, kJac ? dab + 4 * n : dab, n, W, q);
    for (int j = 0; j < W; ++j) sm[W * n + j] = q[j];
  }
}

// Records of order_sum_pair (value only): PAIRV_QUADS float4 per order,
// i.e. PAIRV_VALUES float2 (v, v).  Three threads per order, so that the
// FP64 work of staging is spread over the block.
__device__ void stage_pair_value(const zd* ab, int nmax, float4* sm) {
  float2* r2 = reinterpret_cast<float2*>(sm);
  for (int t = threadIdx.x; t < 3 * (nmax + 1); t += blockDim.x) {
    const int n = t / 3, part = t - 3 * n;
    float v[PAIRV_VALUES];
    pair_value_part(ab + 2 * n, n, part, v);
    const int lo = part == 0 ? 0 : (part == 1 ? 7 : 10);
    const int hi = part == 0 ? 7 : (part == 1 ? 10 : PAIRV_VALUES);
    for (int j = lo; j < hi; ++j) r2[PAIRV_VALUES * n + j] = make_float2(v[j], v[j]);
  }
}

// Records of order_sum_jac_pair: PAIR_QUADS float4 per order, every value
// duplicated into both lanes of a float2.
__device__ void stage_pair(const zd* ab, const zd* dab, int nmax, float4* sm) {
  for (int n = threadIdx.x; n <= nmax; n += blockDim.x) {
    float v[PAIR_VALUES];
    pair_record(ab + 2 * n, dab + 4 * n, n, v);
    for (int j = 0; j < PAIR_QUADS; ++j)
      sm[PAIR_QUADS * n + j] =
          make_float4(v[2 * j], v[2 * j], v[2 * j + 1], v[2 * j + 1]);
  }
}

// ---------------------------------------------------------------------------
// Field / hologram at explicit coordinates, many items, many particles.

template <typename R>
struct FieldOut;
template <>
struct FieldOut<float> {
  typedef float2 C;
};
template <>
struct FieldOut<double> {
  typedef double2 C;
};

// Spherical-aberration phase of one particle at one pixel
// (theory/Aberrated.py:62-79): Phi = c r^4 / (r^2 + z_p^2)^2 with
// c = 4 n_m^3 s / k, r the in-plane distance from the particle (pixels).
template <typename R>
__device__ inline cplx<R> aberration_phase(double c, double dx, double dy,
                                           double zp) {
  const double rsq = dx * dx + dy * dy;
  const double den = rsq + zp * zp;
  const double phi = den > 0. ? c * (rsq / den) * (rsq / den) : 0.;
  return cis(R(reduce_2pi(phi)));
}

// aberr: the coefficient c above, 0 for an ideal instrument.
template <typename R, bool kHologram>
__global__ void __launch_bounds__(256)
k_field(const double* __restrict__ coords, long long npts,
        const lmb_sphere* __restrict__ spheres, const int* __restrict__ item_start,
        const zd* __restrict__ ab, const int* __restrict__ nmax, int nmaxp, double k,
        int flags, double aberr, void* out) {
  extern __shared__ __align__(16) char smem[];
  Quad<R>* coef = reinterpret_cast<Quad<R>*>(smem);
  const int item = blockIdx.y;
  const long long pix = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = pix < npts;
  const bool cart = flags & LMB_CARTESIAN;
  const bool bohren = flags & LMB_BOHREN;
  double x = 0., y = 0., z = 0.;
  if (live) {
    x = coords[pix];
    y = coords[npts + pix];
    z = coords[2 * npts + pix];
  }
  cplx<R> e[3];
  for (int c = 0; c < 3; ++c) e[c] = mk(R(0), R(0));
  const int pb = item_start[item], pe = item_start[item + 1];
  for (int p = pb; p < pe; ++p) {
    const int nm = min(max(nmax[p], 0), nmaxp - 1);
    __syncthreads();
    stage_coef<R, false>(ab + size_t(p) * nmaxp * 2, (const zd*)0, nm, coef);
    __syncthreads();
    if (live) {
      const lmb_sphere sp = spheres[p];
      const Geometry<R> g = geometry<R>(k, x - sp.x_p, y - sp.y_p, z - sp.z_p, z,
                                        sp.z_p, bohren);
      const Sums<R> s = order_sum<R>(g, coef, nm);
      cplx<R> ep[3];
      epilogue<R>(g, s, cart, ep);
      if (aberr != 0.) {
        const cplx<R> ph = aberration_phase<R>(aberr, x - sp.x_p, y - sp.y_p, sp.z_p);
        for (int c = 0; c < 3; ++c) ep[c] = ph * ep[c];
      }
      for (int c = 0; c < 3; ++c) e[c] = e[c] + ep[c];
    }
  }
  if (!live) return;
  if (kHologram) {
    R* o = reinterpret_cast<R*>(out) + (size_t)item * npts;
    o[pix] = intensity<R>(e);
  } else {
    typedef typename FieldOut<R>::C C;
    C* o = reinterpret_cast<C*>(out) + (size_t)item * 3 * npts;
    for (int c = 0; c < 3; ++c) {
      C v;
      v.x = e[c].re;
      v.y = e[c].im;
      o[c * npts + pix] = v;
    }
  }
}

// FP64 re-summation, inside k_field_pair<true>, of the block's pixels whose
// FP32 error bound exceeded HOLO_TOL (mark0/mark1: the thread's two
// pixels).  The particles go in groups of `group` (<= 32), whose FP64
// records (2 Quad<double> per order, nmaxp orders per slot) are staged in
// smem after the marked-pixel list and the FP64 field accumulators.  Two
// ways to spread the work, chosen per block by their cost in order steps:
// - few marked pixels: one warp per marked pixel and one lane per particle,
//   so that a pixel's particles run their recurrences side by side (lanes
//   combined by a fixed shuffle tree);
// - many marked pixels, or few particles (large spheres mark most pixels):
//   one thread per marked pixel, its particles in order.
// The choice depends only on the marked count and the particles' n_max,
// and groups are summed in order, so the result does not depend on
// scheduling.  Every thread of the block calls this.
__device__ void holo_resum64(bool mark0, long long q0, bool mark1, long long q1,
                             long long base, char* smem, int group,
                             const double* __restrict__ coords, long long npts,
                             const lmb_sphere* __restrict__ spheres, int pb, int pe,
                             const zd* __restrict__ ab, const int* __restrict__ nmax,
                             int nmaxp, double k, int flags, double aberr, float* o) {
  __shared__ int s_n;
  if (threadIdx.x == 0) s_n = 0;
  if (!__syncthreads_or(mark0 || mark1)) return;
  int* list = reinterpret_cast<int*>(smem);                      // [2 * blockDim]
  double* acc = reinterpret_cast<double*>(smem + RESUM_LIST_BYTES);  // [.][6]
  Quad<double>* rec =
      reinterpret_cast<Quad<double>*>(smem + RESUM_LIST_BYTES + RESUM_ACC_BYTES);
  if (mark0) list[atomicAdd(&s_n, 1)] = int(q0 - base);
  if (mark1) list[atomicAdd(&s_n, 1)] = int(q1 - base);
  __syncthreads();
  const int F = s_n;
  for (int i = threadIdx.x; i < 6 * F; i += blockDim.x) acc[i] = 0.;
  const bool cart = flags & LMB_CARTESIAN;
  const bool bohren = flags & LMB_BOHREN;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  // order steps of each way: a warp per pixel waits for its group's
  // largest n_max; a thread per pixel walks every particle's orders
  long long by_lane = 0, by_thread = 0;
  for (int g0 = pb; g0 < pe; g0 += group) {
    int mx = 0;
    long long sum = 0;
    for (int j = g0; j < min(g0 + group, pe); ++j) {
      const int nm = min(max(nmax[j], 0), nmaxp - 1);
      mx = max(mx, nm);
      sum += nm;
    }
    by_lane += (long long)((F + nwarps - 1) / nwarps) * mx;
    by_thread += (long long)((F + int(blockDim.x) - 1) / int(blockDim.x)) * sum;
  }
  const bool per_thread = by_thread < by_lane;
  for (int g0 = pb; g0 < pe; g0 += group) {
    const int G = min(group, pe - g0);
    __syncthreads();  // the previous group's records are no longer read
    for (int j = 0; j < G; ++j) {
      const int nm = min(max(nmax[g0 + j], 0), nmaxp - 1);
      stage_coef<double, false>(ab + size_t(g0 + j) * nmaxp * 2, (const zd*)0, nm,
                                rec + size_t(j) * 2 * nmaxp);
    }
    __syncthreads();
    if (per_thread) {
      for (int f = threadIdx.x; f < F; f += blockDim.x) {
        const long long pix = base + list[f];
        const double x = coords[pix], y = coords[npts + pix], z = coords[2 * npts + pix];
        cplx<double> e[3];
        for (int c = 0; c < 3; ++c) e[c] = mk(acc[6 * f + 2 * c], acc[6 * f + 2 * c + 1]);
        for (int j = 0; j < G; ++j) {
          const int p = g0 + j;
          const int nm = min(max(nmax[p], 0), nmaxp - 1);
          const lmb_sphere sp = spheres[p];
          const Geometry<double> g =
              geometry<double>(k, x - sp.x_p, y - sp.y_p, z - sp.z_p, z, sp.z_p, bohren);
          const Sums<double> sm = order_sum<double>(g, rec + size_t(j) * 2 * nmaxp, nm);
          cplx<double> ep[3];
          epilogue<double>(g, sm, cart, ep);
          if (aberr != 0.) {
            const cplx<double> ph =
                aberration_phase<double>(aberr, x - sp.x_p, y - sp.y_p, sp.z_p);
            for (int c = 0; c < 3; ++c) ep[c] = ph * ep[c];
          }
          for (int c = 0; c < 3; ++c) e[c] = e[c] + ep[c];
        }
        for (int c = 0; c < 3; ++c) {
          acc[6 * f + 2 * c] = e[c].re;
          acc[6 * f + 2 * c + 1] = e[c].im;
        }
      }
      continue;
    }
    for (int f = warp; f < F; f += nwarps) {
      const long long pix = base + list[f];
      cplx<double> e[3];
      for (int c = 0; c < 3; ++c) e[c] = mk(0., 0.);
      if (lane < G) {
        const int p = g0 + lane;
        const int nm = min(max(nmax[p], 0), nmaxp - 1);
        const lmb_sphere sp = spheres[p];
        const double x = coords[pix], y = coords[npts + pix], z = coords[2 * npts + pix];
        const Geometry<double> g =
            geometry<double>(k, x - sp.x_p, y - sp.y_p, z - sp.z_p, z, sp.z_p, bohren);
        const Sums<double> sm = order_sum<double>(g, rec + size_t(lane) * 2 * nmaxp, nm);
        epilogue<double>(g, sm, cart, e);
        if (aberr != 0.) {
          const cplx<double> ph = aberration_phase<double>(aberr, x - sp.x_p, y - sp.y_p, sp.z_p);
          for (int c = 0; c < 3; ++c) e[c] = ph * e[c];
        }
      }
      for (int o2 = 16; o2 > 0; o2 >>= 1)
        for (int c = 0; c < 3; ++c) {
          e[c].re += __shfl_xor_sync(0xffffffffu, e[c].re, o2);
          e[c].im += __shfl_xor_sync(0xffffffffu, e[c].im, o2);
        }
      if (lane == 0)
        for (int c = 0; c < 3; ++c) {
          acc[6 * f + 2 * c] += e[c].re;
          acc[6 * f + 2 * c + 1] += e[c].im;
        }
    }
  }
  __syncthreads();
  for (int f = threadIdx.x; f < F; f += blockDim.x) {
    cplx<double> e[3];
    for (int c = 0; c < 3; ++c) e[c] = mk(acc[6 * f + 2 * c], acc[6 * f + 2 * c + 1]);
    o[base + list[f]] = float(intensity<double>(e));
  }
}

// FP32 field / hologram with the packed two-pixel loop: each thread takes
// two adjacent pixels (the last thread of an odd count pairs its pixel with
// itself).  Same inputs and outputs as k_field<float, holo>; the order loop
// runs in f32x2 (order_sum_pair) and the phase in FP64 (phase_turns64).
//
// The particles of an item are summed in groups of up to 32 whose records
// fit the block's shared memory (rec_quads float4): a group's records (and,
// for holograms, the particles' amplitudes A_p, one warp per particle in a
// fixed order) are staged by the whole block at once, so the block passes
// one barrier pair per group rather than per particle.
//
// Holograms also accumulate each pixel's error bound (holo_needs_fp64); the
// block then sums its pixels whose bound exceeds HOLO_TOL again in FP64
// (holo_resum64, particles in groups of resum_group) and writes those.
template <bool kHologram>
__global__ void __launch_bounds__(256)
k_field_pair(const double* __restrict__ coords, long long npts,
             const lmb_sphere* __restrict__ spheres, const int* __restrict__ item_start,
             const zd* __restrict__ ab, const int* __restrict__ nmax, int nmaxp,
             double k, int flags, double aberr, void* out, int rec_quads,
             int resum_group) {
  extern __shared__ __align__(16) char smem[];
  float4* rec = reinterpret_cast<float4*>(smem);
  __shared__ int s_off[33];   // record offsets (float4) of the group's particles
  __shared__ int s_nm[32];
  __shared__ int s_count;     // particles in the group
  __shared__ float s_amp[32];
  const int item = blockIdx.y;
  const long long base = (long long)blockIdx.x * blockDim.x * 2;
  const long long p0 = base + threadIdx.x * 2;
  const bool live0 = p0 < npts;
  const bool live1 = p0 + 1 < npts;
  const long long p1 = live1 ? p0 + 1 : p0;
  const bool cart = flags & LMB_CARTESIAN;
  const bool bohren = flags & LMB_BOHREN;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double x[2] = {0., 0.}, y[2] = {0., 0.}, z[2] = {0., 0.};
  if (live0) {
    x[0] = coords[p0];
    y[0] = coords[npts + p0];
    z[0] = coords[2 * npts + p0];
    x[1] = coords[p1];
    y[1] = coords[npts + p1];
    z[1] = coords[2 * npts + p1];
  }
  cplx<float> e[2][3];
  for (int l = 0; l < 2; ++l)
    for (int c = 0; c < 3; ++c) e[l][c] = mk(0.f, 0.f);
  float m1[2] = {0.f, 0.f}, m0[2] = {0.f, 0.f};  // error bound (holograms)
  const int pb = item_start[item], pe = item_start[item + 1];
  for (int g0 = pb; g0 < pe; g0 += s_count) {
    __syncthreads();  // the previous group's records and s_count are read
    if (warp == 0) {
      // the group: the next particles (up to 32) whose records fit
      const int p = g0 + lane;
      const int nm = p < pe ? min(max(nmax[p], 0), nmaxp - 1) : 0;
      int size = p < pe ? PAIRV_QUADS * (nm + 1) : 0;
      for (int o = 1; o < 32; o <<= 1) {  // inclusive prefix sum
        const int v = __shfl_up_sync(0xffffffffu, size, o);
        if (lane >= o) size += v;
      }
      const unsigned fits = __ballot_sync(0xffffffffu, p < pe && size <= rec_quads);
      const int G = max(1, __popc(fits));  // one particle always fits
      s_nm[lane] = nm;
      const int excl = __shfl_up_sync(0xffffffffu, size, 1);
      const int last = __shfl_sync(0xffffffffu, size, G - 1);
      if (lane < G) s_off[lane] = lane ? excl : 0;
      if (lane == 0) {
        s_count = G;
        s_off[G] = last;
      }
    }
    __syncthreads();
    const int G = s_count;
    {
      // stage: three threads per order over all the group's orders
      float2* r2 = reinterpret_cast<float2*>(rec);
      const int total = 3 * (s_off[G] / PAIRV_QUADS);
      int j = 0;
      for (int t = threadIdx.x; t < total; t += blockDim.x) {
        while (3 * (s_off[j + 1] / PAIRV_QUADS) <= t) ++j;
        const int u = t - 3 * (s_off[j] / PAIRV_QUADS);
        const int n = u / 3, part = u - 3 * n;
        float v[PAIRV_VALUES];
        pair_value_part(ab + size_t(g0 + j) * nmaxp * 2 + 2 * n, n, part, v);
        const int lo = part == 0 ? 0 : (part == 1 ? 7 : 10);
        const int hi = part == 0 ? 7 : (part == 1 ? 10 : PAIRV_VALUES);
        float2* dst = r2 + 2 * s_off[j] + PAIRV_VALUES * n;
        for (int q = lo; q < hi; ++q) dst[q] = make_float2(v[q], v[q]);
      }
      if (kHologram) {
        for (int jj = warp; jj < G; jj += blockDim.x >> 5) {
          const zd* abp = ab + size_t(g0 + jj) * nmaxp * 2;
          float a = 0.f;
          for (int n = 1 + lane; n <= s_nm[jj]; n += 32) a += order_amplitude(abp + 2 * n, n);
          for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
          if (lane == 0) s_amp[jj] = a;
        }
      }
    }
    __syncthreads();
    if (live0) {
      for (int j = 0; j < G; ++j) {
        const lmb_sphere sp = spheres[g0 + j];
        Geometry<float> g[2];
        for (int l = 0; l < 2; ++l)
          g[l] = geometry<float, true>(k, x[l] - sp.x_p, y[l] - sp.y_p, z[l] - sp.z_p,
                                       z[l], sp.z_p, bohren);
        PairSumsV S;
        order_sum_pair(pair_in(g[0], g[1]), rec + s_off[j], s_nm[j], S);
        const float amp = kHologram ? s_amp[j] : 0.f;
#pragma unroll
        for (int l = 0; l < 2; ++l) {
          const Sums<float> sl = pair_lane_value(S, l, g[l].smu);
          cplx<float> ep[3];
          epilogue<float>(g[l], sl, cart, ep);
          if (aberr != 0.) {
            const cplx<float> ph =
                aberration_phase<float>(aberr, x[l] - sp.x_p, y[l] - sp.y_p, sp.z_p);
            for (int c = 0; c < 3; ++c) ep[c] = ph * ep[c];
          }
          for (int c = 0; c < 3; ++c) e[l][c] = e[l][c] + ep[c];
          if (kHologram) holo_bound_add(ep, amp, g[l].ikr, m1[l], m0[l]);
        }
      }
    }
  }
  if constexpr (kHologram) {
    float* o = reinterpret_cast<float*>(out) + (size_t)item * npts;
    bool mark[2] = {false, false};
    for (int l = 0; l < 2; ++l) {
      if (!(l == 0 ? live0 : live1)) continue;
      const float h = intensity<float>(e[l]);
      mark[l] = holo_needs_fp64(h, m1[l], m0[l]);
      if (!mark[l]) o[l ? p1 : p0] = h;
    }
    holo_resum64(mark[0], p0, mark[1], p1, base, smem, resum_group, coords, npts,
                 spheres, pb, pe, ab, nmax, nmaxp, k, flags, aberr, o);
  } else {
    if (!live0) return;
    float2* o = reinterpret_cast<float2*>(out) + (size_t)item * 3 * npts;
    for (int l = 0; l < 2; ++l) {
      if (l == 1 && !live1) break;
      const long long pix = l ? p1 : p0;
      for (int c = 0; c < 3; ++c) o[c * npts + pix] = make_float2(e[l][c].re, e[l][c].im);
    }
  }
}

// ---------------------------------------------------------------------------
// Population chi^2: sum over the pixels of ((H - data) / noise)^2 for each
// of nitems particle lists (the objective of a differential-evolution
// generation), NaN residuals skipped as numpy.nansum does.  Per (item,
// block) partial sums in FP64; k_chi2_reduce adds them in a fixed order.
// With crop_start, item i is compared with the pixels of its own crop
// item_crop[i], [crop_start[c], crop_start[c + 1]) of coords and data (the
// searches of many features in one launch); the grid covers the largest
// crop, and blocks past an item's crop add zeros.  An item whose crop range
// is invalid gets NaN.
template <typename R>
__global__ void __launch_bounds__(256)
k_chi2(const double* __restrict__ coords, long long npts,
       const long long* __restrict__ crop_start, const int* __restrict__ item_crop,
       int ncrops, const lmb_sphere* __restrict__ spheres,
       const int* __restrict__ item_start, const zd* __restrict__ ab,
       const int* __restrict__ nmax, int nmaxp, double k, int flags,
       double aberr, const double* __restrict__ data, double inv_noise,
       double* __restrict__ partial, int* __restrict__ partial_bad) {
  extern __shared__ __align__(16) char smem[];
  __shared__ double red[256 / 32];
  __shared__ int redb[256 / 32];
  Quad<R>* coef = reinterpret_cast<Quad<R>*>(smem);
  const int item = blockIdx.y;
  const size_t slot = (size_t)item * gridDim.x + blockIdx.x;
  long long base = 0, count = npts;
  if (crop_start) {
    const int c = item_crop[item];
    bool ok = c >= 0 && c < ncrops;
    if (ok) {
      base = crop_start[c];
      count = crop_start[c + 1] - base;
      ok = base >= 0 && count >= 0 && base + count <= npts &&
           count <= (long long)gridDim.x * blockDim.x;
    }
    // uniform over the block: before any barrier
    if (!ok || (long long)blockIdx.x * blockDim.x >= count) {
      if (threadIdx.x == 0) {
        partial[slot] = ok ? 0. : __longlong_as_double(0x7ff8000000000000LL);
        partial_bad[slot] = 0;
      }
      return;
    }
  }
  const long long pix = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = pix < count;
  const bool cart = flags & LMB_CARTESIAN;
  const bool bohren = flags & LMB_BOHREN;
  double x = 0., y = 0., z = 0.;
  if (live) {
    x = coords[base + pix];
    y = coords[npts + base + pix];
    z = coords[2 * npts + base + pix];
  }
  cplx<R> e[3];
  for (int c = 0; c < 3; ++c) e[c] = mk(R(0), R(0));
  const int pb = item_start[item], pe = item_start[item + 1];
  for (int p = pb; p < pe; ++p) {
    const int nm = min(max(nmax[p], 0), nmaxp - 1);
    __syncthreads();
    stage_coef<R, false>(ab + size_t(p) * nmaxp * 2, (const zd*)0, nm, coef);
    __syncthreads();
    if (live) {
      const lmb_sphere sp = spheres[p];
      const Geometry<R> g = geometry<R>(k, x - sp.x_p, y - sp.y_p, z - sp.z_p, z,
                                        sp.z_p, bohren);
      const Sums<R> sm = order_sum<R>(g, coef, nm);
      cplx<R> ep[3];
      epilogue<R>(g, sm, cart, ep);
      if (aberr != 0.) {  // spherical aberration, as k_field
        const cplx<R> ph = aberration_phase<R>(aberr, x - sp.x_p, y - sp.y_p, sp.z_p);
        for (int c = 0; c < 3; ++c) ep[c] = ph * ep[c];
      }
      for (int c = 0; c < 3; ++c) e[c] = e[c] + ep[c];
    }
  }
  double v = 0.;
  int bad = 0;
  if (live) {
    const R h = intensity<R>(e);
    bad = isfinite(h) ? 0 : 1;
    const double r = (double(h) - data[base + pix]) * inv_noise;
    if (r == r) v = r * r;  // nansum
  }
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_xor_sync(0xffffffffu, v, o);
    bad += __shfl_xor_sync(0xffffffffu, bad, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[warp] = v;
    redb[warp] = bad;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.;
    int b = 0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) {
      t += red[w];
      b += redb[w];
    }
    partial[slot] = t;
    partial_bad[slot] = b;
  }
}

__global__ void k_chi2_reduce(const double* partial, const int* partial_bad,
                              int nblocks, int nitems, double* chi2,
                              int* nonfinite) {
  const int item = blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= nitems) return;
  double s = 0.;
  int b = 0;
  for (int k = 0; k < nblocks; ++k) {
    s += partial[(size_t)item * nblocks + k];
    b += partial_bad[(size_t)item * nblocks + k];
  }
  chi2[item] = s;
  if (nonfinite) nonfinite[item] = b;
}

// ---------------------------------------------------------------------------
// Hologram + 6-column Jacobian, single sphere per item.

// With kAberr (fits with spherical aberration c = aberr): the phase and
// its gradient at pixel offset (dx, dy) from a particle at height zp enter
// the epilogue and the x_p, y_p, z_p columns.
template <bool kAberr = false>
__device__ inline void holo_jac_pixel(const Geometry<float>& g,
                                      const Quad<float>* coef, int nm, float kf,
                                      float* H, float* dH, double aberr = 0.,
                                      double dx = 0., double dy = 0.,
                                      double zp = 0.) {
  const JacSums<float> A = order_sum_jac<float>(g, coef, nm);
  if constexpr (kAberr) {
    float dphi[3], hphi;
    const cplx<float> w = aberration_wave<float>(aberr, dx, dy, zp, dphi);
    holo_jac_reverse<float, true>(g, A, kf, H, dH, w, &hphi);
    for (int j = 0; j < 3; ++j) dH[j] += hphi * dphi[j];
  } else {
    holo_jac_reverse<float>(g, A, kf, H, dH);
  }
}

// kAberr: the spherical-aberration phase of coefficient aberr in the
// hologram and the x_p, y_p, z_p columns (lmb_jacobian_aberrated).
template <bool kAberr = false>
__global__ void __launch_bounds__(128)
k_jacobian(const double* __restrict__ coords, long long npts,
           const lmb_sphere* __restrict__ spheres, const zd* __restrict__ ab,
           const zd* __restrict__ dab, const int* __restrict__ nmax, int nmaxp,
           double k, int flags, double* holo, double* jac, double aberr = 0.) {
  extern __shared__ __align__(16) char smem[];
  Quad<float>* coef = reinterpret_cast<Quad<float>*>(smem);
  const int item = blockIdx.y;
  const int nm = min(max(nmax[item], 0), nmaxp - 1);
  stage_coef<float, true>(ab + size_t(item) * nmaxp * 2,
                          dab + size_t(item) * nmaxp * 4, nm, coef);
  __syncthreads();
  const long long pix = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= npts) return;
  const lmb_sphere sp = spheres[item];
  const double x = coords[pix], y = coords[npts + pix], z = coords[2 * npts + pix];
  const Geometry<float> g = geometry<float>(k, x - sp.x_p, y - sp.y_p, z - sp.z_p,
                                            z, sp.z_p, flags & LMB_BOHREN);
  float H, dH[6];
  holo_jac_pixel<kAberr>(g, coef, nm, float(k), &H, dH, aberr, x - sp.x_p,
                         y - sp.y_p, sp.z_p);
  if (holo) holo[(size_t)item * npts + pix] = H;
  double* jo = jac + (size_t)item * 6 * npts;
  for (int j = 0; j < 6; ++j) jo[j * npts + pix] = dH[j];
}

// k_jacobian with the packed two-pixel loop: each thread takes two adjacent
// pixels (pair records, stage_pair).
template <bool kAberr = false>
__global__ void __launch_bounds__(128, 3)
k_jacobian_pair(const double* __restrict__ coords, long long npts,
                const lmb_sphere* __restrict__ spheres, const zd* __restrict__ ab,
                const zd* __restrict__ dab, const int* __restrict__ nmax, int nmaxp,
                double k, int flags, double* holo, double* jac, double aberr = 0.) {
  extern __shared__ __align__(16) char smem[];
  float4* rec = reinterpret_cast<float4*>(smem);
  const int item = blockIdx.y;
  const int nm = min(max(nmax[item], 0), nmaxp - 1);
  stage_pair(ab + size_t(item) * nmaxp * 2, dab + size_t(item) * nmaxp * 4, nm, rec);
  __syncthreads();
  const long long p0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 2;
  if (p0 >= npts) return;
  const bool live1 = p0 + 1 < npts;
  const long long p1 = live1 ? p0 + 1 : p0;
  const lmb_sphere sp = spheres[item];
  const double dx[2] = {coords[p0] - sp.x_p, coords[p1] - sp.x_p};
  const double dy[2] = {coords[npts + p0] - sp.y_p, coords[npts + p1] - sp.y_p};
  const double z0 = coords[2 * npts + p0], z1 = coords[2 * npts + p1];
  Geometry<float> g[2];
  g[0] = geometry<float>(k, dx[0], dy[0], z0 - sp.z_p, z0, sp.z_p, flags & LMB_BOHREN);
  g[1] = geometry<float>(k, dx[1], dy[1], z1 - sp.z_p, z1, sp.z_p, flags & LMB_BOHREN);
  PairSums P;
  order_sum_jac_pair(pair_in(g[0], g[1]), rec, nm, P);
  double* jo = jac + (size_t)item * 6 * npts;
  for (int l = 0; l < 2; ++l) {
    if (l == 1 && !live1) break;
    const long long pix = l ? p1 : p0;
    const JacSums<float> A = pair_lane(P, l, g[l].smu);
    float H, dH[6];
    if constexpr (kAberr) {
      float dphi[3], hphi;
      const cplx<float> w = aberration_wave<float>(aberr, dx[l], dy[l], sp.z_p, dphi);
      holo_jac_reverse<float, true>(g[l], A, float(k), &H, dH, w, &hphi);
      for (int j = 0; j < 3; ++j) dH[j] += hphi * dphi[j];
    } else {
      holo_jac_reverse<float>(g[l], A, float(k), &H, dH);
    }
    if (holo) holo[(size_t)item * npts + pix] = H;
    for (int j = 0; j < 6; ++j) jo[j * npts + pix] = dH[j];
  }
}

// ---------------------------------------------------------------------------
// Block reduction of NV floats held by every thread; result in red[0..NV-1]
// of thread 0's view (shared).  Fixed order: deterministic.

template <int NV, int TPB>
__device__ inline void block_reduce(float* v, float* red /* [TPB/32][NV] */) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    float s = v[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    v[j] = s;
  }
  if (lane == 0)
#pragma unroll
    for (int j = 0; j < NV; ++j) red[warp * NV + j] = v[j];
  __syncthreads();
  if (threadIdx.x < NV) {
    float s = 0.f;
    for (int w = 0; w < TPB / 32; ++w) s += red[w * NV + threadIdx.x];
    red[threadIdx.x] = s;  // safe: each thread reads then writes its own column
  }
  __syncthreads();
}

// VJP: per (item, block) partial sums of g * dH/dp.
__global__ void __launch_bounds__(128)
k_vjp(const double* __restrict__ coords, long long npts,
      const lmb_sphere* __restrict__ spheres, const zd* __restrict__ ab,
      const zd* __restrict__ dab, const int* __restrict__ nmax, int nmaxp, double k,
      int flags, const float* __restrict__ gout, double* partial) {
  extern __shared__ __align__(16) char smem[];
  __shared__ float red[(128 / 32) * 6];
  Quad<float>* coef = reinterpret_cast<Quad<float>*>(smem);
  const int item = blockIdx.y;
  const int nm = min(max(nmax[item], 0), nmaxp - 1);
  stage_coef<float, true>(ab + size_t(item) * nmaxp * 2,
                          dab + size_t(item) * nmaxp * 4, nm, coef);
  __syncthreads();
  const long long pix = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (pix < npts) {
    const lmb_sphere sp = spheres[item];
    const double x = coords[pix], y = coords[npts + pix], z = coords[2 * npts + pix];
    const Geometry<float> g = geometry<float>(k, x - sp.x_p, y - sp.y_p,
                                              z - sp.z_p, z, sp.z_p,
                                              flags & LMB_BOHREN);
    float H, dH[6];
    holo_jac_pixel(g, coef, nm, float(k), &H, dH);
    const float go = gout[(size_t)item * npts + pix];
    for (int j = 0; j < 6; ++j) acc[j] = go * dH[j];
  }
  block_reduce<6, 128>(acc, red);
  if (threadIdx.x < 6)
    partial[((size_t)item * gridDim.x + blockIdx.x) * 6 + threadIdx.x] = red[threadIdx.x];
}

// k_vjp with the packed two-pixel loop (two adjacent pixels per thread).
__global__ void __launch_bounds__(128, 3)
k_vjp_pair(const double* __restrict__ coords, long long npts,
           const lmb_sphere* __restrict__ spheres, const zd* __restrict__ ab,
           const zd* __restrict__ dab, const int* __restrict__ nmax, int nmaxp,
           double k, int flags, const float* __restrict__ gout, double* partial) {
  extern __shared__ __align__(16) char smem[];
  __shared__ float red[(128 / 32) * 6];
  float4* rec = reinterpret_cast<float4*>(smem);
  const int item = blockIdx.y;
  const int nm = min(max(nmax[item], 0), nmaxp - 1);
  stage_pair(ab + size_t(item) * nmaxp * 2, dab + size_t(item) * nmaxp * 4, nm, rec);
  __syncthreads();
  const long long p0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 2;
  float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (p0 < npts) {
    const bool live1 = p0 + 1 < npts;
    const long long p1 = live1 ? p0 + 1 : p0;
    const lmb_sphere sp = spheres[item];
    const double z0 = coords[2 * npts + p0], z1 = coords[2 * npts + p1];
    Geometry<float> g[2];
    g[0] = geometry<float>(k, coords[p0] - sp.x_p, coords[npts + p0] - sp.y_p,
                           z0 - sp.z_p, z0, sp.z_p, flags & LMB_BOHREN);
    g[1] = geometry<float>(k, coords[p1] - sp.x_p, coords[npts + p1] - sp.y_p,
                           z1 - sp.z_p, z1, sp.z_p, flags & LMB_BOHREN);
    PairSums P;
    order_sum_jac_pair(pair_in(g[0], g[1]), rec, nm, P);
    for (int l = 0; l < 2; ++l) {
      if (l == 1 && !live1) break;
      const long long pix = l ? p1 : p0;
      const JacSums<float> A = pair_lane(P, l, g[l].smu);
      float H, dH[6];
      holo_jac_reverse<float>(g[l], A, float(k), &H, dH);
      const float go = gout[(size_t)item * npts + pix];
      for (int j = 0; j < 6; ++j) acc[j] += go * dH[j];
    }
  }
  block_reduce<6, 128>(acc, red);
  if (threadIdx.x < 6)
    partial[((size_t)item * gridDim.x + blockIdx.x) * 6 + threadIdx.x] = red[threadIdx.x];
}

__global__ void k_vjp_reduce(const double* partial, int nblocks, int nitems,
                             double* grad) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nitems * 6) return;
  const int item = t / 6, j = t % 6;
  double s = 0.;
  for (int b = 0; b < nblocks; ++b) s += partial[((size_t)item * nblocks + b) * 6 + j];
  grad[t] = s;
}

// ---------------------------------------------------------------------------
// Batched Levenberg-Marquardt.

enum { FIT_NSUM = 28 };  // f^2, J^T J (21), J^T f (6)

struct EvalPoint {
  double p[6];    // parameter vector under evaluation
  int active;     // 1 while an evaluation of this feature is pending
  int pad;
};

struct FitCtx {
  const lmb_feature* features;
  const float* data;
  const float* coords;
  lmb_sphere* params;
  lmb_fit_result* results;
  LMState* state;
  EvalPoint* ev;
  double* base;        // [nf][6] start values (fixed parameters keep them)
  zd* ab;              // [nf][nmaxp][2]
  zd* dab;             // [nf][nmaxp][4]
  Quad<float>* coef32; // [nf][nmaxp][JAC_QUADS or PAIR_QUADS] FP32 records
                       // of the evaluation point (pair layout if pair_records)
  int* nmax;           // [nf]
  int* tile_begin;     // [nf+1]
  int2* tiles;         // [max_tiles]
  double* partial;     // [max_tiles][FIT_NSUM]
  int* counters;       // [0] tile queue, [1] running, [2] ntiles, [3] overflow,
                       // [4] waiting for data, [5] active tiles this round
  int* active_tiles;   // [max_tiles] tiles of the features evaluated this
                       // round (filled by k_fit_step, in no fixed order)
  unsigned long long* work;  // [0] pixels, [1] pixel-orders evaluated
  long long total_pixels;
  int nf, nmax_cap, max_tiles, tile_pixels;
  int nlayers;                // 1: homogeneous spheres
  const double* layer_frac;   // [nf][nlayers-1] inner radii / outer radius
  const double* layer_index;  // [nf][nlayers-1][2] inner layer indices
  double n_m, wavelength, k, inv_noise;
  double aberr;  // spherical-aberration coefficient c (0: ideal optics)
  LMSettings set;
  int variables, flags, max_iterations;
  int pair_records;    // the evaluation kernel reads stage_pair records
  // Streamed admission: features [0, *ready) have their data on the
  // device; the rest wait in LM_PHASE_INIT (counted in counters[4]).  A
  // negative value withdraws the batch.  Null: every feature is ready.
  const int* ready;
};

__device__ inline bool feature_valid(const lmb_feature& ft, long long total) {
  return ft.npix >= 0 && ft.data_offset >= 0 && ft.data_offset + ft.npix <= total &&
         (ft.nx == 0 || (ft.nx > 0 && ft.ny > 0 && (long long)ft.nx * ft.ny == ft.npix));
}

// Tile table and state initialisation; one block.
__global__ void k_fit_setup(FitCtx c) {
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < c.nf; base += blockDim.x) {
    const int f = base + threadIdx.x;
    int nt = 0;
    if (f < c.nf) {
      const lmb_feature ft = c.features[f];
      if (feature_valid(ft, c.total_pixels))
        nt = ft.npix > 0 ? int((ft.npix + c.tile_pixels - 1) / c.tile_pixels) : 0;
    }
    // inclusive scan of nt across the block (Hillis-Steele in shared memory)
    __shared__ int sc[1024];
    sc[threadIdx.x] = nt;
    __syncthreads();
    for (int o = 1; o < blockDim.x; o <<= 1) {
      const int v = threadIdx.x >= o ? sc[threadIdx.x - o] : 0;
      __syncthreads();
      sc[threadIdx.x] += v;
      __syncthreads();
    }
    if (f < c.nf) c.tile_begin[f] = carry + sc[threadIdx.x] - nt;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += sc[threadIdx.x];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    c.tile_begin[c.nf] = carry;
    c.counters[2] = carry > c.max_tiles ? 0 : carry;
    c.counters[3] = carry > c.max_tiles ? 1 : 0;
    c.counters[0] = 0;
    c.counters[1] = 0;
    c.counters[4] = 0;
    c.counters[5] = 0;
    c.work[0] = 0ull;
    c.work[1] = 0ull;
  }
  __syncthreads();
  const int ntiles = carry;
  if (ntiles > c.max_tiles) return;
  for (int f = threadIdx.x; f < c.nf; f += blockDim.x) {
    const int tb = c.tile_begin[f];
    const long long np = c.features[f].npix;
    for (int t = 0; tb + t < c.tile_begin[f + 1]; ++t)
      c.tiles[tb + t] = make_int2(f, t * c.tile_pixels);
    LMState& s = c.state[f];
    const lmb_sphere p0 = c.params[f];
    const double pv[6] = {p0.x_p, p0.y_p, p0.z_p, p0.a_p, p0.n_p, p0.k_p};
    int n = 0;
    for (int j = 0; j < 6; ++j) {
      c.base[f * 6 + j] = pv[j];
      c.ev[f].p[j] = pv[j];
      if (c.variables & (1 << j)) {
        s.slot[n] = j;
        s.x[n] = pv[j];
        ++n;
      }
    }
    s.n = n;
    s.phase = LM_PHASE_INIT;
    s.info = 0;
    s.iter = s.nfev = s.njev = 0;
    s.f2_final = 0.;
    c.ev[f].active = 0;
    if (n == 0 || np < n || !feature_valid(c.features[f], c.total_pixels)) {
      // MINPACK's improper input (m < n), or a feature outside the data
      s.phase = LM_PHASE_DONE;
      s.info = -1;
    }
  }
}

// Evaluation: persistent CTAs pull tiles from an atomic queue.
template <int TPB, int PPT, int MINB, bool kAberr = false>
__global__ void __launch_bounds__(TPB, MINB)
k_fit_eval(FitCtx c) {
  extern __shared__ __align__(16) char smem[];
  Quad<float>* coef = reinterpret_cast<Quad<float>*>(smem);
  __shared__ float red[(TPB / 32) * FIT_NSUM];
  __shared__ int s_tile;
  const int ntiles = c.counters[5];  // tiles of active features
  const int nmaxp = c.nmax_cap + 1;
  const bool bohren = c.flags & LMB_BOHREN;
  const float kf = float(c.k);
  const float inv_noise = float(c.inv_noise);
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(c.counters, 1);
    __syncthreads();
    const int q = s_tile;
    if (q >= ntiles) break;
    const int t = c.active_tiles[q];  // global tile index: fixes partial[]
    const int2 tile = c.tiles[t];
    const int f = tile.x;
    if (!c.ev[f].active) {
      __syncthreads();
      continue;
    }
    const int nm = min(max(c.nmax[f], 0), nmaxp - 1);
    {
      const float4* src =
          reinterpret_cast<const float4*>(c.coef32 + size_t(f) * nmaxp * JAC_QUADS);
      float4* dst = reinterpret_cast<float4*>(coef);
      for (int i = threadIdx.x; i < JAC_QUADS * (nm + 1); i += TPB) dst[i] = src[i];
    }
    const lmb_feature ft = c.features[f];
    const EvalPoint ep = c.ev[f];
    __syncthreads();
    float acc[FIT_NSUM];
#pragma unroll
    for (int j = 0; j < FIT_NSUM; ++j) acc[j] = 0.f;
    for (int q = 0; q < PPT; ++q) {
      const long long i = (long long)tile.y + q * TPB + threadIdx.x;
      if (i >= ft.npix || i >= (long long)tile.y + c.tile_pixels) break;
      double x, y;
      if (ft.nx > 0) {
        const long long row = i / ft.nx;
        x = ft.x0 + double(i - row * ft.nx);
        y = ft.y0 + double(row);
      } else {
        const float2 xy = reinterpret_cast<const float2*>(c.coords)[ft.data_offset + i];
        x = xy.x;
        y = xy.y;
      }
      const float d = c.data[ft.data_offset + i];
      const Geometry<float> g = geometry<float>(c.k, x - ep.p[0], y - ep.p[1],
                                                -ep.p[2], 0., ep.p[2], bohren);
      float H, dH[6];
      holo_jac_pixel<kAberr>(g, coef, nm, kf, &H, dH, c.aberr, x - ep.p[0],
                             y - ep.p[1], ep.p[2]);
      const float r = (H - d) * inv_noise;
      float J[6];
#pragma unroll
      for (int j = 0; j < 6; ++j) J[j] = dH[j] * inv_noise;
      acc[0] += r * r;
      int o = 1;
#pragma unroll
      for (int a = 0; a < 6; ++a)
#pragma unroll
        for (int b = a; b < 6; ++b) acc[o++] += J[a] * J[b];
#pragma unroll
      for (int a = 0; a < 6; ++a) acc[22 + a] += J[a] * r;
    }
    block_reduce<FIT_NSUM, TPB>(acc, red);
    if (threadIdx.x < FIT_NSUM)
      c.partial[(size_t)t * FIT_NSUM + threadIdx.x] = red[threadIdx.x];
    if (threadIdx.x == 0) {
      long long np = ft.npix - tile.y;
      if (np > c.tile_pixels) np = c.tile_pixels;
      atomicAdd(c.work, (unsigned long long)np);
      atomicAdd(c.work + 1, (unsigned long long)np * (unsigned long long)nm);
    }
    __syncthreads();
  }
}

// Two pixels of one sphere through one packed order loop; hologram and
// 6-column Jacobian of each.  (dx, dy, dz): pixel minus particle position.
// With kRecompute the pixel geometry is formed again after the order loop
// instead of being held in registers across it (the empty asm statements
// keep the compiler from merging the two computations).  U: the order
// loop's unroll factor.
template <bool kRecompute, bool kAberr = false, int U = 2>
__device__ inline void holo_jac_pair(double k, const double* dx,
                                     const double* dy, double dz, double zp,
                                     bool bohren, const float4* rec, int nm,
                                     float kf, float* H, float (*dH)[6],
                                     double aberr = 0.) {
  Geometry<float> g[2];
  for (int l = 0; l < 2; ++l)
    g[l] = geometry<float>(k, dx[l], dy[l], dz, 0., zp, bohren);
  PairSums P;
  order_sum_jac_pair<U>(pair_in(g[0], g[1]), rec, nm, P);
  if (kRecompute) {
    for (int l = 0; l < 2; ++l) {
      double x = dx[l], y = dy[l];
      asm volatile("" : "+d"(x), "+d"(y));
      g[l] = geometry<float>(k, x, y, dz, 0., zp, bohren);
    }
  }
#pragma unroll
  for (int lane = 0; lane < 2; ++lane) {
    const Geometry<float>& gl = g[lane];
    const JacSums<float> A = pair_lane(P, lane, gl.smu);
    if constexpr (kAberr) {
      float dphi[3], hphi;
      const cplx<float> w = aberration_wave<float>(aberr, dx[lane], dy[lane], zp, dphi);
      holo_jac_reverse<float, true>(gl, A, kf, &H[lane], dH[lane], w, &hphi);
      for (int j = 0; j < 3; ++j) dH[lane][j] += hphi * dphi[j];
    } else {
      holo_jac_reverse<float>(gl, A, kf, &H[lane], dH[lane]);
    }
  }
}

__device__ inline void fit_pixel_xy(const lmb_feature& ft, const float* coords,
                                    long long i, double* x, double* y) {
  if (ft.nx > 0) {
    const long long row = i / ft.nx;
    *x = ft.x0 + double(i - row * ft.nx);
    *y = ft.y0 + double(row);
  } else {
    const float2 xy = reinterpret_cast<const float2*>(coords)[ft.data_offset + i];
    *x = xy.x;
    *y = xy.y;
  }
}

// Evaluation with the packed two-pixel loop: as k_fit_eval, each thread
// takes pixel pairs (i, i + TPB) of its tile; PPT is even.  The records in
// coef32 are in the pair layout (stage_pair).
template <int TPB, int PPT, int MINB, bool kRecompute, bool kAberr = false>
__global__ void __launch_bounds__(TPB, MINB)
k_fit_eval_pair(FitCtx c) {
  static_assert(PPT % 2 == 0, "pixel pairs");
  extern __shared__ __align__(16) char smem[];
  float4* rec = reinterpret_cast<float4*>(smem);
  __shared__ float red[(TPB / 32) * FIT_NSUM];
  __shared__ int s_tile;
  const int ntiles = c.counters[5];  // tiles of active features
  const int nmaxp = c.nmax_cap + 1;
  const bool bohren = c.flags & LMB_BOHREN;
  const float kf = float(c.k);
  const float inv_noise = float(c.inv_noise);
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(c.counters, 1);
    __syncthreads();
    const int q = s_tile;
    if (q >= ntiles) break;
    const int t = c.active_tiles[q];  // global tile index: fixes partial[]
    const int2 tile = c.tiles[t];
    const int f = tile.x;
    if (!c.ev[f].active) {
      __syncthreads();
      continue;
    }
    const int nm = min(max(c.nmax[f], 0), nmaxp - 1);
    {
      const float4* src =
          reinterpret_cast<const float4*>(c.coef32) + size_t(f) * nmaxp * PAIR_QUADS;
      for (int i = threadIdx.x; i < PAIR_QUADS * (nm + 1); i += TPB) rec[i] = src[i];
    }
    const lmb_feature ft = c.features[f];
    const EvalPoint ep = c.ev[f];
    __syncthreads();
    float acc[FIT_NSUM];
#pragma unroll
    for (int j = 0; j < FIT_NSUM; ++j) acc[j] = 0.f;
    long long lim = (long long)tile.y + c.tile_pixels;
    if (lim > ft.npix) lim = ft.npix;
    for (int q = 0; q < PPT; q += 2) {
      const long long i0 = (long long)tile.y + q * TPB + threadIdx.x;
      if (i0 >= lim) break;
      const long long i1r = i0 + TPB;
      const bool v1 = i1r < lim;
      const long long i1 = v1 ? i1r : i0;
      double x0, y0, x1, y1;
      fit_pixel_xy(ft, c.coords, i0, &x0, &y0);
      fit_pixel_xy(ft, c.coords, i1, &x1, &y1);
      const float d0 = c.data[ft.data_offset + i0];
      const float d1 = c.data[ft.data_offset + i1];
      const double dx[2] = {x0 - ep.p[0], x1 - ep.p[0]};
      const double dy[2] = {y0 - ep.p[1], y1 - ep.p[1]};
      float H[2], dH[2][6];
      // the order loop unrolled by 3 where a thread holds 4 or more pixel
      // pairs (measured faster there), by 2 elsewhere
      holo_jac_pair<kRecompute, kAberr, (PPT >= 8 ? 3 : 2)>(
          c.k, dx, dy, -ep.p[2], ep.p[2], bohren, rec, nm, kf, H, dH, c.aberr);
#pragma unroll
      for (int lane = 0; lane < 2; ++lane) {
        if (lane == 1 && !v1) break;
        const float r = (H[lane] - (lane ? d1 : d0)) * inv_noise;
        float J[6];
#pragma unroll
        for (int j = 0; j < 6; ++j) J[j] = dH[lane][j] * inv_noise;
        acc[0] += r * r;
        int o = 1;
#pragma unroll
        for (int a = 0; a < 6; ++a)
#pragma unroll
          for (int b = a; b < 6; ++b) acc[o++] += J[a] * J[b];
#pragma unroll
        for (int a = 0; a < 6; ++a) acc[22 + a] += J[a] * r;
      }
    }
    block_reduce<FIT_NSUM, TPB>(acc, red);
    if (threadIdx.x < FIT_NSUM)
      c.partial[(size_t)t * FIT_NSUM + threadIdx.x] = red[threadIdx.x];
    if (threadIdx.x == 0) {
      const long long np = lim - tile.y;
      atomicAdd(c.work, (unsigned long long)np);
      atomicAdd(c.work + 1, (unsigned long long)np * (unsigned long long)nm);
    }
    __syncthreads();
  }
}

// Warp-granular evaluation: every warp pulls whole 512-pixel tiles from the
// queue (16 pixels per lane), keeps its own copy of the coefficients of the
// feature it is on, and reduces its 28 sums with shuffles -- no block-wide
// barrier anywhere.  WPB warps per CTA, MINB CTAs per SM at least.
template <int WPB, int MINB, bool kAberr = false>
__global__ void __launch_bounds__(WPB * 32, MINB)
k_fit_eval_warp(FitCtx c) {
  extern __shared__ __align__(16) char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nmaxp = c.nmax_cap + 1;
  Quad<float>* coef = reinterpret_cast<Quad<float>*>(smem) +
                      size_t(warp) * JAC_QUADS * nmaxp;
  const int ntiles = c.counters[5];  // tiles of active features
  const bool bohren = c.flags & LMB_BOHREN;
  const float kf = float(c.k);
  const float inv_noise = float(c.inv_noise);
  constexpr int PPL = 16;  // pixels per lane: 32 x 16 = 512 = one tile
  int cur = -1, nm = 0;
  for (;;) {
    int q = 0;
    if (lane == 0) q = atomicAdd(c.counters, 1);
    q = __shfl_sync(0xffffffffu, q, 0);
    if (q >= ntiles) break;
    const int t = c.active_tiles[q];
    const int2 tile = c.tiles[t];
    const int f = tile.x;
    if (!c.ev[f].active) continue;
    if (f != cur) {
      __syncwarp();
      nm = min(max(c.nmax[f], 0), nmaxp - 1);
      const float4* src =
          reinterpret_cast<const float4*>(c.coef32 + size_t(f) * nmaxp * JAC_QUADS);
      float4* dst = reinterpret_cast<float4*>(coef);
      for (int i = lane; i < JAC_QUADS * (nm + 1); i += 32) dst[i] = src[i];
      __syncwarp();
      cur = f;
    }
    const lmb_feature ft = c.features[f];
    const EvalPoint ep = c.ev[f];
    float acc[FIT_NSUM];
#pragma unroll
    for (int j = 0; j < FIT_NSUM; ++j) acc[j] = 0.f;
    for (int q = 0; q < PPL; ++q) {
      const long long i = (long long)tile.y + q * 32 + lane;
      if (i >= ft.npix || i >= (long long)tile.y + c.tile_pixels) break;
      double x, y;
      if (ft.nx > 0) {
        const long long row = i / ft.nx;
        x = ft.x0 + double(i - row * ft.nx);
        y = ft.y0 + double(row);
      } else {
        const float2 xy = reinterpret_cast<const float2*>(c.coords)[ft.data_offset + i];
        x = xy.x;
        y = xy.y;
      }
      const float d = c.data[ft.data_offset + i];
      const Geometry<float> g = geometry<float>(c.k, x - ep.p[0], y - ep.p[1],
                                                -ep.p[2], 0., ep.p[2], bohren);
      float H, dH[6];
      holo_jac_pixel<kAberr>(g, coef, nm, kf, &H, dH, c.aberr, x - ep.p[0],
                             y - ep.p[1], ep.p[2]);
      const float r = (H - d) * inv_noise;
      float J[6];
#pragma unroll
      for (int j = 0; j < 6; ++j) J[j] = dH[j] * inv_noise;
      acc[0] += r * r;
      int o = 1;
#pragma unroll
      for (int a = 0; a < 6; ++a)
#pragma unroll
        for (int b = a; b < 6; ++b) acc[o++] += J[a] * J[b];
#pragma unroll
      for (int a = 0; a < 6; ++a) acc[22 + a] += J[a] * r;
    }
#pragma unroll
    for (int j = 0; j < FIT_NSUM; ++j) {
      float v = acc[j];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      acc[j] = v;
    }
    // lane j writes sum j (a fixed-order, deterministic reduction)
#pragma unroll
    for (int j = 0; j < FIT_NSUM; ++j)
      if (lane == j) c.partial[(size_t)t * FIT_NSUM + j] = acc[j];
    if (lane == 0) {
      long long np = ft.npix - tile.y;
      if (np > c.tile_pixels) np = c.tile_pixels;
      atomicAdd(c.work, (unsigned long long)np);
      atomicAdd(c.work + 1, (unsigned long long)np * (unsigned long long)nm);
    }
  }
}

// Warp 0 of k_fit_step: gather the feature's sums, advance the LM state
// machine, and write the next evaluation point to p (lane 0).  Returns,
// uniformly over the warp, whether that point's Mie coefficients are needed:
// 0 for a finished, withdrawn or not yet admitted feature.  *phase gets the
// phase the feature was in.
__device__ __forceinline__ int fit_step_advance(const FitCtx& c, int f, int lane, double* p,
                                                int* phase_out) {
  if (c.counters[3]) return 0;  // tile table overflow: nothing ran
  LMState* gs = c.state + f;
  const int phase = gs->phase;
  *phase_out = phase;
  if (phase == LM_PHASE_DONE) return 0;
  if (phase == LM_PHASE_INIT && c.ready) {
    // one read for the whole warp: the flag may change while we look
    int r = 0;
    if (lane == 0) r = *reinterpret_cast<const volatile int*>(c.ready);
    r = __shfl_sync(0xffffffffu, r, 0);
    if (r < 0) {  // withdrawn by the producer: this feature is not fitted
      if (lane == 0) {
        gs->phase = LM_PHASE_DONE;
        gs->info = -4;
        c.ev[f].active = 0;
      }
      return 0;
    }
    if (f >= r) {
      if (lane == 0) atomicAdd(c.counters + 4, 1);
      return 0;
    }
  }
  if (phase == LM_PHASE_INIT) {
    if (lane == 0)
      for (int j = 0; j < 6; ++j) p[j] = c.base[f * 6 + j];
    return 1;
  }
  int need = 0;
  if (phase == LM_PHASE_FIRST || phase == LM_PHASE_TRIAL) {
    double v[FIT_NSUM];
    for (int j = 0; j < FIT_NSUM; ++j) v[j] = 0.;
    const int tb = c.tile_begin[f], te = c.tile_begin[f + 1];
    for (int t = tb + lane; t < te; t += 32)
      for (int j = 0; j < FIT_NSUM; ++j) v[j] += c.partial[(size_t)t * FIT_NSUM + j];
    for (int j = 0; j < FIT_NSUM; ++j)
      for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_xor_sync(0xffffffffu, v[j], o);
    if (lane == 0) {
      LMEval ev;
      ev.f2 = v[0];
      for (int j = 0; j < 21; ++j) ev.jtj[j] = v[1 + j];
      for (int j = 0; j < 6; ++j) ev.jtf[j] = v[22 + j];
      LMState s = *gs;
      const int done = phase == LM_PHASE_FIRST ? lm_start(s, ev, c.set)
                                               : lm_after_trial(s, ev, c.set);
      if (done || s.nfev >= c.max_iterations) {
        if (!done && s.info == 0) s.info = 5;  // evaluation cap reached
        s.phase = LM_PHASE_DONE;
        c.ev[f].active = 0;
      } else {
        s.phase = LM_PHASE_TRIAL;
        for (int j = 0; j < 6; ++j) p[j] = c.base[f * 6 + j];
        for (int a = 0; a < s.n; ++a) p[s.slot[a]] = s.x[a] + s.p[a];
        need = 1;
      }
      *gs = s;
    }
    need = __shfl_sync(0xffffffffu, need, 0);
  }
  return need;
}

// One two-warp block per feature: warp 0 gathers the sums and advances the
// LM state machine; then both warps compute the Mie coefficients of the
// next evaluation point (block_sphere_ab, block_layered_ab) and stage their
// records, and warp 0 lists the feature's tiles.  Both warps pass every
// __syncthreads on every path.
__global__ void __launch_bounds__(64)
k_fit_step(FitCtx c) {
  extern __shared__ __align__(16) char smem[];
  __shared__ double s_p[6];
  __shared__ double s_r[LMB_MAX_LAYERS], s_i[2 * LMB_MAX_LAYERS];
  __shared__ int s_need, s_st;
  const int f = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (f >= c.nf) return;  // the whole block
  LMState* gs = c.state + f;
  int phase = LM_PHASE_DONE;
  if (warp == 0) {
    const int need = fit_step_advance(c, f, lane, s_p, &phase);
    __syncwarp();
    const int L = c.nlayers;
    if (need && L > 1 && lane < L) {
      const bool outer = lane == L - 1;
      s_r[lane] = outer ? s_p[3] : c.layer_frac[size_t(f) * (L - 1) + lane] * s_p[3];
      s_i[2 * lane] = outer ? s_p[4] : c.layer_index[(size_t(f) * (L - 1) + lane) * 2];
      s_i[2 * lane + 1] =
          outer ? s_p[5] : c.layer_index[(size_t(f) * (L - 1) + lane) * 2 + 1];
    }
    if (lane == 0) s_need = need;
  }
  __syncthreads();  // both warps, on every path
  if (!s_need) return;
  const int nmaxp = c.nmax_cap + 1;
  int st;
  if (c.nlayers > 1) {
    st = block_layered_ab(s_r, s_i, c.nlayers, c.n_m, c.wavelength, c.nmax_cap,
                          smem, c.ab + size_t(f) * nmaxp * 2,
                          c.dab + size_t(f) * nmaxp * 4, c.nmax + f);
  } else {
    AbScratch w = carve_ab_scratch(smem, nmaxp);
    st = block_sphere_ab(s_p[3], s_p[4], s_p[5], c.n_m, c.wavelength, c.nmax_cap,
                         w, c.ab + size_t(f) * nmaxp * 2, c.dab + size_t(f) * nmaxp * 4,
                         c.nmax + f);
  }
  // warp 0's status, a_n, b_n (global) and n_max for both warps, which
  // stage the records together
  if (threadIdx.x == 0) s_st = st;
  __syncthreads();
  if (s_st == LMB_OK) {
    const zd* abf = c.ab + size_t(f) * nmaxp * 2;
    const zd* dabf = c.dab + size_t(f) * nmaxp * 4;
    const int nm = min(c.nmax[f], nmaxp - 1);
    if (c.pair_records)
      stage_pair(abf, dabf, nm,
                 reinterpret_cast<float4*>(c.coef32) + size_t(f) * nmaxp * PAIR_QUADS);
    else
      stage_coef<float, true>(abf, dabf, nm, c.coef32 + size_t(f) * nmaxp * JAC_QUADS);
  }
  if (warp != 0) return;
  int base = -1;
  const int tb = c.tile_begin[f], nt = c.tile_begin[f + 1] - tb;
  if (lane == 0) {
    if (st != LMB_OK) {
      gs->phase = LM_PHASE_DONE;
      gs->info = -3;
      c.ev[f].active = 0;
    } else {
      if (phase == LM_PHASE_INIT) gs->phase = LM_PHASE_FIRST;
      for (int j = 0; j < 6; ++j) c.ev[f].p[j] = s_p[j];
      c.ev[f].active = 1;
      atomicAdd(c.counters + 1, 1);
      base = atomicAdd(c.counters + 5, nt);  // this feature's tiles join
    }
  }
  base = __shfl_sync(0xffffffffu, base, 0);
  if (base >= 0)
    for (int j = lane; j < nt; j += 32) c.active_tiles[base + j] = tb + j;
}

// Results: fitted parameters, uncertainties, redchi; one thread per feature.
__global__ void k_fit_finalize(FitCtx c) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= c.nf) return;
  const LMState s = c.state[f];
  lmb_fit_result r;
  for (int j = 0; j < 6; ++j) r.dparams[j] = 0.;
  double pv[6];
  for (int j = 0; j < 6; ++j) pv[j] = c.base[f * 6 + j];
  const long long npix = c.features[f].npix;
  if (c.counters[3]) {
    r.status = -1;
    r.success = 0;
    r.redchi = 0.;
    r.cost = 0.;
    r.nfev = r.njev = 0;
  } else {
    int info = s.info;
    if (s.phase != LM_PHASE_DONE && info == 0) info = 5;
    r.status = lm_scipy_status(info);
    r.success = r.status > 0;
    r.nfev = s.nfev;
    r.njev = s.njev;
    r.cost = 0.5 * s.f2_final;
    r.redchi = 0.;
    if (info > 0 && s.n > 0) {
      for (int a = 0; a < s.n; ++a) pv[s.slot[a]] = s.x[a];
      double dp[LM_NV];
      lm_statistics(s, npix, &r.redchi, dp);
      for (int a = 0; a < s.n; ++a) r.dparams[s.slot[a]] = dp[a];
    }
  }
  lmb_sphere out;
  out.x_p = pv[0];
  out.y_p = pv[1];
  out.z_p = pv[2];
  out.a_p = pv[3];
  out.n_p = pv[4];
  out.k_p = pv[5];
  c.params[f] = out;
  c.results[f] = r;
}

// ---------------------------------------------------------------------------
// Differential evolution on the device: the searches of many features
// stepped together -- k_de_trial forms every search's trial population
// (one thread per candidate) and the sphere records to evaluate, the caller
// evaluates them (lmb_sphere_ab + lmb_chi2_crops), k_de_select keeps the
// better of each pair and tests convergence (one warp per search).  The
// step is scipy's best1bin with deferred updating, dithered mutation and
// binomial crossover; the random numbers come from the SplitMix64 mixing
// function (Steele, Lea and Flood, OOPSLA 2014) of a counter (search key,
// generation, candidate, draw), so a search is reproducible for a seed but
// does not follow scipy's random stream.

__device__ inline unsigned long long splitmix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Uniform in [0, 1) from the top 53 bits of the hash of (key, a, b).
__device__ inline double de_uniform(unsigned long long key,
                                    unsigned long long a,
                                    unsigned long long b) {
  const unsigned long long h = splitmix64(key ^ splitmix64(a ^ splitmix64(b)));
  return double(h >> 11) * (1.0 / 9007199254740992.0);
}

// pop, trial [S][N][P] in [0, 1]; mid, span [S][P]; base [S][6] (the fixed
// sphere parameters); slots [P] (which of the six each variable is).  The
// searches stepped are live[0..L) (indices into the S); spheres [L * N]
// out, search live[k]'s candidates at k * N.  With copy_only, or for a
// finished search, the trial is the population itself.
__global__ void k_de_trial(int S, int L, const int* __restrict__ live, int N,
                           int P, const double* __restrict__ pop,
                           double* __restrict__ trial,
                           const unsigned long long* __restrict__ keys,
                           int generation, double mut_lo, double mut_hi,
                           const double* __restrict__ cr,
                           const double* __restrict__ mid,
                           const double* __restrict__ span,
                           const double* __restrict__ base,
                           const int* __restrict__ slots,
                           const int* __restrict__ done, int copy_only,
                           lmb_sphere* __restrict__ spheres) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)L * N) return;
  const int k = int(i / N), c = int(i - (long long)k * N);
  const int s = live[k];
  if (s < 0 || s >= S) return;  // not a search of this call
  const double* ps = pop + (size_t)s * N * P;
  const size_t row = (size_t)s * N + c;  // the candidate in pop / trial
  const unsigned long long key = keys[s];
  const unsigned long long gen = (unsigned long long)generation;
  const unsigned long long ctr = (unsigned long long)c << 6;
  const bool keep = copy_only || done[s];
  double p[6];
  for (int j = 0; j < 6; ++j) p[j] = base[(size_t)s * 6 + j];
  // best1: pop[0] + F (pop[r0] - pop[r1]), r0 != r1 != c
  const double scale =
      mut_lo + (mut_hi - mut_lo) * de_uniform(key, gen, 0xFFFFFFFFull);
  int r0 = min(int(de_uniform(key, gen, ctr + 1) * (N - 1)), N - 2);
  if (r0 >= c) ++r0;
  int r1 = min(int(de_uniform(key, gen, ctr + 2) * (N - 2)), N - 3);
  const int lo = min(c, r0), hi = max(c, r0);
  if (r1 >= lo) ++r1;
  if (r1 >= hi) ++r1;
  const int fill = min(int(de_uniform(key, gen, ctr + 3) * P), P - 1);
  for (int j = 0; j < P; ++j) {
    double v = ps[(size_t)c * P + j];
    if (!keep) {
      const double b = ps[j] + scale * (ps[(size_t)r0 * P + j] - ps[(size_t)r1 * P + j]);
      if (j == fill || de_uniform(key, gen, ctr + 8 + j) < cr[s]) v = b;
      if (v < 0. || v > 1.) v = de_uniform(key, gen, ctr + 32 + j);
    }
    trial[row * P + j] = v;
    p[slots[j]] = mid[(size_t)s * P + j] + (v - 0.5) * span[(size_t)s * P + j];
  }
  lmb_sphere o;
  o.x_p = p[0];
  o.y_p = p[1];
  o.z_p = p[2];
  o.a_p = p[3];
  o.n_p = p[4];
  o.k_p = p[5];
  spheres[i] = o;
}

// One warp per live search (live[0..L)): deferred selection (the trial
// replaces a candidate whose energy it does not exceed), the best candidate
// moved to index 0, and scipy's convergence test std(E) <= atol +
// tol |mean(E)| (no infinite energy).  etrial [L * N] in the order of
// k_de_trial's spheres.  first: the initial population's energies (no
// selection).  done: 1 converged, 2 maxiter reached.
__global__ void k_de_select(int S, int L, const int* __restrict__ live, int N,
                            int P, double* __restrict__ pop,
                            double* __restrict__ energies,
                            const double* __restrict__ trial,
                            const double* __restrict__ etrial,
                            const double* __restrict__ tol,
                            const double* __restrict__ atol,
                            const int* __restrict__ maxiter,
                            int* __restrict__ nit, int* __restrict__ done,
                            int first) {
  const int lane = threadIdx.x & 31;
  const int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (k >= L) return;
  const int s = live[k];
  if (s < 0 || s >= S || done[s]) return;
  double* e = energies + (size_t)s * N;
  double* ps = pop + (size_t)s * N * P;
  const double* et = etrial + (size_t)k * N;
  const double* ts = trial + (size_t)s * N * P;
  for (int c = lane; c < N; c += 32) {
    if (first || et[c] <= e[c]) {
      e[c] = et[c];
      if (!first)
        for (int j = 0; j < P; ++j) ps[(size_t)c * P + j] = ts[(size_t)c * P + j];
    }
  }
  __syncwarp();
  // the best (the first of equal ones) to index 0; bi == N: none yet
  double bv = 0.;
  int bi = N;
  for (int c = lane; c < N; c += 32)
    if (bi == N || e[c] < bv) {
      bv = e[c];
      bi = c;
    }
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (oi != N && (bi == N || ov < bv || (ov == bv && oi < bi))) {
      bv = ov;
      bi = oi;
    }
  }
  __syncwarp();
  if (lane == 0 && bi > 0 && bi < N) {
    const double t = e[0];
    e[0] = e[bi];
    e[bi] = t;
    for (int j = 0; j < P; ++j) {
      const double u = ps[j];
      ps[j] = ps[(size_t)bi * P + j];
      ps[(size_t)bi * P + j] = u;
    }
  }
  __syncwarp();
  if (first) return;
  // convergence
  double sum = 0.;
  int inf = 0;
  for (int c = lane; c < N; c += 32) {
    sum += e[c];
    inf |= isinf(e[c]) ? 1 : 0;
  }
  for (int o = 16; o > 0; o >>= 1) {
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
    inf |= __shfl_xor_sync(0xffffffffu, inf, o);
  }
  const double mean = sum / N;
  double var = 0.;
  for (int c = lane; c < N; c += 32) var += (e[c] - mean) * (e[c] - mean);
  for (int o = 16; o > 0; o >>= 1) var += __shfl_xor_sync(0xffffffffu, var, o);
  if (lane == 0) {
    const int it = nit[s] + 1;
    nit[s] = it;
    const bool conv = !inf && sqrt(var / N) <= atol[s] + tol[s] * fabs(mean);
    if (conv)
      done[s] = 1;
    else if (it >= maxiter[s])
      done[s] = 2;
  }
}

}  // namespace lmb
