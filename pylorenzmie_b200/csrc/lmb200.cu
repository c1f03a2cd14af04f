// lmb200: C-ABI entry points of the B200 Lorenz-Mie library.
// Declarations and their reference counterparts: include/lmb200.h.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <mutex>
#include <thread>
#include <vector>

#include "lmb200.h"
#include "lmb_kernels.cuh"

using namespace lmb;

namespace {

#define LMB_CK(x)                                    \
  do {                                               \
    cudaError_t e_ = (x);                            \
    if (e_ != cudaSuccess) return LMB_ERR_CUDA;      \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Opt a kernel in to more than 48 KB of dynamic shared memory when needed.
// Per-call host work kept off the path between fits: the shared-memory
// attribute of a kernel is raised once per device to the largest size asked
// for, and persistent grid sizes are looked up once per (device, kernel,
// block, shared memory).
std::mutex g_launch_cache_lock;
struct AttrEntry {
  int device;
  const void* fn;
  size_t value;
  int tpb;
  size_t smem;
};
std::vector<AttrEntry> g_smem_set;    // value: bytes set
std::vector<AttrEntry> g_grid_sizes;  // value: grid

inline int current_device() {
  int dev = -1;
  return cudaGetDevice(&dev) == cudaSuccess ? dev : -1;
}

inline cudaError_t smem_attr(const void* fn, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  const int dev = current_device();
  std::lock_guard<std::mutex> hold(g_launch_cache_lock);
  for (const AttrEntry& e : g_smem_set)
    if (e.device == dev && e.fn == fn && e.value >= bytes) return cudaSuccess;
  const cudaError_t r = cudaFuncSetAttribute(
      fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
  if (r != cudaSuccess || dev < 0) return r;
  for (AttrEntry& e : g_smem_set)
    if (e.device == dev && e.fn == fn) {
      e.value = bytes;
      return r;
    }
  g_smem_set.push_back({dev, fn, bytes, 0, 0});
  return r;
}

inline bool bad_cap(int nmax_cap) { return nmax_cap < 1 || nmax_cap > LMB_NMAX_LIMIT; }

// Fit-evaluation launch shapes: TPB threads, PPT pixels per thread and a
// minimum of MINB resident CTAs per SM (which caps registers per thread).
// Every shape covers a 512-pixel tile, so the tile table and the workspace
// do not depend on the choice.  Index 0 is the default (the fastest on
// B200 for 201x201 crops of 26 orders: 1.62 ms per 256-feature launch).
constexpr int kFitTile = 512;
struct EvalShape {
  int tpb, ppt, minb;
  void (*fn)(FitCtx);
  int warp_tiles;  // 1: each warp owns a tile and a copy of the coefficients
  int pair;        // 1: packed two-pixel loop, pair-layout records
};
const EvalShape kEvalShapes[] = {
    // packed two-pixel loop (default); the geometry is recomputed after the
    // order loop, which frees registers for occupancy
    {64, 8, 6, k_fit_eval_pair<64, 8, 6, true>, 0, 1},
    // scalar loop: also the fallback when pair records do not fit in
    // shared memory (kScalarShape)
    {128, 4, 4, k_fit_eval<128, 4, 4>},
    {128, 4, 3, k_fit_eval_pair<128, 4, 3, true>, 0, 1},
    {64, 8, 5, k_fit_eval_pair<64, 8, 5, true>, 0, 1},
    {32, 16, 12, k_fit_eval_pair<32, 16, 12, true>, 0, 1},
    {64, 8, 4, k_fit_eval_pair<64, 8, 4, false>, 0, 1},
    {128, 4, 2, k_fit_eval_pair<128, 4, 2, false>, 0, 1},
    {256, 2, 2, k_fit_eval_pair<256, 2, 2, false>, 0, 1},
    {64, 8, 8, k_fit_eval<64, 8, 8>},
    {64, 8, 10, k_fit_eval<64, 8, 10>},
    {256, 2, 2, k_fit_eval<256, 2, 2>},
    {128, 16, 4, k_fit_eval_warp<4, 4>, 1},
    {256, 16, 2, k_fit_eval_warp<8, 2>, 1},
};
constexpr int kNumEvalShapes = int(sizeof(kEvalShapes) / sizeof(kEvalShapes[0]));
// The same kernels with the spherical-aberration phase in the epilogue
// (lmb_fit_batch_aberrated): the default packed shape and the scalar
// fallback.
const EvalShape kAberrShapes[] = {
    {64, 8, 6, k_fit_eval_pair<64, 8, 6, true, true>, 0, 1},
    {128, 4, 4, k_fit_eval<128, 4, 4, true>},
};
constexpr int kScalarShape = 1;  // scalar loop, used when pair records do not fit
// pair records take 256 B per order: above this they no longer fit in
// shared memory beside the kernels' own buffers, and the scalar loop runs
constexpr size_t kPairSmemLimit = size_t(200) * 1024;

struct FitLayout {
  size_t state, ev, base, ab, dab, coef32, nmax, tile_begin, tiles,
      active_tiles, partial, counters, total;
  int max_tiles;
};

FitLayout fit_layout(int nf, long long total_pixels, int nmax_cap) {
  FitLayout L;
  const size_t nmaxp = size_t(nmax_cap) + 1;
  long long mt = total_pixels / kFitTile + nf + 1;
  if (mt > (1LL << 30)) mt = 1LL << 30;
  L.max_tiles = int(mt);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    off = align_up(off, 256);
    size_t o = off;
    off += bytes;
    return o;
  };
  L.state = take(sizeof(LMState) * nf);
  L.ev = take(sizeof(EvalPoint) * nf);
  L.base = take(sizeof(double) * 6 * nf);
  L.ab = take(sizeof(zd) * 2 * nmaxp * nf);
  L.dab = take(sizeof(zd) * 4 * nmaxp * nf);
  // room for either record layout (scalar JAC_QUADS or pair PAIR_QUADS)
  L.coef32 = take(sizeof(float4) * PAIR_QUADS * nmaxp * nf);
  L.nmax = take(sizeof(int) * nf);
  L.tile_begin = take(sizeof(int) * (nf + 1));
  L.tiles = take(sizeof(int2) * size_t(L.max_tiles));
  L.active_tiles = take(sizeof(int) * size_t(L.max_tiles));
  L.partial = take(sizeof(double) * FIT_NSUM * size_t(L.max_tiles));
  L.counters = take(sizeof(int) * 16);
  L.total = align_up(off, 256);
  return L;
}

int persistent_grid(const void* fn, int tpb, size_t smem) {
  const int dev = current_device();
  {
    std::lock_guard<std::mutex> hold(g_launch_cache_lock);
    for (const AttrEntry& e : g_grid_sizes)
      if (e.device == dev && e.fn == fn && e.tpb == tpb && e.smem == smem)
        return int(e.value);
  }
  int sms = 148, per = 1;
  if (dev >= 0) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, tpb, smem) != cudaSuccess ||
      per < 1) {
    cudaGetLastError();
    return sms;  // not cached: asked again next time
  }
  std::lock_guard<std::mutex> hold(g_launch_cache_lock);
  g_grid_sizes.push_back({dev, fn, size_t(sms * per), tpb, smem});
  return sms * per;
}

template <typename R, bool kHolo>
int field_launch(const double* coords, long long npts, const lmb_sphere* spheres,
                 const int* item_start, int nitems, const double* ab,
                 const int* nmax, int nmax_cap, double k, int flags, double aberr,
                 void* out, void* stream) {
  const int tpb = 256;
  if constexpr (sizeof(R) == sizeof(float)) {
    // FP32: the packed two-pixel loop, two adjacent pixels per thread.  A
    // ~100 KB block (two blocks per SM, as the registers allow) holds the
    // records of many particles at once (at least one at nmax_cap), and for
    // holograms the FP64 re-summation of the pixels that FP32 cannot
    // resolve: particles in groups whose FP64 records fit.
    const size_t nmaxp = size_t(nmax_cap) + 1;
    const size_t budget = 100 * 1024;
    size_t smem = std::max(budget, sizeof(float4) * PAIRV_QUADS * nmaxp);
    int group = 1;
    if (kHolo) {
      const size_t fixed = RESUM_LIST_BYTES + RESUM_ACC_BYTES;
      const size_t per = 2 * sizeof(Quad<double>) * nmaxp;
      group = int(std::min<size_t>(32, std::max<size_t>(1, (budget - fixed) / per)));
      smem = std::max(smem, fixed + per * size_t(group));
    }
    auto fn = k_field_pair<kHolo>;
    LMB_CK(smem_attr((const void*)fn, smem));
    dim3 grid(unsigned((npts + 2 * tpb - 1) / (2 * tpb)), unsigned(nitems));
    fn<<<grid, tpb, smem, as_stream(stream)>>>(
        coords, npts, spheres, item_start, reinterpret_cast<const zd*>(ab), nmax,
        nmax_cap + 1, k, flags, aberr, out, int(smem / sizeof(float4)), group);
    LMB_CK(cudaGetLastError());
    return LMB_OK;
  }
  const size_t smem = sizeof(Quad<R>) * 2 * (size_t(nmax_cap) + 1);
  auto fn = k_field<R, kHolo>;
  LMB_CK(smem_attr((const void*)fn, smem));
  dim3 grid(unsigned((npts + tpb - 1) / tpb), unsigned(nitems));
  fn<<<grid, tpb, smem, as_stream(stream)>>>(
      coords, npts, spheres, item_start, reinterpret_cast<const zd*>(ab), nmax,
      nmax_cap + 1, k, flags, aberr, out);
  LMB_CK(cudaGetLastError());
  return LMB_OK;
}

int field_common(bool holo, const double* coords, long long npts,
                 const lmb_sphere* spheres, const int* item_start, int nitems,
                 const double* ab, const int* nmax, int nmax_cap, double k,
                 int flags, void* out, void* stream, double aberr = 0.) {
  if (nitems < 0 || npts < 0 || bad_cap(nmax_cap)) return LMB_ERR_ARG;
  if (nitems == 0 || npts == 0) return LMB_OK;
  if (!coords || !spheres || !item_start || !ab || !nmax || !out) return LMB_ERR_ARG;
  if (nitems > 65535 || (npts + 255) / 256 > 0x7fffffffLL) return LMB_ERR_ARG;
  if (flags & LMB_FP64)
    return holo ? field_launch<double, true>(coords, npts, spheres, item_start, nitems,
                                             ab, nmax, nmax_cap, k, flags, aberr, out,
                                             stream)
                : field_launch<double, false>(coords, npts, spheres, item_start, nitems,
                                              ab, nmax, nmax_cap, k, flags, aberr, out,
                                              stream);
  return holo ? field_launch<float, true>(coords, npts, spheres, item_start, nitems, ab,
                                          nmax, nmax_cap, k, flags, aberr, out, stream)
              : field_launch<float, false>(coords, npts, spheres, item_start, nitems, ab,
                                           nmax, nmax_cap, k, flags, aberr, out, stream);
}

}  // namespace

extern "C" {

int lmb_version(void) { return 100; }

const char* lmb_status_string(int status) {
  switch (status) {
    case LMB_OK: return "ok";
    case LMB_ERR_ARG: return "invalid argument";
    case LMB_ERR_CUDA: return "CUDA runtime error";
    case LMB_ERR_NMAX: return "sphere needs more partial-wave orders than nmax_cap";
    case LMB_ERR_WORKSPACE: return "workspace too small";
    case LMB_ERR_UNSUPPORTED: return "unsupported flag combination";
    case LMB_ERR_TIMEOUT: return "streamed fit: no data arrived in time";
    default: return "unknown status";
  }
}

int lmb_sphere_ab(const lmb_sphere* spheres, int nspheres, double n_m,
                  double wavelength, int nmax_cap, double* ab, double* dab,
                  int* nmax, int* status, void* stream) {
  if (nspheres < 0 || bad_cap(nmax_cap)) return LMB_ERR_ARG;
  if (nspheres == 0) return LMB_OK;
  if (!spheres || !ab || !nmax || !status) return LMB_ERR_ARG;
  if (!(wavelength > 0.) || !(n_m > 0.)) return LMB_ERR_ARG;
  const size_t smem = ab_scratch_bytes(nmax_cap + 1);
  LMB_CK(smem_attr((const void*)k_sphere_ab, smem));
  k_sphere_ab<<<nspheres, 64, smem, as_stream(stream)>>>(
      spheres, nspheres, n_m, wavelength, nmax_cap, reinterpret_cast<zd*>(ab),
      reinterpret_cast<zd*>(dab), nmax, status);
  LMB_CK(cudaGetLastError());
  return LMB_OK;
}

int lmb_layered_ab(const double* radii, const double* indices, int nlayers,
                   int nspheres, double n_m, double wavelength, int nmax_cap,
                   double* ab, double* dab, int* nmax, int* status,
                   void* stream) {
  if (nspheres < 0 || bad_cap(nmax_cap)) return LMB_ERR_ARG;
  if (nlayers < 1 || nlayers > LMB_MAX_LAYERS) return LMB_ERR_ARG;
  if (nspheres == 0) return LMB_OK;
  if (!radii || !indices || !ab || !nmax || !status) return LMB_ERR_ARG;
  if (!(wavelength > 0.) || !(n_m > 0.)) return LMB_ERR_ARG;
  const size_t smem = layered_scratch_bytes(nmax_cap + 1, nlayers);
  LMB_CK(smem_attr((const void*)k_layered_ab, smem));
  k_layered_ab<<<nspheres, 64, smem, as_stream(stream)>>>(
      radii, indices, nlayers, nspheres, n_m, wavelength, nmax_cap,
      reinterpret_cast<zd*>(ab), reinterpret_cast<zd*>(dab), nmax, status);
  LMB_CK(cudaGetLastError());
  return LMB_OK;
}

int lmb_field(const double* coords, long long npts, const lmb_sphere* spheres,
              const int* item_start, int nitems, const double* ab,
              const int* nmax, int nmax_cap, double k, int flags, void* out,
              void* stream) {
  return field_common(false, coords, npts, spheres, item_start, nitems, ab, nmax,
                      nmax_cap, k, flags, out, stream);
}

int lmb_hologram(const double* coords, long long npts,
                 const lmb_sphere* spheres, const int* item_start, int nitems,
                 const double* ab, const int* nmax, int nmax_cap, double k,
                 int flags, void* out, void* stream) {
  return field_common(true, coords, npts, spheres, item_start, nitems, ab, nmax,
                      nmax_cap, k, flags, out, stream);
}

int lmb_field_aberrated(const double* coords, long long npts,
                        const lmb_sphere* spheres, const int* item_start,
                        int nitems, const double* ab, const int* nmax,
                        int nmax_cap, double k, int flags, double aberration,
                        void* out, void* stream) {
  if (!(aberration == aberration)) return LMB_ERR_ARG;
  return field_common(false, coords, npts, spheres, item_start, nitems, ab, nmax,
                      nmax_cap, k, flags, out, stream, aberration);
}

int lmb_hologram_aberrated(const double* coords, long long npts,
                           const lmb_sphere* spheres, const int* item_start,
                           int nitems, const double* ab, const int* nmax,
                           int nmax_cap, double k, int flags, double aberration,
                           void* out, void* stream) {
  if (!(aberration == aberration)) return LMB_ERR_ARG;
  return field_common(true, coords, npts, spheres, item_start, nitems, ab, nmax,
                      nmax_cap, k, flags, out, stream, aberration);
}

// Threads (pixels) per k_chi2 block.  Fixed, so that a crop's pixels fall
// into the same blocks whatever else shares the launch (its chi^2 is then
// bit-identical searched alone or beside others); 128 rather than 256
// because a DE crop's ~300 pixels left most of a second 256-thread block
// waiting at its barriers.
constexpr int CHI2_TPB = 128;

size_t lmb_chi2_workspace_bytes(long long npts, int nitems) {
  if (npts <= 0 || nitems <= 0) return 0;
  const size_t n = size_t((npts + CHI2_TPB - 1) / CHI2_TPB) * size_t(nitems);
  return align_up(n * sizeof(double), 256) + n * sizeof(int);
}

// Shared by lmb_chi2_batch (one pixel set) and lmb_chi2_crops (a crop per
// item): grid (blocks over the largest pixel set) x items.
static int chi2_launch(const double* coords, long long npts, const double* data,
                       double noise, const long long* crop_start, int ncrops,
                       const int* item_crop, long long span,
                       const lmb_sphere* spheres, const int* item_start,
                       int nitems, const double* ab, const int* nmax,
                       int nmax_cap, double k, int flags, double* chi2,
                       int* nonfinite, void* workspace, size_t workspace_bytes,
                       void* stream, double aberr = 0.) {
  if (nitems < 0 || npts < 0 || span < 0 || bad_cap(nmax_cap)) return LMB_ERR_ARG;
  if (!isfinite(aberr)) return LMB_ERR_ARG;
  if (nitems == 0) return LMB_OK;
  if (!chi2 || !(noise > 0.)) return LMB_ERR_ARG;
  cudaStream_t st = as_stream(stream);
  if (span == 0) {
    LMB_CK(cudaMemsetAsync(chi2, 0, sizeof(double) * nitems, st));
    if (nonfinite) LMB_CK(cudaMemsetAsync(nonfinite, 0, sizeof(int) * nitems, st));
    return LMB_OK;
  }
  if (!coords || !data || !spheres || !item_start || !ab || !nmax) return LMB_ERR_ARG;
  if (nitems > 65535 || (span + CHI2_TPB - 1) / CHI2_TPB > 0x7fffffffLL)
    return LMB_ERR_ARG;
  if (!workspace || workspace_bytes < lmb_chi2_workspace_bytes(span, nitems))
    return LMB_ERR_WORKSPACE;
  const int tpb = CHI2_TPB;
  const int nb = int((span + tpb - 1) / tpb);
  double* partial = reinterpret_cast<double*>(workspace);
  int* partial_bad = reinterpret_cast<int*>(
      reinterpret_cast<char*>(workspace) +
      align_up(size_t(nb) * size_t(nitems) * sizeof(double), 256));
  const dim3 grid{unsigned(nb), unsigned(nitems)};
  if (flags & LMB_FP64) {
    const size_t smem = sizeof(Quad<double>) * 2 * (size_t(nmax_cap) + 1);
    LMB_CK(smem_attr((const void*)k_chi2<double>, smem));
    k_chi2<double><<<grid, tpb, smem, st>>>(
        coords, npts, crop_start, item_crop, ncrops, spheres, item_start,
        reinterpret_cast<const zd*>(ab), nmax, nmax_cap + 1, k, flags, aberr,
        data, 1. / noise, partial, partial_bad);
  } else {
    const size_t smem = sizeof(Quad<float>) * 2 * (size_t(nmax_cap) + 1);
    LMB_CK(smem_attr((const void*)k_chi2<float>, smem));
    k_chi2<float><<<grid, tpb, smem, st>>>(
        coords, npts, crop_start, item_crop, ncrops, spheres, item_start,
        reinterpret_cast<const zd*>(ab), nmax, nmax_cap + 1, k, flags, aberr,
        data, 1. / noise, partial, partial_bad);
  }
  LMB_CK(cudaGetLastError());
  k_chi2_reduce<<<(nitems + 127) / 128, 128, 0, st>>>(partial, partial_bad, nb,
                                                       nitems, chi2, nonfinite);
  LMB_CK(cudaGetLastError());
  return LMB_OK;
}

int lmb_chi2_batch(const double* coords, long long npts, const double* data,
                   double noise, const lmb_sphere* spheres,
                   const int* item_start, int nitems, const double* ab,
                   const int* nmax, int nmax_cap, double k, int flags,
                   double* chi2, int* nonfinite, void* workspace,
                   size_t workspace_bytes, void* stream) {
  return chi2_launch(coords, npts, data, noise, nullptr, 0, nullptr, npts,
                     spheres, item_start, nitems, ab, nmax, nmax_cap, k, flags,
                     chi2, nonfinite, workspace, workspace_bytes, stream);
}

int lmb_chi2_crops(const double* coords, long long npts, const double* data,
                   double noise, const long long* crop_start, int ncrops,
                   const int* item_crop, long long max_crop_npts,
                   const lmb_sphere* spheres, const int* item_start, int nitems,
                   const double* ab, const int* nmax, int nmax_cap, double k,
                   int flags, double* chi2, int* nonfinite, void* workspace,
                   size_t workspace_bytes, void* stream, double aberration) {
  if (ncrops <= 0 || !crop_start || !item_crop || max_crop_npts > npts)
    return nitems == 0 ? LMB_OK : LMB_ERR_ARG;
  return chi2_launch(coords, npts, data, noise, crop_start, ncrops, item_crop,
                     max_crop_npts, spheres, item_start, nitems, ab, nmax,
                     nmax_cap, k, flags, chi2, nonfinite, workspace,
                     workspace_bytes, stream, aberration);
}

}  // extern "C"

namespace {

// Hologram + Jacobian launch for lmb_jacobian (kAberr false) and
// lmb_jacobian_aberrated.
template <bool kAberr>
int jacobian_launch(const double* coords, long long npts,
                    const lmb_sphere* spheres, int nitems, const double* ab,
                    const double* dab, const int* nmax, int nmax_cap, double k,
                    int flags, double* holo, double* jac, void* stream,
                    double aberr) {
  if (nitems < 0 || npts < 0 || bad_cap(nmax_cap)) return LMB_ERR_ARG;
  if (!isfinite(aberr)) return LMB_ERR_ARG;
  if (nitems == 0 || npts == 0) return LMB_OK;
  if (!coords || !spheres || !ab || !dab || !nmax || !jac) return LMB_ERR_ARG;
  if (!(flags & LMB_CARTESIAN) || (flags & LMB_FP64)) return LMB_ERR_UNSUPPORTED;
  if (nitems > 65535) return LMB_ERR_ARG;
  const int tpb = 128;
  const size_t psmem = sizeof(float4) * PAIR_QUADS * (size_t(nmax_cap) + 1);
  if (psmem <= kPairSmemLimit) {  // packed two-pixel loop
    LMB_CK(smem_attr((const void*)k_jacobian_pair<kAberr>, psmem));
    dim3 grid(unsigned((npts + 2 * tpb - 1) / (2 * tpb)), unsigned(nitems));
    k_jacobian_pair<kAberr><<<grid, tpb, psmem, as_stream(stream)>>>(
        coords, npts, spheres, reinterpret_cast<const zd*>(ab),
        reinterpret_cast<const zd*>(dab), nmax, nmax_cap + 1, k, flags, holo, jac,
        aberr);
    LMB_CK(cudaGetLastError());
    return LMB_OK;
  }
  const size_t smem = sizeof(Quad<float>) * JAC_QUADS * (size_t(nmax_cap) + 1);
  LMB_CK(smem_attr((const void*)k_jacobian<kAberr>, smem));
  dim3 grid(unsigned((npts + tpb - 1) / tpb), unsigned(nitems));
  k_jacobian<kAberr><<<grid, tpb, smem, as_stream(stream)>>>(
      coords, npts, spheres, reinterpret_cast<const zd*>(ab),
      reinterpret_cast<const zd*>(dab), nmax, nmax_cap + 1, k, flags, holo, jac,
      aberr);
  LMB_CK(cudaGetLastError());
  return LMB_OK;
}

}  // namespace

extern "C" {

int lmb_de_trial(int nsearch, int nlive, const int* live, int npop,
                 int nparam, const double* pop, double* trial,
                 const unsigned long long* keys, int generation,
                 double mutation_lo, double mutation_hi,
                 const double* recombination, const double* mid,
                 const double* span, const double* base, const int* slots,
                 const int* done, int copy_only, lmb_sphere* spheres,
                 void* stream) {
  if (nsearch < 0 || nlive < 0 || nlive > nsearch || npop < 3 || nparam < 1 ||
      nparam > 6)
    return LMB_ERR_ARG;
  if (nlive == 0) return LMB_OK;
  if (!live || !pop || !trial || !keys || !recombination || !mid || !span ||
      !base || !slots || !done || !spheres)
    return LMB_ERR_ARG;
  if (!(mutation_lo >= 0.) || !(mutation_hi >= mutation_lo) || !(mutation_hi < 2.) ||
      generation < 0)
    return LMB_ERR_ARG;
  const long long n = (long long)nlive * npop;
  const int tpb = 128;
  k_de_trial<<<unsigned((n + tpb - 1) / tpb), tpb, 0, as_stream(stream)>>>(
      nsearch, nlive, live, npop, nparam, pop, trial, keys, generation,
      mutation_lo,
      mutation_hi, recombination, mid, span, base, slots, done, copy_only,
      spheres);
  LMB_CK(cudaGetLastError());
  return LMB_OK;
}

int lmb_de_select(int nsearch, int nlive, const int* live, int npop,
                  int nparam, double* pop, double* energies,
                  const double* trial, const double* trial_energies,
                  const double* tol, const double* atol, const int* maxiter,
                  int* nit, int* done, int first, void* stream) {
  if (nsearch < 0 || nlive < 0 || nlive > nsearch || npop < 3 || nparam < 1 ||
      nparam > 6)
    return LMB_ERR_ARG;
  if (nlive == 0) return LMB_OK;
  if (!live || !pop || !energies || !trial || !trial_energies || !tol ||
      !atol || !maxiter || !nit || !done)
    return LMB_ERR_ARG;
  const int wpb = 4;  // warps (searches) per block
  k_de_select<<<unsigned((nlive + wpb - 1) / wpb), 32 * wpb, 0,
                as_stream(stream)>>>(nsearch, nlive, live, npop, nparam, pop,
                                     energies,
                                     trial, trial_energies, tol, atol, maxiter,
                                     nit, done, first);
  LMB_CK(cudaGetLastError());
  return LMB_OK;
}

int lmb_jacobian(const double* coords, long long npts,
                 const lmb_sphere* spheres, int nitems, const double* ab,
                 const double* dab, const int* nmax, int nmax_cap, double k,
                 int flags, double* holo, double* jac, void* stream) {
  return jacobian_launch<false>(coords, npts, spheres, nitems, ab, dab, nmax,
                                nmax_cap, k, flags, holo, jac, stream, 0.);
}

int lmb_jacobian_aberrated(const double* coords, long long npts,
                           const lmb_sphere* spheres, int nitems,
                           const double* ab, const double* dab,
                           const int* nmax, int nmax_cap, double k, int flags,
                           double aberration, double* holo, double* jac,
                           void* stream) {
  return jacobian_launch<true>(coords, npts, spheres, nitems, ab, dab, nmax,
                               nmax_cap, k, flags, holo, jac, stream,
                               aberration);
}

size_t lmb_vjp_workspace_bytes(long long npts, int nitems) {
  if (npts <= 0 || nitems <= 0) return 0;
  const long long nb = (npts + 127) / 128;
  return size_t(nb) * size_t(nitems) * 6 * sizeof(double);
}

int lmb_hologram_vjp(const double* coords, long long npts,
                     const lmb_sphere* spheres, int nitems, const double* ab,
                     const double* dab, const int* nmax, int nmax_cap,
                     double k, int flags, const float* gout, double* grad,
                     void* workspace, size_t workspace_bytes, void* stream) {
  if (nitems < 0 || npts < 0 || bad_cap(nmax_cap)) return LMB_ERR_ARG;
  if (nitems == 0) return LMB_OK;
  if (!grad) return LMB_ERR_ARG;
  if (npts == 0) {
    LMB_CK(cudaMemsetAsync(grad, 0, sizeof(double) * 6 * nitems, as_stream(stream)));
    return LMB_OK;
  }
  if (!coords || !spheres || !ab || !dab || !nmax || !gout) return LMB_ERR_ARG;
  if (!(flags & LMB_CARTESIAN) || (flags & LMB_FP64)) return LMB_ERR_UNSUPPORTED;
  if (nitems > 65535) return LMB_ERR_ARG;
  if (!workspace || workspace_bytes < lmb_vjp_workspace_bytes(npts, nitems))
    return LMB_ERR_WORKSPACE;
  const int tpb = 128;
  double* partial = reinterpret_cast<double*>(workspace);
  const size_t psmem = sizeof(float4) * PAIR_QUADS * (size_t(nmax_cap) + 1);
  int nb;
  if (psmem <= kPairSmemLimit) {  // packed two-pixel loop: 256 pixels a block
    nb = int((npts + 2 * tpb - 1) / (2 * tpb));
    LMB_CK(smem_attr((const void*)k_vjp_pair, psmem));
    k_vjp_pair<<<dim3(nb, nitems), tpb, psmem, as_stream(stream)>>>(
        coords, npts, spheres, reinterpret_cast<const zd*>(ab),
        reinterpret_cast<const zd*>(dab), nmax, nmax_cap + 1, k, flags, gout,
        partial);
  } else {
    nb = int((npts + tpb - 1) / tpb);
    const size_t smem = sizeof(Quad<float>) * JAC_QUADS * (size_t(nmax_cap) + 1);
    LMB_CK(smem_attr((const void*)k_vjp, smem));
    k_vjp<<<dim3(nb, nitems), tpb, smem, as_stream(stream)>>>(
        coords, npts, spheres, reinterpret_cast<const zd*>(ab),
        reinterpret_cast<const zd*>(dab), nmax, nmax_cap + 1, k, flags, gout,
        partial);
  }
  LMB_CK(cudaGetLastError());
  const int nt = nitems * 6;
  k_vjp_reduce<<<(nt + 127) / 128, 128, 0, as_stream(stream)>>>(partial, nb, nitems, grad);
  LMB_CK(cudaGetLastError());
  return LMB_OK;
}

int lmb_fit_tile_config(int index, int* threads, int* pixels_per_thread,
                        int* min_blocks) {
  if (index < 0 || index >= kNumEvalShapes) return LMB_ERR_ARG;
  if (threads) *threads = kEvalShapes[index].tpb;
  if (pixels_per_thread) *pixels_per_thread = kEvalShapes[index].ppt;
  if (min_blocks) *min_blocks = kEvalShapes[index].minb;
  return LMB_OK;
}

size_t lmb_fit_workspace_bytes(int nfeatures, long long total_pixels,
                               int nmax_cap) {
  if (nfeatures <= 0 || total_pixels < 0 || bad_cap(nmax_cap)) return 0;
  return fit_layout(nfeatures, total_pixels, nmax_cap).total;
}

}  // extern "C"

namespace {

// Host-side resources of the pipelined round loop, one set per host thread
// and device: a ring of pinned slots, each taking a copy of the fit's
// counters (8 ints) and work totals (2 x 64 bit) after a round, and an
// event per slot (32 slots of 64 bytes and 32 events), plus the timing
// events of the fits that ask for stats.  Made on a thread's first fit on
// a device and released when that thread exits.
constexpr int kRingSlots = 32;
constexpr int kSlotInts = 16;
constexpr size_t kSlotCopyBytes = 8 * sizeof(int) + 2 * sizeof(unsigned long long);
constexpr int kRingDevices = 64;
struct RoundRing {
  int* slots = nullptr;
  cudaEvent_t done[kRingSlots] = {};
  ~RoundRing() {
    if (!slots) return;
    // a fit may return with copies into its last slots still queued
    for (int i = 0; i < kRingSlots; ++i) {
      cudaEventSynchronize(done[i]);
      cudaEventDestroy(done[i]);
    }
    cudaFreeHost(slots);
  }
};

struct EventPool {
  std::vector<cudaEvent_t> events;
  ~EventPool() {
    for (cudaEvent_t e : events) cudaEventDestroy(e);
  }
};

std::vector<cudaEvent_t>* timing_pool() {
  static thread_local EventPool pools[kRingDevices];
  const int dev = current_device();
  if (dev < 0 || dev >= kRingDevices) return nullptr;
  return &pools[dev].events;
}

RoundRing* round_ring() {
  static thread_local RoundRing rings[kRingDevices];
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kRingDevices)
    return nullptr;
  RoundRing& r = rings[dev];
  if (r.slots) return &r;
  void* p = nullptr;
  if (cudaHostAlloc(&p, sizeof(int) * kSlotInts * kRingSlots,
                    cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  for (int i = 0; i < kRingSlots; ++i) {
    if (cudaEventCreateWithFlags(&r.done[i], cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      for (int j = 0; j < i; ++j) cudaEventDestroy(r.done[j]);
      cudaFreeHost(p);
      return nullptr;
    }
  }
  r.slots = static_cast<int*>(p);
  return &r;
}

int fit_batch_impl(const lmb_feature* features, int nfeatures,
                   long long total_pixels, const float* data,
                   const float* coords, lmb_sphere* params, double n_m,
                   double wavelength, double magnification, double noise,
                   int nmax_cap, const lmb_fit_settings* settings,
                   lmb_fit_result* results, void* workspace,
                   size_t workspace_bytes, lmb_fit_stats* stats, void* stream,
                   int nlayers, const double* layer_frac,
                   const double* layer_index, const int* ready = nullptr,
                   double wait_seconds = 0., bool sync_rounds = false,
                   double aberr = 0.) {
  if (nlayers < 1 || nlayers > LMB_MAX_LAYERS) return LMB_ERR_ARG;
  if (nlayers > 1 && nfeatures > 0 && (!layer_frac || !layer_index))
    return LMB_ERR_ARG;
  if (nfeatures < 0 || total_pixels < 0 || bad_cap(nmax_cap) || !settings)
    return LMB_ERR_ARG;
  if (nfeatures == 0) return LMB_OK;
  if (!features || !data || !params || !results) return LMB_ERR_ARG;
  if (!(wavelength > 0.) || !(n_m > 0.) || !(magnification > 0.) || !(noise > 0.))
    return LMB_ERR_ARG;
  const FitLayout L = fit_layout(nfeatures, total_pixels, nmax_cap);
  if (!workspace || workspace_bytes < L.total) return LMB_ERR_WORKSPACE;
  cudaStream_t st = as_stream(stream);
  char* ws = reinterpret_cast<char*>(workspace);

  FitCtx c;
  c.features = features;
  c.data = data;
  c.coords = coords;
  c.params = params;
  c.results = results;
  c.state = reinterpret_cast<LMState*>(ws + L.state);
  c.ev = reinterpret_cast<EvalPoint*>(ws + L.ev);
  c.base = reinterpret_cast<double*>(ws + L.base);
  c.ab = reinterpret_cast<zd*>(ws + L.ab);
  c.dab = reinterpret_cast<zd*>(ws + L.dab);
  c.coef32 = reinterpret_cast<Quad<float>*>(ws + L.coef32);
  c.nmax = reinterpret_cast<int*>(ws + L.nmax);
  c.tile_begin = reinterpret_cast<int*>(ws + L.tile_begin);
  c.tiles = reinterpret_cast<int2*>(ws + L.tiles);
  c.active_tiles = reinterpret_cast<int*>(ws + L.active_tiles);
  c.partial = reinterpret_cast<double*>(ws + L.partial);
  c.counters = reinterpret_cast<int*>(ws + L.counters);
  c.work = reinterpret_cast<unsigned long long*>(ws + L.counters + 8 * sizeof(int));
  c.total_pixels = total_pixels;
  c.ready = ready;
  c.nlayers = nlayers;
  c.layer_frac = layer_frac;
  c.layer_index = layer_index;
  c.nf = nfeatures;
  c.nmax_cap = nmax_cap;
  c.max_tiles = L.max_tiles;
  c.tile_pixels = kFitTile;
  c.n_m = n_m;
  c.wavelength = wavelength;
  // Instrument.wavenumber, theory/Instrument.py:65-70 (same operation order)
  double k = 2. * 3.141592653589793 / wavelength;
  k *= n_m;
  k *= magnification;
  c.k = k;
  c.inv_noise = 1. / noise;
  if (!isfinite(aberr)) return LMB_ERR_ARG;
  c.aberr = aberr;
  c.set.ftol = settings->ftol;
  c.set.xtol = settings->xtol;
  c.set.gtol = settings->gtol;
  c.set.factor = settings->factor > 0. ? settings->factor : 100.;
  c.set.maxfev = settings->max_nfev > 0 ? settings->max_nfev : 2000;
  c.variables = settings->variables & 63;
  c.flags = settings->flags;
  c.max_iterations = settings->max_iterations > 0 ? settings->max_iterations : 1;
  if (c.max_iterations > c.set.maxfev) c.max_iterations = c.set.maxfev;

  const size_t ab_smem = nlayers > 1 ? layered_scratch_bytes(nmax_cap + 1, nlayers)
                                     : ab_scratch_bytes(nmax_cap + 1);
  const int shape_index = settings->tile_config;
  if (shape_index < 0 || shape_index >= kNumEvalShapes) return LMB_ERR_ARG;
  EvalShape shape = aberr != 0. ? kAberrShapes[0] : kEvalShapes[shape_index];
  // pair records take 256 B per order: above ~800 orders they no longer fit
  // in shared memory next to the reduction buffer, so such batches use the
  // scalar loop
  if (shape.pair && sizeof(float4) * PAIR_QUADS * (size_t(nmax_cap) + 1) >
                        kPairSmemLimit)
    shape = aberr != 0. ? kAberrShapes[1] : kEvalShapes[kScalarShape];
  c.pair_records = shape.pair;
  const size_t coef_smem = (shape.pair ? sizeof(float4) * PAIR_QUADS
                                       : sizeof(Quad<float>) * JAC_QUADS) *
                           (size_t(nmax_cap) + 1);
  auto eval = shape.fn;
  const size_t eval_smem = shape.warp_tiles ? coef_smem * (shape.tpb / 32) : coef_smem;
  LMB_CK(smem_attr((const void*)k_fit_step, ab_smem));
  LMB_CK(smem_attr((const void*)eval, eval_smem));
  const int egrid = persistent_grid((const void*)eval, shape.tpb, eval_smem);

  // Optional timing: one event pair per evaluation launch, plus the span;
  // the events come from a per-thread, per-device pool kept across calls.
  std::vector<cudaEvent_t> ev;
  std::vector<cudaEvent_t>* pool = stats ? timing_pool() : nullptr;
  if (stats && !pool) return LMB_ERR_CUDA;
  auto mark = [&](void) -> cudaError_t {
    if (ev.size() == pool->size()) {
      cudaEvent_t e;
      const cudaError_t r = cudaEventCreate(&e);
      if (r != cudaSuccess) return r;
      pool->push_back(e);
    }
    cudaEvent_t e = (*pool)[ev.size()];
    ev.push_back(e);
    return cudaEventRecord(e, st);
  };
  auto release = [&]() { ev.clear(); };
  int launches = 0, evals = 0, iterations = 0;
  int counted_evals = -1;  // evaluations that found work (pipelined loop)
  int status = LMB_OK;
  // counters[1] (features with an evaluation pending) and counters[4]
  // (features still waiting for their data) after each step
  int cnt[5] = {0, 0, 0, 0, 0};
  int overflow = 0;
  unsigned long long work[2] = {0ull, 0ull};
  auto read_counts = [&]() -> bool {
    return cudaMemcpyAsync(cnt, c.counters, sizeof(cnt), cudaMemcpyDeviceToHost,
                           st) == cudaSuccess &&
           cudaStreamSynchronize(st) == cudaSuccess;
  };
  auto launch_eval = [&]() -> bool {
    if (cudaMemsetAsync(c.counters + 0, 0, sizeof(int), st) != cudaSuccess) return false;
    if (stats && mark() != cudaSuccess) return false;
    eval<<<egrid, shape.tpb, eval_smem, st>>>(c);
    if (stats && mark() != cudaSuccess) return false;
    launches += 1;
    ++evals;
    return true;
  };
  auto launch_step = [&]() {
    cudaMemsetAsync(c.counters + 1, 0, sizeof(int), st);
    cudaMemsetAsync(c.counters + 4, 0, 2 * sizeof(int), st);  // [4], [5]
    k_fit_step<<<nfeatures, 64, ab_smem, st>>>(c);
    launches += 1;
    ++iterations;
  };
  // The pipelined loop (below) keeps rounds queued ahead of the host; it
  // needs pinned counter slots, so the callers that may not allocate, and
  // streamed admission (whose rounds wait for data), take this loop.
  RoundRing* ring = (sync_rounds || ready) ? nullptr : round_ring();
  bool pipelined = ring != nullptr;
  do {
    if (stats && mark() != cudaSuccess) { status = LMB_ERR_CUDA; break; }
    k_fit_setup<<<1, 1024, 0, st>>>(c);
    k_fit_step<<<nfeatures, 64, ab_smem, st>>>(c);
    launches += 2;
    if (pipelined) {
      // Round r's counters (and the work totals after them) land in slot
      // r of a ring of pinned buffers, with an event; the host reads round
      // r while round r + 1 (and, in the tail, up to 15 more) already run,
      // so the GPU does not wait for the host between rounds.  A round
      // issued after one that left no feature running finds no tiles and
      // only finished features: it changes nothing.
      auto issue_copy = [&](int r) -> bool {
        int* slot = ring->slots + size_t(r % kRingSlots) * kSlotInts;
        return cudaMemcpyAsync(slot, c.counters, kSlotCopyBytes,
                               cudaMemcpyDeviceToHost, st) == cudaSuccess &&
               cudaEventRecord(ring->done[r % kRingSlots], st) == cudaSuccess;
      };
      if (cudaGetLastError() != cudaSuccess || !issue_copy(0)) {
        status = LMB_ERR_CUDA;
        break;
      }
      // Rounds in flight outside the tail: 2 for large batches, whose
      // rounds outlast the host's turnaround; 4 for small ones (at most
      // 128 features), whose rounds take tens of microseconds.
      const int base_depth = nfeatures <= 128 ? 4 : 2;
      int issued = 1, consumed = 0, depth = base_depth, eval_rounds = 0;
      bool capped = false;
      for (;;) {
        while (!capped && issued - consumed < depth) {
          // the step kernel caps every feature's evaluations at
          // max_iterations, so this bound is a safety net only
          if (++eval_rounds > c.max_iterations + 1) {
            capped = true;
            break;
          }
          if (!launch_eval()) { status = LMB_ERR_CUDA; break; }
          launch_step();
          if (cudaGetLastError() != cudaSuccess || !issue_copy(issued)) {
            status = LMB_ERR_CUDA;
            break;
          }
          ++issued;
        }
        if (status != LMB_OK) break;
        // with the rounds capped, wait for the last one issued
        const int r = capped ? issued - 1 : consumed;
        if (cudaEventSynchronize(ring->done[r % kRingSlots]) != cudaSuccess) {
          status = LMB_ERR_CUDA;
          break;
        }
        const int* slot = ring->slots + size_t(r % kRingSlots) * kSlotInts;
        memcpy(cnt, slot, sizeof(cnt));
        overflow = slot[3];
        memcpy(work, slot + 8, sizeof(work));
        consumed = r + 1;
        // rounds 1..r evaluated; later ones only found nothing to do
        counted_evals = r;
        if (capped || cnt[1] == 0) break;
        const bool tail = cnt[1] * 16 <= nfeatures;
        depth = tail ? std::min(2 * depth, 16) : base_depth;
      }
      if (status != LMB_OK) break;
    } else {
      if (cudaGetLastError() != cudaSuccess || !read_counts()) {
        status = LMB_ERR_CUDA;
        break;
      }
      // Every evaluation advances each running feature's nfev, which the
      // step kernel caps at max_iterations, so the rounds after the last
      // admission are bounded by max_iterations; waiting for data is
      // bounded by wait_seconds without progress.
      int since_admission = 0, pending = cnt[4];
      auto wait_start = std::chrono::steady_clock::now();
      // In the tail (every feature admitted, at most 1/16 of them running)
      // several rounds go out per read of the counters: a round with
      // nothing left to do is an evaluation launch that finds no tiles and
      // a step launch whose features are all done, cheaper than the host
      // round trip.  The burst doubles while the tail lasts, from 2 up to 16.
      int burst = 1;
      bool capped = false;
      while (cnt[1] > 0 || cnt[4] > 0) {
        const bool tail = cnt[4] == 0 && cnt[1] > 0 && cnt[1] * 16 <= nfeatures;
        burst = tail ? std::min(2 * burst, 16) : 1;
        for (int r = 0; r < burst && status == LMB_OK; ++r) {
          if (cnt[1] > 0) {
            if (++since_admission > c.max_iterations + 1) {
              capped = true;
              break;
            }
            if (!launch_eval()) { status = LMB_ERR_CUDA; break; }
          } else {
            const double waited = std::chrono::duration<double>(
                std::chrono::steady_clock::now() - wait_start).count();
            if (waited > wait_seconds) { status = LMB_ERR_TIMEOUT; break; }
            std::this_thread::sleep_for(std::chrono::microseconds(20));
          }
          launch_step();
        }
        if (status != LMB_OK || capped) break;
        if (cudaGetLastError() != cudaSuccess || !read_counts()) {
          status = LMB_ERR_CUDA;
          break;
        }
        if (cnt[4] < pending) {  // new features admitted
          pending = cnt[4];
          since_admission = 0;
          wait_start = std::chrono::steady_clock::now();
        }
      }
      if (status != LMB_OK) break;
    }
    k_fit_finalize<<<(nfeatures + 127) / 128, 128, 0, st>>>(c);
    launches += 1;
    if (cudaGetLastError() != cudaSuccess) { status = LMB_ERR_CUDA; break; }
    if (stats && mark() != cudaSuccess) { status = LMB_ERR_CUDA; break; }
  } while (0);
  if (status == LMB_OK && !pipelined) {
    if (cudaMemcpyAsync(&overflow, c.counters + 3, sizeof(int),
                        cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(work, c.work, sizeof(work), cudaMemcpyDeviceToHost,
                        st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      status = LMB_ERR_CUDA;
  }
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    // events: [span start] then pairs around each evaluation, then end.
    // The pipelined loop's productive evaluations ended before the last
    // counter read, so their events are complete and the call need not
    // wait for the rounds queued after them or for k_fit_finalize: its
    // span ends with the last productive evaluation.
    const int useful = counted_evals >= 0 ? counted_evals : evals;
    if (status == LMB_OK && ev.size() >= 2) {
      float ms = 0.f;
      if (!pipelined)
        cudaEventElapsedTime(&ms, ev.front(), ev.back());
      else if (useful > 0)
        cudaEventElapsedTime(&ms, ev.front(), ev[size_t(2 * useful)]);
      stats->total_ms = ms;
      for (size_t q = 1; q + 1 < ev.size() && int(q / 2) < useful; q += 2) {
        float e = 0.f;
        cudaEventElapsedTime(&e, ev[q], ev[q + 1]);
        stats->eval_ms += e;
      }
    }
    stats->pixels = double(work[0]);
    stats->pixel_orders = double(work[1]);
    stats->eval_launches = counted_evals >= 0 ? counted_evals : evals;
    stats->kernel_launches = launches;
    stats->iterations = iterations;
  }
  release();
  if (status != LMB_OK) return status;
  return overflow ? LMB_ERR_WORKSPACE : LMB_OK;
}

}  // namespace

extern "C" {

int lmb_fit_batch(const lmb_feature* features, int nfeatures,
                  long long total_pixels, const float* data,
                  const float* coords, lmb_sphere* params, double n_m,
                  double wavelength, double magnification, double noise,
                  int nmax_cap, const lmb_fit_settings* settings,
                  lmb_fit_result* results, void* workspace,
                  size_t workspace_bytes, lmb_fit_stats* stats, void* stream) {
  return fit_batch_impl(features, nfeatures, total_pixels, data, coords, params,
                        n_m, wavelength, magnification, noise, nmax_cap,
                        settings, results, workspace, workspace_bytes, stats,
                        stream, 1, nullptr, nullptr);
}

int lmb_fit_batch_streamed(const lmb_feature* features, int nfeatures,
                           long long total_pixels, const float* data,
                           const float* coords, lmb_sphere* params,
                           int nlayers, const double* layer_fractions,
                           const double* layer_indices, double n_m,
                           double wavelength, double magnification,
                           double noise, int nmax_cap,
                           const lmb_fit_settings* settings, const int* ready,
                           double wait_seconds, lmb_fit_result* results,
                           void* workspace, size_t workspace_bytes,
                           lmb_fit_stats* stats, void* stream,
                           double aberration) {
  if (!ready || !(wait_seconds >= 0.)) return LMB_ERR_ARG;
  return fit_batch_impl(features, nfeatures, total_pixels, data, coords, params,
                        n_m, wavelength, magnification, noise, nmax_cap,
                        settings, results, workspace, workspace_bytes, stats,
                        stream, nlayers, layer_fractions, layer_indices, ready,
                        wait_seconds, false, aberration);
}
int lmb_fit_batch_aberrated(const lmb_feature* features, int nfeatures,
                            long long total_pixels, const float* data,
                            const float* coords, lmb_sphere* params,
                            int nlayers, const double* layer_fractions,
                            const double* layer_indices, double n_m,
                            double wavelength, double magnification,
                            double noise, int nmax_cap, double aberration,
                            const lmb_fit_settings* settings,
                            lmb_fit_result* results, void* workspace,
                            size_t workspace_bytes, lmb_fit_stats* stats,
                            void* stream) {
  return fit_batch_impl(features, nfeatures, total_pixels, data, coords, params,
                        n_m, wavelength, magnification, noise, nmax_cap,
                        settings, results, workspace, workspace_bytes, stats,
                        stream, nlayers, layer_fractions, layer_indices, nullptr,
                        0., false, aberration);
}

int lmb_fit_batch_layered(const lmb_feature* features, int nfeatures,
                          long long total_pixels, const float* data,
                          const float* coords, lmb_sphere* params, int nlayers,
                          const double* layer_fractions,
                          const double* layer_indices, double n_m,
                          double wavelength, double magnification,
                          double noise, int nmax_cap,
                          const lmb_fit_settings* settings,
                          lmb_fit_result* results, void* workspace,
                          size_t workspace_bytes, lmb_fit_stats* stats,
                          void* stream) {
  return fit_batch_impl(features, nfeatures, total_pixels, data, coords, params,
                        n_m, wavelength, magnification, noise, nmax_cap,
                        settings, results, workspace, workspace_bytes, stats,
                        stream, nlayers, layer_fractions, layer_indices);
}

}  // extern "C"

namespace {
__device__ float g_fma_sink;

__global__ void k_fma_peak_sink(int iters) {
  float a0 = threadIdx.x * 1e-7f, a1 = a0 + 1e-3f, a2 = a0 + 2e-3f, a3 = a0 + 3e-3f;
  float a4 = a0 + 4e-3f, a5 = a0 + 5e-3f, a6 = a0 + 6e-3f, a7 = a0 + 7e-3f;
  const float m = 0.9999f, b = 1e-4f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      a0 = fmaf(a0, m, b); a1 = fmaf(a1, m, b); a2 = fmaf(a2, m, b); a3 = fmaf(a3, m, b);
      a4 = fmaf(a4, m, b); a5 = fmaf(a5, m, b); a6 = fmaf(a6, m, b); a7 = fmaf(a7, m, b);
    }
  }
  const float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 1234.5f) g_fma_sink = s;
}
}  // namespace

extern "C" int lmb_measure_fp32_peak(double* flops, void* stream) {
  if (!flops) return LMB_ERR_ARG;
  cudaStream_t st = as_stream(stream);
  int dev = 0, sms = 148;
  LMB_CK(cudaGetDevice(&dev));
  LMB_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int tpb = 256, bps = 8, iters = 2048;
  const int grid = sms * bps;
  cudaEvent_t e0, e1;
  LMB_CK(cudaEventCreate(&e0));
  LMB_CK(cudaEventCreate(&e1));
  k_fma_peak_sink<<<grid, tpb, 0, st>>>(iters);  // warm-up
  double best = 0.;
  for (int rep = 0; rep < 3; ++rep) {
    cudaEventRecord(e0, st);
    k_fma_peak_sink<<<grid, tpb, 0, st>>>(iters);
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    const double f = 2.0 * 8.0 * 16.0 * double(iters) * double(grid) * tpb / (ms * 1e-3);
    if (f > best) best = f;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  LMB_CK(cudaGetLastError());
  *flops = best;
  return best > 0. ? LMB_OK : LMB_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// lmb_fit_batch_noalloc: the batched fit with its scratch in a static device
// array instead of a caller workspace, for callers that cannot allocate
// device memory (declaration and contract in include/lmb200.h).

namespace {

static __device__ __align__(256) unsigned char
    g_fit_scratch[LMB_FIT_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_lock;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_fit_scratch on the current device, looked up once per
// device (the host-side symbol is not a device address).
int scratch_address(void** out) {
  int dev = -1;
  LMB_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return LMB_ERR_ARG;
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    LMB_CK(cudaGetSymbolAddress(&p, g_fit_scratch));
    if (!p) return LMB_ERR_CUDA;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return LMB_OK;
}

}  // namespace

extern "C" int lmb_fit_batch_noalloc(const lmb_feature* features, int nfeatures,
                                     long long total_pixels, const float* data,
                                     const float* coords, lmb_sphere* params,
                                     double n_m, double wavelength,
                                     double magnification, double noise,
                                     int nmax_cap,
                                     const lmb_fit_settings* settings,
                                     lmb_fit_result* results, void* stream) {
  if (nfeatures < 0 || total_pixels < 0 || bad_cap(nmax_cap) || !settings)
    return LMB_ERR_ARG;
  std::lock_guard<std::mutex> hold(g_noalloc_lock);
  void* scratch = nullptr;
  const int st = scratch_address(&scratch);
  if (st != LMB_OK) return st;
  if (nfeatures == 0) return LMB_OK;
  const FitLayout L = fit_layout(nfeatures, total_pixels, nmax_cap);
  if (L.total > size_t(LMB_FIT_NOALLOC_SCRATCH_BYTES)) return LMB_ERR_WORKSPACE;
  // counters must start at zero; the setup kernel writes them too
  LMB_CK(cudaMemsetAsync(reinterpret_cast<char*>(scratch) + L.counters, 0,
                         sizeof(int) * 16, as_stream(stream)));
  // the synchronous round loop: the pipelined one pins host memory
  const int status =
      fit_batch_impl(features, nfeatures, total_pixels, data, coords, params,
                     n_m, wavelength, magnification, noise, nmax_cap, settings,
                     results, scratch, size_t(LMB_FIT_NOALLOC_SCRATCH_BYTES),
                     nullptr, stream, 1, nullptr, nullptr, nullptr, 0., true);
  // An error can leave kernels that write the array queued; wait for them
  // before the lock lets the next call in (this allocates nothing).
  const cudaError_t drained = cudaStreamSynchronize(as_stream(stream));
  if (status == LMB_OK && drained != cudaSuccess) return LMB_ERR_CUDA;
  return status;
}
