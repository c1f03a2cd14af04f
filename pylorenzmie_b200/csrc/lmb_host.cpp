// Host-side packing of hologram crops for the batched fit: conversion of
// many crops to float32 into one (pinned) staging buffer, on a persistent
// pool of native threads so that the caller's interpreter lock is not
// involved and small portions of a streamed batch convert at full speed.
#include <stddef.h>
#include <stdint.h>

#include <algorithm>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

#include "lmb200.h"

namespace {

template <typename T>
__attribute__((target("avx2"))) void convert_avx2(const T* s, float* d,
                                                  size_t n) {
  for (size_t i = 0; i < n; ++i) d[i] = static_cast<float>(s[i]);
}

template <typename T>
void convert_base(const T* s, float* d, size_t n) {
  for (size_t i = 0; i < n; ++i) d[i] = static_cast<float>(s[i]);
}

bool have_avx2() {
  static const bool v = __builtin_cpu_supports("avx2");
  return v;
}

struct PackJob {
  const void* const* sources;
  const long long* first;  // [n + 1] prefix sums of the counts
  int nsources;
  int src_type;
  float* dst;
  long long total;
  int parts;
};

// Convert elements [a, b) of the concatenated sources.
void run_part(const PackJob& j, long long a, long long b) {
  if (a >= b) return;
  int i = int(std::upper_bound(j.first, j.first + j.nsources + 1, a) - j.first) - 1;
  const bool avx2 = have_avx2();
  while (a < b && i < j.nsources) {
    const long long lo = a - j.first[i];
    const long long hi = std::min(b, j.first[i + 1]) - j.first[i];
    if (hi > lo) {
      float* d = j.dst + j.first[i] + lo;
      const size_t n = size_t(hi - lo);
      if (j.src_type == LMB_PACK_F64) {
        const double* s = static_cast<const double*>(j.sources[i]) + lo;
        avx2 ? convert_avx2(s, d, n) : convert_base(s, d, n);
      } else {
        const float* s = static_cast<const float*>(j.sources[i]) + lo;
        avx2 ? convert_avx2(s, d, n) : convert_base(s, d, n);
      }
      a = j.first[i] + hi;
    }
    ++i;
  }
}

// Persistent workers; part 0 of every job runs on the calling thread.
class Pool {
 public:
  void run(const PackJob& job) {
    std::unique_lock<std::mutex> call(call_mutex_);  // one job at a time
    grow(job.parts - 1);
    {
      std::lock_guard<std::mutex> g(m_);
      job_ = &job;
      pending_ = job.parts - 1;
      ++generation_;
    }
    cv_work_.notify_all();
    do_part(job, 0);
    std::unique_lock<std::mutex> g(m_);
    cv_done_.wait(g, [&] { return pending_ == 0; });
    job_ = nullptr;
  }

  ~Pool() {
    {
      std::lock_guard<std::mutex> g(m_);
      stop_ = true;
    }
    cv_work_.notify_all();
    for (auto& t : threads_) t.join();
  }

 private:
  static void do_part(const PackJob& j, int p) {
    const long long a = j.total * p / j.parts;
    const long long b = j.total * (p + 1) / j.parts;
    run_part(j, a, b);
  }

  // Called by run() before it publishes a job: a new worker starts from
  // the current generation, so it takes part in the job about to come.
  void grow(int workers) {
    while (int(threads_.size()) < workers) {
      const int id = int(threads_.size()) + 1;  // its part index
      const uint64_t g0 = generation_;
      threads_.emplace_back([this, id, g0] { loop(id, g0); });
    }
  }

  void loop(int id, uint64_t seen) {
    for (;;) {
      const PackJob* job;
      {
        std::unique_lock<std::mutex> g(m_);
        cv_work_.wait(g, [&] { return stop_ || generation_ != seen; });
        if (stop_) return;
        seen = generation_;
        job = job_;
        if (!job || id >= job->parts) continue;
      }
      do_part(*job, id);
      {
        std::lock_guard<std::mutex> g(m_);
        --pending_;
      }
      cv_done_.notify_one();
    }
  }

  std::mutex call_mutex_, m_;
  std::condition_variable cv_work_, cv_done_;
  std::vector<std::thread> threads_;
  const PackJob* job_ = nullptr;
  int pending_ = 0;
  uint64_t generation_ = 0;
  bool stop_ = false;
};

Pool& pool() {
  static Pool* p = new Pool();  // never destroyed: workers live with the process
  return *p;
}

}  // namespace

extern "C" int lmb_pack_crops(const void* const* sources,
                              const long long* counts, int nsources,
                              int src_type, float* dst, int nthreads) {
  if (nsources < 0 || nthreads < 1 || nthreads > 256) return LMB_ERR_ARG;
  if (src_type != LMB_PACK_F64 && src_type != LMB_PACK_F32) return LMB_ERR_ARG;
  if (nsources == 0) return LMB_OK;
  if (!sources || !counts || !dst) return LMB_ERR_ARG;
  std::vector<long long> first(size_t(nsources) + 1, 0);
  for (int i = 0; i < nsources; ++i) {
    if (counts[i] < 0 || (counts[i] > 0 && !sources[i])) return LMB_ERR_ARG;
    first[i + 1] = first[i] + counts[i];
  }
  PackJob job{sources, first.data(), nsources, src_type, dst, first.back(), 1};
  // at least ~256 k elements per part: below that, waking threads costs
  // more than it saves
  const long long want = std::max(1LL, job.total / (256LL << 10));
  job.parts = int(std::min<long long>(nthreads, want));
  if (job.parts == 1) {
    run_part(job, 0, job.total);
    return LMB_OK;
  }
  pool().run(job);
  return LMB_OK;
}

// ---------------------------------------------------------------------------
// Differential-evolution sample draws on numpy's own bit generator.
//
// numpy's bitgen_t (numpy/random/bitgen.h), as BitGenerator.ctypes
// .bit_generator points to it: the generator's state and its draw
// functions.
namespace {

struct NpBitgen {
  void* state;
  uint64_t (*next_uint64)(void*);
  uint32_t (*next_uint32)(void*);
  double (*next_double)(void*);
  uint64_t (*next_raw)(void*);
};

// numpy's random_interval (random/src/distributions/distributions.c): an
// integer uniform on [0, max] by rejection of the draws masked to the
// smallest all-ones mask >= max; 32-bit draws while max fits in 32 bits.
uint64_t np_interval(NpBitgen* g, uint64_t max) {
  if (max == 0) return 0;
  uint64_t mask = max;
  mask |= mask >> 1;
  mask |= mask >> 2;
  mask |= mask >> 4;
  mask |= mask >> 8;
  mask |= mask >> 16;
  mask |= mask >> 32;
  uint64_t v;
  if (max <= 0xffffffffULL) {
    do {
      v = g->next_uint32(g->state) & mask;
    } while (v > max);
  } else {
    do {
      v = g->next_uint64(g->state) & mask;
    } while (v > max);
  }
  return v;
}

}  // namespace

extern "C" int lmb_de_shuffles(void* bitgen, long long* index, long long n,
                               long long count, int keep, long long* out) {
  if (!bitgen || n < 0 || count < 0 || keep < 0 || keep > n) return LMB_ERR_ARG;
  if ((n > 0 && !index) || (count > 0 && keep > 0 && !out)) return LMB_ERR_ARG;
  NpBitgen* g = static_cast<NpBitgen*>(bitgen);
  for (long long c = 0; c < count; ++c) {
    // Generator.shuffle / RandomState.shuffle of a 1-d array: Fisher-Yates
    // from the last entry down, partner drawn on [0, i]
    for (long long i = n - 1; i >= 1; --i) {
      const long long j = (long long)np_interval(g, (uint64_t)i);
      const long long t = index[i];
      index[i] = index[j];
      index[j] = t;
    }
    for (int k = 0; k < keep; ++k) out[c * keep + k] = index[k];
  }
  return LMB_OK;
}

namespace {

// numpy's bounded integers on [0, rng] for rng < 2^32 (the 32-bit branch
// of random_bounded_uint64_fill): masked rejection for RandomState,
// Lemire's multiply-shift rejection (Lemire 2019) for Generator.
uint64_t np_bounded32(NpBitgen* g, uint32_t rng, bool masked) {
  if (rng == 0) return 0;
  if (rng == 0xffffffffu) return g->next_uint32(g->state);
  if (masked) {
    uint32_t mask = rng;
    mask |= mask >> 1;
    mask |= mask >> 2;
    mask |= mask >> 4;
    mask |= mask >> 8;
    mask |= mask >> 16;
    uint32_t v;
    do {
      v = g->next_uint32(g->state) & mask;
    } while (v > rng);
    return v;
  }
  const uint32_t excl = rng + 1;
  uint64_t m = uint64_t(g->next_uint32(g->state)) * excl;
  uint32_t left = uint32_t(m);
  if (left < excl) {
    const uint32_t threshold = (0xffffffffu - rng) % excl;
    while (left < threshold) {
      m = uint64_t(g->next_uint32(g->state)) * excl;
      left = uint32_t(m);
    }
  }
  return m >> 32;
}

}  // namespace

extern "C" int lmb_de_draws(void* bitgen, int masked, int dither, double dlo,
                            double dhi, double* scale, long long* index,
                            long long n, int keep, long long* first,
                            int nparam, double cr, long long* fill,
                            unsigned char* cross) {
  if (!bitgen || n < 1 || keep < 0 || keep > n || nparam < 1) return LMB_ERR_ARG;
  if (!index || (keep > 0 && !first) || !fill || !cross) return LMB_ERR_ARG;
  if (dither && !scale) return LMB_ERR_ARG;
  NpBitgen* g = static_cast<NpBitgen*>(bitgen);
  // rng.uniform(lo, hi): lower + range * next_double
  if (dither) *scale = dlo + (dhi - dlo) * g->next_double(g->state);
  const int st = lmb_de_shuffles(bitgen, index, n, n, keep, first);
  if (st != LMB_OK) return st;
  // rng.integers(nparam, size=n) / rng.randint(nparam, size=n)
  for (long long c = 0; c < n; ++c)
    fill[c] = (long long)np_bounded32(g, uint32_t(nparam - 1), masked != 0);
  // rng.uniform(size=(n, nparam)) < cr
  for (long long k = 0; k < n * nparam; ++k)
    cross[k] = g->next_double(g->state) < cr;
  return LMB_OK;
}

extern "C" int lmb_de_draws_many(int nsearch, void* const* bitgens,
                                 const int* masked, const int* dither,
                                 const double* dlo, const double* dhi,
                                 double* scale, long long* const* index,
                                 long long n, int keep, long long* first,
                                 int nparam, const double* cr,
                                 long long* fill, unsigned char* cross) {
  if (nsearch < 0) return LMB_ERR_ARG;
  if (nsearch == 0) return LMB_OK;
  if (!bitgens || !masked || !dither || !dlo || !dhi || !scale || !index ||
      !cr)
    return LMB_ERR_ARG;
  // search by search, each search's draws complete before the next: the
  // order of lmb_de_draws called in turn, also where searches share a
  // generator
  for (int s = 0; s < nsearch; ++s) {
    const int st = lmb_de_draws(
        bitgens[s], masked[s], dither[s], dlo[s], dhi[s], scale + s, index[s],
        n, keep, first ? first + size_t(s) * n * keep : nullptr, nparam, cr[s],
        fill ? fill + size_t(s) * n : nullptr,
        cross ? cross + size_t(s) * n * nparam : nullptr);
    if (st != LMB_OK) return st;
  }
  return LMB_OK;
}

// ---------------------------------------------------------------------------
// The random pixel subset of Mask (analysis/Mask.py:64-72, 82-105) on
// numpy's own bit generator: one uniform per pixel, in pixel order -- the
// draws of RandomState.random_sample, which np.random.rand(*shape) makes
// -- and pixel i kept when its draw is below fraction and exclude[i] (when
// given) is zero.  index receives the kept pixels in increasing order
// (room for n), *count their number.
//
// layout 0 draws through the generator's next_double.  layout 1 is for
// numpy's MT19937 state (624 32-bit words and a position), which it
// advances itself: the Mersenne Twister of M. Matsumoto and T. Nishimura
// (ACM TOMACS 8, 3 (1998)) -- a block of 624 words regenerated when used
// up, each word tempered on output -- with a double made of two words,
// (a >> 5) 2^26 + (b >> 6) over 2^53, as numpy's next_double makes it.
// Tempering a block's words in one loop costs a fraction of a function
// call per word; the caller checks once that both layouts agree.
namespace {

constexpr int kMtN = 624, kMtM = 397;

struct MtState {
  uint32_t key[kMtN];
  int pos;
};

// The block loops below are data-parallel; they are built for AVX2 and for
// the baseline ISA, and the loader picks the clone the CPU supports.
#if defined(__GNUC__) && !defined(__clang__) && defined(__x86_64__)
#define LMB_CLONES __attribute__((target_clones("avx2", "default")))
#else
#define LMB_CLONES
#endif

LMB_CLONES void mt_regenerate(MtState* s) {
  const uint32_t upper = 0x80000000u, lower = 0x7fffffffu, a = 0x9908b0dfu;
  int i = 0;
  for (; i < kMtN - kMtM; ++i) {
    const uint32_t y = (s->key[i] & upper) | (s->key[i + 1] & lower);
    s->key[i] = s->key[i + kMtM] ^ (y >> 1) ^ ((0u - (y & 1u)) & a);
  }
  for (; i < kMtN - 1; ++i) {
    const uint32_t y = (s->key[i] & upper) | (s->key[i + 1] & lower);
    s->key[i] = s->key[i + kMtM - kMtN] ^ (y >> 1) ^ ((0u - (y & 1u)) & a);
  }
  const uint32_t y = (s->key[kMtN - 1] & upper) | (s->key[0] & lower);
  s->key[kMtN - 1] = s->key[kMtM - 1] ^ (y >> 1) ^ ((0u - (y & 1u)) & a);
  s->pos = 0;
}

inline uint32_t mt_temper(uint32_t y) {
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

inline double mt_double(uint32_t a, uint32_t b) {
  return (double(a >> 5) * 67108864.0 + double(b >> 6)) / 9007199254740992.0;
}

inline uint32_t mt_word(MtState* s) {
  if (s->pos >= kMtN) mt_regenerate(s);
  return mt_temper(s->key[s->pos++]);
}

// keep[j] = (the double of words w[2j], w[2j+1]) < fraction, j < m.
LMB_CLONES void mt_keep_block(const uint32_t* w, long long m, double fraction,
                              unsigned char* keep) {
  for (long long j = 0; j < m; ++j)
    keep[j] = mt_double(mt_temper(w[2 * j]), mt_temper(w[2 * j + 1])) < fraction;
}

}  // namespace

extern "C" int lmb_mask_select(void* bitgen, long long n, double fraction,
                               const unsigned char* exclude, int layout,
                               long long* index, long long* count) {
  if (!bitgen || n < 0 || !index || !count || layout < 0 || layout > 1)
    return LMB_ERR_ARG;
  NpBitgen* g = static_cast<NpBitgen*>(bitgen);
  long long k = 0;
  if (layout == 0) {
    for (long long i = 0; i < n; ++i) {
      const bool keep = g->next_double(g->state) < fraction;
      if (keep && !(exclude && exclude[i])) index[k++] = i;
    }
    *count = k;
    return LMB_OK;
  }
  MtState* s = static_cast<MtState*>(g->state);
  if (s->pos < 0 || s->pos > kMtN) return LMB_ERR_ARG;
  long long i = 0;
  while (i < n) {
    if (s->pos >= kMtN) mt_regenerate(s);
    const long long pairs = std::min<long long>((kMtN - s->pos) / 2, n - i);
    if (pairs == 0) {  // one word left in the block: the draw straddles it
      const uint32_t a = mt_word(s);
      const uint32_t b = mt_word(s);
      if (mt_double(a, b) < fraction && !(exclude && exclude[i])) index[k++] = i;
      ++i;
      continue;
    }
    unsigned char keep[kMtN / 2];
    mt_keep_block(s->key + s->pos, pairs, fraction, keep);
    // branch-free compaction: every slot is written, k advances on a keep
    // (index has room for n, and k <= i + j)
    if (exclude) {
      for (long long j = 0; j < pairs; ++j) {
        index[k] = i + j;
        k += keep[j] & (exclude[i + j] == 0);
      }
    } else {
      for (long long j = 0; j < pairs; ++j) {
        index[k] = i + j;
        k += keep[j];
      }
    }
    s->pos += int(2 * pairs);
    i += pairs;
  }
  *count = k;
  return LMB_OK;
}
