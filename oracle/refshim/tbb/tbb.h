// Stand-in for the four Intel TBB entry points the libWetCloth Core uses.
//
// Test infrastructure only: this header exists so that the reference Core
// (used as the checker and as the timed CPU baseline) compiles without TBB,
// which is not installed in this image.  It provides exactly
//   tbb::blocked_range<T>
//   tbb::parallel_for(first, last, step, f)
//   tbb::parallel_reduce(blocked_range<T*>, init, body, join)
//   tbb::parallel_sort(first, last [, cmp])
// which is the complete set named by `grep tbb::` over libWetCloth/Core.
//
// Two variants:
//   * default (serial): plain loops and std::sort.  Every result is bitwise
//     reproducible; this is the build the golden fixtures come from.
//   * WCREF_OMP: OpenMP loops (schedule(dynamic,64)), per-thread partials for
//     parallel_reduce joined in thread order, and __gnu_parallel::sort.  This is
//     the timed CPU baseline.  The arithmetic of every loop body is unchanged;
//     parallel_reduce is only used for the particle bounding box (min/max, order
//     independent) and every parallel_sort call sorts unique keys.
#ifndef WCREF_TBB_SHIM_H
#define WCREF_TBB_SHIM_H

#include <algorithm>
#include <cstddef>
#include <vector>

#ifdef WCREF_OMP
#include <omp.h>
#include <parallel/algorithm>
#endif

namespace tbb {

template <typename T>
class blocked_range {
 public:
  blocked_range(T b, T e) : b_(b), e_(e) {}
  T begin() const { return b_; }
  T end() const { return e_; }
  bool empty() const { return !(b_ < e_); }

 private:
  T b_, e_;
};

template <typename I, typename F>
void parallel_for(I first, I last, I step, const F& f) {
#ifdef WCREF_OMP
  if (step == (I)1) {
    long long n = (long long)last - (long long)first;
#pragma omp parallel for schedule(dynamic, 64)
    for (long long t = 0; t < n; ++t) f((I)(first + (I)t));
    return;
  }
#endif
  for (I i = first; i < last; i += step) f(i);
}

template <typename T, typename V, typename Body, typename Join>
V parallel_reduce(const blocked_range<T*>& r, const V& init, const Body& body,
                  const Join& join) {
#ifdef WCREF_OMP
  const long long n = (long long)(r.end() - r.begin());
  const int nt = omp_get_max_threads();
  if (n > 4096 && nt > 1) {
    std::vector<V> part(nt, init);
    std::vector<char> used(nt, 0);
#pragma omp parallel num_threads(nt)
    {
      const int t = omp_get_thread_num();
      const long long chunk = (n + nt - 1) / nt;
      const long long lo = (long long)t * chunk;
      const long long hi = std::min(n, lo + chunk);
      if (lo < hi) {
        part[t] = body(blocked_range<T*>(r.begin() + lo, r.begin() + hi), init);
        used[t] = 1;
      }
    }
    V acc = init;
    for (int t = 0; t < nt; ++t)
      if (used[t]) acc = join(acc, part[t]);
    return acc;
  }
#endif
  return body(r, init);
}

template <typename It>
void parallel_sort(It first, It last) {
#ifdef WCREF_OMP
  __gnu_parallel::sort(first, last);
#else
  std::sort(first, last);
#endif
}

template <typename It, typename Cmp>
void parallel_sort(It first, It last, const Cmp& cmp) {
#ifdef WCREF_OMP
  __gnu_parallel::sort(first, last, cmp);
#else
  std::sort(first, last, cmp);
#endif
}

}  // namespace tbb

#endif
