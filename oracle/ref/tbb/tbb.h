/* OpenMP stand-in for the handful of oneTBB symbols the MSBG core uses.
 *
 * Oracle-only build support: this header lets the reference MSBG sources be
 * compiled here without oneTBB, so that the reference CPU solver can serve as
 * the parity checker and the timed CPU baseline.  It is not part of the GPU
 * product.  Only the forms the reference calls are provided:
 *   tbb::blocked_range<T>, tbb::parallel_for(range, body),
 *   tbb::parallel_sort(first, last, cmp),
 *   tbb::this_task_arena::{current_thread_index, max_concurrency},
 *   tbb::global_control(max_allowed_parallelism, n).
 */
#ifndef MSBG_ORACLE_TBB_SHIM_H
#define MSBG_ORACLE_TBB_SHIM_H

#include <omp.h>
#include <algorithm>
#include <cstddef>

namespace tbb {

template <typename T>
class blocked_range {
 public:
  blocked_range(T b, T e, size_t grain = 1) : b_(b), e_(e), grain_(grain) {}
  T begin() const { return b_; }
  T end() const { return e_; }
  size_t size() const { return (size_t)(e_ - b_); }
  size_t grainsize() const { return grain_; }
  bool empty() const { return !(b_ < e_); }

 private:
  T b_, e_;
  size_t grain_;
};

/* Dynamic schedule over unit sub-ranges: block tasks have uneven cost. */
template <typename T, typename Body>
void parallel_for(const blocked_range<T>& r, const Body& body) {
  const long long n = (long long)(r.end() - r.begin());
  const T b = r.begin();
#pragma omp parallel for schedule(dynamic, 1)
  for (long long i = 0; i < n; i++) {
    blocked_range<T> sub(b + (T)i, b + (T)i + 1);
    body(sub);
  }
}

template <typename It, typename Cmp>
void parallel_sort(It first, It last, const Cmp& cmp) {
  std::sort(first, last, cmp);
}

namespace this_task_arena {
inline int current_thread_index() { return omp_get_thread_num(); }
inline int max_concurrency() { return omp_get_max_threads(); }
}  // namespace this_task_arena

class global_control {
 public:
  enum parameter { max_allowed_parallelism };
  global_control(parameter, size_t n) {
    if (n > 0) omp_set_num_threads((int)n);
  }
};

}  // namespace tbb

#endif
