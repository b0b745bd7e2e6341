// Stand-in for the oneTBB calls the reference uses (parallel_for over an index
// range or a blocked_range, parallel_sort), used only to build the reference's
// own sources into oracle/_ref.
//  * default (the parity build): serial, in index order.  The reference's
//    parallel loops write disjoint cells, except its FLIP P2G splat (racy under
//    TBB), which serial execution runs in particle order;
//  * SIMCRAFT_REF_PARALLEL (the timing build): the loops are split over OpenMP
//    threads in contiguous static chunks, as TBB splits a range.  Only the
//    pressure solve is timed with it; its parallel loops (applyCompressedMatrix,
//    saxpy, scaleAndAdd) write disjoint cells.
#pragma once
#include <algorithm>
#ifdef SIMCRAFT_REF_PARALLEL
#include <omp.h>
#endif
namespace tbb {
template <class T> class blocked_range {
 public:
  blocked_range(T b, T e) : b_(b), e_(e) {}
  T begin() const { return b_; }
  T end() const { return e_; }
 private:
  T b_, e_;
};
#ifdef SIMCRAFT_REF_PARALLEL
template <class T, class F> void parallel_for(const blocked_range<T>& r, const F& f) {
#pragma omp parallel
  {
    const T n = r.end() - r.begin();
    const int nt = omp_get_num_threads(), t = omp_get_thread_num();
    const T lo = r.begin() + (T)((long long)n * t / nt), hi = r.begin() + (T)((long long)n * (t + 1) / nt);
    if (lo < hi) f(blocked_range<T>(lo, hi));
  }
}
template <class F> void parallel_for(int b, int e, const F& f) {
#pragma omp parallel for schedule(static)
  for (int i = b; i < e; i++) f(i);
}
#else
template <class T, class F> void parallel_for(const blocked_range<T>& r, const F& f) { f(r); }
template <class F> void parallel_for(int b, int e, const F& f) { for (int i = b; i < e; i++) f(i); }
#endif
template <class It, class C> void parallel_sort(It b, It e, const C& c) { std::sort(b, e, c); }
template <class It> void parallel_sort(It b, It e) { std::sort(b, e); }
}  // namespace tbb
