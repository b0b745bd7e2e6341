// Serial stand-in for the oneTBB calls the reference uses (parallel_for over an
// index range or a blocked_range, parallel_sort), used only to build the
// reference's own sources into oracle/_ref.  The reference's parallel loops
// write disjoint cells, except its FLIP P2G splat (racy under TBB); serial
// execution gives that splat in particle order.
#pragma once
#include <algorithm>
namespace tbb {
template <class T> class blocked_range {
 public:
  blocked_range(T b, T e) : b_(b), e_(e) {}
  T begin() const { return b_; }
  T end() const { return e_; }
 private:
  T b_, e_;
};
template <class T, class F> void parallel_for(const blocked_range<T>& r, const F& f) { f(r); }
template <class F> void parallel_for(int b, int e, const F& f) { for (int i = b; i < e; i++) f(i); }
template <class It, class C> void parallel_sort(It b, It e, const C& c) { std::sort(b, e, c); }
template <class It> void parallel_sort(It b, It e) { std::sort(b, e); }
}  // namespace tbb
