// TBB-compatible parallel_for over blocked_range for the oracle build.
// The range is cut into pieces no larger than its grain size (as TBB's
// recursive splitting does) and the pieces are spread over the shim pool.
#pragma once
#include <algorithm>
#include "tbb/blocked_range.h"
#include "tbb/shim_pool.h"

namespace tbb {

struct simple_partitioner {};
struct auto_partitioner {};

template <typename Value, typename Body>
void parallel_for(const blocked_range<Value>& r, const Body& body) {
  if (r.empty()) return;
  const long n = long(r.size());
  const long g = long(r.grainsize());
  const long n_pieces = (n + g - 1) / g;
  const long base = n / n_pieces, extra = n % n_pieces;
  tbbshim::run_tasks(int(n_pieces), [&](int i) {
    const long off = i * base + std::min<long>(i, extra);
    const long len = base + (i < extra ? 1 : 0);
    blocked_range<Value> sub(Value(r.begin() + off), Value(r.begin() + off + len), r.grainsize());
    body(sub);
  });
}

template <typename Value, typename Body, typename Partitioner>
void parallel_for(const blocked_range<Value>& r, const Body& body, const Partitioner&) {
  parallel_for(r, body);
}

template <typename Index, typename Func>
void parallel_for(Index first, Index last, const Func& f) {
  parallel_for(blocked_range<Index>(first, last, 1),
               [&](const blocked_range<Index>& sub) {
                 for (Index i = sub.begin(); i != sub.end(); ++i) f(i);
               });
}

}  // namespace tbb
