// TBB-compatible parallel_for over blocked_range for the oracle build.
// The range is cut into pieces and the pieces are spread over the shim
// pool. The cut, chosen by tbbshim::split_mode():
//   0 (default): ceil(n / grain) pieces of near-equal size;
//   1: recursive halving while a piece is larger than the grain, the cut of
//      TBB's simple_partitioner (blocked_range splits at begin + size / 2);
//   2: ceil(n / (2 grain)) near-equal pieces, and
//   3: the whole range as one piece -- TBB's default auto_partitioner
//      stops splitting once every thread has work, so pieces larger than
//      the grain are cuts a TBB run makes too;
//   4: pieces of random sizes between half the grain and the grain, from
//      tbbshim::split_seed() (TBB's proportional splits cut ranges
//      unevenly).
// The reference's results depend on the cut only where its per-task
// batching (NN-wide groups, record insertion order under std::sort)
// decides.
#pragma once
#include <algorithm>
#include <vector>
#include "tbb/blocked_range.h"
#include "tbb/shim_pool.h"

namespace tbbshim {
inline int& split_mode() {
  static int mode = 0;
  return mode;
}
inline unsigned& split_seed() {
  static unsigned seed = 1;
  return seed;
}
}  // namespace tbbshim

namespace tbb {

struct simple_partitioner {};
struct auto_partitioner {};

template <typename Value, typename Body>
void parallel_for(const blocked_range<Value>& r, const Body& body) {
  if (r.empty()) return;
  const long n = long(r.size());
  const long g = long(r.grainsize());
  std::vector<std::pair<long, long>> pieces;  // (offset, length)
  if (tbbshim::split_mode() == 1) {
    std::vector<std::pair<long, long>> todo{{0, n}};
    while (!todo.empty()) {
      const auto p = todo.back();
      todo.pop_back();
      if (p.second > g) {
        const long half = p.second / 2;
        todo.push_back({p.first + half, p.second - half});
        todo.push_back({p.first, half});
      } else {
        pieces.push_back(p);
      }
    }
  } else if (tbbshim::split_mode() == 3) {
    pieces.push_back({0, n});
  } else if (tbbshim::split_mode() == 4) {
    unsigned x = tbbshim::split_seed() * 2654435761u + unsigned(n) * 40503u + unsigned(g);
    const long lo = (g + 1) / 2;
    for (long off = 0; off < n;) {
      x = x * 1664525u + 1013904223u;
      const long len = std::min(n - off, lo + long((x >> 8) % unsigned(g - lo + 1)));
      pieces.push_back({off, len});
      off += len;
    }
  } else {
    const long gg = tbbshim::split_mode() == 2 ? 2 * g : g;
    const long n_pieces = (n + gg - 1) / gg;
    const long base = n / n_pieces, extra = n % n_pieces;
    for (long i = 0; i < n_pieces; ++i)
      pieces.push_back({i * base + std::min<long>(i, extra), base + (i < extra ? 1 : 0)});
  }
  tbbshim::run_tasks(int(pieces.size()), [&](int i) {
    blocked_range<Value> sub(Value(r.begin() + pieces[i].first),
                             Value(r.begin() + pieces[i].first + pieces[i].second), r.grainsize());
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
