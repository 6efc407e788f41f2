// TBB-compatible parallel_for_each for the oracle build.
#pragma once
#include <iterator>
#include <vector>
#include "tbb/shim_pool.h"

namespace tbb {

template <typename Iterator, typename Body>
void parallel_for_each(Iterator first, Iterator last, const Body& body) {
  std::vector<Iterator> items;
  for (Iterator it = first; it != last; ++it) items.push_back(it);
  tbbshim::run_tasks(int(items.size()), [&](int i) { body(*items[i]); });
}

}  // namespace tbb
