// TBB-compatible task_arena for the oracle build: execute() runs the functor
// on the calling thread; the thread count comes from the shim pool.
#pragma once
#include "tbb/shim_pool.h"

namespace tbb {

class task_arena {
 public:
  explicit task_arena(int = -1) {}
  template <typename F>
  auto execute(const F& f) -> decltype(f()) { return f(); }
};

}  // namespace tbb
