// TBB-compatible concurrent_queue (mutex + deque) for the oracle build.
#pragma once
#include <deque>
#include <mutex>

namespace tbb {

template <typename T>
class concurrent_queue {
 public:
  void push(const T& v) {
    std::lock_guard<std::mutex> lk(m_mtx);
    m_q.push_back(v);
  }
  bool try_pop(T& out) {
    std::lock_guard<std::mutex> lk(m_mtx);
    if (m_q.empty()) return false;
    out = m_q.front();
    m_q.pop_front();
    return true;
  }
  std::size_t unsafe_size() const { return m_q.size(); }
  bool empty() const { return m_q.empty(); }

 private:
  std::deque<T> m_q;
  mutable std::mutex m_mtx;
};

}  // namespace tbb
