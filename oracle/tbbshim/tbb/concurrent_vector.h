// TBB-compatible concurrent_vector subset (mutex-guarded growth) for the
// oracle build. Only the reference's vestigial seeding path names it.
#pragma once
#include <mutex>
#include <vector>

namespace tbb {

template <typename T>
class concurrent_vector {
 public:
  using iterator = typename std::vector<T>::iterator;
  using const_iterator = typename std::vector<T>::const_iterator;
  void push_back(const T& v) {
    std::lock_guard<std::mutex> lk(m_mtx);
    m_v.push_back(v);
  }
  std::size_t size() const { return m_v.size(); }
  T& operator[](std::size_t i) { return m_v[i]; }
  const T& operator[](std::size_t i) const { return m_v[i]; }
  iterator begin() { return m_v.begin(); }
  iterator end() { return m_v.end(); }
  const_iterator begin() const { return m_v.begin(); }
  const_iterator end() const { return m_v.end(); }
  void clear() { m_v.clear(); }
  void reserve(std::size_t n) { m_v.reserve(n); }

 private:
  std::vector<T> m_v;
  std::mutex m_mtx;
};

}  // namespace tbb
