// TBB-compatible blocked_range for the oracle build (scheduling only).
#pragma once
#include <cstddef>

namespace tbb {

template <typename Value>
class blocked_range {
 public:
  using const_iterator = Value;
  blocked_range() = default;
  blocked_range(Value b, Value e, std::size_t grain = 1)
      : m_begin(b), m_end(e), m_grain(grain ? grain : 1) {}
  Value begin() const { return m_begin; }
  Value end() const { return m_end; }
  std::size_t size() const { return std::size_t(m_end - m_begin); }
  std::size_t grainsize() const { return m_grain; }
  bool empty() const { return !(m_begin < m_end); }
  bool is_divisible() const { return size() > m_grain; }

 private:
  Value m_begin{}, m_end{};
  std::size_t m_grain = 1;
};

}  // namespace tbb
