// printVector helper (src/swatlib/vector.hpp).
#ifndef IPUMA_B200_SWATLIB_VECTOR_HPP
#define IPUMA_B200_SWATLIB_VECTOR_HPP
#include <sstream>
#include <string>
#include <vector>

namespace swatlib {
template <typename T>
std::string printVector(const std::vector<T>& v) {
  std::ostringstream ss;
  ss << "[";
  for (size_t i = 0; i < v.size(); ++i) ss << (i ? ", " : "") << +v[i];
  ss << "]";
  return ss.str();
}
}  // namespace swatlib
#endif
