// swatlib::Matrix -- small dense row-major matrix, the container the
// reference uses for substitution tables and profiles
// (src/swatlib/matrix.h:10-62).  Header-only.
#ifndef IPUMA_B200_SWATLIB_MATRIX_H
#define IPUMA_B200_SWATLIB_MATRIX_H

#include <cstddef>
#include <sstream>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

namespace swatlib {

template <typename T>
class Matrix {
 protected:
  std::vector<T> vdata;
  size_t m = 0, n = 0;

 public:
  Matrix() = default;
  Matrix(size_t m_, size_t n_) : vdata(m_ * n_), m(m_), n(n_) {}
  Matrix(size_t m_, size_t n_, T v) : vdata(m_ * n_, v), m(m_), n(n_) {}
  Matrix(size_t m_, size_t n_, std::vector<T> v) : vdata(std::move(v)), m(m_), n(n_) {
    if (vdata.size() != m * n) throw std::runtime_error("Matrix: data size does not match shape");
  }

  std::tuple<size_t, size_t> shape() const { return {m, n}; }
  size_t getM() const { return m; }
  size_t getN() const { return n; }

  T& get(int i, int j) { return vdata.at((size_t)i * n + j); }
  void set(int i, int j, T v) { vdata.at((size_t)i * n + j) = v; }

  // Index of the largest element; the first one in row-major order on ties.
  std::tuple<int, int> argmax() const {
    size_t best = 0;
    for (size_t k = 1; k < vdata.size(); ++k)
      if (vdata[k] > vdata[best]) best = k;
    return {static_cast<int>(best / n), static_cast<int>(best % n)};
  }

  void copyValues(std::vector<T> newData) {
    if (newData.size() != vdata.size()) throw std::runtime_error("Matrix: size mismatch");
    vdata = std::move(newData);
  }

  Matrix copy() const { return *this; }
  T* data() { return vdata.data(); }
  const T* data() const { return vdata.data(); }
  typename std::vector<T>::iterator begin() { return vdata.begin(); }
  typename std::vector<T>::iterator end() { return vdata.end(); }

  T& operator()(int i, int j) { return vdata[(size_t)i * n + j]; }
  T operator()(int i, int j) const { return vdata[(size_t)i * n + j]; }

  const std::vector<T> vector() const { return vdata; }

  std::string toString() const {
    std::ostringstream ss;
    for (size_t i = 0; i < m; ++i) {
      for (size_t j = 0; j < n; ++j) ss << (j ? " " : "") << +vdata[i * n + j];
      ss << "\n";
    }
    return ss.str();
  }

  std::vector<std::vector<T>> toVector() const {
    std::vector<std::vector<T>> out(m);
    for (size_t i = 0; i < m; ++i) out[i].assign(vdata.begin() + i * n, vdata.begin() + (i + 1) * n);
    return out;
  }
};

}  // namespace swatlib
#endif
