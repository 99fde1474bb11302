// Host-side stand-in for the few Poplar vertex field types that the ipuma
// codelets use (Vertex, MultiVertex, Input, Output, Vector).  Written for this
// oracle so that the reference codelet sources compile unmodified with g++;
// it contains no Poplar code.  TEST INFRASTRUCTURE ONLY.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>

namespace poplar {

enum class VectorLayout { ONE_PTR, SPAN, COMPACT_PTR, SCALED_PTR32, SCALED_PTR64 };

class Vertex {
 public:
  virtual ~Vertex() = default;
};

class MultiVertex {
 public:
  virtual ~MultiVertex() = default;
  static unsigned numWorkers() { return 6; }
};

// A vector field: a bare pointer that the harness points at host memory.
template <typename T, VectorLayout L = VectorLayout::SPAN, unsigned Align = alignof(T)>
class Vector {
 public:
  T* ptr_ = nullptr;
  T& operator[](std::size_t i) const { return ptr_[i]; }
  void bind(T* p) { ptr_ = p; }
};

// Scalar field: converts to its value; `*field` also yields the value.
template <typename T>
class Input {
 public:
  T value_{};
  operator T() const { return value_; }
  const T& operator*() const { return value_; }
  void set(T v) { value_ = v; }
};

template <typename E, VectorLayout L, unsigned A>
class Input<Vector<E, L, A>> : public Vector<E, L, A> {};

template <typename T>
class Output;

template <typename E, VectorLayout L, unsigned A>
class Output<Vector<E, L, A>> : public Vector<E, L, A> {};

}  // namespace poplar
