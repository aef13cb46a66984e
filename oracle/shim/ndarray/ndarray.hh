// Minimal stand-in for hguo/ndarray's `ftk::ndarray<T>`, written for this repository.
//
// TEST INFRASTRUCTURE ONLY: it exists so the reference engine headers
// (include/ftk2/core/engine.hpp and friends) compile unmodified for the CPU
// oracle build under oracle/_ref.  It is never linked into the product.
//
// The real ndarray library is not vendored by the reference
// (CMakeLists.txt:18 `find_package(ndarray REQUIRED)`, no version pin).  What
// the engine needs from it is Fortran ("first index fastest") indexing, as the
// reference documents in docs/MULTICOMPONENT_ARRAYS.md:84,248: an array of
// shape [M, nx, ny, nt] stores element (j, x, y, t) at
// j + M*(x + nx*(y + ny*t)).
#pragma once

#include <cstddef>
#include <cstring>
#include <cstdint>
#include <vector>
#include <initializer_list>

namespace ftk {

template <typename T>
class ndarray {
public:
  ndarray() = default;
  explicit ndarray(const std::vector<size_t>& dims) { reshapef(dims); }
  ndarray(std::initializer_list<size_t> dims) { reshapef(std::vector<size_t>(dims)); }

  void reshapef(const std::vector<size_t>& dims) {
    dims_ = dims;
    size_t n = 1;
    for (size_t d : dims_) n *= d;
    buf_.assign(n, T(0));
  }

  size_t nd() const { return dims_.size(); }
  size_t dimf(size_t i) const { return i < dims_.size() ? dims_[i] : 1; }
  std::vector<size_t> shapef() const { return dims_; }
  size_t nelem() const { return buf_.size(); }
  size_t size() const { return buf_.size(); }
  void fill(T v) { for (auto& x : buf_) x = v; }

  T* data() { return buf_.data(); }
  const T* data() const { return buf_.data(); }
  T* pdata() { return buf_.data(); }
  const T* pdata() const { return buf_.data(); }

  T& operator[](size_t i) { return buf_[i]; }
  const T& operator[](size_t i) const { return buf_[i]; }

  // Fortran-order element access; arguments may arrive as doubles from the
  // engine's coordinate vectors and are truncated to indices, as an integer
  // parameter would do.
  template <typename... Idx>
  T& f(Idx... idx) { return buf_[offset({static_cast<size_t>(idx)...})]; }
  template <typename... Idx>
  const T& f(Idx... idx) const { return buf_[offset({static_cast<size_t>(idx)...})]; }

private:
  size_t offset(std::initializer_list<size_t> idx) const {
    size_t off = 0, mul = 1, k = 0;
    for (size_t i : idx) {
      off += i * mul;
      mul *= dimf(k);
      ++k;
    }
    return off;
  }

  std::vector<size_t> dims_;
  std::vector<T> buf_;
};

}  // namespace ftk
