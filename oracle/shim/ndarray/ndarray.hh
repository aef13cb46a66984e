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

#ifdef __CUDACC__
#include <cuda_runtime.h>
#endif

namespace ftk {

#ifdef __CUDACC__
// Device copies for the reference's CUDA engine (engine.hpp:327-345), built
// only into the incumbent-GPU timing driver: copy_to_device / to_device keep
// one device copy of the buffer, get_devptr returns it, get_lattice().prod_
// holds the Fortran strides in the reversed order the engine indexes them.
enum { NDARRAY_DEVICE_CUDA = 1 };
struct lattice_t {
  std::vector<size_t> prod_;
};
#endif

template <typename T>
class ndarray {
public:
  ndarray() = default;
#ifdef __CUDACC__
  ndarray(const ndarray& o) : dims_(o.dims_), buf_(o.buf_) {}
  ndarray(ndarray&& o) noexcept : dims_(std::move(o.dims_)), buf_(std::move(o.buf_)), dev_(o.dev_) { o.dev_ = nullptr; }
  ndarray& operator=(const ndarray& o) {
    if (this != &o) {
      dims_ = o.dims_;
      buf_ = o.buf_;
      release();
    }
    return *this;
  }
  ndarray& operator=(ndarray&& o) noexcept {
    if (this != &o) {
      release();
      dims_ = std::move(o.dims_);
      buf_ = std::move(o.buf_);
      dev_ = o.dev_;
      o.dev_ = nullptr;
    }
    return *this;
  }
  ~ndarray() { release(); }
  void copy_to_device(int, int) {
    release();
    if (cudaMalloc(&dev_, sizeof(T) * (buf_.size() ? buf_.size() : 1)) != cudaSuccess) {
      dev_ = nullptr;
      return;
    }
    cudaMemcpy(dev_, buf_.data(), sizeof(T) * buf_.size(), cudaMemcpyHostToDevice);
  }
  void to_device(int a, int b) { copy_to_device(a, b); }
  void* get_devptr() const { return dev_; }
  lattice_t get_lattice() const {
    lattice_t l;
    const size_t n = dims_.size();
    l.prod_.assign(n, 1);
    for (size_t k = 0; k < n; ++k) {
      size_t p = 1;
      for (size_t j = 0; j + 1 + k < n; ++j) p *= dims_[j];
      l.prod_[k] = p;
    }
    return l;
  }
  void release() {
    if (dev_) cudaFree(dev_);
    dev_ = nullptr;
  }
#endif
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
#ifdef __CUDACC__
  void* dev_ = nullptr;
#endif
};

}  // namespace ftk
