// Stub of hguo/ndarray's stream interface, enough for the reference engine's
// execute_stream() (engine.hpp:214-270) to compile.  TEST INFRASTRUCTURE ONLY.
// The oracle build never streams from files; it calls execute() on arrays.
#pragma once

#include <ndarray/ndarray.hh>
#include <map>
#include <memory>
#include <string>

namespace ftk {

struct native_storage {};

struct ndarray_group {
  template <typename T>
  const ndarray<T>& get_ref(const std::string&) const {
    static ndarray<T> empty;
    return empty;
  }
};

template <typename Storage = native_storage>
struct stream {
  int total_timesteps() const { return 0; }
  std::shared_ptr<ndarray_group> read(int) { return std::make_shared<ndarray_group>(); }
  void parse_yaml(const std::string&) {}
};

}  // namespace ftk
