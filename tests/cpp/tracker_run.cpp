// Runs the high-level tracker of include/ftk2b/feature_tracker.hpp the way a
// reference caller runs ftk2::FeatureTracker: load a YAML configuration,
// hand it the arrays, let it write its outputs.
//
//   tracker_run CONFIG.yaml [--dump OUT] NAME=FILE:DTYPE:d0,d1,... [NAME=...]
//
// Each array is raw little-endian data (f32 or f64) in Fortran order with the
// given dims (first fastest), e.g. vec=vec.bin:f64:2,64,64,10.  Prints the
// number of features, then "ok".  --dump writes the returned complex, one
// feature per line: "F vertex ids | float barycentrics | track_id | 16
// attributes" (floats as hexadecimal bit patterns), then "E lo hi" per edge.
// With --config-only it parses the
// configuration and prints it back as YAML (the round trip of to_yaml).
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "ftk2b/feature_tracker.hpp"

namespace {

struct Arr {
  std::vector<size_t> dims;
  std::vector<double> buf;
  size_t nd() const { return dims.size(); }
  size_t dimf(size_t i) const { return i < dims.size() ? dims[i] : 1; }
  size_t nelem() const { return buf.size(); }
  const double* pdata() const { return buf.data(); }
};

Arr load(const std::string& spec) {
  // FILE:DTYPE:d0,d1,...
  const size_t a = spec.find(':'), b = spec.find(':', a + 1);
  const std::string file = spec.substr(0, a), dt = spec.substr(a + 1, b - a - 1);
  Arr r;
  std::stringstream ds(spec.substr(b + 1));
  std::string tok;
  size_t n = 1;
  while (std::getline(ds, tok, ',')) {
    r.dims.push_back(std::stoull(tok));
    n *= r.dims.back();
  }
  std::ifstream in(file, std::ios::binary);
  if (!in) throw std::runtime_error("cannot read " + file);
  r.buf.resize(n);
  if (dt == "f64") {
    in.read(reinterpret_cast<char*>(r.buf.data()), (std::streamsize)(8 * n));
  } else {
    std::vector<float> f(n);
    in.read(reinterpret_cast<char*>(f.data()), (std::streamsize)(4 * n));
    for (size_t i = 0; i < n; ++i) r.buf[i] = f[i];
  }
  return r;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s CONFIG.yaml [--config-only] NAME=FILE:DTYPE:dims ...\n", argv[0]);
    return 2;
  }
  try {
    if (argc >= 3 && std::string(argv[2]) == "--config-only") {
      std::cout << ftk2b::TrackingConfig::from_yaml(argv[1]).to_yaml_string();
      return 0;
    }
    if (argc >= 3 && std::string(argv[2]) == "--config-dump") {
      // the parsed fields, one "key=value" per line
      const auto c = ftk2b::TrackingConfig::from_yaml(argv[1]);
      using TC = ftk2b::TrackingConfig;
      std::cout << "feature=" << TC::feature_type_to_string(c.feature) << "\n";
      std::cout << "dimension=" << c.dimension << "\n";
      std::cout << "input.type=" << TC::input_type_to_string(c.input.type) << "\n";
      for (const auto& v : c.input.variables) std::cout << "input.variable=" << v << "\n";
      std::cout << "input.field_type=" << c.input.field_type << "\n";
      std::cout << "data.source=" << TC::data_source_type_to_string(c.data.source) << "\n";
      std::cout << "data.inline_stream=" << (c.data.inline_stream ? 1 : 0) << "\n";
      std::cout << "mesh.type=" << TC::mesh_type_to_string(c.mesh.type) << "\n";
      for (auto d : c.mesh.dimensions) std::cout << "mesh.dimension=" << d << "\n";
      std::cout << "execution.backend=" << TC::backend_to_string(c.execution.backend) << "\n";
      std::cout << "execution.precision=" << TC::precision_to_string(c.execution.precision) << "\n";
      std::cout << "execution.threads=" << c.execution.num_threads << "\n";
      std::cout << "output.trajectories=" << c.output.trajectories << "\n";
      std::cout << "output.statistics=" << c.output.statistics << "\n";
      std::cout << "output.format=" << c.output.format << "\n";
      for (const auto& a : c.output.attributes)
        std::cout << "output.attribute=" << a.name << "," << a.source << "," << a.type << "," << a.component << "\n";
      return 0;
    }
    auto tracker = ftk2b::FeatureTracker::from_yaml(argv[1]);
    std::map<std::string, Arr> data;
    std::string dump;
    for (int i = 2; i < argc; ++i) {
      const std::string s = argv[i];
      if (s == "--dump" && i + 1 < argc) {
        dump = argv[++i];
        continue;
      }
      const size_t eq = s.find('=');
      data[s.substr(0, eq)] = load(s.substr(eq + 1));
    }
    auto res = tracker->execute_with_data(data);
    if (!dump.empty()) {
      std::ofstream out(dump);
      const auto& c = res.get_complex();
      auto bits = [](float f) {
        uint32_t u;
        std::memcpy(&u, &f, 4);
        char b[16];
        std::snprintf(b, sizeof(b), "%08x", u);
        return std::string(b);
      };
      for (const auto& e : c.vertices) {
        out << "F";
        for (int v = 0; v <= e.simplex.dimension; ++v) out << " " << e.simplex.vertices[v];
        out << " |";
        for (int v = 0; v <= e.simplex.dimension; ++v) out << " " << bits(e.barycentric_coords[0][v]);
        out << " | " << e.track_id << " |";
        for (int a = 0; a < 16; ++a) out << " " << bits(e.attributes[a]);
        out << "\n";
      }
      for (const auto& cn : c.connectivity)
        if (cn.dimension == 1)
          for (size_t k = 0; k + 1 < cn.indices.size(); k += 2) out << "E " << cn.indices[k] << " " << cn.indices[k + 1] << "\n";
    }
    std::cout << res.num_vertices() << "\nok\n";
  } catch (const std::exception& e) {
    std::cerr << "error: " << e.what() << "\n";
    return 1;
  }
  return 0;
}
