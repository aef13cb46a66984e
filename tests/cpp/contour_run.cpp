// Level sets through the C++ drop-in header, as a reference caller writes
// them (tests/test_examples.cpp:225-256 of the reference): a
// RegularSimplicialMesh, a ContourPredicate<T> on one scalar array,
// SimplicialEngine::execute and get_complex.  Dumps the complex as text:
//   F v0 v1 | bary0 bary1 (float bits, hex) | track_id | scalar bits
//   C dim i0 i1 ...
// Usage: contour_run <field.bin> <f32|f64> <d0,d1,...> <threshold> <sos_q> <out.txt>
//        contour_run fiber <f.bin> <g.bin> <f32|f64> <d0,...> <t0> <t1> <sos_q> <out.txt>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "ftk2b/engine.hpp"

template <typename T>
struct Array {
  std::vector<size_t> dims;
  std::vector<T> buf;
  size_t nd() const { return dims.size(); }
  size_t dimf(size_t i) const { return i < dims.size() ? dims[i] : 1; }
  size_t nelem() const { return buf.size(); }
  const T* pdata() const { return buf.data(); }
};

static uint32_t fbits(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  return u;
}

template <typename T>
static int run(const char* path, const std::vector<size_t>& dims, double thr, double q, const char* out) {
  Array<T> a;
  a.dims = dims;
  size_t n = 1;
  for (size_t d : dims) n *= d;
  a.buf.resize(n);
  FILE* f = std::fopen(path, "rb");
  if (!f || std::fread(a.buf.data(), sizeof(T), n, f) != n) {
    std::fprintf(stderr, "cannot read %s\n", path);
    return 2;
  }
  std::fclose(f);
  std::vector<uint64_t> md(dims.begin(), dims.end());
  auto mesh = std::make_shared<ftk2b::RegularSimplicialMesh>(md);
  ftk2b::ContourPredicate<T> pred;
  pred.var_name = "S";
  pred.threshold = (T)thr;
  pred.sos_q = q;
  ftk2b::SimplicialEngine<T, ftk2b::ContourPredicate<T>> engine(mesh, pred);
  std::map<std::string, Array<T>> data;
  data["S"] = a;
  engine.execute(data, {"S"});
  ftk2b::FeatureComplex c = engine.get_complex();
  FILE* o = std::fopen(out, "w");
  if (!o) return 2;
  for (const auto& el : c.vertices)
    std::fprintf(o, "F %" PRIu64 " %" PRIu64 " | %08x %08x | %" PRIu64 " | %08x\n", el.simplex.vertices[0],
                 el.simplex.vertices[1], fbits(el.barycentric_coords[0][0]), fbits(el.barycentric_coords[0][1]),
                 el.track_id, fbits(el.scalar));
  for (const auto& conn : c.connectivity) {
    const size_t k = conn.dimension + 1;
    for (size_t i = 0; i + k <= conn.indices.size(); i += k) {
      std::fprintf(o, "C %d", conn.dimension);
      for (size_t j = 0; j < k; ++j) std::fprintf(o, " %u", conn.indices[i + j]);
      std::fprintf(o, "\n");
    }
  }
  std::fclose(o);
  return 0;
}

// fibers: contour_run fiber <f.bin> <g.bin> <f32|f64> <d0,...> <t0> <t1> <sos_q> <out.txt>
//   F v0 v1 v2 | bary bits | track_id     C dim i0 i1 [i2]
template <typename T>
static int run_fiber(char** argv, const std::vector<size_t>& dims) {
  Array<T> a[2];
  size_t n = 1;
  for (size_t d : dims) n *= d;
  for (int j = 0; j < 2; ++j) {
    a[j].dims = dims;
    a[j].buf.resize(n);
    FILE* f = std::fopen(argv[2 + j], "rb");
    if (!f || std::fread(a[j].buf.data(), sizeof(T), n, f) != n) {
      std::fprintf(stderr, "cannot read %s\n", argv[2 + j]);
      return 2;
    }
    std::fclose(f);
  }
  std::vector<uint64_t> md(dims.begin(), dims.end());
  auto mesh = std::make_shared<ftk2b::RegularSimplicialMesh>(md);
  ftk2b::FiberPredicate<T> pred;
  pred.var_names[0] = "F";
  pred.var_names[1] = "G";
  pred.thresholds[0] = (T)std::atof(argv[6]);
  pred.thresholds[1] = (T)std::atof(argv[7]);
  pred.sos_q = std::atof(argv[8]);
  ftk2b::SimplicialEngine<T, ftk2b::FiberPredicate<T>> engine(mesh, pred);
  std::map<std::string, Array<T>> data;
  data["F"] = a[0];
  data["G"] = a[1];
  engine.execute(data, {"F", "G"});
  ftk2b::FeatureComplex c = engine.get_complex();
  FILE* o = std::fopen(argv[9], "w");
  if (!o) return 2;
  for (const auto& el : c.vertices)
    std::fprintf(o, "F %" PRIu64 " %" PRIu64 " %" PRIu64 " | %08x %08x %08x | %" PRIu64 "\n", el.simplex.vertices[0],
                 el.simplex.vertices[1], el.simplex.vertices[2], fbits(el.barycentric_coords[0][0]),
                 fbits(el.barycentric_coords[0][1]), fbits(el.barycentric_coords[0][2]), el.track_id);
  for (const auto& conn : c.connectivity) {
    const size_t k = conn.dimension + 1;
    for (size_t i = 0; i + k <= conn.indices.size(); i += k) {
      std::fprintf(o, "C %d", conn.dimension);
      for (size_t j = 0; j < k; ++j) std::fprintf(o, " %u", conn.indices[i + j]);
      std::fprintf(o, "\n");
    }
  }
  std::fclose(o);
  return 0;
}

int main(int argc, char** argv) {
  if (argc == 10 && std::strcmp(argv[1], "fiber") == 0) {
    std::vector<size_t> dims;
    std::stringstream ss(argv[5]);
    std::string tok;
    while (std::getline(ss, tok, ',')) dims.push_back(std::stoul(tok));
    try {
      return std::strcmp(argv[4], "f64") == 0 ? run_fiber<double>(argv, dims) : run_fiber<float>(argv, dims);
    } catch (const std::exception& e) {
      std::fprintf(stderr, "%s\n", e.what());
      return 1;
    }
  }
  if (argc != 7) {
    std::fprintf(stderr, "usage: contour_run <field.bin> <f32|f64> <d0,d1,...> <threshold> <sos_q> <out.txt>\n");
    return 2;
  }
  std::vector<size_t> dims;
  std::stringstream ss(argv[3]);
  std::string tok;
  while (std::getline(ss, tok, ',')) dims.push_back(std::stoul(tok));
  const double thr = std::atof(argv[4]), q = std::atof(argv[5]);
  try {
    return std::strcmp(argv[2], "f64") == 0 ? run<double>(argv[1], dims, thr, q, argv[6])
                                            : run<float>(argv[1], dims, thr, q, argv[6]);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
}
