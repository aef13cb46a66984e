// Drives include/ftk2b/vtk.hpp without a GPU.
//
//   vtk_run write <case.txt> <outdir>   one complex and mesh, every writer form
//   vtk_run read <file.vtu>             read_vtu, printed as text
//
// case.txt (whitespace-separated):
//   mesh regular <nd> <local dims> <offset> <global dims>
//   mesh extruded <spatial_dim> <cell_dim> <n_verts> <3 n_verts coords> <n_cells> <cells...> <n_layers>
//   mesh extruded_regular <nd> <global dims> <n_layers>
//   features <n>, then per feature: <dim> <dim+1 vertex ids> <dim+1 float barycentrics> <track> <type> <scalar>
//   connectivity <n>, then per entry: <dim> <count> <count indices>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>

#include "ftk2b/vtk.hpp"

using namespace ftk2b;

static std::shared_ptr<Mesh> read_mesh(std::istream& in) {
  std::string tag, kind;
  in >> tag >> kind;
  if (kind == "regular") {
    int nd;
    in >> nd;
    std::vector<uint64_t> l(nd), o(nd), g(nd);
    for (auto& v : l) in >> v;
    for (auto& v : o) in >> v;
    for (auto& v : g) in >> v;
    return std::make_shared<RegularSimplicialMesh>(l, o, g);
  }
  if (kind == "extruded") {
    int sd, cd;
    uint64_t nv, nc, nl;
    in >> sd >> cd >> nv;
    std::vector<double> coords(3 * nv);
    for (auto& v : coords) in >> v;
    in >> nc;
    std::vector<uint64_t> cells(nc * (cd + 1));
    for (auto& v : cells) in >> v;
    in >> nl;
    return std::make_shared<ExtrudedSimplicialMesh>(std::make_shared<UnstructuredSimplicialMesh>(sd, cd, coords, cells),
                                                    nl);
  }
  int nd;
  uint64_t nl;
  in >> nd;
  std::vector<uint64_t> g(nd);
  for (auto& v : g) in >> v;
  in >> nl;
  return std::make_shared<ExtrudedSimplicialMesh>(std::make_shared<RegularSimplicialMesh>(g), nl);
}

static FeatureComplex read_complex(std::istream& in) {
  FeatureComplex c;
  std::string tag;
  size_t n;
  in >> tag >> n;
  c.vertices.resize(n);
  for (auto& el : c.vertices) {
    in >> el.simplex.dimension;
    for (int v = 0; v <= el.simplex.dimension; ++v) in >> el.simplex.vertices[v];
    for (int v = 0; v <= el.simplex.dimension; ++v) {
      std::string s;
      in >> s;
      el.barycentric_coords[0][v] = std::strtof(s.c_str(), nullptr);
    }
    std::string sc;
    in >> el.track_id >> el.type >> sc;
    el.scalar = std::strtof(sc.c_str(), nullptr);
  }
  in >> tag >> n;
  for (size_t i = 0; i < n; ++i) {
    FeatureComplex::SimplexIndices s;
    size_t cnt;
    in >> s.dimension >> cnt;
    s.indices.resize(cnt);
    for (auto& v : s.indices) in >> v;
    c.connectivity.push_back(std::move(s));
  }
  return c;
}

int main(int argc, char** argv) {
  try {
    if (argc == 4 && std::string(argv[1]) == "write") {
      std::ifstream in(argv[2]);
      std::shared_ptr<Mesh> mesh = read_mesh(in);
      const FeatureComplex c = read_complex(in);
      const std::string d = argv[3];
      write_complex_to_vtp(c, *mesh, d + "/all_ascii.vtp", -1, true);
      write_complex_to_vtp(c, *mesh, d + "/all_bin.vtp");
      write_complex_to_vtp(c, *mesh, d + "/dim1_ascii.vtp", 1, true);
      write_complex_to_vtu(c, *mesh, d + "/all_ascii.vtu", -1, true);
      write_complex_to_vtu(c, *mesh, d + "/all_bin.vtu");
      write_complex_to_vtu(c, *mesh, d + "/dim0_bin.vtu", 0);
      write_complex_to_vtu(c, *mesh, d + "/dim3_ascii.vtu", 3, true);
      return 0;
    }
    if (argc == 3 && std::string(argv[1]) == "read") {
      std::shared_ptr<UnstructuredSimplicialMesh> m = read_vtu(argv[2]);
      if (!m) {
        std::printf("none\n");
        return 0;
      }
      std::printf("%d %d %llu %zu\n", m->get_spatial_dimension(), m->cell_dim(),
                  (unsigned long long)m->get_num_vertices(), m->cells().size());
      for (double v : m->coords()) std::printf("%.17g\n", v);
      for (uint64_t v : m->cells()) std::printf("%llu\n", (unsigned long long)v);
      return 0;
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 2;
  }
  std::fprintf(stderr, "usage: vtk_run write <case.txt> <outdir> | vtk_run read <file.vtu>\n");
  return 1;
}
