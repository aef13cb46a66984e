// Drop-in check written the way the reference's own examples are
// (examples/critical_point_2d.cpp, tests/test_examples.cpp): the config-1
// field through ftk2b::SimplicialEngine, result dumped for the pytest side to
// compare with the reference engine's fixture.
//
// usage: dropin_c1 <field.f64 raw [2,64,64,10] Fortran> <out.bin>
#include <cstdio>
#include <fstream>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include <ndarray/ndarray.hh>  // any ndarray with nd()/dimf()/pdata(); the oracle shim here
#include <ftk2b/engine.hpp>

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  ftk::ndarray<double> vec({2, 64, 64, 10});
  std::ifstream in(argv[1], std::ios::binary);
  in.read(reinterpret_cast<char*>(vec.data()), vec.nelem() * sizeof(double));
  if (!in) return 3;
  std::map<std::string, ftk::ndarray<double>> data = {{"vec", vec}};

  auto mesh = std::make_shared<ftk2b::RegularSimplicialMesh>(std::vector<uint64_t>{64, 64, 10});
  ftk2b::CriticalPointPredicate<2, double> pred;
  pred.vector_var_name = "vec";
  ftk2b::SimplicialEngine<double, ftk2b::CriticalPointPredicate<2, double>> engine(mesh, pred);
  engine.execute(data);
  ftk2b::FeatureComplex fc = engine.get_complex();

  std::ofstream out(argv[2], std::ios::binary);
  uint64_t n = fc.vertices.size();
  out.write(reinterpret_cast<const char*>(&n), 8);
  for (const auto& el : fc.vertices) {
    out.write(reinterpret_cast<const char*>(el.simplex.vertices), 3 * 8);
    out.write(reinterpret_cast<const char*>(el.barycentric_coords[0]), 3 * 4);
    out.write(reinterpret_cast<const char*>(&el.track_id), 8);
  }
  uint64_t ne = fc.connectivity.empty() ? 0 : fc.connectivity[0].indices.size() / 2;
  out.write(reinterpret_cast<const char*>(&ne), 8);
  if (ne) out.write(reinterpret_cast<const char*>(fc.connectivity[0].indices.data()), ne * 8);
  std::printf("features %llu edges %llu\n", (unsigned long long)n, (unsigned long long)ne);
  return 0;
}
