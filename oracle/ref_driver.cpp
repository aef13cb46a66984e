// Driver that runs the reference's own CPU critical-point engine.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile into
// oracle/_ref/libftk2ref.so from the reference headers where they lie (the
// reference's include/ tree) plus the ndarray shim in oracle/shim; no reference
// source is copied into this repository.
//
// Per call it builds the mesh and predicate exactly as the reference's own
// tests and examples do (tests/test_examples.cpp:79-100, 162-184;
// examples/critical_point_2d.cpp:65-84), runs
// SimplicialEngine<T, CriticalPointPredicate<M,T>>::execute() and
// get_complex() (engine.hpp:96-99, 822-996) and flattens the returned
// FeatureComplex.  As a side channel it re-runs the reference's
// ZeroCrossingSolver<M,T>::solve (zero_crossing.hpp:20-47) on every returned
// simplex, gathering values the way extract_simplex does
// (engine.hpp:1096-1124, get_value 999-1009), so double-precision barycentrics
// can be compared even though FeatureElement stores floats (feature.hpp:26).
#include <ftk2/core/engine.hpp>
#include <ftk2/core/mesh.hpp>
#include <ftk2/core/predicate.hpp>
#include <ftk2/core/unstructured_mesh.hpp>

#include <cstdlib>
#include <cstring>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "oracle_api.h"

#ifdef FTK2REF_SINGLE_THREAD
// One-worker build: the reference's parallel_for and get_num_threads
// (parallel.hpp:14-67) size their pools by std::thread::hardware_concurrency(),
// which answers 1 here, as on a one-core host, so every engine loop runs
// sequentially.  Linked with -Bsymbolic-functions so the engine's calls bind
// to this definition.  Used for the level-set path, whose multi-threaded
// patching reads active_nodes_ without its lock while other workers insert
// (engine.hpp:1229-1244) and numbers boundary nodes in thread-arrival order.
unsigned int std::thread::hardware_concurrency() noexcept { return 1; }
#endif

namespace {

template <typename T>
ftk::ndarray<T> make_array(const void* src, int nd, const uint64_t* dims, size_t lead = 0) {
  std::vector<size_t> shape;
  if (lead) shape.push_back(lead);
  for (int i = 0; i < nd; ++i) shape.push_back((size_t)dims[i]);
  ftk::ndarray<T> a(shape);
  std::memcpy(a.data(), src, a.nelem() * sizeof(T));
  return a;
}

template <typename T, int M>
int run(const orc_mesh* mesh, const orc_field* field, orc_result* out) {
  using namespace ftk2;
  std::shared_ptr<Mesh> mesh_ptr;
  std::shared_ptr<RegularSimplicialMesh> reg;
  if (mesh->kind == ORC_MESH_REGULAR) {
    std::vector<uint64_t> dims, off, glob;
    for (int i = 0; i < mesh->ndims; ++i) {
      dims.push_back(mesh->local_dims[i]);
      off.push_back(mesh->offset[i]);
      glob.push_back(mesh->global_dims[i]);
    }
    reg = std::make_shared<RegularSimplicialMesh>(dims, off, glob);
    mesh_ptr = reg;
  } else {
    std::vector<double> coords(mesh->base_coords, mesh->base_coords + 3 * mesh->n_base_verts);
    size_t nc = (size_t)mesh->n_base_cells * (mesh->base_cell_dim + 1);
    std::vector<uint64_t> cells(mesh->base_cells, mesh->base_cells + nc);
    auto base = std::make_shared<UnstructuredSimplicialMesh>(
        mesh->base_cell_dim, mesh->base_cell_dim, coords, cells);
    mesh_ptr = std::make_shared<ExtrudedSimplicialMesh>(base, mesh->n_layers);
  }

  CriticalPointPredicate<M, T> pred;
  pred.sos_q = field->sos_q;
  std::map<std::string, ftk::ndarray<T>> data;
  static const char* names[4] = {"U", "V", "W", "S"};
  if (field->layout == ORC_LAYOUT_MULTI) {
    pred.use_multicomponent = true;
    pred.vector_var_name = "vec";
    data["vec"] = make_array<T>(field->comp[0], field->nd, field->dims, (size_t)M);
  } else {
    pred.use_multicomponent = false;
    for (int j = 0; j < M; ++j) {
      pred.var_names[j] = names[j];
      data[names[j]] = make_array<T>(field->comp[j], field->nd, field->dims);
    }
  }
  if (field->scalar) {
    pred.scalar_var_name = "S";
    data["S"] = make_array<T>(field->scalar, field->scalar_nd, field->scalar_dims);
  }

  SimplicialEngine<T, CriticalPointPredicate<M, T>> engine(mesh_ptr, pred);
  // The engine reports progress on stdout; keep it out of the caller's stream.
  std::streambuf* saved = std::cout.rdbuf();
  std::ostringstream sink;
  std::cout.rdbuf(sink.rdbuf());
  engine.execute(data);
  FeatureComplex complex = engine.get_complex();
  std::cout.rdbuf(saved);

  const uint64_t n = complex.vertices.size();
  out->m = M;
  out->n = n;
  out->simplices = (uint64_t*)std::malloc(sizeof(uint64_t) * (n * (M + 1) + 1));
  out->bary = (float*)std::malloc(sizeof(float) * (n * (M + 1) + 1));
  out->lambda = (double*)std::malloc(sizeof(double) * (n * (M + 1) + 1));
  out->track_id = (uint64_t*)std::malloc(sizeof(uint64_t) * (n + 1));
  out->type = (uint32_t*)std::malloc(sizeof(uint32_t) * (n + 1));
  out->scalar = (float*)std::malloc(sizeof(float) * (n + 1));
  out->n_tested = 0;

  for (uint64_t i = 0; i < n; ++i) {
    const FeatureElement& el = complex.vertices[i];
    T values[M + 1][M];
    for (int v = 0; v <= M; ++v) {
      out->simplices[i * (M + 1) + v] = el.simplex.vertices[v];
      out->bary[i * (M + 1) + v] = el.barycentric_coords[0][v];
      std::vector<double> coords = mesh_ptr->get_vertex_coordinates(el.simplex.vertices[v]);
      for (int j = 0; j < M; ++j) {
        if (field->layout == ORC_LAYOUT_MULTI) {
          const auto& a = data.at("vec");
          if (coords.size() == 3) values[v][j] = a.f(j, coords[0], coords[1], coords[2]);
          else values[v][j] = a.f(j, coords[0], coords[1], coords[2], coords[3]);
        } else {
          const auto& a = data.at(names[j]);
          if (a.nd() == 1) { values[v][j] = a[el.simplex.vertices[v]]; continue; }
          std::vector<double> lc = coords;
          if (reg) for (size_t k = 0; k < lc.size(); ++k) lc[k] -= (double)reg->get_offset()[k];
          if (lc.size() == 3) values[v][j] = a.f(lc[0], lc[1], lc[2]);
          else values[v][j] = a.f(lc[0], lc[1], lc[2], lc[3]);
        }
      }
    }
    T lambda[M + 1];
    bool ok = ZeroCrossingSolver<M, T>::solve(values, lambda);
    for (int v = 0; v <= M; ++v) out->lambda[i * (M + 1) + v] = ok ? (double)lambda[v] : NAN;
    out->track_id[i] = el.track_id;
    out->type[i] = el.type;
    out->scalar[i] = el.scalar;
  }

  std::vector<uint32_t> edges;
  for (const auto& conn : complex.connectivity)
    if (conn.dimension == 1) edges = conn.indices;
  out->n_edges = edges.size() / 2;
  out->edges = (uint32_t*)std::malloc(sizeof(uint32_t) * (edges.size() + 2));
  if (!edges.empty()) std::memcpy(out->edges, edges.data(), sizeof(uint32_t) * edges.size());
  return 0;
}


// The high-level flow: the engine on the extruded regular spatial mesh, with
// attributes; results flattened as run() does.
template <typename T, int M>
int run_tracked(const orc_tracked* in, orc_result* out, float** attrs) {
  using namespace ftk2;
  std::vector<uint64_t> sdims(in->dims, in->dims + M);
  auto base = std::make_shared<RegularSimplicialMesh>(sdims);
  std::shared_ptr<Mesh> mesh_ptr = std::make_shared<ExtrudedSimplicialMesh>(base, in->nt - 1);
  CriticalPointPredicate<M, T> pred;
  pred.use_multicomponent = true;
  pred.vector_var_name = "vec";
  std::map<std::string, ftk::ndarray<T>> data;
  std::vector<uint64_t> vdims(in->dims, in->dims + M);
  vdims.push_back(in->nt);
  data["vec"] = make_array<T>(in->vec, M + 1, vdims.data(), (size_t)M);
  for (int a = 0; a < in->n_attr; ++a) {
    const std::string name = "attr" + std::to_string(a);
    data[name] = make_array<T>(in->attr_data[a], in->attr_nd[a], in->attr_dims[a]);
    AttributeSpec spec;
    spec.name = name;
    spec.source = name;
    spec.type = in->attr_magnitude[a] ? "magnitude" : "scalar";
    spec.component = in->attr_component[a];
    spec.slot = a;
    pred.attributes.push_back(spec);
  }
  SimplicialEngine<T, CriticalPointPredicate<M, T>> engine(mesh_ptr, pred);
  std::streambuf* saved = std::cout.rdbuf();
  std::ostringstream sink;
  std::cout.rdbuf(sink.rdbuf());
  engine.execute(data);
  FeatureComplex complex = engine.get_complex();
  std::cout.rdbuf(saved);
  const uint64_t n = complex.vertices.size();
  out->m = M;
  out->n = n;
  out->simplices = (uint64_t*)std::malloc(sizeof(uint64_t) * (n * (M + 1) + 1));
  out->bary = (float*)std::malloc(sizeof(float) * (n * (M + 1) + 1));
  out->lambda = (double*)std::malloc(sizeof(double) * (n * (M + 1) + 1));
  out->track_id = (uint64_t*)std::malloc(sizeof(uint64_t) * (n + 1));
  out->type = (uint32_t*)std::malloc(sizeof(uint32_t) * (n + 1));
  out->scalar = (float*)std::malloc(sizeof(float) * (n + 1));
  out->n_tested = 0;
  *attrs = (float*)std::malloc(sizeof(float) * (n * 16 + 1));
  for (uint64_t i = 0; i < n; ++i) {
    const FeatureElement& el = complex.vertices[i];
    for (int v = 0; v <= M; ++v) {
      out->simplices[i * (M + 1) + v] = el.simplex.vertices[v];
      out->bary[i * (M + 1) + v] = el.barycentric_coords[0][v];
      out->lambda[i * (M + 1) + v] = NAN;
    }
    out->track_id[i] = el.track_id;
    out->type[i] = el.type;
    out->scalar[i] = el.scalar;
    for (int a = 0; a < 16; ++a) (*attrs)[i * 16 + a] = el.attributes[a];
  }
  std::vector<uint32_t> edges;
  for (const auto& conn : complex.connectivity)
    if (conn.dimension == 1) edges = conn.indices;
  out->n_edges = edges.size() / 2;
  out->edges = (uint32_t*)std::malloc(sizeof(uint32_t) * (edges.size() + 2));
  if (!edges.empty()) std::memcpy(out->edges, edges.data(), sizeof(uint32_t) * edges.size());
  return 0;
}

// Level sets: SimplicialEngine<T, ContourPredicate<T>> on a regular mesh
// (the reference's tests/test_examples.cpp:225-256 set-up), features and the
// manifold cells of get_complex flattened.
template <typename T>
int run_contour(const orc_mesh* mesh, const orc_field* field, double threshold, orc_result* out, orc_conn* conn) {
  using namespace ftk2;
  std::vector<uint64_t> dims, off, glob;
  std::shared_ptr<Mesh> mesh_ptr;
  std::shared_ptr<RegularSimplicialMesh> reg;
  if (mesh->kind == ORC_MESH_REGULAR) {
    for (int i = 0; i < mesh->ndims; ++i) {
      dims.push_back(mesh->local_dims[i]);
      off.push_back(mesh->offset[i]);
      glob.push_back(mesh->global_dims[i]);
    }
    reg = std::make_shared<RegularSimplicialMesh>(dims, off, glob);
    mesh_ptr = reg;
  } else {
    // ExtrudedSimplicialMesh over an UnstructuredSimplicialMesh: the field is
    // per vertex (a 1-D array indexed by vertex id, engine.hpp:1000)
    std::vector<double> coords(mesh->base_coords, mesh->base_coords + 3 * mesh->n_base_verts);
    size_t nc = (size_t)mesh->n_base_cells * (mesh->base_cell_dim + 1);
    std::vector<uint64_t> cells(mesh->base_cells, mesh->base_cells + nc);
    auto base = std::make_shared<UnstructuredSimplicialMesh>(mesh->base_cell_dim, mesh->base_cell_dim, coords, cells);
    mesh_ptr = std::make_shared<ExtrudedSimplicialMesh>(base, mesh->n_layers);
  }
  ContourPredicate<T> pred;
  pred.var_name = "S";
  pred.threshold = (T)threshold;
  pred.sos_q = field->sos_q;
  std::map<std::string, ftk::ndarray<T>> data;
  data["S"] = make_array<T>(field->comp[0], field->nd, field->dims);
  SimplicialEngine<T, ContourPredicate<T>> engine(mesh_ptr, pred);
  std::streambuf* saved = std::cout.rdbuf();
  std::ostringstream sink;
  std::cout.rdbuf(sink.rdbuf());
  engine.execute(data, {"S"});
  FeatureComplex complex = engine.get_complex();
  std::cout.rdbuf(saved);

  const uint64_t n = complex.vertices.size();
  const auto& a = data.at("S");
  out->m = 1;
  out->n = n;
  out->simplices = (uint64_t*)std::malloc(sizeof(uint64_t) * (2 * n + 1));
  out->bary = (float*)std::malloc(sizeof(float) * (2 * n + 1));
  out->lambda = (double*)std::malloc(sizeof(double) * (2 * n + 1));
  out->track_id = (uint64_t*)std::malloc(sizeof(uint64_t) * (n + 1));
  out->type = (uint32_t*)std::malloc(sizeof(uint32_t) * (n + 1));
  out->scalar = (float*)std::malloc(sizeof(float) * (n + 1));
  out->n_tested = 0;
  for (uint64_t i = 0; i < n; ++i) {
    const FeatureElement& el = complex.vertices[i];
    T values[2][1];
    for (int v = 0; v < 2; ++v) {
      out->simplices[2 * i + v] = el.simplex.vertices[v];
      out->bary[2 * i + v] = el.barycentric_coords[0][v];
      T x;
      if (a.nd() == 1 || !reg) {
        x = a[el.simplex.vertices[v]];
      } else {
        std::vector<double> c = reg->get_vertex_coordinates(el.simplex.vertices[v]);
        for (size_t k = 0; k < c.size(); ++k) c[k] -= (double)off[k];
        x = c.size() == 3 ? a.f(c[0], c[1], c[2]) : a.f(c[0], c[1], c[2], c[3]);
      }
      values[v][0] = x - pred.threshold;
    }
    // the barycentrics ContourPredicate::extract_it stores (predicate.hpp:149)
    T lambda[2];
    if (!ZeroCrossingSolver<1, T>::solve(values, lambda)) lambda[0] = lambda[1] = (T)0.5;
    out->lambda[2 * i] = (double)lambda[0];
    out->lambda[2 * i + 1] = (double)lambda[1];
    out->track_id[i] = el.track_id;
    out->type[i] = el.type;
    out->scalar[i] = el.scalar;
  }
  out->n_edges = 0;
  out->edges = (uint32_t*)std::malloc(sizeof(uint32_t) * 2);
  conn->dim = mesh->ndims - 1;
  conn->n = 0;
  std::vector<uint32_t> cells;
  for (const auto& c : complex.connectivity)
    if (c.dimension == conn->dim) cells = c.indices;
  conn->n = cells.size() / (conn->dim + 1);
  conn->idx = (uint32_t*)std::malloc(sizeof(uint32_t) * (cells.size() + 1));
  if (!cells.empty()) std::memcpy(conn->idx, cells.data(), sizeof(uint32_t) * cells.size());
  return 0;
}

// Fibers: SimplicialEngine<T, FiberPredicate<T>> on a regular mesh with the
// two scalar fields F and G (the reference's tests/test_examples.cpp fiber
// set-up), flattened as run() does.  lambda: the barycentrics the predicate
// stores (solver output, or 1/3 where it falls back, predicate.hpp:354).
template <typename T>
int run_fiber(const orc_mesh* mesh, const orc_field* field, const double* thr, orc_result* out,
              orc_conn* conn = nullptr) {
  using namespace ftk2;
  std::vector<uint64_t> dims, off, glob;
  std::shared_ptr<Mesh> mesh_ptr;
  std::shared_ptr<RegularSimplicialMesh> reg;
  if (mesh->kind == ORC_MESH_REGULAR) {
    for (int i = 0; i < mesh->ndims; ++i) {
      dims.push_back(mesh->local_dims[i]);
      off.push_back(mesh->offset[i]);
      glob.push_back(mesh->global_dims[i]);
    }
    reg = std::make_shared<RegularSimplicialMesh>(dims, off, glob);
    mesh_ptr = reg;
  } else {
    std::vector<double> coords(mesh->base_coords, mesh->base_coords + 3 * mesh->n_base_verts);
    size_t nc = (size_t)mesh->n_base_cells * (mesh->base_cell_dim + 1);
    std::vector<uint64_t> cells(mesh->base_cells, mesh->base_cells + nc);
    auto base = std::make_shared<UnstructuredSimplicialMesh>(mesh->base_cell_dim, mesh->base_cell_dim, coords, cells);
    mesh_ptr = std::make_shared<ExtrudedSimplicialMesh>(base, mesh->n_layers);
  }
  FiberPredicate<T> pred;
  pred.var_names[0] = "F";
  pred.var_names[1] = "G";
  pred.thresholds[0] = (T)thr[0];
  pred.thresholds[1] = (T)thr[1];
  pred.sos_q = field->sos_q;
  std::map<std::string, ftk::ndarray<T>> data;
  data["F"] = make_array<T>(field->comp[0], field->nd, field->dims);
  data["G"] = make_array<T>(field->comp[1], field->nd, field->dims);
  SimplicialEngine<T, FiberPredicate<T>> engine(mesh_ptr, pred);
  std::streambuf* saved = std::cout.rdbuf();
  std::ostringstream sink;
  std::cout.rdbuf(sink.rdbuf());
  engine.execute(data, {"F", "G"});
  FeatureComplex complex = engine.get_complex();
  std::cout.rdbuf(saved);

  const uint64_t n = complex.vertices.size();
  out->m = 2;
  out->n = n;
  out->simplices = (uint64_t*)std::malloc(sizeof(uint64_t) * (3 * n + 1));
  out->bary = (float*)std::malloc(sizeof(float) * (3 * n + 1));
  out->lambda = (double*)std::malloc(sizeof(double) * (3 * n + 1));
  out->track_id = (uint64_t*)std::malloc(sizeof(uint64_t) * (n + 1));
  out->type = (uint32_t*)std::malloc(sizeof(uint32_t) * (n + 1));
  out->scalar = (float*)std::malloc(sizeof(float) * (n + 1));
  out->n_tested = 0;
  for (uint64_t i = 0; i < n; ++i) {
    const FeatureElement& el = complex.vertices[i];
    T values[3][2];
    for (int v = 0; v < 3; ++v) {
      out->simplices[3 * i + v] = el.simplex.vertices[v];
      out->bary[3 * i + v] = el.barycentric_coords[0][v];
      for (int j = 0; j < 2; ++j) {
        const auto& a = data.at(j == 0 ? "F" : "G");
        T x;
        if (!reg || a.nd() == 1) {
          x = a[el.simplex.vertices[v]];
        } else {
          std::vector<double> c = reg->get_vertex_coordinates(el.simplex.vertices[v]);
          for (size_t k = 0; k < c.size(); ++k) c[k] -= (double)off[k];
          x = c.size() == 3 ? a.f(c[0], c[1], c[2]) : a.f(c[0], c[1], c[2], c[3]);
        }
        values[v][j] = (T)(x - pred.thresholds[j]);
      }
    }
    T lambda[3];
    if (!ZeroCrossingSolver<2, T>::solve(values, lambda))
      for (int v = 0; v < 3; ++v) lambda[v] = (T)1.0 / 3.0;
    for (int v = 0; v < 3; ++v) out->lambda[3 * i + v] = (double)lambda[v];
    out->track_id[i] = el.track_id;
    out->type[i] = el.type;
    out->scalar[i] = el.scalar;
  }
  std::vector<uint32_t> edges, tris;
  for (const auto& cc : complex.connectivity) {
    if (cc.dimension == 1) edges = cc.indices;
    if (cc.dimension == 2) tris = cc.indices;
  }
  out->n_edges = edges.size() / 2;
  out->edges = (uint32_t*)std::malloc(sizeof(uint32_t) * (edges.size() + 2));
  if (!edges.empty()) std::memcpy(out->edges, edges.data(), sizeof(uint32_t) * edges.size());
  if (conn) {
    conn->dim = 2;
    conn->n = tris.size() / 3;
    conn->idx = (uint32_t*)std::malloc(sizeof(uint32_t) * (tris.size() + 1));
    if (!tris.empty()) std::memcpy(conn->idx, tris.data(), sizeof(uint32_t) * tris.size());
  }
  return 0;
}

}  // namespace

// Fiber surfaces: FiberPredicate<T> on a regular 3D+t mesh, or on an extruded
// mesh over tets (per-vertex arrays); conn receives the star-fan triangles of
// get_complex (form_general_manifold_patches, k = 2).
extern "C" int ftk2ref_run_fiber_surface(const orc_mesh* mesh, const orc_field* field, const double* thresholds,
                                         orc_result* out, orc_conn* conn) {
  std::memset(out, 0, sizeof(*out));
  std::memset(conn, 0, sizeof(*conn));
  if (mesh->ndims != 4 || field->layout != ORC_LAYOUT_SEPARATE) return 3;
  if (mesh->kind == ORC_MESH_EXTRUDED && (mesh->base_cell_dim != 3 || field->nd != 1)) return 3;
  try {
    return field->dtype == ORC_F64 ? run_fiber<double>(mesh, field, thresholds, out, conn)
                                   : run_fiber<float>(mesh, field, thresholds, out, conn);
  } catch (const std::exception& e) {
    std::cerr << "ftk2ref_run_fiber_surface: " << e.what() << std::endl;
    return 1;
  }
}

extern "C" int ftk2ref_run_fiber(const orc_mesh* mesh, const orc_field* field, const double* thresholds,
                                 orc_result* out) {
  std::memset(out, 0, sizeof(*out));
  if (mesh->ndims != 3 || field->layout != ORC_LAYOUT_SEPARATE) return 3;
  if (mesh->kind == ORC_MESH_EXTRUDED && field->nd != 1) return 3;
  try {
    return field->dtype == ORC_F64 ? run_fiber<double>(mesh, field, thresholds, out)
                                   : run_fiber<float>(mesh, field, thresholds, out);
  } catch (const std::exception& e) {
    std::cerr << "ftk2ref_run_fiber: " << e.what() << std::endl;
    return 1;
  }
}

extern "C" int ftk2ref_run_contour(const orc_mesh* mesh, const orc_field* field, double threshold,
                                   orc_result* out, orc_conn* conn) {
  std::memset(out, 0, sizeof(*out));
  std::memset(conn, 0, sizeof(*conn));
  if (mesh->ndims != 3 && mesh->ndims != 4) return 3;
  if (mesh->kind == ORC_MESH_EXTRUDED && field->nd != 1) return 3;
  try {
    return field->dtype == ORC_F64 ? run_contour<double>(mesh, field, threshold, out, conn)
                                   : run_contour<float>(mesh, field, threshold, out, conn);
  } catch (const std::exception& e) {
    std::cerr << "ftk2ref_run_contour: " << e.what() << std::endl;
    return 1;
  }
}

extern "C" void ftk2ref_free_conn(orc_conn* c) {
  std::free(c->idx);
  std::memset(c, 0, sizeof(*c));
}

extern "C" int ftk2ref_run(const orc_mesh* mesh, const orc_field* field, orc_result* out) {
  std::memset(out, 0, sizeof(*out));
  try {
    const bool f64 = field->dtype == ORC_F64;
    if (field->ncomp == 2) return f64 ? run<double, 2>(mesh, field, out) : run<float, 2>(mesh, field, out);
    if (field->ncomp == 3) return f64 ? run<double, 3>(mesh, field, out) : run<float, 3>(mesh, field, out);
    return 2;
  } catch (const std::exception& e) {
    std::cerr << "ftk2ref_run: " << e.what() << std::endl;
    return 1;
  }
}

extern "C" void ftk2ref_free(orc_result* r) {
  std::free(r->simplices);
  std::free(r->bary);
  std::free(r->lambda);
  std::free(r->track_id);
  std::free(r->type);
  std::free(r->scalar);
  std::free(r->edges);
  std::memset(r, 0, sizeof(*r));
}

extern "C" int ftk2ref_run_tracked(const orc_tracked* in, orc_result* out, float** attrs) {
  std::memset(out, 0, sizeof(*out));
  *attrs = nullptr;
  try {
    if (in->m == 2) return in->dtype == ORC_F64 ? run_tracked<double, 2>(in, out, attrs)
                                                : run_tracked<float, 2>(in, out, attrs);
    if (in->m == 3) return in->dtype == ORC_F64 ? run_tracked<double, 3>(in, out, attrs)
                                                : run_tracked<float, 3>(in, out, attrs);
    return 2;
  } catch (const std::exception& e) {
    std::cerr << "ftk2ref_run_tracked: " << e.what() << std::endl;
    return 1;
  }
}

extern "C" void ftk2ref_free_attrs(float* attrs) { std::free(attrs); }
