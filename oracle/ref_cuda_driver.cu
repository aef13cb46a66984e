// Driver that runs the reference's own GPU engine (execute_cuda,
// engine.hpp:273-425 with cuda_engine.hpp:366-493) for timing the incumbent
// GPU path on the same device as the B200 path.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile (target refcuda) into
// oracle/_ref/libftk2refcuda.so from the reference headers where they lie,
// against the ndarray shim in oracle/shim.  The reference's GPU path reads
// separate per-component arrays only (predicate.hpp:112) and falls back to
// the centroid where its solve fails (predicate.hpp:115), so it is a timing
// baseline, not the oracle.
#include <ftk2/core/engine.hpp>
#include <ftk2/core/mesh.hpp>
#include <ftk2/core/predicate.hpp>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "oracle_api.h"

namespace {

template <typename T>
ftk::ndarray<T> make_array(const void* src, int nd, const uint64_t* dims) {
  std::vector<size_t> shape;
  for (int i = 0; i < nd; ++i) shape.push_back((size_t)dims[i]);
  ftk::ndarray<T> a(shape);
  std::memcpy(a.data(), src, a.nelem() * sizeof(T));
  return a;
}

template <typename T, int M>
int run(const orc_mesh* mesh, const orc_field* field, orc_result* out, double* exec_ms, double* complex_ms) {
  using namespace ftk2;
  std::vector<uint64_t> dims, off, glob;
  for (int i = 0; i < mesh->ndims; ++i) {
    dims.push_back(mesh->local_dims[i]);
    off.push_back(mesh->offset[i]);
    glob.push_back(mesh->global_dims[i]);
  }
  auto reg = std::make_shared<RegularSimplicialMesh>(dims, off, glob);
  CriticalPointPredicate<M, T> pred;
  pred.sos_q = field->sos_q;
  pred.use_multicomponent = false;
  std::map<std::string, ftk::ndarray<T>> data;
  static const char* names[3] = {"U", "V", "W"};
  for (int j = 0; j < M; ++j) {
    pred.var_names[j] = names[j];
    data[names[j]] = make_array<T>(field->comp[j], field->nd, field->dims);
  }
  SimplicialEngine<T, CriticalPointPredicate<M, T>> engine(reg, pred);
  std::streambuf* saved = std::cout.rdbuf();
  std::ostringstream sink;
  std::cout.rdbuf(sink.rdbuf());
  const auto t0 = std::chrono::steady_clock::now();
  engine.execute_cuda(data);
  const auto t1 = std::chrono::steady_clock::now();
  FeatureComplex complex = engine.get_complex();
  const auto t2 = std::chrono::steady_clock::now();
  std::cout.rdbuf(saved);
  *exec_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  *complex_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
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
    for (int v = 0; v <= M; ++v) {
      out->simplices[i * (M + 1) + v] = el.simplex.vertices[v];
      out->bary[i * (M + 1) + v] = el.barycentric_coords[0][v];
      out->lambda[i * (M + 1) + v] = NAN;
    }
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

// The reference kernel alone: the device mesh, views and result buffers set
// up as execute_cuda_regular does (engine.hpp:306-370), one untimed launch to
// size the node and connectivity buffers, then `reps` launches each timed
// with CUDA events on the default stream.
template <typename T, int M>
int time_kernel(const orc_mesh* mesh, const orc_field* field, int reps, double* kernel_ms, int* n_nodes) {
  using namespace ftk2;
  RegularSimplicialMeshDevice dm;
  std::memset(&dm, 0, sizeof(dm));
  dm.ndims = mesh->ndims;
  for (int i = 0; i < 4; ++i) {
    dm.local_dims[i] = i < mesh->ndims ? mesh->local_dims[i] : 1;
    dm.offset[i] = i < mesh->ndims ? mesh->offset[i] : 0;
    dm.global_dims[i] = i < mesh->ndims ? mesh->global_dims[i] : 1;
  }
  CriticalPointPredicate<M, T> pred;
  pred.sos_q = field->sos_q;
  size_t ne = 1;
  for (int i = 0; i < field->nd; ++i) ne *= field->dims[i];
  CudaDataView<T> hv[M];
  std::vector<void*> allocs;
  auto alloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    allocs.push_back(p);
    return p;
  };
  auto cleanup = [&]() {
    for (void* p : allocs) cudaFree(p);
    allocs.clear();
  };
  for (int j = 0; j < M; ++j) {
    void* d = alloc(ne * sizeof(T));
    if (!d) return cleanup(), 4;
    cudaMemcpy(d, field->comp[j], ne * sizeof(T), cudaMemcpyHostToDevice);
    std::memset(&hv[j], 0, sizeof(hv[j]));
    hv[j].data = static_cast<const T*>(d);
    hv[j].ndims = field->nd;
    uint64_t stride = 1;
    for (int i = 0; i < 4; ++i) {
      hv[j].dims[i] = i < field->nd ? field->dims[i] : 1;
      hv[j].s[i] = i < field->nd ? stride : 0;
      if (i < field->nd) stride *= field->dims[i];
    }
  }
  auto* dv = static_cast<CudaDataView<T>*>(alloc(sizeof(hv)));
  if (!dv) return cleanup(), 4;
  cudaMemcpy(dv, hv, sizeof(hv), cudaMemcpyHostToDevice);
  int* counts = static_cast<int*>(alloc(4 * sizeof(int)));
  if (!counts) return cleanup(), 4;
  const uint64_t n_hc = dm.get_num_hypercubes();
  const int n_types = get_num_simplex_types(dm.ndims, M);
  const uint64_t total = n_hc * (uint64_t)n_types;
  const unsigned grid = (unsigned)((total + 255) / 256);
  using Dev = typename CriticalPointPredicate<M, T>::Device;
  int max_nodes = 1000000, max_conn = 3000000;
  CudaExtractionResult<uint64_t> res;
  float total_ms = 0.f;
  int h[4] = {0, 0, 0, 0};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int attempt = 0; attempt < 2; ++attempt) {
    res.max_nodes = max_nodes;
    res.max_conn = max_conn;
    res.nodes = static_cast<FeatureElement*>(alloc((size_t)max_nodes * sizeof(FeatureElement)));
    res.edges = static_cast<DeviceManifoldSimplex<uint64_t, 1>*>(alloc((size_t)max_conn * sizeof(DeviceManifoldSimplex<uint64_t, 1>)));
    res.faces = static_cast<DeviceManifoldSimplex<uint64_t, 2>*>(alloc((size_t)max_conn * sizeof(DeviceManifoldSimplex<uint64_t, 2>)));
    res.volumes = static_cast<DeviceManifoldSimplex<uint64_t, 3>*>(alloc((size_t)max_conn * sizeof(DeviceManifoldSimplex<uint64_t, 3>)));
    if (!res.nodes || !res.edges || !res.faces || !res.volumes) return cleanup(), 4;
    res.node_count = counts;
    res.edge_count = counts + 1;
    res.face_count = counts + 2;
    res.volume_count = counts + 3;
    bool overflow = false;
    for (int r = -1; r < reps; ++r) {
      cudaMemset(counts, 0, 4 * sizeof(int));
      cudaEventRecord(e0);
      extraction_kernel<RegularSimplicialMeshDevice, Dev, T, uint64_t><<<grid, 256>>>(dm, pred.get_device(), dv, M, res);
      cudaEventRecord(e1);
      if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) return cleanup(), 5;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (r >= 0) total_ms += ms;
      cudaMemcpy(h, counts, sizeof(h), cudaMemcpyDeviceToHost);
      if (h[0] > max_nodes || std::max({h[1], h[2], h[3]}) > max_conn) {
        overflow = true;
        break;
      }
    }
    if (!overflow) break;
    max_nodes = h[0] + 1000;
    max_conn = std::max({h[1], h[2], h[3]}) + 1000;
    total_ms = 0.f;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cleanup();
  *kernel_ms = reps > 0 ? total_ms / reps : 0.0;
  *n_nodes = h[0];
  return 0;
}

}  // namespace

extern "C" int ftk2refcuda_time_kernel(const orc_mesh* mesh, const orc_field* field, int reps, double* kernel_ms,
                                       int* n_nodes) {
  if (mesh->kind != ORC_MESH_REGULAR || field->layout != ORC_LAYOUT_SEPARATE) return 3;
  if (field->ncomp == 2) return field->dtype == ORC_F64 ? time_kernel<double, 2>(mesh, field, reps, kernel_ms, n_nodes)
                                                        : time_kernel<float, 2>(mesh, field, reps, kernel_ms, n_nodes);
  if (field->ncomp == 3) return field->dtype == ORC_F64 ? time_kernel<double, 3>(mesh, field, reps, kernel_ms, n_nodes)
                                                        : time_kernel<float, 3>(mesh, field, reps, kernel_ms, n_nodes);
  return 2;
}

// Regular mesh, separate component arrays; exec_ms = execute_cuda (uploads,
// the extraction kernel and the host-side node bookkeeping), complex_ms =
// get_complex.
extern "C" int ftk2refcuda_run(const orc_mesh* mesh, const orc_field* field, orc_result* out, double* exec_ms,
                               double* complex_ms) {
  std::memset(out, 0, sizeof(*out));
  if (mesh->kind != ORC_MESH_REGULAR || field->layout != ORC_LAYOUT_SEPARATE) return 3;
  try {
    if (field->ncomp == 2) return field->dtype == ORC_F64 ? run<double, 2>(mesh, field, out, exec_ms, complex_ms)
                                                          : run<float, 2>(mesh, field, out, exec_ms, complex_ms);
    if (field->ncomp == 3) return field->dtype == ORC_F64 ? run<double, 3>(mesh, field, out, exec_ms, complex_ms)
                                                          : run<float, 3>(mesh, field, out, exec_ms, complex_ms);
    return 2;
  } catch (const std::exception& e) {
    std::cerr << "ftk2refcuda_run: " << e.what() << std::endl;
    return 1;
  }
}

extern "C" void ftk2refcuda_free(orc_result* r) {
  std::free(r->simplices);
  std::free(r->bary);
  std::free(r->lambda);
  std::free(r->track_id);
  std::free(r->type);
  std::free(r->scalar);
  std::free(r->edges);
  std::memset(r, 0, sizeof(*r));
}
