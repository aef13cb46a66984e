// C++ drop-in for the reference's critical-point engine, backed by the
// B200 C ABI (include/ftk2b.h).
//
// It mirrors the reference interface for this path so that a caller switches
// by changing the namespace and the include:
//
//   reference (include/ftk2/core/engine.hpp)      this header
//   ftk2::RegularSimplicialMesh(dims, off, glob)   ftk2b::RegularSimplicialMesh   (mesh.hpp:256-265)
//   ftk2::UnstructuredSimplicialMesh(...)          ftk2b::UnstructuredSimplicialMesh (unstructured_mesh.hpp:16)
//   ftk2::ExtrudedSimplicialMesh(base, layers)     ftk2b::ExtrudedSimplicialMesh  (mesh.hpp:544)
//   ftk2::CriticalPointPredicate<M,T>              ftk2b::CriticalPointPredicate<M,T> (predicate.hpp:49-64)
//   ftk2::SimplicialEngine<T,Pred>(mesh, pred)     ftk2b::SimplicialEngine<T,Pred> (engine.hpp:84-85)
//     .execute(data, vars) / .execute_cuda(...)      .execute / .execute_cuda      (engine.hpp:96-99, 273)
//     .get_complex() -> FeatureComplex               .get_complex()                (engine.hpp:822-996)
//
// `data` is any std::map<std::string, Array> whose Array exposes the
// reference ndarray's nd(), dimf(i) and pdata() (Fortran order, first index
// fastest), e.g. ftk::ndarray<T>.  Errors are thrown as ftk2b::Error carrying
// the ABI status (the reference throws from std::map::at and exits on CUDA
// errors, engine.hpp:29-37); there is no CPU fallback.
#pragma once

#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../ftk2b.h"

namespace ftk2b {

class Error : public std::runtime_error {
 public:
  Error(ftk2b_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
  ftk2b_status status;
};

// ---- meshes (descriptors only: the GPU derives every simplex implicitly)

class Mesh {
 public:
  virtual ~Mesh() = default;
  virtual int get_total_dimension() const = 0;
  virtual ftk2b_mesh_desc desc() const = 0;
};

class RegularSimplicialMesh : public Mesh {
 public:
  RegularSimplicialMesh(const std::vector<uint64_t>& dims, const std::vector<uint64_t>& offset = {},
                        const std::vector<uint64_t>& global_dims = {})
      : dims_(dims), offset_(offset), global_dims_(global_dims) {
    if (offset_.empty()) offset_.assign(dims_.size(), 0);
    if (global_dims_.empty()) global_dims_ = dims_;
  }
  int get_total_dimension() const override { return (int)dims_.size(); }
  const std::vector<uint64_t>& get_local_dims() const { return dims_; }
  const std::vector<uint64_t>& get_offset() const { return offset_; }
  const std::vector<uint64_t>& get_global_dims() const { return global_dims_; }
  ftk2b_mesh_desc desc() const override {
    ftk2b_mesh_desc d;
    std::memset(&d, 0, sizeof(d));
    d.kind = FTK2B_MESH_REGULAR;
    d.ndims = (int)dims_.size();
    for (size_t i = 0; i < dims_.size() && i < 4; ++i) {
      d.local_dims[i] = dims_[i];
      d.offset[i] = offset_[i];
      d.global_dims[i] = global_dims_[i];
    }
    return d;
  }

 private:
  std::vector<uint64_t> dims_, offset_, global_dims_;
};

class UnstructuredSimplicialMesh : public Mesh {
 public:
  UnstructuredSimplicialMesh(int spatial_dim, int cell_dim, const std::vector<double>& coords,
                             const std::vector<uint64_t>& cells)
      : spatial_dim_(spatial_dim), cell_dim_(cell_dim), coords_(coords), cells_(cells) {}
  int get_total_dimension() const override { return cell_dim_; }
  uint64_t get_num_vertices() const { return coords_.size() / 3; }
  int cell_dim() const { return cell_dim_; }
  const std::vector<uint64_t>& cells() const { return cells_; }
  ftk2b_mesh_desc desc() const override {
    throw Error(FTK2B_UNSUPPORTED, "a bare unstructured mesh has no time axis; extrude it");
  }

 private:
  int spatial_dim_, cell_dim_;
  std::vector<double> coords_;
  std::vector<uint64_t> cells_;
};

class ExtrudedSimplicialMesh : public Mesh {
 public:
  ExtrudedSimplicialMesh(std::shared_ptr<UnstructuredSimplicialMesh> base, uint64_t n_layers)
      : base_(std::move(base)), n_layers_(n_layers) {}
  int get_total_dimension() const override { return base_->get_total_dimension() + 1; }
  uint64_t get_n_layers() const { return n_layers_; }
  ftk2b_mesh_desc desc() const override {
    ftk2b_mesh_desc d;
    std::memset(&d, 0, sizeof(d));
    d.kind = FTK2B_MESH_EXTRUDED;
    d.ndims = base_->cell_dim() + 1;
    d.n_base_verts = base_->get_num_vertices();
    d.base_cells = base_->cells().data();
    d.base_cell_dim = base_->cell_dim();
    d.n_base_cells = base_->cells().size() / (base_->cell_dim() + 1);
    d.n_layers = n_layers_;
    return d;
  }

 private:
  std::shared_ptr<UnstructuredSimplicialMesh> base_;
  uint64_t n_layers_;
};

// ---- predicate (the CP knobs of predicate.hpp:22-64)

template <int M, typename T = double>
struct CriticalPointPredicate {
  static constexpr int codimension = M;
  double sos_q = 1000000.0;
  std::string vector_var_name;
  std::string var_names[M];
  std::string scalar_var_name;
  bool use_multicomponent = true;
  int precision = FTK2B_PRECISION_EXACT;  // new: refined-FP32 reporting
  bool classify = false;                  // new: Jacobian classification
};

// ---- output (feature.hpp:22-39, complex.hpp:14-58)

enum class FeatureGeometryType { Point, Segment, Polygon };

struct Simplex {
  int dimension;
  uint64_t vertices[5];
};

struct FeatureElement {
  Simplex simplex;
  FeatureGeometryType geometry_type;
  float barycentric_coords[3][16];
  uint64_t track_id;
  uint32_t type;
  float scalar;
  float attributes[16];
  FeatureElement() {
    std::memset(this, 0, sizeof(FeatureElement));
    geometry_type = FeatureGeometryType::Point;
  }
};

struct FeatureComplex {
  std::vector<FeatureElement> vertices;
  struct SimplexIndices {
    int dimension;
    std::vector<uint32_t> indices;
  };
  std::vector<SimplexIndices> connectivity;
  // new: double-precision barycentrics and classification, per vertex
  std::vector<double> lambda;
  std::vector<uint32_t> cp_class;
};

// ---- engine

template <typename T, typename PredicateType>
class SimplicialEngine {
 public:
  static constexpr int m = PredicateType::codimension;

  SimplicialEngine(std::shared_ptr<Mesh> mesh, PredicateType pred = PredicateType(), int device = 0)
      : mesh_(std::move(mesh)), pred_(pred) {
    ftk2b_ctx* c = nullptr;
    ftk2b_status s = ftk2b_ctx_create(device, &c);
    if (s != FTK2B_OK) throw Error(s, "ftk2b_ctx_create failed");
    ctx_.reset(c);
  }

  template <typename Array>
  void execute(const std::map<std::string, Array>& data, const std::vector<std::string>& = {}) {
    ftk2b_mesh_desc md = mesh_->desc();
    ftk2b_field_desc fd;
    std::memset(&fd, 0, sizeof(fd));
    fd.dtype = sizeof(T) == 8 ? FTK2B_F64 : FTK2B_F32;
    fd.ncomp = m;
    fd.location = FTK2B_HOST;
    const bool extruded = md.kind == FTK2B_MESH_EXTRUDED;
    if (pred_.use_multicomponent && !pred_.vector_var_name.empty()) {
      const Array& a = data.at(pred_.vector_var_name);
      fd.layout = FTK2B_LAYOUT_MULTICOMPONENT;
      fd.comp[0] = a.pdata();
      fd.nd = (int)a.nd() - 1;
      for (int i = 0; i < fd.nd && i < 4; ++i) fd.dims[i] = a.dimf(i + 1);
    } else {
      fd.layout = extruded ? FTK2B_LAYOUT_PER_VERTEX : FTK2B_LAYOUT_SEPARATE;
      for (int j = 0; j < m; ++j) {
        const Array& a = data.at(pred_.var_names[j]);
        fd.comp[j] = a.pdata();
        fd.nd = (int)a.nd();
        for (int i = 0; i < fd.nd && i < 4; ++i) fd.dims[i] = a.dimf(i);
        if (extruded) {
          fd.nd = 1;
          fd.dims[0] = a.nelem();
        }
      }
    }
    if (!pred_.scalar_var_name.empty()) {
      const Array& s = data.at(pred_.scalar_var_name);
      fd.scalar = s.pdata();
      fd.scalar_nd = (int)s.nd();
      for (int i = 0; i < fd.scalar_nd && i < 4; ++i) fd.scalar_dims[i] = s.dimf(i);
    }
    ftk2b_cp_params p = ftk2b_cp_params_default();
    p.sos_q = pred_.sos_q;
    p.precision = pred_.precision;
    p.classify = pred_.classify ? 1 : 0;
    ftk2b_cp_result* r = nullptr;
    ftk2b_status st = ftk2b_cp_extract(ctx_.get(), &md, &fd, &p, &r);
    if (st != FTK2B_OK) throw Error(st, ftk2b_last_error(ctx_.get()));
    result_.reset(r);
  }

  template <typename Array>
  void execute_cuda(const std::map<std::string, Array>& data, const std::vector<std::string>& v = {}) {
    execute(data, v);
  }

  FeatureComplex get_complex() const {
    FeatureComplex fc;
    const ftk2b_cp_result* r = result_.get();
    if (!r) return fc;
    const int k = r->m + 1;
    fc.vertices.resize(r->n_features);
    fc.lambda.assign(r->lambda, r->lambda + r->n_features * k);
    fc.cp_class.assign(r->cp_class, r->cp_class + r->n_features);
    for (uint64_t i = 0; i < r->n_features; ++i) {
      FeatureElement& el = fc.vertices[i];
      el.simplex.dimension = r->m;
      for (int v = 0; v < k; ++v) {
        el.simplex.vertices[v] = r->simplices[i * k + v];
        el.barycentric_coords[0][v] = r->barycentric[i * k + v];
      }
      el.track_id = r->track_id[i];
      el.type = r->type[i];
      el.scalar = r->scalar[i];
    }
    if (r->n_edges) {
      FeatureComplex::SimplexIndices e;
      e.dimension = 1;
      e.indices.assign(r->edges, r->edges + 2 * r->n_edges);
      fc.connectivity.push_back(std::move(e));
    }
    return fc;
  }

 private:
  struct CtxDel {
    void operator()(ftk2b_ctx* c) const { ftk2b_ctx_destroy(c); }
  };
  struct ResDel {
    void operator()(ftk2b_cp_result* r) const { ftk2b_cp_result_free(r); }
  };
  std::shared_ptr<Mesh> mesh_;
  PredicateType pred_;
  std::unique_ptr<ftk2b_ctx, CtxDel> ctx_;
  std::unique_ptr<ftk2b_cp_result, ResDel> result_;
};

}  // namespace ftk2b
