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
//   ftk2::ContourPredicate<T> (level sets)         ftk2b::ContourPredicate<T>     (predicate.hpp:135-183)
//   ftk2::FiberPredicate<T> (fibers)               ftk2b::FiberPredicate<T>       (predicate.hpp:341-362)
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

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <type_traits>
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
  virtual int get_spatial_dimension() const = 0;
  virtual int get_total_dimension() const = 0;
  // grid or physical coordinates of a vertex, time last on extruded meshes
  // (mesh.hpp:374-378, 714-720; unstructured_mesh.hpp:100-107)
  virtual std::vector<double> get_vertex_coordinates(uint64_t vertex_id) const = 0;
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
  int get_spatial_dimension() const override { return (int)dims_.size(); }
  int get_total_dimension() const override { return (int)dims_.size(); }
  // the global grid index of the id, one coordinate per axis
  std::vector<double> get_vertex_coordinates(uint64_t id) const override {
    std::vector<double> c(global_dims_.size());
    for (size_t i = 0; i < global_dims_.size(); ++i) {
      c[i] = (double)(id % global_dims_[i]);
      id /= global_dims_[i];
    }
    return c;
  }
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
  int get_spatial_dimension() const override { return spatial_dim_; }
  int get_total_dimension() const override { return cell_dim_; }
  // the first spatial_dim of the vertex's three stored coordinates; empty
  // past the last vertex
  std::vector<double> get_vertex_coordinates(uint64_t id) const override {
    if (id >= get_num_vertices()) return {};
    return std::vector<double>(coords_.begin() + 3 * id, coords_.begin() + 3 * id + spatial_dim_);
  }
  uint64_t get_num_vertices() const { return coords_.size() / 3; }
  const std::vector<double>& coords() const { return coords_; }
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
  // Over a regular spatial mesh, as the reference's high-level caller builds
  // its spacetime mesh (feature_tracker.cpp:520): the base cells are the
  // spatial grid's Kuhn simplices (one per axis order, d! per cube, as
  // RegularSimplicialMesh enumerates them) and the vertex id of spatial vertex
  // s at timestep t is s + t * S with S = the base's grid_index_to_id(global
  // dims), which is what ExtrudedSimplicialMesh's constructor takes as its
  // spatial vertex count (mesh.hpp:544-560).
  ExtrudedSimplicialMesh(std::shared_ptr<RegularSimplicialMesh> base, uint64_t n_layers)
      : n_layers_(n_layers), regular_(std::move(base)) {
    const std::vector<uint64_t>& g = regular_->get_global_dims();
    const int d = (int)g.size();
    if (d != 2 && d != 3) throw Error(FTK2B_UNSUPPORTED, "regular spatial meshes are 2D or 3D");
    for (int k = 0; k < d; ++k)
      if (regular_->get_offset()[k] != 0 || regular_->get_local_dims()[k] != g[k])
        throw Error(FTK2B_UNSUPPORTED, "an extruded regular base must cover its global grid");
    stride_ = 0;
    uint64_t mul = 1;
    for (int k = 0; k < d; ++k) {
      stride_ += g[k] * mul;
      mul *= g[k];
    }
    int perm[3] = {0, 1, 2};
    std::vector<std::vector<int>> orders;
    do {
      orders.push_back(std::vector<int>(perm, perm + d));
    } while (std::next_permutation(perm, perm + d));
    const uint64_t nz = d == 3 ? g[2] : 1;
    for (uint64_t z = 0; z + (d == 3 ? 1 : 0) < nz; ++z)
      for (uint64_t y = 0; y + 1 < g[1]; ++y)
        for (uint64_t x = 0; x + 1 < g[0]; ++x)
          for (const auto& o : orders) {
            uint64_t c[3] = {x, y, z};
            cells_.push_back(c[0] + g[0] * (c[1] + g[1] * c[2]));
            for (int i = 0; i < d; ++i) {
              c[o[i]]++;
              cells_.push_back(c[0] + g[0] * (c[1] + g[1] * c[2]));
            }
          }
  }
  int get_spatial_dimension() const override {
    return regular_ ? regular_->get_spatial_dimension() : base_->get_spatial_dimension();
  }
  int get_total_dimension() const override {
    return (regular_ ? (int)regular_->get_global_dims().size() : base_->get_total_dimension()) + 1;
  }
  // the base vertex's coordinates, then the layer (vertex id s + t * S)
  std::vector<double> get_vertex_coordinates(uint64_t id) const override {
    const uint64_t S = regular_ ? stride_ : base_->get_num_vertices();
    if (S == 0) return {};
    std::vector<double> c = regular_ ? regular_->get_vertex_coordinates(id % S)
                                     : base_->get_vertex_coordinates(id % S);
    c.push_back((double)(id / S));
    return c;
  }
  uint64_t get_n_layers() const { return n_layers_; }
  // regular base: its spatial grid and the per-timestep vertex id stride
  const RegularSimplicialMesh* regular_base() const { return regular_.get(); }
  uint64_t vertex_stride() const { return stride_; }
  ftk2b_mesh_desc desc() const override {
    ftk2b_mesh_desc d;
    std::memset(&d, 0, sizeof(d));
    d.kind = FTK2B_MESH_EXTRUDED;
    d.n_layers = n_layers_;
    if (regular_) {
      const int sd = (int)regular_->get_global_dims().size();
      d.ndims = sd + 1;
      d.n_base_verts = stride_;
      d.base_cells = cells_.data();
      d.base_cell_dim = sd;
      d.n_base_cells = cells_.size() / (sd + 1);
      return d;
    }
    d.ndims = base_->cell_dim() + 1;
    d.n_base_verts = base_->get_num_vertices();
    d.base_cells = base_->cells().data();
    d.base_cell_dim = base_->cell_dim();
    d.n_base_cells = base_->cells().size() / (base_->cell_dim() + 1);
    return d;
  }

 private:
  std::shared_ptr<UnstructuredSimplicialMesh> base_;
  uint64_t n_layers_;
  std::shared_ptr<RegularSimplicialMesh> regular_;
  uint64_t stride_ = 0;
  std::vector<uint64_t> cells_;
};

// ---- predicate (the CP knobs of predicate.hpp:22-64)

// An array value to record at every feature (predicate.hpp:34-40): type
// "magnitude" or "scalar", component >= 0 for one component of a
// multicomponent source, slot 0..15 of FeatureElement::attributes.
struct AttributeSpec {
  std::string name;
  std::string source;
  std::string type = "scalar";
  int component = -1;
  int slot = -1;
};

template <int M, typename T = double>
struct CriticalPointPredicate {
  static constexpr int codimension = M;
  double sos_q = 1000000.0;
  std::string vector_var_name;
  std::string var_names[M];
  std::string scalar_var_name;
  bool use_multicomponent = true;
  std::vector<AttributeSpec> attributes;
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
    const auto* ext = dynamic_cast<const ExtrudedSimplicialMesh*>(mesh_.get());
    if (ext && ext->regular_base()) {
      execute_extruded_regular(data, *ext);
      return;
    }
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
    record_attributes(data);
  }

  template <typename Array>
  void execute_cuda(const std::map<std::string, Array>& data, const std::vector<std::string>& v = {}) {
    execute(data, v);
  }

  FeatureComplex get_complex() const {
    FeatureComplex fc;
    const ftk2b_cp_result* r = result_.get();
    if (!r) return fc;
    const bool with_attrs = attrs_.size() == 16 * (size_t)r->n_features;
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
      if (with_attrs)
        for (int a = 0; a < 16; ++a) el.attributes[a] = attrs_[16 * (size_t)i + a];
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
  template <typename Array>
  using elem_t = std::remove_cv_t<std::remove_pointer_t<decltype(std::declval<const Array&>().pdata())>>;

  // FeatureElement::attributes at each feature (engine.hpp:1143-1199),
  // interpolated on the device by ftk2b_cp_attributes with the float
  // barycentrics the elements store, in the field precision T.  The kind of
  // each spec follows the reference: a source whose first dimension is 1..16
  // is multicomponent, read as one component (component >= 0) or as its
  // magnitude (type "magnitude"); anything else is read as a plain value.
  template <typename Array>
  void record_attributes(const std::map<std::string, Array>& data) {
    attrs_.clear();
    const ftk2b_cp_result* r = result_.get();
    if (!r || pred_.attributes.empty()) return;
    std::vector<ftk2b_attribute_desc> descs;
    std::vector<std::vector<T>> conv;
    conv.reserve(pred_.attributes.size());
    for (const AttributeSpec& spec : pred_.attributes) {
      if (spec.slot < 0 || spec.slot >= 16) continue;
      auto it = data.find(spec.source);
      if (it == data.end()) continue;
      const Array& a = it->second;
      if (a.nd() < 1 || a.nd() > 6) throw Error(FTK2B_UNSUPPORTED, "attribute arrays have 1 to 6 dimensions");
      const bool multicomp = a.nd() >= 2 && a.dimf(0) >= 1 && a.dimf(0) <= 16;
      ftk2b_attribute_desc d;
      std::memset(&d, 0, sizeof(d));
      d.kind = (multicomp && spec.component >= 0) ? FTK2B_ATTR_COMPONENT
               : (multicomp && spec.type == "magnitude") ? FTK2B_ATTR_MAGNITUDE
                                                         : FTK2B_ATTR_VALUE;
      d.component = spec.component;
      d.slot = spec.slot;
      d.location = FTK2B_HOST;
      d.nd = (int)a.nd();
      for (int q = 0; q < d.nd; ++q) d.dims[q] = a.dimf(q);
      if (std::is_same<elem_t<Array>, T>::value) {
        d.data = a.pdata();
      } else {
        conv.emplace_back(a.pdata(), a.pdata() + a.nelem());
        d.data = conv.back().data();
      }
      descs.push_back(d);
    }
    const auto* ext = dynamic_cast<const ExtrudedSimplicialMesh*>(mesh_.get());
    const ftk2b_mesh_desc md = mesh_->desc();
    std::vector<uint64_t> bg;
    if (ext && ext->regular_base()) bg = ext->regular_base()->get_global_dims();
    attrs_.assign(16 * (size_t)r->n_features, 0.f);
    const ftk2b_status st = ftk2b_cp_attributes(ctx_.get(), &md, bg.empty() ? nullptr : bg.data(),
                                                (uint32_t)descs.size(), descs.data(), attrs_.data());
    if (st != FTK2B_OK) throw Error(st, ftk2b_last_error(ctx_.get()));
  }

  // The extruded mesh over a regular base: the reference reads the arrays at
  // each vertex's grid coordinates (multicomponent f(j, x, y, [z,] t), legacy
  // f(x, y, [z,] t)), so they are laid out here as per-vertex arrays indexed
  // by the extruded vertex id s + t * S (the gap ids of each timestep, which no
  // simplex uses, hold zeros).
  template <typename Array>
  void execute_extruded_regular(const std::map<std::string, Array>& data, const ExtrudedSimplicialMesh& ext) {
    const std::vector<uint64_t>& g = ext.regular_base()->get_global_dims();
    uint64_t nxy = 1;
    for (uint64_t d : g) nxy *= d;
    const uint64_t S = ext.vertex_stride(), nt = ext.get_n_layers() + 1;
    std::vector<std::vector<T>> comps(m);
    auto lay_out = [&](const Array& a, int j, int ncomp, std::vector<T>& dst) {
      dst.assign(S * nt, T(0));
      const uint64_t have = (uint64_t)a.nelem() / (uint64_t)ncomp;
      for (uint64_t t = 0; t < nt; ++t)
        for (uint64_t sv = 0; sv < nxy; ++sv) {
          const uint64_t e = sv + nxy * t;
          if (e < have) dst[sv + S * t] = (T)a.pdata()[(uint64_t)j + (uint64_t)ncomp * e];
        }
    };
    if (pred_.use_multicomponent && !pred_.vector_var_name.empty()) {
      const Array& a = data.at(pred_.vector_var_name);
      for (int j = 0; j < m; ++j) lay_out(a, j, m, comps[j]);
    } else {
      for (int j = 0; j < m; ++j) {
        const Array& a = data.at(pred_.var_names[j]);
        if (a.nd() == 1) {
          comps[j].assign(a.pdata(), a.pdata() + a.nelem());
          comps[j].resize(std::max<size_t>(comps[j].size(), S * nt), T(0));
        } else {
          lay_out(a, 0, 1, comps[j]);
        }
      }
    }
    std::vector<T> scal;
    ftk2b_mesh_desc md = ext.desc();
    ftk2b_field_desc fd;
    std::memset(&fd, 0, sizeof(fd));
    fd.dtype = sizeof(T) == 8 ? FTK2B_F64 : FTK2B_F32;
    fd.ncomp = m;
    fd.location = FTK2B_HOST;
    fd.layout = FTK2B_LAYOUT_PER_VERTEX;
    fd.nd = 1;
    fd.dims[0] = S * nt;
    for (int j = 0; j < m; ++j) fd.comp[j] = comps[j].data();
    if (!pred_.scalar_var_name.empty() && !pred_.use_multicomponent) {
      const Array& sa = data.at(pred_.scalar_var_name);
      if (sa.nd() == 1) scal.assign(sa.pdata(), sa.pdata() + sa.nelem());
      else lay_out(sa, 0, 1, scal);
      scal.resize(std::max<size_t>(scal.size(), S * nt), T(0));
      fd.scalar = scal.data();
      fd.scalar_nd = 1;
      fd.scalar_dims[0] = S * nt;
    }
    ftk2b_cp_params p = ftk2b_cp_params_default();
    p.sos_q = pred_.sos_q;
    p.precision = pred_.precision;
    ftk2b_cp_result* r = nullptr;
    ftk2b_status st = ftk2b_cp_extract(ctx_.get(), &md, &fd, &p, &r);
    if (st != FTK2B_OK) throw Error(st, ftk2b_last_error(ctx_.get()));
    result_.reset(r);
    record_attributes(data);
  }

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
  std::vector<float> attrs_;  // 16 per feature when attributes were recorded
};

// ---- level sets (ContourPredicate<T>, predicate.hpp:135-183)

template <typename T = double>
struct ContourPredicate {
  static constexpr int codimension = 1;
  double sos_q = 1000000.0;
  std::string var_name;
  T threshold = (T)0.0;
};

// SimplicialEngine<T, ContourPredicate<T>> on a regular mesh or an extruded
// mesh over an unstructured base (one value per vertex id): execute runs
// ftk2b_contour_extract on the scalar array (the predicate's var_name, or the
// first name passed); get_complex returns the edge features in simplex order
// and the manifold cells (dimension 2 on 2D+t meshes, 3 on 3D+t meshes) as
// the reference's get_complex lists them (engine.hpp:822-996).
template <typename T>
class SimplicialEngine<T, ContourPredicate<T>> {
 public:
  static constexpr int m = 1;

  SimplicialEngine(std::shared_ptr<Mesh> mesh, ContourPredicate<T> pred = ContourPredicate<T>(), int device = 0)
      : mesh_(std::move(mesh)), pred_(pred) {
    ftk2b_ctx* c = nullptr;
    ftk2b_status s = ftk2b_ctx_create(device, &c);
    if (s != FTK2B_OK) throw Error(s, "ftk2b_ctx_create failed");
    ctx_.reset(c);
  }

  template <typename Array>
  void execute(const std::map<std::string, Array>& data, const std::vector<std::string>& vars = {}) {
    const std::string& name = vars.empty() ? pred_.var_name : vars[0];
    const Array& a = data.at(name);
    ftk2b_mesh_desc md = mesh_->desc();
    if (md.kind == FTK2B_MESH_EXTRUDED) {
      // extruded meshes over unstructured bases, one value per vertex id; a
      // regular base's vertex ids leave gaps that carry no vertex
      const auto* ext = dynamic_cast<const ExtrudedSimplicialMesh*>(mesh_.get());
      if (!ext || ext->regular_base())
        throw Error(FTK2B_UNSUPPORTED, "level sets on extruded meshes need an unstructured base");
    }
    using E = std::remove_cv_t<std::remove_pointer_t<decltype(a.pdata())>>;
    std::vector<T> conv;
    const void* p = a.pdata();
    if (!std::is_same<E, T>::value) {
      conv.assign(a.pdata(), a.pdata() + a.nelem());
      p = conv.data();
    }
    ftk2b_field_desc fd;
    std::memset(&fd, 0, sizeof(fd));
    fd.dtype = sizeof(T) == 8 ? FTK2B_F64 : FTK2B_F32;
    fd.ncomp = 1;
    fd.layout = FTK2B_LAYOUT_SEPARATE;
    fd.location = FTK2B_HOST;
    fd.comp[0] = p;
    fd.nd = (int)a.nd();
    for (int i = 0; i < fd.nd && i < 4; ++i) fd.dims[i] = a.dimf(i);
    if (md.kind == FTK2B_MESH_EXTRUDED) {
      fd.nd = 1;
      fd.dims[0] = a.nelem();
    }
    ftk2b_contour_result* r = nullptr;
    ftk2b_status st = ftk2b_contour_extract(ctx_.get(), &md, &fd, (double)pred_.threshold, pred_.sos_q, &r);
    if (st != FTK2B_OK) throw Error(st, ftk2b_last_error(ctx_.get()));
    result_.reset(r);
  }

  template <typename Array>
  void execute_cuda(const std::map<std::string, Array>& data, const std::vector<std::string>& v = {}) {
    execute(data, v);
  }

  FeatureComplex get_complex() const {
    FeatureComplex fc;
    const ftk2b_contour_result* r = result_.get();
    if (!r) return fc;
    fc.vertices.resize(r->n_features);
    fc.lambda.assign(r->lambda, r->lambda + 2 * r->n_features);
    for (uint64_t i = 0; i < r->n_features; ++i) {
      FeatureElement& el = fc.vertices[i];
      el.simplex.dimension = 1;
      for (int v = 0; v < 2; ++v) {
        el.simplex.vertices[v] = r->simplices[2 * i + v];
        el.barycentric_coords[0][v] = r->barycentric[2 * i + v];
      }
      el.track_id = r->track_id[i];
      el.scalar = r->scalar[i];
    }
    if (r->n_cells) {
      FeatureComplex::SimplexIndices c;
      c.dimension = r->cell_dim;
      c.indices.assign(r->cells, r->cells + (size_t)(r->cell_dim + 1) * r->n_cells);
      fc.connectivity.push_back(std::move(c));
    }
    return fc;
  }

 private:
  struct CtxDel {
    void operator()(ftk2b_ctx* c) const { ftk2b_ctx_destroy(c); }
  };
  struct ResDel {
    void operator()(ftk2b_contour_result* r) const { ftk2b_contour_result_free(r); }
  };
  std::shared_ptr<Mesh> mesh_;
  ContourPredicate<T> pred_;
  std::unique_ptr<ftk2b_ctx, CtxDel> ctx_;
  std::unique_ptr<ftk2b_contour_result, ResDel> result_;
};

// ---- fibers (FiberPredicate<T>, predicate.hpp:341-362)

template <typename T = double>
struct FiberPredicate {
  static constexpr int codimension = 2;
  double sos_q = 1000000.0;
  std::string var_names[2];
  T thresholds[2] = {(T)0.0, (T)0.0};
};

// SimplicialEngine<T, FiberPredicate<T>> on a regular mesh or an
// ExtrudedSimplicialMesh (per-vertex arrays): 2D+t meshes give triangle
// features joined by star edges (ftk2b_fiber_extract), 3D+t meshes triangle
// features of the 4-D mesh with the star-fan triangles of get_complex
// (ftk2b_fiber_surface_extract).
template <typename T>
class SimplicialEngine<T, FiberPredicate<T>> {
 public:
  static constexpr int m = 2;

  SimplicialEngine(std::shared_ptr<Mesh> mesh, FiberPredicate<T> pred = FiberPredicate<T>(), int device = 0)
      : mesh_(std::move(mesh)), pred_(pred) {
    ftk2b_ctx* c = nullptr;
    ftk2b_status s = ftk2b_ctx_create(device, &c);
    if (s != FTK2B_OK) throw Error(s, "ftk2b_ctx_create failed");
    ctx_.reset(c);
  }

  template <typename Array>
  void execute(const std::map<std::string, Array>& data, const std::vector<std::string>& vars = {}) {
    const std::string n0 = vars.size() >= 2 ? vars[0] : pred_.var_names[0];
    const std::string n1 = vars.size() >= 2 ? vars[1] : pred_.var_names[1];
    const Array* a[2] = {&data.at(n0), &data.at(n1)};
    ftk2b_mesh_desc md = mesh_->desc();
    using E = std::remove_cv_t<std::remove_pointer_t<decltype(a[0]->pdata())>>;
    std::vector<T> conv[2];
    ftk2b_field_desc fd;
    std::memset(&fd, 0, sizeof(fd));
    fd.dtype = sizeof(T) == 8 ? FTK2B_F64 : FTK2B_F32;
    fd.ncomp = 2;
    fd.layout = FTK2B_LAYOUT_SEPARATE;
    fd.location = FTK2B_HOST;
    for (int j = 0; j < 2; ++j) {
      fd.comp[j] = a[j]->pdata();
      if (!std::is_same<E, T>::value) {
        conv[j].assign(a[j]->pdata(), a[j]->pdata() + a[j]->nelem());
        fd.comp[j] = conv[j].data();
      }
    }
    fd.nd = (int)a[0]->nd();
    for (int i = 0; i < fd.nd && i < 4; ++i) fd.dims[i] = a[0]->dimf(i);
    const double thr[2] = {(double)pred_.thresholds[0], (double)pred_.thresholds[1]};
    cp_.reset();
    fs_.reset();
    ftk2b_status st;
    if (md.ndims == 4) {
      ftk2b_fiber_surface_result* r = nullptr;
      st = ftk2b_fiber_surface_extract(ctx_.get(), &md, &fd, thr, pred_.sos_q, &r);
      fs_.reset(r);
    } else {
      ftk2b_cp_result* r = nullptr;
      st = ftk2b_fiber_extract(ctx_.get(), &md, &fd, thr, pred_.sos_q, &r);
      cp_.reset(r);
    }
    if (st != FTK2B_OK) throw Error(st, ftk2b_last_error(ctx_.get()));
  }

  template <typename Array>
  void execute_cuda(const std::map<std::string, Array>& data, const std::vector<std::string>& v = {}) {
    execute(data, v);
  }

  FeatureComplex get_complex() const {
    FeatureComplex fc;
    uint64_t n = 0;
    const uint64_t* simp = nullptr;
    const double* lam = nullptr;
    const float* bary = nullptr;
    const uint64_t* track = nullptr;
    if (cp_) n = cp_->n_features, simp = cp_->simplices, lam = cp_->lambda, bary = cp_->barycentric,
             track = cp_->track_id;
    if (fs_) n = fs_->n_features, simp = fs_->simplices, lam = fs_->lambda, bary = fs_->barycentric,
             track = fs_->track_id;
    fc.vertices.resize(n);
    if (n) fc.lambda.assign(lam, lam + 3 * n);
    for (uint64_t i = 0; i < n; ++i) {
      FeatureElement& el = fc.vertices[i];
      el.simplex.dimension = 2;
      for (int v = 0; v < 3; ++v) {
        el.simplex.vertices[v] = simp[3 * i + v];
        el.barycentric_coords[0][v] = bary[3 * i + v];
      }
      el.track_id = track[i];
    }
    if (cp_ && cp_->n_edges) {
      FeatureComplex::SimplexIndices e;
      e.dimension = 1;
      e.indices.assign(cp_->edges, cp_->edges + 2 * cp_->n_edges);
      fc.connectivity.push_back(std::move(e));
    }
    if (fs_ && fs_->n_cells) {
      FeatureComplex::SimplexIndices c;
      c.dimension = 2;
      c.indices.assign(fs_->cells, fs_->cells + 3 * fs_->n_cells);
      fc.connectivity.push_back(std::move(c));
    }
    return fc;
  }

 private:
  struct CtxDel {
    void operator()(ftk2b_ctx* c) const { ftk2b_ctx_destroy(c); }
  };
  struct CpDel {
    void operator()(ftk2b_cp_result* r) const { ftk2b_cp_result_free(r); }
  };
  struct FsDel {
    void operator()(ftk2b_fiber_surface_result* r) const { ftk2b_fiber_surface_result_free(r); }
  };
  std::shared_ptr<Mesh> mesh_;
  FiberPredicate<T> pred_;
  std::unique_ptr<ftk2b_ctx, CtxDel> ctx_;
  std::unique_ptr<ftk2b_cp_result, CpDel> cp_;
  std::unique_ptr<ftk2b_fiber_surface_result, FsDel> fs_;
};

}  // namespace ftk2b
