// High-level feature tracker for the critical-point path, configured by the
// same YAML files as the reference's FeatureTracker
// (include/ftk2/high_level/feature_tracker.hpp, src/high_level/
// feature_tracker.cpp) and running on the B200 engine of ftk2b/engine.hpp.
//
//   reference                                     this header
//   ftk2::FeatureTracker::from_yaml(path)         ftk2b::FeatureTracker::from_yaml(path)
//   ftk2::FeatureTracker::create(config)          ftk2b::FeatureTracker::create(config)
//   tracker->execute()                            tracker->execute_with_data(arrays)
//   FeatureTrackerImpl<T>::execute_with_predicate the same flow, on the GPU
//
// What the flow does, step for step as the reference (feature_tracker.cpp:
// 255-363 and 420-560): derive the spatial dimension and the regular mesh's
// dimensions from the first array when the configuration leaves them out;
// extrude the regular spatial mesh over the timesteps of the data (the
// reference always tracks on ExtrudedSimplicialMesh(spatial, nt - 1)); pick
// the first array whose leading dimension equals the number of components as
// the multicomponent vector field, else the configured variables as separate
// arrays; record the configured attributes in slots 0..15; run the engine;
// write the feature list as text (and JSON statistics) exactly as the
// reference's write_results does.
//
// Differences, all because the reference's inputs for them are missing here:
// the data arrays are passed in (the reference's "arrays" source is the
// announced execute_with_data and its own execute() throws for it; ndarray
// YAML streams, VTU series and synthetic generators come from the
// un-vendored ndarray library and are reported as unsupported), every
// backend runs on the GPU (the reference runs its CPU engine whatever
// execution.backend says), and only critical points are tracked here.  A VTP
// file (plain XML PolyData: feature positions, star edges as lines, track id,
// scalar and attributes per point) is written when output.format is "vtp"
// and output.filename is set.
#pragma once

#include <cstdio>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "engine.hpp"
#include "tracking_config.hpp"

namespace ftk2b {

class TrackingResults {
 public:
  TrackingResults() = default;
  explicit TrackingResults(FeatureComplex c) : complex_(std::move(c)) {}
  const FeatureComplex& get_complex() const { return complex_; }
  FeatureComplex& get_complex() { return complex_; }
  size_t num_vertices() const { return complex_.vertices.size(); }

 private:
  FeatureComplex complex_;
};

template <typename T>
class FeatureTrackerImpl;

class FeatureTracker {
 public:
  static std::unique_ptr<FeatureTracker> from_yaml(const std::string& path) {
    return create(TrackingConfig::from_yaml(path));
  }
  static std::unique_ptr<FeatureTracker> create(const TrackingConfig& config);
  virtual ~FeatureTracker() = default;

  // The reference's execute(): its data sources (ndarray streams, VTU,
  // synthetic generators) are not available here; pass the arrays instead.
  TrackingResults execute() {
    throw Error(FTK2B_UNSUPPORTED,
                "data source '" + TrackingConfig::data_source_type_to_string(config_.data.source) +
                    "' needs the ndarray library; pass the arrays with execute_with_data()");
  }
  // Tracks the features of `data` (name -> Fortran-order array exposing nd(),
  // dimf(i), nelem() and pdata()), writes the configured outputs and returns
  // the complex.  Arrays of another element type are converted to the
  // configured precision first.
  template <typename Array>
  TrackingResults execute_with_data(const std::map<std::string, Array>& data);

  const TrackingConfig& get_config() const { return config_; }
  std::string get_output_path() const { return config_.output.trajectories; }

 protected:
  explicit FeatureTracker(const TrackingConfig& c) : config_(c) {}
  TrackingConfig config_;
};

namespace detail {

// A Fortran-order array of the configured precision (the ndarray shape the
// engine reads), filled from any array type.
template <typename T>
struct HostArray {
  std::vector<size_t> dims;
  std::vector<T> buf;
  size_t nd() const { return dims.size(); }
  size_t dimf(size_t i) const { return i < dims.size() ? dims[i] : 1; }
  size_t nelem() const { return buf.size(); }
  const T* pdata() const { return buf.data(); }
};

}  // namespace detail

template <typename T>
class FeatureTrackerImpl : public FeatureTracker {
 public:
  explicit FeatureTrackerImpl(const TrackingConfig& c) : FeatureTracker(c) {}

  template <typename Array>
  TrackingResults run(const std::map<std::string, Array>& raw) {
    std::map<std::string, detail::HostArray<T>> data;
    for (const auto& kv : raw) {
      detail::HostArray<T> a;
      for (size_t i = 0; i < kv.second.nd(); ++i) a.dims.push_back(kv.second.dimf(i));
      const auto* p = kv.second.pdata();
      a.buf.assign(p, p + kv.second.nelem());
      data.emplace(kv.first, std::move(a));
    }
    if (data.empty()) throw Error(FTK2B_INVALID_ARG, "Cannot infer dimension from empty data");
    if (config_.dimension == 0) config_.dimension = infer_dimension(data);
    if (config_.feature != FeatureType::CriticalPoints)
      throw Error(FTK2B_UNSUPPORTED, "feature '" + TrackingConfig::feature_type_to_string(config_.feature) +
                                         "' is not on the B200 path (critical points only)");
    if (config_.input.type == InputType::Scalar)
      throw Error(FTK2B_UNSUPPORTED, "Gradient computation from scalar field not yet implemented.");
    if (config_.input.type != InputType::Vector && config_.input.type != InputType::GradientVector)
      throw Error(FTK2B_UNSUPPORTED, "input type '" + TrackingConfig::input_type_to_string(config_.input.type) +
                                         "' does not feed critical points");
    // The reference's unstructured route (read_vtu, feature_tracker.cpp:46-57)
    // feeds the multicomponent gather physical vertex coordinates as array
    // indices (engine.hpp:1107-1122 with mesh.hpp:714-720); the meshes it
    // serves are loaded with ftk2b::read_vtu (vtk.hpp) and run through
    // SimplicialEngine with per-vertex arrays instead.
    if (config_.mesh.type != MeshType::Regular)
      throw Error(FTK2B_UNSUPPORTED, "mesh type '" + TrackingConfig::mesh_type_to_string(config_.mesh.type) +
                                         "' is not on the tracker's GPU route; load it with read_vtu and run "
                                         "SimplicialEngine on ExtrudedSimplicialMesh");
    // regular spatial mesh: configured dims, or the first array's shape
    const detail::HostArray<T>& first = data.begin()->second;
    std::vector<uint64_t> dims = config_.mesh.dimensions;
    if (dims.empty()) {
      const int nd = (int)first.nd();
      const int start = (first.dimf(0) >= 1 && first.dimf(0) <= 3) ? 1 : 0;
      const int end = (nd - start >= 3) ? nd - 1 : nd;
      for (int d = start; d < end; ++d) dims.push_back(first.dimf(d));
    }
    last_dims_ = dims;
    uint64_t nt = 1;
    if (first.nd() >= 4) nt = first.dimf(first.nd() - 1);
    auto spatial = std::make_shared<RegularSimplicialMesh>(dims);
    auto mesh = std::make_shared<ExtrudedSimplicialMesh>(spatial, nt - 1);
    TrackingResults res;
    if (config_.dimension == 2) res = execute_with_predicate<CriticalPointPredicate<2, T>>(mesh, data);
    else if (config_.dimension == 3) res = execute_with_predicate<CriticalPointPredicate<3, T>>(mesh, data);
    else throw Error(FTK2B_INVALID_ARG, "Invalid dimension for critical points");
    write_results(res);
    return res;
  }

 private:
  template <typename A>
  static int infer_dimension(const std::map<std::string, A>& data) {
    const A& f = data.begin()->second;
    const int nd = (int)f.nd();
    const bool comps = nd >= 3 && f.dimf(0) >= 1 && f.dimf(0) <= 3;
    const int sd = comps ? nd - 2 : nd - 1;
    if (sd < 2 || sd > 3)
      throw Error(FTK2B_INVALID_ARG, "Inferred spatial dimension must be 2D or 3D, got " + std::to_string(sd) + "D");
    return sd;
  }

  template <typename Pred, typename A>
  TrackingResults execute_with_predicate(std::shared_ptr<Mesh> mesh, const std::map<std::string, A>& data) {
    Pred pred;
    pred.use_multicomponent = true;
    bool found = false;
    for (const auto& kv : data)
      if (kv.second.nd() >= 3 && (int)kv.second.dimf(0) == Pred::codimension) {
        pred.vector_var_name = kv.first;
        found = true;
        break;
      }
    if (!found) {
      pred.use_multicomponent = false;
      if ((int)config_.input.variables.size() >= Pred::codimension)
        for (int i = 0; i < Pred::codimension; ++i) pred.var_names[i] = config_.input.variables[i];
    }
    for (const auto& ac : config_.output.attributes) {
      if (data.find(ac.source) == data.end()) continue;
      AttributeSpec spec;
      spec.name = ac.name;
      spec.source = ac.source;
      spec.type = ac.type;
      spec.component = ac.component;
      spec.slot = (int)pred.attributes.size();
      if (spec.slot >= 16) break;
      pred.attributes.push_back(spec);
    }
    SimplicialEngine<T, Pred> engine(mesh, pred);
    engine.execute(data);
    return TrackingResults(engine.get_complex());
  }

  // write_results of the reference (feature_tracker.cpp:541-611), plus VTP
  void write_results(const TrackingResults& results) const {
    const FeatureComplex& c = results.get_complex();
    const std::vector<AttributeConfig>& attrs = config_.output.attributes;
    if (!config_.output.trajectories.empty()) {
      std::ofstream f(config_.output.trajectories);
      if (!f) throw Error(FTK2B_INVALID_ARG, "Cannot open output file: " + config_.output.trajectories);
      f << "# FTK2 Feature Complex\n";
      f << "# Feature: " << TrackingConfig::feature_type_to_string(config_.feature) << "\n";
      f << "# Num vertices: " << c.vertices.size() << "\n";
      if (!attrs.empty()) {
        f << "# Attributes: ";
        for (size_t i = 0; i < attrs.size(); ++i) {
          f << attrs[i].name;
          if (i < attrs.size() - 1) f << ", ";
        }
        f << "\n";
      }
      f << "\n";
      f << "# Feature Elements:\n";
      for (size_t i = 0; i < c.vertices.size(); ++i) {
        const FeatureElement& e = c.vertices[i];
        f << i << ": track_id=" << e.track_id << " type=" << e.type << " scalar=" << e.scalar;
        if (!attrs.empty()) {
          f << " attrs=[";
          for (size_t j = 0; j < attrs.size(); ++j)
            if (j < 16) {
              f << e.attributes[j];
              if (j < attrs.size() - 1) f << ", ";
            }
          f << "]";
        }
        f << "\n";
      }
    }
    if (!config_.output.statistics.empty()) {
      std::ofstream f(config_.output.statistics);
      if (!f) throw Error(FTK2B_INVALID_ARG, "Cannot open statistics file: " + config_.output.statistics);
      f << "{\n";
      f << "  \"feature\": \"" << TrackingConfig::feature_type_to_string(config_.feature) << "\",\n";
      f << "  \"dimension\": " << config_.dimension << ",\n";
      f << "  \"num_vertices\": " << c.vertices.size() << ",\n";
      f << "  \"precision\": \"" << (std::is_same<T, double>::value ? "double" : "float") << "\",\n";
      f << "  \"backend\": \"" << TrackingConfig::backend_to_string(config_.execution.backend) << "\"\n";
      f << "}\n";
    }
    if (TrackingConfig::lower(config_.output.format) == "vtp" && !config_.output.filename.empty())
      write_vtp(c, config_.output.filename);
  }

  // Feature positions = sum_i lambda_i * grid coordinates of vertex i (the
  // double barycentrics), spaced and offset by mesh.spacing / mesh.origin;
  // time as the last coordinate of 2D features, a point-data array in 3D.
  void write_vtp(const FeatureComplex& c, const std::string& path) const {
    std::ofstream f(path);
    if (!f) throw Error(FTK2B_INVALID_ARG, "Cannot open output file: " + path);
    const int sd = config_.dimension;
    const size_t n = c.vertices.size();
    const int k = n ? c.vertices[0].simplex.dimension + 1 : 0;
    uint64_t S = 0, mul = 1;
    for (uint64_t d : last_dims_) {
      S += d * mul;
      mul *= d;
    }
    std::vector<double> pos(3 * n, 0.0), tim(n, 0.0);
    for (size_t i = 0; i < n; ++i)
      for (int v = 0; v < k; ++v) {
        const uint64_t vid = c.vertices[i].simplex.vertices[v];
        const double lam = c.lambda.empty() ? (double)c.vertices[i].barycentric_coords[0][v] : c.lambda[i * k + v];
        uint64_t s = S ? vid % S : vid, t = S ? vid / S : 0;
        for (int d = 0; d < sd && d < (int)last_dims_.size(); ++d) {
          const double sp = d < (int)config_.mesh.spacing.size() ? config_.mesh.spacing[d] : 1.0;
          const double og = d < (int)config_.mesh.origin.size() ? config_.mesh.origin[d] : 0.0;
          pos[3 * i + d] += lam * (og + sp * (double)(s % last_dims_[d]));
          s /= last_dims_[d];
        }
        tim[i] += lam * (double)t;
      }
    if (sd == 2)
      for (size_t i = 0; i < n; ++i) pos[3 * i + 2] = tim[i];
    std::vector<uint32_t> lines;
    for (const auto& cn : c.connectivity)
      if (cn.dimension == 1) lines = cn.indices;
    f << "<?xml version=\"1.0\"?>\n";
    f << "<VTKFile type=\"PolyData\" version=\"1.0\" byte_order=\"LittleEndian\">\n";
    f << "  <PolyData>\n";
    f << "    <Piece NumberOfPoints=\"" << n << "\" NumberOfVerts=\"0\" NumberOfLines=\"" << lines.size() / 2
      << "\" NumberOfStrips=\"0\" NumberOfPolys=\"0\">\n";
    f << "      <Points>\n        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n";
    char b[96];
    for (size_t i = 0; i < n; ++i) {
      std::snprintf(b, sizeof(b), "          %.17g %.17g %.17g\n", pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
      f << b;
    }
    f << "        </DataArray>\n      </Points>\n";
    f << "      <PointData>\n";
    f << "        <DataArray type=\"UInt64\" Name=\"track_id\" format=\"ascii\">\n";
    for (size_t i = 0; i < n; ++i) f << "          " << c.vertices[i].track_id << "\n";
    f << "        </DataArray>\n";
    f << "        <DataArray type=\"Float32\" Name=\"scalar\" format=\"ascii\">\n";
    for (size_t i = 0; i < n; ++i) f << "          " << c.vertices[i].scalar << "\n";
    f << "        </DataArray>\n";
    if (sd == 3) {
      f << "        <DataArray type=\"Float64\" Name=\"time\" format=\"ascii\">\n";
      for (size_t i = 0; i < n; ++i) {
        std::snprintf(b, sizeof(b), "          %.17g\n", tim[i]);
        f << b;
      }
      f << "        </DataArray>\n";
    }
    const auto& attrs = config_.output.attributes;
    for (size_t a = 0; a < attrs.size() && a < 16; ++a) {
      f << "        <DataArray type=\"Float32\" Name=\"" << attrs[a].name << "\" format=\"ascii\">\n";
      for (size_t i = 0; i < n; ++i) f << "          " << c.vertices[i].attributes[a] << "\n";
      f << "        </DataArray>\n";
    }
    f << "      </PointData>\n";
    f << "      <Lines>\n        <DataArray type=\"Int64\" Name=\"connectivity\" format=\"ascii\">\n";
    for (size_t e = 0; e + 1 < lines.size(); e += 2) f << "          " << lines[e] << " " << lines[e + 1] << "\n";
    f << "        </DataArray>\n        <DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\">\n";
    for (size_t e = 0; e < lines.size() / 2; ++e) f << "          " << 2 * (e + 1) << "\n";
    f << "        </DataArray>\n      </Lines>\n";
    f << "    </Piece>\n  </PolyData>\n</VTKFile>\n";
  }

 public:
  std::vector<uint64_t> last_dims_;  // spatial dims of the last run's mesh
};

inline std::unique_ptr<FeatureTracker> FeatureTracker::create(const TrackingConfig& config) {
  if (config.execution.precision == Precision::Double)
    return std::unique_ptr<FeatureTracker>(new FeatureTrackerImpl<double>(config));
  return std::unique_ptr<FeatureTracker>(new FeatureTrackerImpl<float>(config));
}

template <typename Array>
TrackingResults FeatureTracker::execute_with_data(const std::map<std::string, Array>& data) {
  if (config_.execution.precision == Precision::Double)
    return static_cast<FeatureTrackerImpl<double>*>(this)->run(data);
  return static_cast<FeatureTrackerImpl<float>*>(this)->run(data);
}

}  // namespace ftk2b
