// Tracking configuration of the high-level caller, read from the same YAML
// files as the reference's TrackingConfig (include/ftk2/high_level/
// tracking_config.hpp, src/high_level/tracking_config.cpp): same keys, same
// enum spellings and aliases, same defaults and validation.  The reference
// parses with yaml-cpp; this header carries a small reader of the YAML subset
// those files use (block mappings and sequences by indentation, flow
// sequences `[a, b]`, quoted and plain scalars, `~` / `null`, comments), so it
// has no dependency beyond the C++ standard library.
#pragma once

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <functional>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace ftk2b {

// ---------------------------------------------------------------------------
// YAML subset

namespace yaml {

class Node {
 public:
  enum Kind { Null, Scalar, Sequence, Map };
  Node() = default;
  static Node scalar(const std::string& v) {
    Node n;
    n.kind_ = Scalar;
    n.value_ = v;
    return n;
  }
  Kind kind() const { return kind_; }
  bool defined() const { return kind_ != Null; }
  explicit operator bool() const { return defined(); }
  bool IsScalar() const { return kind_ == Scalar; }
  bool IsSequence() const { return kind_ == Sequence; }
  bool IsMap() const { return kind_ == Map; }
  // missing keys give a null node (like yaml-cpp's operator[] on a const node)
  const Node& operator[](const std::string& key) const {
    static const Node none;
    if (kind_ != Map) return none;
    for (const auto& kv : map_)
      if (kv.first == key) return kv.second;
    return none;
  }
  const std::vector<Node>& items() const { return seq_; }
  const std::vector<std::pair<std::string, Node>>& entries() const { return map_; }
  const std::string& str() const {
    if (kind_ != Scalar) throw std::invalid_argument("YAML: expected a scalar");
    return value_;
  }
  std::string as_string() const { return str(); }
  int as_int() const { return std::stoi(str()); }
  double as_double() const { return std::stod(str()); }
  uint64_t as_u64() const { return std::stoull(str()); }
  std::vector<std::string> as_strings() const {
    std::vector<std::string> v;
    if (kind_ == Scalar) {
      v.push_back(value_);
      return v;
    }
    for (const Node& n : seq_) v.push_back(n.str());
    return v;
  }
  std::map<std::string, std::string> as_string_map() const {
    std::map<std::string, std::string> m;
    for (const auto& kv : map_) m[kv.first] = kv.second.str();
    return m;
  }

  Kind kind_ = Null;
  std::string value_;
  std::vector<Node> seq_;
  std::vector<std::pair<std::string, Node>> map_;
};

namespace detail {

struct Line {
  int indent;
  std::string text;  // without indentation and comment
  int number;
};

inline std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

// a '#' starts a comment outside quotes when it opens the text or follows blank
inline std::string strip_comment(const std::string& s) {
  char q = 0;
  for (size_t i = 0; i < s.size(); ++i) {
    const char c = s[i];
    if (q) {
      if (c == q) q = 0;
    } else if (c == '"' || c == '\'') {
      q = c;
    } else if (c == '#' && (i == 0 || std::isspace((unsigned char)s[i - 1]))) {
      return s.substr(0, i);
    }
  }
  return s;
}

inline Node plain(const std::string& raw) {
  const std::string v = trim(raw);
  if (v.empty() || v == "~" || v == "null" || v == "Null" || v == "NULL") return Node();
  if (v.size() >= 2 && ((v.front() == '"' && v.back() == '"') || (v.front() == '\'' && v.back() == '\'')))
    return Node::scalar(v.substr(1, v.size() - 2));
  if (v.front() == '[') {
    if (v.back() != ']') throw std::invalid_argument("YAML: unterminated flow sequence: " + v);
    Node n;
    n.kind_ = Node::Sequence;
    const std::string body = trim(v.substr(1, v.size() - 2));
    if (body.empty()) return n;
    std::string cur;
    char q = 0;
    for (char c : body) {
      if (q) {
        if (c == q) q = 0;
        cur += c;
      } else if (c == '"' || c == '\'') {
        q = c;
        cur += c;
      } else if (c == ',') {
        n.seq_.push_back(plain(cur));
        cur.clear();
      } else {
        cur += c;
      }
    }
    n.seq_.push_back(plain(cur));
    return n;
  }
  return Node::scalar(v);
}

// position of the ':' that separates a mapping key (followed by blank or end)
inline size_t key_colon(const std::string& t) {
  char q = 0;
  for (size_t i = 0; i < t.size(); ++i) {
    const char c = t[i];
    if (q) {
      if (c == q) q = 0;
    } else if (c == '"' || c == '\'') {
      q = c;
    } else if (c == ':' && (i + 1 == t.size() || std::isspace((unsigned char)t[i + 1]))) {
      return i;
    } else if (c == '[' || c == '{') {
      return std::string::npos;
    }
  }
  return std::string::npos;
}

class Parser {
 public:
  explicit Parser(const std::string& text) {
    std::istringstream in(text);
    std::string raw;
    int no = 0;
    while (std::getline(in, raw)) {
      ++no;
      if (!raw.empty() && raw.back() == '\r') raw.pop_back();
      if (trim(raw) == "---") continue;
      const std::string s = strip_comment(raw);
      if (trim(s).empty()) continue;
      int ind = 0;
      while (ind < (int)s.size() && s[ind] == ' ') ++ind;
      if (ind < (int)s.size() && s[ind] == '\t') throw std::invalid_argument("YAML: tab indentation");
      lines_.push_back({ind, trim(s), no});
    }
  }
  Node parse() {
    if (lines_.empty()) return Node();
    Node n = block(lines_[0].indent);
    if (pos_ != lines_.size())
      throw std::invalid_argument("YAML: unexpected indentation at line " + std::to_string(lines_[pos_].number));
    return n;
  }

 private:
  bool is_item(const std::string& t) const { return t == "-" || (t.size() > 1 && t[0] == '-' && t[1] == ' '); }

  // a block at exactly `ind`: a sequence if it starts with "- ", else a map
  Node block(int ind) {
    if (pos_ < lines_.size() && is_item(lines_[pos_].text)) return sequence(ind);
    return mapping(ind);
  }

  Node sequence(int ind) {
    Node n;
    n.kind_ = Node::Sequence;
    while (pos_ < lines_.size() && lines_[pos_].indent == ind && is_item(lines_[pos_].text)) {
      Line l = lines_[pos_];
      const std::string rest = l.text.size() > 1 ? trim(l.text.substr(1)) : std::string();
      if (rest.empty()) {
        ++pos_;
        if (pos_ < lines_.size() && lines_[pos_].indent > ind) n.seq_.push_back(block(lines_[pos_].indent));
        else n.seq_.push_back(Node());
        continue;
      }
      if (key_colon(rest) != std::string::npos) {
        // "- key: value" opens a mapping whose keys sit at the item's text column
        const int col = ind + (int)(l.text.size() - rest.size());
        lines_[pos_].indent = col;
        lines_[pos_].text = rest;
        n.seq_.push_back(mapping(col));
        continue;
      }
      ++pos_;
      n.seq_.push_back(plain(rest));
    }
    return n;
  }

  Node mapping(int ind) {
    Node n;
    n.kind_ = Node::Map;
    while (pos_ < lines_.size() && lines_[pos_].indent == ind && !is_item(lines_[pos_].text)) {
      const Line l = lines_[pos_];
      const size_t c = key_colon(l.text);
      if (c == std::string::npos) throw std::invalid_argument("YAML: expected 'key: value' at line " + std::to_string(l.number));
      std::string key = trim(l.text.substr(0, c));
      if (key.size() >= 2 && (key.front() == '"' || key.front() == '\'')) key = key.substr(1, key.size() - 2);
      const std::string rest = trim(l.text.substr(c + 1));
      ++pos_;
      Node value;
      if (!rest.empty()) {
        value = plain(rest);
      } else if (pos_ < lines_.size() && (lines_[pos_].indent > ind ||
                                          (lines_[pos_].indent == ind && is_item(lines_[pos_].text)))) {
        value = block(lines_[pos_].indent);
      }
      n.map_.push_back({key, value});
    }
    return n;
  }

  std::vector<Line> lines_;
  size_t pos_ = 0;
};

}  // namespace detail

inline Node Load(const std::string& text) { return detail::Parser(text).parse(); }

inline Node LoadFile(const std::string& path) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("cannot open " + path);
  std::stringstream ss;
  ss << in.rdbuf();
  return Load(ss.str());
}

}  // namespace yaml

// ---------------------------------------------------------------------------
// configuration (the reference's types and fields)

enum class FeatureType {
  CriticalPoints,
  Levelsets,
  Fibers,
  TDGLVortex,
  ApproxParallelVectors,
  SujadiHaimes,
  LevyDeganiSeginer
};
enum class InputType { Scalar, Vector, GradientVector, MultiScalar, Complex, PairedVectors };
enum class DataSourceType { Stream, Arrays, VTU, Synthetic };
enum class Backend { CPU, CUDA, MPI };
enum class Precision { Float, Double };
enum class MeshType { Regular, Unstructured, Extruded };
enum class OutputType { Discrete, Traced, Sliced, Intercepted };

struct InputConfig {
  InputType type = InputType::Scalar;
  std::vector<std::string> variables;
  std::string field_type = "gradient";
  std::string scalar_field;
  std::map<std::string, std::string> field_map;
  std::string vector_u, vector_v;
  void validate() const {
    if (variables.empty()) throw std::invalid_argument("Input variables cannot be empty");
    if (field_type != "gradient" && field_type != "flow")
      throw std::invalid_argument("field_type must be 'gradient' or 'flow'");
  }
};

struct DataConfig {
  DataSourceType source = DataSourceType::Arrays;
  std::string stream_yaml;
  yaml::Node inline_stream;
  std::string vtu_pattern;
  std::string generator;
  std::map<std::string, double> generator_params;
  void validate() const {
    if (source == DataSourceType::Stream && stream_yaml.empty() && !inline_stream)
      throw std::invalid_argument("stream_yaml or inline stream config required for Stream source");
    if (source == DataSourceType::VTU && vtu_pattern.empty())
      throw std::invalid_argument("vtu_pattern required for VTU source");
    if (source == DataSourceType::Synthetic && generator.empty())
      throw std::invalid_argument("generator required for Synthetic source");
  }
};

struct MeshConfig {
  MeshType type = MeshType::Regular;
  std::vector<uint64_t> dimensions;
  std::vector<double> spacing = {1.0, 1.0, 1.0};
  std::vector<double> origin = {0.0, 0.0, 0.0};
  std::string mesh_file;
  void validate() const {
    if (type == MeshType::Regular && !dimensions.empty() && (dimensions.size() < 2 || dimensions.size() > 3))
      throw std::invalid_argument("dimensions must be 2D or 3D");
    if (type == MeshType::Unstructured && mesh_file.empty())
      throw std::invalid_argument("mesh_file required for Unstructured mesh");
  }
};

struct ExecutionConfig {
  Backend backend = Backend::CPU;
  Precision precision = Precision::Double;
  int num_threads = -1;
  void validate() const {}
};

struct AttributeConfig {
  std::string name;
  std::string source;
  std::string type = "scalar";
  int component = -1;
  void validate() const {
    if (name.empty()) throw std::invalid_argument("Attribute name cannot be empty");
    if (source.empty()) throw std::invalid_argument("Attribute source cannot be empty");
  }
};

struct OutputConfig {
  OutputType type = OutputType::Traced;
  std::string filename;
  std::string trajectories;
  std::string format = "auto";
  std::string statistics;
  std::vector<AttributeConfig> attributes;
  void validate() const {
    if (filename.empty() && trajectories.empty()) throw std::invalid_argument("Output filename cannot be empty");
    for (const auto& a : attributes) a.validate();
  }
};

struct FeatureOptions {
  std::string line_type = "ridge";
  std::string integrator = "rk4";
  int num_steps = 1000;
  double dt = 0.01;
  std::map<std::string, std::string> seeding;
  int min_winding = 1;
  double threshold = 0.0;
  double w2_threshold = 0.1;
  bool auto_compute_vorticity = false;
  std::string filter_mode = "absolute";
  double filter_percentile = 0.1;
};

class TrackingConfig {
 public:
  FeatureType feature = FeatureType::CriticalPoints;
  int dimension = 0;
  InputConfig input;
  DataConfig data;
  MeshConfig mesh;
  ExecutionConfig execution;
  OutputConfig output;
  FeatureOptions options;

  void validate() const {
    if (dimension != 0 && dimension != 2 && dimension != 3)
      throw std::invalid_argument("dimension must be 0 (auto-derive), 2, or 3");
    input.validate();
    data.validate();
    mesh.validate();
    execution.validate();
    output.validate();
  }

  static std::string lower(std::string s) {
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    return s;
  }

  static FeatureType parse_feature_type(const std::string& str) {
    const std::string l = lower(str);
    if (l == "critical_points" || l == "cp") return FeatureType::CriticalPoints;
    if (l == "levelsets" || l == "contour" || l == "iso") return FeatureType::Levelsets;
    if (l == "fibers") return FeatureType::Fibers;
    if (l == "tdgl_vortex" || l == "tdgl") return FeatureType::TDGLVortex;
    if (l == "approx_parallel_vectors" || l == "approx_pv" || l == "apv") return FeatureType::ApproxParallelVectors;
    if (l == "sujudi_haimes" || l == "sujudi-haimes" || l == "sh") return FeatureType::SujadiHaimes;
    if (l == "levy_degani_seginer" || l == "levy-degani-seginer" || l == "lds") return FeatureType::LevyDeganiSeginer;
    throw std::invalid_argument("Unknown feature type: " + str);
  }
  static std::string feature_type_to_string(FeatureType t) {
    switch (t) {
      case FeatureType::CriticalPoints: return "critical_points";
      case FeatureType::Levelsets: return "levelsets";
      case FeatureType::Fibers: return "fibers";
      case FeatureType::TDGLVortex: return "tdgl_vortex";
      case FeatureType::ApproxParallelVectors: return "approx_parallel_vectors";
      case FeatureType::SujadiHaimes: return "sujudi_haimes";
      case FeatureType::LevyDeganiSeginer: return "levy_degani_seginer";
    }
    return "unknown";
  }
  static InputType parse_input_type(const std::string& str) {
    const std::string l = lower(str);
    if (l == "scalar") return InputType::Scalar;
    if (l == "vector") return InputType::Vector;
    if (l == "gradient_vector") return InputType::GradientVector;
    if (l == "multi_scalar") return InputType::MultiScalar;
    if (l == "complex") return InputType::Complex;
    if (l == "paired_vectors" || l == "paired") return InputType::PairedVectors;
    throw std::invalid_argument("Unknown input type: " + str);
  }
  static std::string input_type_to_string(InputType t) {
    switch (t) {
      case InputType::Scalar: return "scalar";
      case InputType::Vector: return "vector";
      case InputType::GradientVector: return "gradient_vector";
      case InputType::MultiScalar: return "multi_scalar";
      case InputType::Complex: return "complex";
      case InputType::PairedVectors: return "paired_vectors";
    }
    return "unknown";
  }
  static DataSourceType parse_data_source_type(const std::string& str) {
    const std::string l = lower(str);
    if (l == "stream") return DataSourceType::Stream;
    if (l == "arrays") return DataSourceType::Arrays;
    if (l == "vtu") return DataSourceType::VTU;
    if (l == "synthetic") return DataSourceType::Synthetic;
    throw std::invalid_argument("Unknown data source type: " + str);
  }
  static std::string data_source_type_to_string(DataSourceType t) {
    switch (t) {
      case DataSourceType::Stream: return "stream";
      case DataSourceType::Arrays: return "arrays";
      case DataSourceType::VTU: return "vtu";
      case DataSourceType::Synthetic: return "synthetic";
    }
    return "unknown";
  }
  static Backend parse_backend(const std::string& str) {
    const std::string l = lower(str);
    if (l == "cpu") return Backend::CPU;
    if (l == "cuda" || l == "gpu") return Backend::CUDA;
    if (l == "mpi") return Backend::MPI;
    throw std::invalid_argument("Unknown backend: " + str);
  }
  static std::string backend_to_string(Backend b) {
    switch (b) {
      case Backend::CPU: return "cpu";
      case Backend::CUDA: return "cuda";
      case Backend::MPI: return "mpi";
    }
    return "unknown";
  }
  static Precision parse_precision(const std::string& str) {
    const std::string l = lower(str);
    if (l == "float" || l == "single") return Precision::Float;
    if (l == "double") return Precision::Double;
    throw std::invalid_argument("Unknown precision: " + str);
  }
  static std::string precision_to_string(Precision p) { return p == Precision::Float ? "float" : "double"; }
  static MeshType parse_mesh_type(const std::string& str) {
    const std::string l = lower(str);
    if (l == "regular") return MeshType::Regular;
    if (l == "unstructured") return MeshType::Unstructured;
    if (l == "extruded") return MeshType::Extruded;
    throw std::invalid_argument("Unknown mesh type: " + str);
  }
  static std::string mesh_type_to_string(MeshType t) {
    switch (t) {
      case MeshType::Regular: return "regular";
      case MeshType::Unstructured: return "unstructured";
      case MeshType::Extruded: return "extruded";
    }
    return "unknown";
  }
  static OutputType parse_output_type(const std::string& str) {
    const std::string l = lower(str);
    if (l == "discrete") return OutputType::Discrete;
    if (l == "traced") return OutputType::Traced;
    if (l == "sliced") return OutputType::Sliced;
    if (l == "intercepted") return OutputType::Intercepted;
    throw std::invalid_argument("Unknown output type: " + str);
  }
  static std::string output_type_to_string(OutputType t) {
    switch (t) {
      case OutputType::Discrete: return "discrete";
      case OutputType::Traced: return "traced";
      case OutputType::Sliced: return "sliced";
      case OutputType::Intercepted: return "intercepted";
    }
    return "unknown";
  }

  // the keys the reference reads (tracking_config.cpp:167-390)
  static TrackingConfig from_yaml_node(const yaml::Node& node) {
    TrackingConfig c;
    if (node["feature"]) c.feature = parse_feature_type(node["feature"].str());
    if (node["dimension"]) c.dimension = node["dimension"].as_int();
    if (const yaml::Node& in = node["input"]) {
      if (in["type"]) c.input.type = parse_input_type(in["type"].str());
      if (in["variables"]) c.input.variables = in["variables"].as_strings();
      if (in["field_type"]) c.input.field_type = in["field_type"].str();
      if (in["scalar_field"]) c.input.scalar_field = in["scalar_field"].str();
      if (in["field_map"]) c.input.field_map = in["field_map"].as_string_map();
      if (in["vector_u"]) c.input.vector_u = in["vector_u"].str();
      if (in["vector_v"]) c.input.vector_v = in["vector_v"].str();
    }
    if (const yaml::Node& d = node["data"]) {
      if (d["source"]) c.data.source = parse_data_source_type(d["source"].str());
      if (d["stream_yaml"]) c.data.stream_yaml = d["stream_yaml"].str();
      else if (d["stream_config"]) c.data.stream_yaml = d["stream_config"].str();
      if (d["stream"]) c.data.inline_stream = d["stream"];
      if (d["vtu_pattern"]) c.data.vtu_pattern = d["vtu_pattern"].str();
      if (d["generator"]) c.data.generator = d["generator"].str();
      if (d["generator_params"])
        for (const auto& kv : d["generator_params"].entries()) c.data.generator_params[kv.first] = kv.second.as_double();
    }
    if (const yaml::Node& m = node["mesh"]) {
      if (m["type"]) c.mesh.type = parse_mesh_type(m["type"].str());
      if (m["dimensions"]) {
        c.mesh.dimensions.clear();
        for (const auto& v : m["dimensions"].items()) c.mesh.dimensions.push_back(v.as_u64());
      }
      if (m["spacing"]) {
        c.mesh.spacing.clear();
        for (const auto& v : m["spacing"].items()) c.mesh.spacing.push_back(v.as_double());
      }
      if (m["origin"]) {
        c.mesh.origin.clear();
        for (const auto& v : m["origin"].items()) c.mesh.origin.push_back(v.as_double());
      }
      if (m["mesh_file"]) c.mesh.mesh_file = m["mesh_file"].str();
    }
    if (const yaml::Node& e = node["execution"]) {
      if (e["backend"]) c.execution.backend = parse_backend(e["backend"].str());
      if (e["precision"]) c.execution.precision = parse_precision(e["precision"].str());
      if (e["threads"]) c.execution.num_threads = e["threads"].as_int();
    }
    if (const yaml::Node& o = node["output"]) {
      if (o["filename"]) c.output.filename = o["filename"].str();
      if (o["trajectories"]) c.output.trajectories = o["trajectories"].str();
      if (o["statistics"]) c.output.statistics = o["statistics"].str();
      if (o["format"]) c.output.format = o["format"].str();
      if (o["type"]) c.output.type = parse_output_type(o["type"].str());
      if (o["attributes"].IsSequence())
        for (const yaml::Node& a : o["attributes"].items()) {
          AttributeConfig ac;
          if (a.IsScalar()) {
            ac.name = a.str();
            ac.source = ac.name;
          } else if (a.IsMap()) {
            if (a["name"]) ac.name = a["name"].str();
            if (a["source"]) ac.source = a["source"].str();
            else if (!ac.name.empty()) ac.source = ac.name;
            if (a["type"]) ac.type = a["type"].str();
            if (a["component"]) ac.component = a["component"].as_int();
          }
          c.output.attributes.push_back(ac);
        }
    }
    if (const yaml::Node& op = node["options"]) {
      if (op["line_type"]) c.options.line_type = op["line_type"].str();
      if (op["integrator"]) c.options.integrator = op["integrator"].str();
      if (op["num_steps"]) c.options.num_steps = op["num_steps"].as_int();
      if (op["dt"]) c.options.dt = op["dt"].as_double();
      if (op["min_winding"]) c.options.min_winding = op["min_winding"].as_int();
      if (op["threshold"]) c.options.threshold = op["threshold"].as_double();
      if (op["seeding"]) c.options.seeding = op["seeding"].as_string_map();
      if (op["w2_threshold"]) c.options.w2_threshold = op["w2_threshold"].as_double();
      if (op["auto_compute_vorticity"])
        c.options.auto_compute_vorticity = lower(op["auto_compute_vorticity"].str()) == "true";
      if (op["filter_mode"]) c.options.filter_mode = op["filter_mode"].str();
      if (op["filter_percentile"]) c.options.filter_percentile = op["filter_percentile"].as_double();
    }
    c.validate();
    return c;
  }

  // The reference's to_yaml layout (tracking_config.cpp:416-488, emitted the
  // way yaml-cpp writes block style: two-space indentation, sequences as
  // "- item" lines, a missing inline stream as "~").
  std::string to_yaml_string() const {
    std::ostringstream o;
    auto num = [](double v) {
      char b[64];
      std::snprintf(b, sizeof(b), "%.17g", v);
      return std::string(b);
    };
    auto seq = [&](const std::string& ind, const std::string& key, const std::vector<std::string>& v) {
      if (v.empty()) {
        o << ind << key << ": []\n";
        return;
      }
      o << ind << key << ":\n";
      for (const auto& x : v) o << ind << "  - " << x << "\n";
    };
    std::function<void(const yaml::Node&, const std::string&)> emit_block;
    emit_block = [&](const yaml::Node& n, const std::string& ind) {
      if (n.IsMap()) {
        for (const auto& kv : n.entries()) {
          if (kv.second.IsScalar()) o << ind << kv.first << ": " << kv.second.str() << "\n";
          else if (!kv.second.defined()) o << ind << kv.first << ": ~\n";
          else {
            o << ind << kv.first << ":\n";
            emit_block(kv.second, ind + "  ");
          }
        }
      } else if (n.IsSequence()) {
        for (const auto& it : n.items()) {
          if (it.IsScalar()) o << ind << "- " << it.str() << "\n";
          else {
            o << ind << "-\n";
            emit_block(it, ind + "  ");
          }
        }
      }
    };
    o << "tracking:\n";
    o << "  feature: " << feature_type_to_string(feature) << "\n";
    o << "  dimension: " << dimension << "\n";
    o << "  input:\n";
    o << "    type: " << input_type_to_string(input.type) << "\n";
    seq("    ", "variables", input.variables);
    o << "    field_type: " << input.field_type << "\n";
    if (!input.scalar_field.empty()) o << "    scalar_field: " << input.scalar_field << "\n";
    if (!input.field_map.empty()) {
      o << "    field_map:\n";
      for (const auto& kv : input.field_map) o << "      " << kv.first << ": " << kv.second << "\n";
    }
    o << "  data:\n";
    o << "    source: " << data_source_type_to_string(data.source) << "\n";
    if (!data.stream_yaml.empty()) o << "    stream_config: " << data.stream_yaml << "\n";
    if (data.inline_stream.IsMap() || data.inline_stream.IsSequence()) {
      o << "    stream:\n";
      emit_block(data.inline_stream, "      ");
    } else if (data.inline_stream.IsScalar()) {
      o << "    stream: " << data.inline_stream.str() << "\n";
    } else {
      o << "    stream: ~\n";
    }
    if (!data.vtu_pattern.empty()) o << "    vtu_pattern: " << data.vtu_pattern << "\n";
    if (!data.generator.empty()) o << "    generator: " << data.generator << "\n";
    if (!data.generator_params.empty()) {
      o << "    generator_params:\n";
      for (const auto& kv : data.generator_params) o << "      " << kv.first << ": " << num(kv.second) << "\n";
    }
    o << "  mesh:\n";
    o << "    type: " << mesh_type_to_string(mesh.type) << "\n";
    if (!mesh.dimensions.empty()) {
      std::vector<std::string> d;
      for (uint64_t v : mesh.dimensions) d.push_back(std::to_string(v));
      seq("    ", "dimensions", d);
    }
    std::vector<std::string> sp, og;
    for (double v : mesh.spacing) sp.push_back(num(v));
    for (double v : mesh.origin) og.push_back(num(v));
    seq("    ", "spacing", sp);
    seq("    ", "origin", og);
    if (!mesh.mesh_file.empty()) o << "    mesh_file: " << mesh.mesh_file << "\n";
    o << "  execution:\n";
    o << "    backend: " << backend_to_string(execution.backend) << "\n";
    o << "    precision: " << precision_to_string(execution.precision) << "\n";
    if (execution.num_threads != -1) o << "    threads: " << execution.num_threads << "\n";
    o << "  output:\n";
    o << "    trajectories: " << output.trajectories << "\n";
    if (!output.statistics.empty()) o << "    statistics: " << output.statistics << "\n";
    o << "    format: " << output.format;
    return o.str();
  }

  void to_yaml(const std::string& path) const {
    std::ofstream out(path);
    if (!out) throw std::runtime_error("Cannot open file for writing: " + path);
    out << to_yaml_string();
  }

  static TrackingConfig from_yaml_string(const std::string& text) {
    const yaml::Node root = yaml::Load(text);
    if (!root["tracking"]) throw std::invalid_argument("YAML file must contain 'tracking' key");
    return from_yaml_node(root["tracking"]);
  }

  static TrackingConfig from_yaml(const std::string& path) {
    const yaml::Node root = yaml::LoadFile(path);
    if (!root["tracking"]) throw std::invalid_argument("YAML file must contain 'tracking' key");
    return from_yaml_node(root["tracking"]);
  }
};

}  // namespace ftk2b
