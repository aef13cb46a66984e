// VTK XML output of feature complexes and input of base meshes, written as
// plain XML with no VTK library (utils/vtk.hpp of hguo/ftk2 needs VTK):
//
//   write_complex_to_vtp(complex, mesh, file, target_dim = -1, use_ascii = false)
//   write_complex_to_vtu(complex, mesh, file, target_dim = -1, use_ascii = false)
//   read_vtu(file) -> shared_ptr<UnstructuredSimplicialMesh>
//
// Content follows utils/vtk.hpp:26-160: one point per feature at
// sum_i (double)(float barycentric_i) * mesh.get_vertex_coordinates(v_i),
// its first three coordinates stored as Float32 (the precision of a default
// vtkPoints); point arrays "Scalar" (Float32), "TrackID" (Int32), "Type"
// (Int32) and "Time" (Float32: the last coordinate where the mesh's total
// dimension exceeds its spatial one, else 0).  VTP: connectivity of
// dimension 0 / 1 / 2 as verts / lines / polys.  VTU: dimension 0..3 as
// VTK_VERTEX / LINE / TRIANGLE / TETRA cells, or one VTK_VERTEX per feature
// for target_dim 0.  A target_dim other than -1 keeps that dimension only.
//
// Encoding: ASCII when use_ascii is set or FTK_DEBUG is in the environment,
// else appended data encoded as base64 with UInt64 block headers and no
// compression, as the reference configures VTK's writer (SetDataModeToAppended,
// SetEncodeAppendedData(1), SetCompressorTypeToNone; utils/vtk.hpp:102-108,
// 150-156): per array, the base64 of its 8-byte length header followed by the
// base64 of its bytes, each padded on its own, offsets counted in characters
// of the encoded text after the '_' marker.  read_vtu reads single-piece
// little-endian files in ASCII, inline base64, appended base64 and appended
// raw form, uncompressed, as utils/vtk.hpp:165-192 does through VTK: points,
// and the triangles and tetrahedra among the cells (other cells skipped),
// into UnstructuredSimplicialMesh(cell_dim, cell_dim, coords, cells).
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "engine.hpp"

namespace ftk2b {
namespace vtk_detail {

enum : uint8_t { kVertex = 1, kLine = 3, kTriangle = 5, kTetra = 10 };

struct Points {
  std::vector<float> xyz, scalar, time;
  std::vector<int32_t> track, type;
};

inline Points complex_points(const FeatureComplex& c, const Mesh& mesh) {
  Points p;
  const size_t n = c.vertices.size();
  const int td = mesh.get_total_dimension();
  const bool has_time = td > mesh.get_spatial_dimension();
  p.xyz.assign(3 * n, 0.f);
  p.scalar.resize(n);
  p.time.resize(n);
  p.track.resize(n);
  p.type.resize(n);
  std::vector<double> pos(td > 0 ? td : 0);
  for (size_t i = 0; i < n; ++i) {
    const FeatureElement& el = c.vertices[i];
    std::fill(pos.begin(), pos.end(), 0.0);
    for (int v = 0; v <= el.simplex.dimension && v < 5; ++v) {
      const std::vector<double> vc = mesh.get_vertex_coordinates(el.simplex.vertices[v]);
      for (size_t j = 0; j < pos.size() && j < vc.size(); ++j)
        pos[j] += (double)el.barycentric_coords[0][v] * vc[j];
    }
    for (size_t j = 0; j < 3 && j < pos.size(); ++j) p.xyz[3 * i + j] = (float)pos[j];
    p.scalar[i] = el.scalar;
    p.track[i] = (int32_t)el.track_id;
    p.type[i] = (int32_t)el.type;
    p.time[i] = has_time && !pos.empty() ? (float)pos.back() : 0.0f;
  }
  return p;
}

// DataArray elements, inline ASCII or appended raw blocks
class Writer {
 public:
  explicit Writer(bool ascii) : ascii_(ascii) {}
  std::ostringstream body;

  template <typename E>
  void array(const char* type, const char* name, int ncomp, const std::vector<E>& a, const char* indent) {
    body << indent << "<DataArray type=\"" << type << "\" Name=\"" << name << "\"";
    if (ncomp > 1) body << " NumberOfComponents=\"" << ncomp << "\"";
    if (!ascii_) {
      body << " format=\"appended\" offset=\"" << appended_.size() << "\"/>\n";
      const uint64_t nb = a.size() * sizeof(E);
      b64(reinterpret_cast<const uint8_t*>(&nb), 8);
      b64(reinterpret_cast<const uint8_t*>(a.data()), nb);
      return;
    }
    body << " format=\"ascii\">\n";
    char b[32];
    for (size_t i = 0; i < a.size(); ++i) {
      if (i % 6 == 0) body << indent << "  ";
      fmt(b, a[i]);
      body << b << ((i % 6 == 5 || i + 1 == a.size()) ? "\n" : " ");
    }
    body << indent << "</DataArray>\n";
  }

  void save(const std::string& path, const char* type) const {
    std::ofstream f(path, std::ios::binary);
    if (!f) throw Error(FTK2B_INVALID_ARG, "Cannot open output file: " + path);
    f << "<?xml version=\"1.0\"?>\n<VTKFile type=\"" << type
      << "\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n";
    f << body.str();
    if (!ascii_) {
      f << "  <AppendedData encoding=\"base64\">\n   _";
      f.write(appended_.data(), (std::streamsize)appended_.size());
      f << "\n  </AppendedData>\n";
    }
    f << "</VTKFile>\n";
    if (!f) throw Error(FTK2B_INVALID_ARG, "Cannot write output file: " + path);
  }

 private:
  // appends the base64 text of n bytes, padded with '=' to whole quanta
  void b64(const uint8_t* d, uint64_t n) {
    static const char* A = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
    for (uint64_t i = 0; i < n; i += 3) {
      const uint32_t b0 = d[i], b1 = i + 1 < n ? d[i + 1] : 0, b2 = i + 2 < n ? d[i + 2] : 0;
      const uint32_t w = b0 << 16 | b1 << 8 | b2;
      appended_.push_back(A[(w >> 18) & 63]);
      appended_.push_back(A[(w >> 12) & 63]);
      appended_.push_back(i + 1 < n ? A[(w >> 6) & 63] : '=');
      appended_.push_back(i + 2 < n ? A[w & 63] : '=');
    }
  }
  static void fmt(char* b, float v) { std::snprintf(b, 32, "%.9g", (double)v); }
  static void fmt(char* b, int32_t v) { std::snprintf(b, 32, "%d", v); }
  static void fmt(char* b, int64_t v) { std::snprintf(b, 32, "%lld", (long long)v); }
  static void fmt(char* b, uint8_t v) { std::snprintf(b, 32, "%u", (unsigned)v); }
  bool ascii_;
  std::vector<char> appended_;
};

inline bool want_ascii(bool use_ascii) { return use_ascii || std::getenv("FTK_DEBUG") != nullptr; }

inline void point_data(Writer& w, const Points& p) {
  w.body << "      <PointData>\n";
  w.array("Float32", "Scalar", 1, p.scalar, "        ");
  w.array("Int32", "TrackID", 1, p.track, "        ");
  w.array("Int32", "Type", 1, p.type, "        ");
  w.array("Float32", "Time", 1, p.time, "        ");
  w.body << "      </PointData>\n      <CellData>\n      </CellData>\n      <Points>\n";
  w.array("Float32", "Points", 3, p.xyz, "        ");
  w.body << "      </Points>\n";
}

struct CellList {
  std::vector<int64_t> conn, offsets;
  std::vector<uint8_t> types;
  void add(const uint32_t* idx, int n, uint8_t type) {
    for (int j = 0; j < n; ++j) conn.push_back((int64_t)idx[j]);
    offsets.push_back((int64_t)conn.size());
    types.push_back(type);
  }
};

// ---- reading

struct Xml {
  std::string s;
  // the value of attribute key inside the tag that starts at pos
  std::string attr(size_t pos, const std::string& key) const {
    const size_t end = s.find('>', pos);
    const std::string pat = " " + key + "=\"";
    const size_t a = s.find(pat, pos);
    if (a == std::string::npos || a > end) return "";
    const size_t b = a + pat.size();
    return s.substr(b, s.find('"', b) - b);
  }
};

inline int b64val(char c) {
  if (c >= 'A' && c <= 'Z') return c - 'A';
  if (c >= 'a' && c <= 'z') return c - 'a' + 26;
  if (c >= '0' && c <= '9') return c - '0' + 52;
  if (c == '+') return 62;
  if (c == '/') return 63;
  return -1;
}

// Decodes base64 quanta from p until want bytes are out; '=' padding may end
// a quantum in the middle of the text (a header encoded apart from its data).
// Returns the position after the last quantum read.
inline size_t b64decode(const std::string& s, size_t p, size_t want, std::vector<uint8_t>& out) {
  int q[4], nq = 0, pad = 0;
  while (out.size() < want && p < s.size()) {
    const char c = s[p++];
    if (c == '=') {
      q[nq++] = 0;
      ++pad;
    } else {
      const int v = b64val(c);
      if (v < 0) {
        if (c == '<') break;
        continue;  // whitespace
      }
      q[nq++] = v;
    }
    if (nq == 4) {
      const uint32_t w = (uint32_t)q[0] << 18 | (uint32_t)q[1] << 12 | (uint32_t)q[2] << 6 | (uint32_t)q[3];
      const uint8_t b[3] = {(uint8_t)(w >> 16), (uint8_t)(w >> 8), (uint8_t)w};
      for (int k = 0; k < 3 - pad; ++k) out.push_back(b[k]);
      nq = pad = 0;
    }
  }
  return p;
}

// One DataArray (the tag at pos) as doubles.
inline std::vector<double> read_array(const Xml& x, size_t pos, size_t count, size_t appended, bool raw,
                                      int header_bytes) {
  const std::string type = x.attr(pos, "type"), format = x.attr(pos, "format");
  int esz = 0;
  if (type == "Float32" || type == "Int32" || type == "UInt32") esz = 4;
  else if (type == "Float64" || type == "Int64" || type == "UInt64") esz = 8;
  else if (type == "Int8" || type == "UInt8") esz = 1;
  else if (type == "Int16" || type == "UInt16") esz = 2;
  else throw Error(FTK2B_UNSUPPORTED, "VTU data type " + type);
  std::vector<double> out;
  out.reserve(count);
  if (format == "ascii") {
    size_t p = x.s.find('>', pos) + 1;
    const char* c = x.s.c_str() + p;
    for (size_t i = 0; i < count; ++i) {
      char* e = nullptr;
      const double v = std::strtod(c, &e);
      if (e == c) throw Error(FTK2B_INVALID_ARG, "short ASCII DataArray in VTU");
      out.push_back(esz == 4 && type == "Float32" ? (double)(float)v : v);  // the array's own precision
      c = e;
    }
    return out;
  }
  std::vector<uint8_t> bytes;
  const size_t need = (size_t)header_bytes + count * esz;
  if (format == "binary") {
    b64decode(x.s, x.s.find('>', pos) + 1, need, bytes);
  } else if (format == "appended") {
    if (appended == std::string::npos) throw Error(FTK2B_INVALID_ARG, "VTU has no AppendedData");
    const size_t off = appended + (size_t)std::strtoull(x.attr(pos, "offset").c_str(), nullptr, 10);
    if (raw) {
      if (off + need > x.s.size()) throw Error(FTK2B_INVALID_ARG, "truncated appended data in VTU");
      bytes.assign(x.s.begin() + off, x.s.begin() + off + need);
    } else {
      b64decode(x.s, off, need, bytes);
    }
  } else {
    throw Error(FTK2B_UNSUPPORTED, "VTU DataArray format " + format);
  }
  if (bytes.size() < need) throw Error(FTK2B_INVALID_ARG, "truncated DataArray in VTU");
  const uint8_t* d = bytes.data() + header_bytes;
  for (size_t i = 0; i < count; ++i) {
    const uint8_t* e = d + i * esz;
    double v = 0;
    if (type == "Float32") { float f; std::memcpy(&f, e, 4); v = f; }
    else if (type == "Float64") { std::memcpy(&v, e, 8); }
    else if (type == "Int32") { int32_t t; std::memcpy(&t, e, 4); v = t; }
    else if (type == "UInt32") { uint32_t t; std::memcpy(&t, e, 4); v = t; }
    else if (type == "Int64") { int64_t t; std::memcpy(&t, e, 8); v = (double)t; }
    else if (type == "UInt64") { uint64_t t; std::memcpy(&t, e, 8); v = (double)t; }
    else if (type == "Int16") { int16_t t; std::memcpy(&t, e, 2); v = t; }
    else if (type == "UInt16") { uint16_t t; std::memcpy(&t, e, 2); v = t; }
    else if (type == "Int8") { v = (int8_t)*e; }
    else { v = *e; }
    out.push_back(v);
  }
  return out;
}

// the DataArray inside [from, to) whose Name is name (or the first one)
inline size_t find_array(const Xml& x, size_t from, size_t to, const char* name) {
  for (size_t p = x.s.find("<DataArray", from); p != std::string::npos && p < to;
       p = x.s.find("<DataArray", p + 1))
    if (!name || x.attr(p, "Name") == name) return p;
  throw Error(FTK2B_INVALID_ARG, std::string("VTU lacks DataArray ") + (name ? name : "Points"));
}

}  // namespace vtk_detail

inline void write_complex_to_vtp(const FeatureComplex& complex, const Mesh& mesh, const std::string& filename,
                                 int target_dim = -1, bool use_ascii = false) {
  using namespace vtk_detail;
  const Points p = complex_points(complex, mesh);
  CellList sec[3];
  for (const auto& cn : complex.connectivity) {
    if (target_dim != -1 && cn.dimension != target_dim) continue;
    if (cn.dimension < 0 || cn.dimension > 2) continue;
    const int k = cn.dimension + 1;
    for (size_t i = 0; i + k <= cn.indices.size(); i += k) sec[cn.dimension].add(&cn.indices[i], k, 0);
  }
  Writer w(want_ascii(use_ascii));
  w.body << "  <PolyData>\n    <Piece NumberOfPoints=\"" << p.scalar.size() << "\" NumberOfVerts=\""
         << sec[0].types.size() << "\" NumberOfLines=\"" << sec[1].types.size()
         << "\" NumberOfStrips=\"0\" NumberOfPolys=\"" << sec[2].types.size() << "\">\n";
  point_data(w, p);
  const char* tag[4] = {"Verts", "Lines", "Strips", "Polys"};
  const CellList none;
  for (int s = 0; s < 4; ++s) {
    const CellList& c = s == 0 ? sec[0] : s == 1 ? sec[1] : s == 3 ? sec[2] : none;
    w.body << "      <" << tag[s] << ">\n";
    w.array("Int64", "connectivity", 1, c.conn, "        ");
    w.array("Int64", "offsets", 1, c.offsets, "        ");
    w.body << "      </" << tag[s] << ">\n";
  }
  w.body << "    </Piece>\n  </PolyData>\n";
  w.save(filename, "PolyData");
}

inline void write_complex_to_vtu(const FeatureComplex& complex, const Mesh& mesh, const std::string& filename,
                                 int target_dim = -1, bool use_ascii = false) {
  using namespace vtk_detail;
  const Points p = complex_points(complex, mesh);
  CellList cells;
  if (target_dim == 0) {
    for (size_t i = 0; i < complex.vertices.size(); ++i) {
      const uint32_t v = (uint32_t)i;
      cells.add(&v, 1, kVertex);
    }
  } else {
    const uint8_t types[4] = {kVertex, kLine, kTriangle, kTetra};
    for (const auto& cn : complex.connectivity) {
      if (target_dim != -1 && cn.dimension != target_dim) continue;
      if (cn.dimension < 0 || cn.dimension > 3) continue;
      const int k = cn.dimension + 1;
      for (size_t i = 0; i + k <= cn.indices.size(); i += k) cells.add(&cn.indices[i], k, types[cn.dimension]);
    }
  }
  Writer w(want_ascii(use_ascii));
  w.body << "  <UnstructuredGrid>\n    <Piece NumberOfPoints=\"" << p.scalar.size() << "\" NumberOfCells=\""
         << cells.types.size() << "\">\n";
  point_data(w, p);
  w.body << "      <Cells>\n";
  w.array("Int64", "connectivity", 1, cells.conn, "        ");
  w.array("Int64", "offsets", 1, cells.offsets, "        ");
  w.array("UInt8", "types", 1, cells.types, "        ");
  w.body << "      </Cells>\n    </Piece>\n  </UnstructuredGrid>\n";
  w.save(filename, "UnstructuredGrid");
}

inline std::shared_ptr<UnstructuredSimplicialMesh> read_vtu(const std::string& filename) {
  using namespace vtk_detail;
  std::ifstream f(filename, std::ios::binary);
  if (!f) return nullptr;
  Xml x;
  x.s.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  const size_t root = x.s.find("<VTKFile");
  if (root == std::string::npos || x.attr(root, "type") != "UnstructuredGrid")
    throw Error(FTK2B_INVALID_ARG, "not a VTK UnstructuredGrid file: " + filename);
  if (x.attr(root, "byte_order") == "BigEndian") throw Error(FTK2B_UNSUPPORTED, "big-endian VTU");
  if (!x.attr(root, "compressor").empty()) throw Error(FTK2B_UNSUPPORTED, "compressed VTU");
  const int hb = x.attr(root, "header_type") == "UInt64" ? 8 : 4;
  size_t app = x.s.find("<AppendedData");
  bool raw = false;
  if (app != std::string::npos) {
    raw = x.attr(app, "encoding") == "raw";
    app = x.s.find('_', x.s.find('>', app)) + 1;
  }
  const size_t piece = x.s.find("<Piece");
  if (piece == std::string::npos) throw Error(FTK2B_INVALID_ARG, "VTU without a Piece");
  const size_t np = std::strtoull(x.attr(piece, "NumberOfPoints").c_str(), nullptr, 10);
  const size_t nc = std::strtoull(x.attr(piece, "NumberOfCells").c_str(), nullptr, 10);
  const size_t pts = x.s.find("<Points", piece), cs = x.s.find("<Cells", piece);
  if (pts == std::string::npos || cs == std::string::npos) throw Error(FTK2B_INVALID_ARG, "VTU lacks Points/Cells");
  const size_t pa = find_array(x, pts, x.s.find("</Points>", pts), nullptr);
  const int ncomp = std::atoi(x.attr(pa, "NumberOfComponents").c_str());
  const int pc = ncomp > 0 ? ncomp : 1;
  const std::vector<double> xyz = read_array(x, pa, np * pc, app, raw, hb);
  std::vector<double> coords(3 * np, 0.0);
  for (size_t i = 0; i < np; ++i)
    for (int j = 0; j < 3 && j < pc; ++j) coords[3 * i + j] = xyz[i * pc + j];
  const size_t ce = x.s.find("</Cells>", cs);
  const std::vector<double> off = read_array(x, find_array(x, cs, ce, "offsets"), nc, app, raw, hb);
  const std::vector<double> typ = read_array(x, find_array(x, cs, ce, "types"), nc, app, raw, hb);
  const size_t nconn = nc ? (size_t)off[nc - 1] : 0;
  const std::vector<double> conn = read_array(x, find_array(x, cs, ce, "connectivity"), nconn, app, raw, hb);
  std::vector<uint64_t> cells;
  int cell_dim = 0;
  for (size_t i = 0; i < nc; ++i) {
    const size_t b = i ? (size_t)off[i - 1] : 0, e = (size_t)off[i];
    if ((int)typ[i] == kTriangle) cell_dim = 2;
    else if ((int)typ[i] == kTetra) cell_dim = 3;
    else continue;
    if (e > conn.size() || b > e) throw Error(FTK2B_INVALID_ARG, "VTU cell offsets out of range");
    for (size_t j = b; j < e; ++j) cells.push_back((uint64_t)conn[j]);
  }
  return std::make_shared<UnstructuredSimplicialMesh>(cell_dim, cell_dim, coords, cells);
}

}  // namespace ftk2b
