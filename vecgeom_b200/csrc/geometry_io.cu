// geometry_io.cu -- geometry ingestion and export formats.
//
//   flat image   the recorded object graph (shape records and constructor
//                arguments, transformations, logical volumes with labels,
//                placements, world) as one checksummed little-endian blob;
//                loading replays the placements, so the tables derived at close
//                come out identical.
//   C++ source   a function `generateDetector()` that rebuilds the geometry
//                with VecGeom's own API, in the layout of
//                GeomCppExporter::DumpGeometry (source/CppExporter.cpp:436-486):
//                transformations, logical volumes over `new Unplaced*(...)`,
//                PlaceDaughter calls, the world placement.  Numbers carry 17
//                significant digits (the reference's exporter prints 15, which
//                does not round-trip a double); every shape this library
//                builds is written (the reference's exporter knows box, tube,
//                cone, trapezoid, torus, polycone, polyhedron, trd, boolean).
//
// Host code only.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "geometry.h"
#include "shapes.cuh"

using namespace vgb;

namespace {

constexpr char kMagic[8] = {'V', 'G', 'B', 'G', 'E', 'O', 'M', '1'};
constexpr uint32_t kVersion = 3;  // 2: polyhedron quadrilaterals of 33 doubles; 3: polycone sections of 41

uint64_t fnv1a(const uint8_t *p, size_t n) {
  uint64_t h = 1469598103934665603ull;
  for (size_t i = 0; i < n; ++i) {
    h ^= p[i];
    h *= 1099511628211ull;
  }
  return h;
}

struct Writer {
  std::vector<uint8_t> b;
  void bytes(const void *p, size_t n) {
    const uint8_t *c = static_cast<const uint8_t *>(p);
    b.insert(b.end(), c, c + n);
  }
  template <class T> void put(const T &v) { bytes(&v, sizeof(T)); }
};

struct Reader {
  const uint8_t *p, *end;
  bool bytes(void *out, size_t n) {
    if ((size_t)(end - p) < n) return false;
    std::memcpy(out, p, n);
    p += n;
    return true;
  }
  template <class T> bool get(T &v) { return bytes(&v, sizeof(T)); }
  size_t left() const { return (size_t)(end - p); }
};

// the logical volume each placed volume is a daughter of (-1: none)
std::vector<int32_t> mothers_of(const vgb_geometry *g) {
  std::vector<int32_t> m(g->placed.size(), -1);
  for (size_t l = 0; l < g->logical_daughters.size(); ++l)
    for (int32_t d : g->logical_daughters[l]) m[d] = (int32_t)l;
  return m;
}

// %.17g, or false for a value C++ source cannot spell as a literal
bool num(std::string &out, double v) {
  if (!std::isfinite(v)) return false;
  char buf[40];
  std::snprintf(buf, sizeof buf, "%.17g", v);
  out += buf;
  return true;
}

std::string quoted(const std::string &s) {
  std::string q = "\"";
  for (unsigned char c : s) {
    if (c == '"' || c == '\\') {
      q += '\\';
      q += (char)c;
    } else if (c < 0x20 || c >= 0x7f) {
      char buf[8];
      std::snprintf(buf, sizeof buf, "\\%03o", c);
      q += buf;
    } else {
      q += (char)c;
    }
  }
  return q + "\"";
}

const char *shape_header(int type) {
  switch (type) {
    case VGB_SHAPE_BOX: return "volumes/UnplacedBox.h";
    case VGB_SHAPE_TUBE: return "volumes/UnplacedTube.h";
    case VGB_SHAPE_CONE: return "volumes/UnplacedCone.h";
    case VGB_SHAPE_SPHERE: return "volumes/UnplacedSphere.h";
    case VGB_SHAPE_TORUS: return "volumes/UnplacedTorus.h";
    case VGB_SHAPE_TRD: return "volumes/UnplacedTrd.h";
    case VGB_SHAPE_POLYCONE: return "volumes/UnplacedPolycone.h";
    case VGB_SHAPE_POLYHEDRON: return "volumes/UnplacedPolyhedron.h";
    case VGB_SHAPE_BOOLEAN: return "volumes/UnplacedBooleanVolume.h";
    case VGB_SHAPE_ORB: return "volumes/UnplacedOrb.h";
    case VGB_SHAPE_PARALLELEPIPED: return "volumes/UnplacedParallelepiped.h";
    case VGB_SHAPE_PARABOLOID: return "volumes/UnplacedParaboloid.h";
    case VGB_SHAPE_TRAPEZOID: return "volumes/UnplacedTrapezoid.h";
    default: return nullptr;
  }
}

const char *shape_class(int type) {
  switch (type) {
    case VGB_SHAPE_BOX: return "UnplacedBox";
    case VGB_SHAPE_TUBE: return "UnplacedTube";
    case VGB_SHAPE_CONE: return "UnplacedCone";
    case VGB_SHAPE_SPHERE: return "UnplacedSphere";
    case VGB_SHAPE_TORUS: return "UnplacedTorus";
    case VGB_SHAPE_TRD: return "UnplacedTrd";
    case VGB_SHAPE_POLYCONE: return "UnplacedPolycone";
    case VGB_SHAPE_POLYHEDRON: return "UnplacedPolyhedron";
    case VGB_SHAPE_ORB: return "UnplacedOrb";
    case VGB_SHAPE_PARALLELEPIPED: return "UnplacedParallelepiped";
    case VGB_SHAPE_PARABOLOID: return "UnplacedParaboloid";
    case VGB_SHAPE_TRAPEZOID: return "UnplacedTrapezoid";
    default: return nullptr;
  }
}

// "a , b , c" of args[first, last)
bool num_list(std::string &out, const std::vector<double> &a, size_t first, size_t last) {
  for (size_t i = first; i < last; ++i) {
    if (i > first) out += " , ";
    if (!num(out, a[i])) return false;
  }
  return true;
}

// the reference's DumpVector form, &std::vector<double>{...}[0]
bool vec_literal(std::string &out, const std::vector<double> &a, size_t first, size_t n) {
  out += "&std::vector<double>{";
  if (!num_list(out, a, first, first + n)) return false;
  out += "}[0]";
  return true;
}

// `new Unplaced*( ... )` of a non-boolean shape; `pre` receives statements the
// expression needs first (the trapezoid's corner array)
vgb_status shape_expr(const vgb_geometry *g, int32_t u, const std::string &tag, std::string &pre,
                      std::string &e) {
  const int type = g->unplaced[u].type;
  const std::vector<double> &a = g->ctor_args[u];
  const char *cls = shape_class(type);
  auto bad = [&]() {
    return set_error(VGB_EINVAL, "vgb_geometry_export_cpp: shape %d (type %d) has a value C++ "
                                 "cannot spell or no recorded constructor", u, type);
  };
  if (!cls || a.empty()) return bad();
  if (type == VGB_SHAPE_POLYCONE || type == VGB_SHAPE_POLYHEDRON) {
    // polycone (sphi, dphi, nz, rmin[], rmax[], z[]); polyhedron (phi start,
    // phi delta, sides, nz, z[], rmin[], rmax[]) -- the arrays as recorded
    const size_t head = type == VGB_SHAPE_POLYCONE ? 3 : 4;
    if (a.size() < head) return bad();
    const size_t nz = (size_t)a[head - 1];
    if (a.size() != head + 3 * nz) return bad();
    e += std::string("new ") + cls + "( ";
    if (!num_list(e, a, 0, 2)) return bad();
    for (size_t k = 2; k < head; ++k) e += " , " + std::to_string((long long)a[k]);
    for (size_t k = 0; k < 3; ++k) {
      e += " , ";
      if (!vec_literal(e, a, head + k * nz, nz)) return bad();
    }
    e += " )";
    return VGB_OK;
  }
  if (type == VGB_SHAPE_TRAPEZOID && g->ctor_form[u] == kCtorCorners) {
    if (a.size() != 24) return bad();
    pre += "Vector3D<Precision> " + tag + "_corners[8] = {";
    for (int k = 0; k < 8; ++k) {
      pre += k ? " , Vector3D<Precision>(" : "Vector3D<Precision>(";
      if (!num_list(pre, a, 3 * k, 3 * k + 3)) return bad();
      pre += ")";
    }
    pre += "};\n";
    e += "new UnplacedTrapezoid( " + tag + "_corners )";
    return VGB_OK;
  }
  std::string args;
  if (!num_list(args, a, 0, a.size())) return bad();
  if (type == VGB_SHAPE_ORB) {
    // UnplacedOrb(r) computes its tolerance from a member it has not yet set
    // (source/UnplacedOrb.cpp:33-44); SetRadius recomputes the cached values
    e += "[]{ UnplacedOrb * o = new UnplacedOrb( " + args + " ); o->SetRadius( " + args +
         " ); return o; }()";
    return VGB_OK;
  }
  e += std::string("new ") + cls + "( " + args + " )";
  return VGB_OK;
}

vgb_status export_cpp(const vgb_geometry *g, std::string &out) {
  if (g->world < 0) return set_error(VGB_EINVAL, "vgb_geometry_export_cpp: no world set");
  const int32_t nl = (int32_t)g->logicals.size();
  std::vector<std::string> headers;
  auto need = [&](int type) {
    const char *h = shape_header(type);
    if (h && std::find(headers.begin(), headers.end(), h) == headers.end()) headers.push_back(h);
  };
  std::vector<int32_t> order;  // our placed ids in the order the function creates them
  std::string trans, lvols, tree;
  // transformations, as Transformation3D(tx, ty, tz, r0..r8): with SetProperties
  // (source/Transformation3D.cpp:46-55) giving the flags the angle form gives
  for (size_t t = 0; t < g->raw_xforms.size(); ++t) {
    const RawXform &x = g->raw_xforms[t];
    std::string line = "Transformation3D * transf" + std::to_string(t) + " = new Transformation3D(";
    for (int i = 0; i < 12; ++i) {
      line += i ? " , " : " ";
      if (!num(line, i < 3 ? x.t[i] : x.r[i - 3]))
        return set_error(VGB_EINVAL, "vgb_geometry_export_cpp: transformation %zu is not finite",
                         t);
    }
    trans += line + " );\n";
  }
  // logical volumes in id order: a boolean's components come from logical
  // volumes made before it; their placements are statements of their own so
  // the creation order (and the reference's placed-volume ids) is fixed
  for (int32_t l = 0; l < nl; ++l) {
    const int32_t u = g->logicals[l].unplaced;
    const int type = g->unplaced[u].type;
    const std::string tag = "lvol" + std::to_string(l);
    need(type);
    std::string pre, e;
    if (type == VGB_SHAPE_BOOLEAN) {
      const std::vector<double> &a = g->ctor_args[u];
      if (a.size() != 3)
        return set_error(VGB_EINVAL, "vgb_geometry_export_cpp: boolean %d has no recorded "
                                     "constructor", u);
      static const char *ops[3] = {"kUnion", "kIntersection", "kSubtraction"};
      const int op = (int)a[0];
      if (op < 0 || op > 2 || a[1] < 0 || a[2] < 0 || a[1] >= (double)g->placed.size() ||
          a[2] >= (double)g->placed.size())
        return set_error(VGB_EINVAL, "vgb_geometry_export_cpp: boolean %d is malformed", u);
      std::string comp[2];
      for (int k = 0; k < 2; ++k) {
        const int32_t pv = (int32_t)a[1 + k];
        const PlacedRec &p = g->placed[pv];
        comp[k] = tag + (k ? "_right" : "_left");
        pre += "VPlacedVolume const * " + comp[k] + " = lvol" + std::to_string(p.logical) +
               "->Place( transf" + std::to_string(p.raw_xform) + " );\n";
        order.push_back(pv);
      }
      e = std::string("new UnplacedBooleanVolume( ") + ops[op] + " , " + comp[0] + " , " +
          comp[1] + " )";
    } else {
      vgb_status s = shape_expr(g, u, tag, pre, e);
      if (s != VGB_OK) return s;
    }
    lvols += pre + "LogicalVolume * " + tag + " = new LogicalVolume ( " + quoted(g->labels[l]) +
             " , " + e + " );\n";
  }
  for (int32_t l = 0; l < nl; ++l)
    for (int32_t d : g->logical_daughters[l]) {
      const PlacedRec &p = g->placed[d];
      tree += "lvol" + std::to_string(l) + "->PlaceDaughter( lvol" + std::to_string(p.logical) +
              " , transf" + std::to_string(p.raw_xform) + " );\n";
      order.push_back(d);
    }
  const PlacedRec &w = g->placed[g->world];
  order.push_back(g->world);

  out += "// Geometry source in the layout of VecGeom's GeomCppExporter\n";
  out += "// (source/CppExporter.cpp), written by vgb_geometry_export_cpp.\n";
  out += "#include \"base/Global.h\"\n#include \"volumes/PlacedVolume.h\"\n";
  out += "#include \"volumes/LogicalVolume.h\"\n#include \"base/Transformation3D.h\"\n";
  out += "#include \"management/GeoManager.h\"\n#include <vector>\n";
  for (const std::string &h : headers) out += "#include \"" + h + "\"\n";
  out += "using namespace vecgeom;\n\n";
  out += "// placed-volume ids of the exported geometry, in the order generateDetector()\n";
  out += "// creates the placements:";
  for (int32_t id : order) out += " " + std::to_string(id);
  out += "\n";
  out += "VPlacedVolume const * generateDetector() {\n";
  out += trans + lvols + tree;
  out += "VPlacedVolume const * world = lvol" + std::to_string(w.logical) + "->Place( transf" +
         std::to_string(w.raw_xform) + " );\n";
  out += "return world;\n}\n";
  return VGB_OK;
}

vgb_status serialize(const vgb_geometry *g, Writer &w) {
  const std::vector<int32_t> mother = mothers_of(g);
  w.bytes(kMagic, 8);
  w.put(kVersion);
  w.put((uint32_t)0);
  w.put((uint32_t)g->unplaced.size());
  w.put((uint32_t)g->raw_xforms.size());
  w.put((uint32_t)g->logicals.size());
  w.put((uint32_t)g->placed.size());
  w.put((uint64_t)g->params.size());
  w.put((int32_t)g->world);
  w.put((int32_t)0);
  for (size_t u = 0; u < g->unplaced.size(); ++u) {
    w.put(g->unplaced[u]);
    w.put(g->ctor_form[u]);
    w.put((uint32_t)g->ctor_args[u].size());
    w.bytes(g->ctor_args[u].data(), g->ctor_args[u].size() * sizeof(double));
  }
  w.bytes(g->params.data(), g->params.size() * sizeof(double));
  for (const RawXform &x : g->raw_xforms) {
    w.bytes(x.t, sizeof x.t);
    w.bytes(x.r, sizeof x.r);
  }
  for (size_t l = 0; l < g->logicals.size(); ++l) {
    w.put(g->logicals[l].unplaced);
    w.put((uint32_t)g->labels[l].size());
    w.bytes(g->labels[l].data(), g->labels[l].size());
  }
  for (size_t p = 0; p < g->placed.size(); ++p) {
    w.put(g->placed[p].logical);
    w.put(g->placed[p].raw_xform);
    w.put(mother[p]);
  }
  w.put(fnv1a(w.b.data(), w.b.size()));
  return VGB_OK;
}

vgb_status deserialize(const uint8_t *data, size_t len, vgb_geometry *g) {
  auto bad = [](const char *what) {
    return set_error(VGB_EINVAL, "vgb_geometry_deserialize: %s", what);
  };
  if (len < 8 + 8 + 4 * 4 + 8 + 8 + 8) return bad("image too short");
  uint64_t sum;
  std::memcpy(&sum, data + len - 8, 8);
  if (fnv1a(data, len - 8) != sum) return bad("checksum mismatch");
  Reader r{data, data + len - 8};
  char magic[8];
  uint32_t version, flags, nu, nx, nl, np;
  uint64_t nparams;
  int32_t world, pad;
  r.bytes(magic, 8);
  if (std::memcmp(magic, kMagic, 8) != 0) return bad("not a vgb geometry image");
  r.get(version);
  r.get(flags);
  if (version != kVersion) return bad("unknown image version");
  (void)flags;
  if (!(r.get(nu) && r.get(nx) && r.get(nl) && r.get(np) && r.get(nparams) && r.get(world) &&
        r.get(pad)))
    return bad("truncated header");
  (void)pad;
  if (nparams > r.left() / sizeof(double)) return bad("parameter pool larger than the image");
  g->unplaced.resize(nu);
  g->ctor_form.resize(nu);
  g->ctor_args.resize(nu);
  for (uint32_t u = 0; u < nu; ++u) {
    uint32_t na;
    if (!(r.get(g->unplaced[u]) && r.get(g->ctor_form[u]) && r.get(na)))
      return bad("truncated shape table");
    if (na > r.left() / sizeof(double)) return bad("truncated constructor arguments");
    g->ctor_args[u].resize(na);
    r.bytes(g->ctor_args[u].data(), na * sizeof(double));
    const UnplacedRec &ur = g->unplaced[u];
    if (ur.type < VGB_SHAPE_BOX || ur.type > VGB_SHAPE_TRAPEZOID || ur.param_off < 0 ||
        ur.param_len < 0 || (uint64_t)ur.param_off + (uint64_t)ur.param_len > nparams ||
        ur.param_off % 2)
      return bad("shape record out of range");
  }
  g->params.resize(nparams);
  if (!r.bytes(g->params.data(), nparams * sizeof(double))) return bad("truncated parameters");
  for (uint32_t t = 0; t < nx; ++t) {
    double v[12];
    if (!r.bytes(v, sizeof v)) return bad("truncated transformations");
    int32_t id;
    vgb_status s = vgb_transformation_matrix(g, v[0], v[1], v[2], v + 3, &id);
    if (s != VGB_OK) return s;
  }
  for (uint32_t l = 0; l < nl; ++l) {
    int32_t u;
    uint32_t n;
    if (!(r.get(u) && r.get(n)) || n > r.left()) return bad("truncated logical volumes");
    std::string label((const char *)r.p, n);
    r.p += n;
    int32_t id;
    vgb_status s = vgb_logical_volume(g, label.c_str(), u, &id);
    if (s != VGB_OK) return s;
  }
  for (uint32_t p = 0; p < np; ++p) {
    int32_t l, x, m, id;
    if (!(r.get(l) && r.get(x) && r.get(m))) return bad("truncated placements");
    if (m < -1 || m >= (int32_t)nl) return bad("mother logical volume out of range");
    vgb_status s = m < 0 ? vgb_place(g, l, x, &id) : vgb_place_daughter(g, m, l, x, &id);
    if (s != VGB_OK) return s;
  }
  for (uint32_t u = 0; u < nu; ++u)
    if (g->unplaced[u].type == VGB_SHAPE_BOOLEAN &&
        (g->unplaced[u].extra < 0 || g->unplaced[u].extra >= (int32_t)np))
      return bad("boolean component out of range");
  if (r.left() != 0) return bad("trailing bytes");
  if (world >= (int32_t)np || world < -1) return bad("world out of range");
  g->world = world;
  return VGB_OK;
}

vgb_status copy_out(const std::string &s, char *buf, size_t cap, size_t *len) {
  if (len) *len = s.size();
  if (buf && cap < s.size()) return set_error(VGB_ENOSPC, "buffer of %zu bytes, %zu needed", cap,
                                              s.size());
  if (buf) std::memcpy(buf, s.data(), s.size());
  return VGB_OK;
}

}  // namespace

extern "C" {

vgb_status vgb_geometry_serialize(const vgb_geometry *g, void *buf, size_t cap, size_t *len) {
  if (!g) return set_error(VGB_EINVAL, "vgb_geometry_serialize: geometry is NULL");
  Writer w;
  vgb_status s = serialize(g, w);
  if (s != VGB_OK) return s;
  return copy_out(std::string(w.b.begin(), w.b.end()), static_cast<char *>(buf), cap, len);
}

vgb_status vgb_geometry_deserialize(const void *buf, size_t len, vgb_geometry **out) {
  if (!buf || !out) return set_error(VGB_EINVAL, "vgb_geometry_deserialize: NULL argument");
  vgb_geometry *g = nullptr;
  vgb_status s = vgb_geometry_create(&g);
  if (s != VGB_OK) return s;
  s = deserialize(static_cast<const uint8_t *>(buf), len, g);
  if (s != VGB_OK) {
    vgb_geometry_destroy(g);
    return s;
  }
  *out = g;
  return VGB_OK;
}

vgb_status vgb_geometry_save(const vgb_geometry *g, const char *path) {
  if (!g || !path) return set_error(VGB_EINVAL, "vgb_geometry_save: NULL argument");
  Writer w;
  vgb_status s = serialize(g, w);
  if (s != VGB_OK) return s;
  FILE *f = std::fopen(path, "wb");
  if (!f) return set_error(VGB_EINVAL, "vgb_geometry_save: cannot open %s", path);
  const size_t n = std::fwrite(w.b.data(), 1, w.b.size(), f);
  const int c = std::fclose(f);
  if (n != w.b.size() || c != 0) return set_error(VGB_EINVAL, "vgb_geometry_save: write failed");
  return VGB_OK;
}

vgb_status vgb_geometry_load(const char *path, vgb_geometry **out) {
  if (!path || !out) return set_error(VGB_EINVAL, "vgb_geometry_load: NULL argument");
  FILE *f = std::fopen(path, "rb");
  if (!f) return set_error(VGB_EINVAL, "vgb_geometry_load: cannot open %s", path);
  std::vector<uint8_t> data;
  uint8_t chunk[1 << 16];
  size_t n;
  while ((n = std::fread(chunk, 1, sizeof chunk, f)) > 0) data.insert(data.end(), chunk, chunk + n);
  std::fclose(f);
  return vgb_geometry_deserialize(data.data(), data.size(), out);
}

vgb_status vgb_geometry_export_cpp(const vgb_geometry *g, char *buf, size_t cap, size_t *len) {
  if (!g) return set_error(VGB_EINVAL, "vgb_geometry_export_cpp: geometry is NULL");
  std::string s;
  vgb_status st = export_cpp(g, s);
  if (st != VGB_OK) return st;
  return copy_out(s, buf, cap, len);
}

}  // extern "C"
