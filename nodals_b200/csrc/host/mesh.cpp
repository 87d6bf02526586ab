#include "mesh.hpp"

#include <algorithm>
#include <cerrno>
#ifdef _OPENMP
#include <parallel/algorithm>
#endif
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <unordered_map>

namespace nds {

const char* const kCanonicalPatches[3] = {"patch_0_0", "patch_2_0", "patch_1_0"};

int Mesh::patch_index(const std::string& name) const {
  for (size_t i = 0; i < patches.size(); ++i)
    if (patches[i].name == name) return (int)i;
  return -1;
}

double det3(const double J[3][3]) {
  return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
         J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
         J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}

void inv3(const double J[3][3], double I[3][3]) {
  const double d = det3(J);
  if (std::abs(d) < 1e-30) throw std::runtime_error("singular tetrahedron");
  I[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / d;
  I[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / d;
  I[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / d;
  I[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / d;
  I[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / d;
  I[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / d;
  I[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / d;
  I[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / d;
  I[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / d;
}

void tet_jacobian(const Mesh& m, const std::array<int32_t, 4>& t, double J[3][3]) {
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) J[r][k] = m.xyz[3 * (size_t)t[k + 1] + r] - m.xyz[3 * (size_t)t[0] + r];
}

namespace {

// ---------------------------------------------------------------------------
// cells from faces (the reference reader's rule)
// ---------------------------------------------------------------------------
void build_cells(Mesh& m) {
  if (m.owner.size() != m.faces.size()) throw std::runtime_error("owner size != faces size");
  int maxc = -1;
  for (int32_t c : m.owner) maxc = std::max(maxc, (int)c);
  for (int32_t c : m.neighbour) maxc = std::max(maxc, (int)c);
  const int nc = maxc + 1;
  if (nc <= 0) throw std::runtime_error("mesh has no cells");
  std::vector<int32_t> cnt((size_t)nc + 1, 0);
  for (int32_t c : m.owner) ++cnt[(size_t)c + 1];
  for (int32_t c : m.neighbour) ++cnt[(size_t)c + 1];
  for (int c = 0; c < nc; ++c) cnt[(size_t)c + 1] += cnt[(size_t)c];
  std::vector<int32_t> cf((size_t)cnt[(size_t)nc]);
  std::vector<int32_t> pos(cnt.begin(), cnt.end() - 1);
  for (int f = 0; f < (int)m.owner.size(); ++f) cf[(size_t)pos[(size_t)m.owner[(size_t)f]]++] = f;
  for (int f = 0; f < (int)m.neighbour.size(); ++f) cf[(size_t)pos[(size_t)m.neighbour[(size_t)f]]++] = f;
  m.tets.assign((size_t)nc, {});
  m.opp.assign((size_t)nc, {});
  for (int c = 0; c < nc; ++c) {
    const int b = cnt[(size_t)c], e = cnt[(size_t)c + 1];
    if (e - b != 4) throw std::runtime_error("non-tetrahedral cell " + std::to_string(c));
    int32_t vs[12];
    int k = 0;
    for (int q = b; q < e; ++q)
      for (int j = 0; j < 3; ++j) vs[k++] = m.faces[(size_t)cf[(size_t)q]][(size_t)j];
    std::sort(vs, vs + 12);
    int u = (int)(std::unique(vs, vs + 12) - vs);
    if (u != 4) throw std::runtime_error("tetrahedron vertex count mismatch in cell " + std::to_string(c));
    std::array<int32_t, 4> t{vs[0], vs[1], vs[2], vs[3]};
    double J[3][3];
    tet_jacobian(m, t, J);
    if (det3(J) < 0) std::swap(t[1], t[2]);
    m.tets[(size_t)c] = t;
    for (int i = 0; i < 4; ++i) {
      int found = -1;
      for (int q = b; q < e; ++q) {
        const auto& F = m.faces[(size_t)cf[(size_t)q]];
        if (F[0] != t[(size_t)i] && F[1] != t[(size_t)i] && F[2] != t[(size_t)i]) {
          if (found >= 0) throw std::runtime_error("multiple opposite faces in cell " + std::to_string(c));
          found = cf[(size_t)q];
        }
      }
      if (found < 0) throw std::runtime_error("missing opposite face in cell " + std::to_string(c));
      m.opp[(size_t)c][(size_t)i] = found;
    }
  }
  m.face_patch.assign(m.faces.size(), -1);
  for (int p = 0; p < (int)m.patches.size(); ++p) {
    const auto& P = m.patches[(size_t)p];
    for (int f = P.start; f < P.start + P.count; ++f) {
      if (f < 0 || f >= (int)m.faces.size()) throw std::runtime_error("patch range out of bounds");
      m.face_patch[(size_t)f] = p;
    }
  }
}

// ---------------------------------------------------------------------------
// canonical faces for meshes given as cells + tagged boundary triangles
// ---------------------------------------------------------------------------
struct FaceRec {
  int32_t a, b, c, cell;
};
inline bool tri_less(const FaceRec& x, const FaceRec& y) {
  if (x.a != y.a) return x.a < y.a;
  if (x.b != y.b) return x.b < y.b;
  if (x.c != y.c) return x.c < y.c;
  return x.cell < y.cell;
}
inline void sort3(int32_t& a, int32_t& b, int32_t& c) {
  if (a > b) std::swap(a, b);
  if (b > c) std::swap(b, c);
  if (a > b) std::swap(a, b);
}

void canonical_faces(Mesh& m, const std::vector<std::array<int32_t, 4>>& cells,
                     const std::vector<std::array<int32_t, 3>>& btri, const std::vector<int32_t>& bpatch,
                     int npatch) {
  const int nc = (int)cells.size();
  std::vector<FaceRec> f;
  f.reserve((size_t)nc * 4);
  static const int L[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
  for (int c = 0; c < nc; ++c)
    for (int k = 0; k < 4; ++k) {
      FaceRec r{cells[(size_t)c][(size_t)L[k][0]], cells[(size_t)c][(size_t)L[k][1]], cells[(size_t)c][(size_t)L[k][2]], c};
      sort3(r.a, r.b, r.c);
      f.push_back(r);
    }
  // the keys are unique up to the two cells of an internal face, whose order
  // the pairing below does not use: a parallel sort gives the same faces
#ifdef _OPENMP
  __gnu_parallel::sort(f.begin(), f.end(), tri_less);
#else
  std::sort(f.begin(), f.end(), tri_less);
#endif
  struct Internal { int32_t own, nei, a, b, c; };
  std::vector<Internal> in;
  std::vector<FaceRec> bd;
  in.reserve(f.size() / 2);
  for (size_t i = 0; i < f.size();) {
    size_t j = i + 1;
    while (j < f.size() && f[j].a == f[i].a && f[j].b == f[i].b && f[j].c == f[i].c) ++j;
    if (j - i == 2) {
      in.push_back({std::min(f[i].cell, f[i + 1].cell), std::max(f[i].cell, f[i + 1].cell), f[i].a, f[i].b, f[i].c});
    } else if (j - i == 1) {
      bd.push_back(f[i]);
    } else {
      throw std::runtime_error("non-manifold face shared by more than two cells");
    }
    i = j;
  }
  // (owner, neighbour) pairs are unique
  const auto own_nei = [](const Internal& x, const Internal& y) {
    return x.own != y.own ? x.own < y.own : x.nei < y.nei;
  };
#ifdef _OPENMP
  __gnu_parallel::sort(in.begin(), in.end(), own_nei);
#else
  std::sort(in.begin(), in.end(), own_nei);
#endif
  // boundary tags
  std::vector<FaceRec> tags(btri.size());
  for (size_t i = 0; i < btri.size(); ++i) {
    FaceRec r{btri[i][0], btri[i][1], btri[i][2], bpatch[i]};
    sort3(r.a, r.b, r.c);
    if (r.cell < 0 || r.cell >= npatch) throw std::runtime_error("boundary triangle patch index out of range");
    tags[i] = r;
  }
  std::sort(tags.begin(), tags.end(), tri_less);
  if (tags.size() != bd.size())
    throw std::runtime_error("tagged boundary triangles (" + std::to_string(tags.size()) +
                             ") do not match the mesh boundary (" + std::to_string(bd.size()) + ")");
  struct Bnd { int32_t patch, own, a, b, c; };
  std::vector<Bnd> bb(bd.size());
  for (size_t i = 0; i < bd.size(); ++i) {
    auto it = std::lower_bound(tags.begin(), tags.end(), FaceRec{bd[i].a, bd[i].b, bd[i].c, INT_MIN}, tri_less);
    if (it == tags.end() || it->a != bd[i].a || it->b != bd[i].b || it->c != bd[i].c)
      throw std::runtime_error("boundary face without a patch tag");
    bb[i] = {it->cell, bd[i].cell, bd[i].a, bd[i].b, bd[i].c};
  }
  std::sort(bb.begin(), bb.end(), [](const Bnd& x, const Bnd& y) {
    if (x.patch != y.patch) return x.patch < y.patch;
    if (x.own != y.own) return x.own < y.own;
    if (x.a != y.a) return x.a < y.a;
    if (x.b != y.b) return x.b < y.b;
    return x.c < y.c;
  });
  m.faces.clear();
  m.owner.clear();
  m.neighbour.clear();
  m.faces.reserve(in.size() + bb.size());
  for (const auto& q : in) {
    m.faces.push_back({q.a, q.b, q.c});
    m.owner.push_back(q.own);
    m.neighbour.push_back(q.nei);
  }
  std::vector<int> count((size_t)npatch, 0);
  for (const auto& q : bb) {
    m.faces.push_back({q.a, q.b, q.c});
    m.owner.push_back(q.own);
    ++count[(size_t)q.patch];
  }
  int s = (int)in.size();
  for (int p = 0; p < npatch; ++p) {
    m.patches[(size_t)p].start = s;
    m.patches[(size_t)p].count = count[(size_t)p];
    s += count[(size_t)p];
  }
  // orient every face out of its owner
  for (size_t i = 0; i < m.faces.size(); ++i) {
    auto& F = m.faces[i];
    const auto& t = cells[(size_t)m.owner[i]];
    double cc[3] = {0, 0, 0}, fc[3], e1[3], e2[3], n[3];
    for (int k = 0; k < 4; ++k)
      for (int d = 0; d < 3; ++d) cc[d] += 0.25 * m.xyz[3 * (size_t)t[(size_t)k] + d];
    for (int d = 0; d < 3; ++d) {
      const double a = m.xyz[3 * (size_t)F[0] + d], b = m.xyz[3 * (size_t)F[1] + d], c = m.xyz[3 * (size_t)F[2] + d];
      fc[d] = (a + b + c) / 3.0;
      e1[d] = b - a;
      e2[d] = c - a;
    }
    n[0] = e1[1] * e2[2] - e1[2] * e2[1];
    n[1] = e1[2] * e2[0] - e1[0] * e2[2];
    n[2] = e1[0] * e2[1] - e1[1] * e2[0];
    if (n[0] * (fc[0] - cc[0]) + n[1] * (fc[1] - cc[1]) + n[2] * (fc[2] - cc[2]) < 0) std::swap(F[1], F[2]);
  }
}

// ---------------------------------------------------------------------------
// OpenFOAM ASCII tokenizer
// ---------------------------------------------------------------------------
class FoamScanner {
 public:
  explicit FoamScanner(const std::string& path) : path_(path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("cannot open " + path);
    std::ostringstream ss;
    ss << in.rdbuf();
    buf_ = ss.str();
  }
  // next token: punctuation ( ) { } ; as single chars, quoted strings, words
  bool next(std::string& tok) {
    skip();
    if (p_ >= buf_.size()) return false;
    const char c = buf_[p_];
    if (c == '(' || c == ')' || c == '{' || c == '}' || c == ';') {
      tok.assign(1, c);
      ++p_;
      return true;
    }
    if (c == '"') {
      size_t e = buf_.find('"', p_ + 1);
      if (e == std::string::npos) throw std::runtime_error("unterminated quote in " + path_);
      tok = buf_.substr(p_ + 1, e - p_ - 1);
      p_ = e + 1;
      return true;
    }
    size_t b = p_;
    while (p_ < buf_.size()) {
      const char d = buf_[p_];
      if (std::isspace((unsigned char)d) || d == '(' || d == ')' || d == '{' || d == '}' || d == ';') break;
      if (d == '/' && p_ + 1 < buf_.size() && (buf_[p_ + 1] == '/' || buf_[p_ + 1] == '*')) break;
      ++p_;
    }
    tok.assign(buf_, b, p_ - b);
    return true;
  }
  std::string need() {
    std::string t;
    if (!next(t)) throw std::runtime_error("unexpected end of " + path_);
    return t;
  }
  void expect(const char* w) {
    std::string t = need();
    if (t != w) throw std::runtime_error("expected '" + std::string(w) + "' but got '" + t + "' in " + path_);
  }
  long long integer() {
    std::string t = need();
    char* e = nullptr;
    errno = 0;
    long long v = std::strtoll(t.c_str(), &e, 10);
    if (errno || !e || *e) throw std::runtime_error("invalid integer '" + t + "' in " + path_);
    return v;
  }
  double real() {
    std::string t = need();
    char* e = nullptr;
    errno = 0;
    double v = std::strtod(t.c_str(), &e);
    if (errno || !e || *e) throw std::runtime_error("invalid number '" + t + "' in " + path_);
    return v;
  }
  // first "N (" pair outside the FoamFile header dictionary
  int list_start() {
    std::string t, prev;
    int depth = 0;
    while (next(t)) {
      if (t == "{") { ++depth; continue; }
      if (t == "}") { --depth; continue; }
      if (depth == 0 && t == "(" && !prev.empty()) {
        char* e = nullptr;
        long long v = std::strtoll(prev.c_str(), &e, 10);
        if (e && !*e && v >= 0 && v <= INT_MAX) return (int)v;
      }
      prev = t;
    }
    throw std::runtime_error("cannot find list count in " + path_);
  }
  const std::string& path() const { return path_; }

 private:
  void skip() {
    while (p_ < buf_.size()) {
      const char c = buf_[p_];
      if (std::isspace((unsigned char)c)) { ++p_; continue; }
      if (c == '/' && p_ + 1 < buf_.size() && buf_[p_ + 1] == '/') {
        while (p_ < buf_.size() && buf_[p_] != '\n') ++p_;
        continue;
      }
      if (c == '/' && p_ + 1 < buf_.size() && buf_[p_ + 1] == '*') {
        size_t e = buf_.find("*/", p_ + 2);
        if (e == std::string::npos) throw std::runtime_error("unterminated comment in " + path_);
        p_ = e + 2;
        continue;
      }
      break;
    }
  }
  std::string path_, buf_;
  size_t p_ = 0;
};

}  // namespace

Mesh read_polymesh(const std::string& dirIn) {
  std::string dir = dirIn;
  while (dir.size() > 1 && dir.back() == '/') dir.pop_back();
  Mesh m;
  {
    FoamScanner s(dir + "/points");
    const int n = s.list_start();
    m.xyz.resize(3 * (size_t)n);
    for (int i = 0; i < n; ++i) {
      s.expect("(");
      for (int d = 0; d < 3; ++d) m.xyz[3 * (size_t)i + d] = s.real();
      s.expect(")");
    }
    s.expect(")");
  }
  {
    FoamScanner s(dir + "/faces");
    const int n = s.list_start();
    m.faces.resize((size_t)n);
    for (int i = 0; i < n; ++i) {
      if (s.integer() != 3) throw std::runtime_error("non-triangular face in " + s.path());
      s.expect("(");
      for (int j = 0; j < 3; ++j) {
        long long v = s.integer();
        if (v < 0 || v >= m.n_points()) throw std::runtime_error("face vertex out of range in " + s.path());
        m.faces[(size_t)i][(size_t)j] = (int32_t)v;
      }
      s.expect(")");
    }
    s.expect(")");
  }
  auto labels = [&](const std::string& name, std::vector<int32_t>& out) {
    FoamScanner s(dir + "/" + name);
    const int n = s.list_start();
    out.resize((size_t)n);
    for (int i = 0; i < n; ++i) {
      long long v = s.integer();
      if (v < INT_MIN || v > INT_MAX) throw std::runtime_error("label out of range in " + s.path());
      out[(size_t)i] = (int32_t)v;
    }
    s.expect(")");
  };
  labels("owner", m.owner);
  labels("neighbour", m.neighbour);
  {
    FoamScanner s(dir + "/boundary");
    const int n = s.list_start();
    for (int i = 0; i < n; ++i) {
      Patch P;
      P.name = s.need();
      if (P.name == ")") throw std::runtime_error("missing patch name in " + s.path());
      s.expect("{");
      long long nf = -1, sf = -1;
      int depth = 1;
      while (depth) {
        std::string t = s.need();
        if (t == "{") { ++depth; continue; }
        if (t == "}") { --depth; continue; }
        if (depth != 1) continue;
        if (t == "nFaces") { nf = s.integer(); s.expect(";"); }
        else if (t == "startFace") { sf = s.integer(); s.expect(";"); }
      }
      if (nf < 0 || sf < 0) throw std::runtime_error("invalid patch range " + P.name);
      P.start = (int)sf;
      P.count = (int)nf;
      m.patches.push_back(P);
    }
    s.expect(")");
  }
  build_cells(m);
  return m;
}

Mesh mesh_from_arrays(int np, const double* xyz, int nc, const int32_t* tets, int nb, const int32_t* btri,
                      const int32_t* bpatch, const std::vector<std::string>& patch_names) {
  if (np <= 0 || nc <= 0 || nb <= 0) throw std::runtime_error("mesh arrays are empty");
  Mesh m;
  m.xyz.assign(xyz, xyz + 3 * (size_t)np);
  std::vector<std::array<int32_t, 4>> cells((size_t)nc);
  for (int c = 0; c < nc; ++c)
    for (int k = 0; k < 4; ++k) {
      const int32_t v = tets[4 * (size_t)c + k];
      if (v < 0 || v >= np) throw std::runtime_error("tetrahedron vertex out of range");
      cells[(size_t)c][(size_t)k] = v;
    }
  std::vector<std::array<int32_t, 3>> tri((size_t)nb);
  std::vector<int32_t> tag((size_t)nb);
  for (int i = 0; i < nb; ++i) {
    for (int k = 0; k < 3; ++k) {
      const int32_t v = btri[3 * (size_t)i + k];
      if (v < 0 || v >= np) throw std::runtime_error("boundary vertex out of range");
      tri[(size_t)i][(size_t)k] = v;
    }
    tag[(size_t)i] = bpatch[i];
  }
  for (const auto& n : patch_names) m.patches.push_back({n, 0, 0});
  canonical_faces(m, cells, tri, tag, (int)patch_names.size());
  build_cells(m);
  return m;
}

Mesh read_msh2(const std::string& path) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("cannot open " + path);
  std::string line;
  std::unordered_map<long long, int> id2idx;
  std::vector<double> xyz;
  std::vector<int32_t> tets, btri, bpatch;
  bool fmt = false;
  while (std::getline(in, line)) {
    if (line.rfind("$MeshFormat", 0) == 0) {
      std::getline(in, line);
      std::istringstream h(line);
      double ver = 0;
      int ft = -1;
      h >> ver >> ft;
      if (!(ver >= 2.0 && ver < 3.0) || ft != 0) throw std::runtime_error("MSH reader supports ASCII format 2.x only: " + path);
      fmt = true;
    } else if (line.rfind("$Nodes", 0) == 0) {
      long long n = 0;
      in >> n;
      xyz.resize(3 * (size_t)n);
      for (long long i = 0; i < n; ++i) {
        long long id;
        in >> id >> xyz[3 * (size_t)i] >> xyz[3 * (size_t)i + 1] >> xyz[3 * (size_t)i + 2];
        if (!in) throw std::runtime_error("bad $Nodes block in " + path);
        id2idx[id] = (int)i;
      }
    } else if (line.rfind("$Elements", 0) == 0) {
      long long n = 0;
      in >> n;
      for (long long e = 0; e < n; ++e) {
        long long id, type, ntag;
        in >> id >> type >> ntag;
        std::vector<long long> tg((size_t)std::max(0LL, ntag));
        for (auto& q : tg) in >> q;
        int nn = (type == 4) ? 4 : (type == 2) ? 3 : (type == 15) ? 1 : (type == 1) ? 2 : -1;
        if (nn < 0) throw std::runtime_error("unsupported MSH element type " + std::to_string(type) + " in " + path);
        long long v[4];
        for (int k = 0; k < nn; ++k) in >> v[k];
        if (!in) throw std::runtime_error("bad $Elements block in " + path);
        const long long phys = tg.empty() ? 0 : tg[0];
        auto idx = [&](long long q) {
          auto it = id2idx.find(q);
          if (it == id2idx.end()) throw std::runtime_error("element references unknown node in " + path);
          return (int32_t)it->second;
        };
        if (type == 4) {
          for (int k = 0; k < 4; ++k) tets.push_back(idx(v[k]));
        } else if (type == 2) {
          int p = -1;
          if (phys == 3) p = 0;       // wall   -> patch_0_0
          else if (phys == 1) p = 1;  // inlet  -> patch_2_0
          else if (phys == 2) p = 2;  // outlet -> patch_1_0
          else throw std::runtime_error("boundary triangle with unknown physical tag " + std::to_string(phys));
          for (int k = 0; k < 3; ++k) btri.push_back(idx(v[k]));
          bpatch.push_back(p);
        }
      }
    }
  }
  if (!fmt) throw std::runtime_error("missing $MeshFormat in " + path);
  if (tets.empty()) throw std::runtime_error("no tetrahedra in " + path);
  std::vector<std::string> names(kCanonicalPatches, kCanonicalPatches + 3);
  return mesh_from_arrays((int)(xyz.size() / 3), xyz.data(), (int)(tets.size() / 4), tets.data(),
                          (int)bpatch.size(), btri.data(), bpatch.data(), names);
}

// HXT1 layout (hxt1_mesh.hpp:19-103, writer hybrid_hxt1/prepare_hxt1.py):
// 8-byte magic, u32 version, u32 reserved, 13 u64 counts
//   nv nhex ntet nhexface ntetface nvel npressure ninterface
//   nwallhex ninhex nintet nouthex nouttet,
// then, little-endian and packed: points (3 f64), hexes (8 i32), tets (4 i32),
// hex velocity dofs (14 i32), tet velocity dofs (8 i32), hex and tet
// pressure ids (i32), hex geometry (82 f64), tet geometry (12 f64),
// interface records (9 i32) and the wall-hex, inlet-hex, inlet-tet,
// outlet-hex, outlet-tet boundary records (cell, local face, bubble: 3 i32),
// and nothing after them.  Local face lf of a tet is its vertices
// kTetFace[lf] (the face opposite vertex lf).
Mesh read_hxt1(const std::string& path) {
  static const int kTetFace[4][3] = {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}};
  std::ifstream in(path, std::ios::binary);
  if (!in) throw std::runtime_error("cannot open " + path);
  char magic[8];
  in.read(magic, 8);
  if (!in || std::memcmp(magic, "HXT1BIN1", 8) != 0) throw std::runtime_error("bad HXT1 magic in " + path);
  uint32_t version = 0, reserved = 0;
  in.read(reinterpret_cast<char*>(&version), 4);
  in.read(reinterpret_cast<char*>(&reserved), 4);
  if (!in) throw std::runtime_error("short read: HXT1 version in " + path);
  if (version != 1) throw std::runtime_error("unsupported HXT1 version " + std::to_string(version) + " in " + path);
  uint64_t h[13];
  in.read(reinterpret_cast<char*>(h), sizeof(h));
  if (!in) throw std::runtime_error("short read: HXT1 header counts in " + path);
  const uint64_t nv = h[0], nhex = h[1], ntet = h[2], nwallhex = h[8], ninhex = h[9], nintet = h[10],
                 nouthex = h[11], nouttet = h[12], ninterface = h[7];
  if (nhex || ninterface || nwallhex || ninhex || nouthex)
    throw std::runtime_error("HXT1 mesh " + path + " has " + std::to_string(nhex) +
                             " hex cells: the tetrahedral solver needs a pure-tet HXT1 file");
  if (ntet == 0) throw std::runtime_error("no tetrahedra in " + path);
  if (nv > (uint64_t)INT32_MAX || ntet > (uint64_t)INT32_MAX) throw std::runtime_error("HXT1 mesh too large: " + path);
  auto read = [&](void* dst, uint64_t n, size_t size, const char* what) {
    if (n) in.read(reinterpret_cast<char*>(dst), (std::streamsize)(n * size));
    if (!in) throw std::runtime_error(std::string("short read: HXT1 ") + what + " in " + path);
  };
  auto skip = [&](uint64_t n, size_t size, const char* what) {
    std::vector<char> junk(n * size);
    read(junk.data(), n, size, what);
  };
  std::vector<double> xyz(3 * (size_t)nv);
  read(xyz.data(), nv, 3 * sizeof(double), "points");
  std::vector<int32_t> tets(4 * (size_t)ntet);
  read(tets.data(), ntet, 4 * sizeof(int32_t), "tets");
  skip(ntet, 8 * sizeof(int32_t), "tet velocity dofs");
  skip(ntet, sizeof(int32_t), "tet pressure ids");
  skip(ntet, 12 * sizeof(double), "tet geometry");
  std::vector<int32_t> inrec(3 * (size_t)nintet), outrec(3 * (size_t)nouttet);
  read(inrec.data(), nintet, 3 * sizeof(int32_t), "inlet tet records");
  read(outrec.data(), nouttet, 3 * sizeof(int32_t), "outlet tet records");
  char extra = 0;
  in.read(&extra, 1);
  if (in.gcount() != 0) throw std::runtime_error("trailing bytes in HXT1 mesh " + path);
  for (int32_t v : tets)
    if (v < 0 || (uint64_t)v >= nv) throw std::runtime_error("HXT1 tet references an unknown point in " + path);
  // exterior faces: used by exactly one tet
  using Key = std::array<int32_t, 3>;
  auto key_of = [&](int c, int lf) {
    Key k{tets[4 * (size_t)c + kTetFace[lf][0]], tets[4 * (size_t)c + kTetFace[lf][1]],
          tets[4 * (size_t)c + kTetFace[lf][2]]};
    std::sort(k.begin(), k.end());
    return k;
  };
  std::vector<std::pair<Key, int64_t>> all;  // face, 4 cell + lf
  all.reserve(4 * (size_t)ntet);
  for (int c = 0; c < (int)ntet; ++c)
    for (int lf = 0; lf < 4; ++lf) all.push_back({key_of(c, lf), 4 * (int64_t)c + lf});
  std::sort(all.begin(), all.end());
  std::vector<int8_t> label(4 * (size_t)ntet, -1);  // patch of each exterior (cell, lf); -2 interior
  for (size_t a = 0; a < all.size();) {
    size_t b = a;
    while (b < all.size() && all[b].first == all[a].first) ++b;
    if (b - a > 2) throw std::runtime_error("non-manifold face in HXT1 mesh " + path);
    for (size_t q = a; q < b; ++q) label[(size_t)all[q].second] = (b - a == 1) ? 0 : -2;  // exterior: wall unless tagged
    a = b;
  }
  auto tag = [&](const std::vector<int32_t>& rec, int patch, const char* what) {
    for (size_t r = 0; r < rec.size() / 3; ++r) {
      const int32_t c = rec[3 * r], lf = rec[3 * r + 1];
      if (c < 0 || (uint64_t)c >= ntet || lf < 0 || lf > 3)
        throw std::runtime_error(std::string("HXT1 ") + what + " record out of range in " + path);
      int8_t& l = label[4 * (size_t)c + (size_t)lf];
      if (l != 0) throw std::runtime_error(std::string("HXT1 ") + what + " face is not an untagged exterior face in " + path);
      l = (int8_t)patch;
    }
  };
  tag(inrec, 1, "inlet");
  tag(outrec, 2, "outlet");
  std::vector<int32_t> btri, bpatch;
  for (int c = 0; c < (int)ntet; ++c)
    for (int lf = 0; lf < 4; ++lf) {
      const int8_t l = label[4 * (size_t)c + (size_t)lf];
      if (l < 0) continue;
      for (int k = 0; k < 3; ++k) btri.push_back(tets[4 * (size_t)c + kTetFace[lf][k]]);
      bpatch.push_back(l);
    }
  std::vector<std::string> names(kCanonicalPatches, kCanonicalPatches + 3);
  return mesh_from_arrays((int)nv, xyz.data(), (int)ntet, tets.data(), (int)bpatch.size(), btri.data(), bpatch.data(),
                          names);
}

}  // namespace nds
