#include "hybrid.hpp"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <fstream>
#include <map>
#include <stdexcept>
#include <tuple>

#include "../../../include/nodals_b200.h"
#include "fem.hpp"

namespace nds {
namespace {

// Reference hexahedron [-1,1]^3: vertex a sits at kHexSign[a]; local face f
// is kHexFace[f] (z-, z+, y-, x+, y+, x-), bubble 8 + f lives on it.  A
// tet's local face lf is kTetFace[lf], the face opposite vertex lf.
// (hybrid_hxt2/hxt2_main.cu:18-27, hybrid_hxt1/prepare_hxt1.py)
const int kHexSign[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                            {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
const int kHexFace[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}};
const int kTetFace[4][3] = {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}};

// trilinear (Q1) values and reference gradients
void hex_q1(double x, double y, double z, double phi[8], double g[8][3]) {
  for (int a = 0; a < 8; ++a) {
    const double sx = kHexSign[a][0], sy = kHexSign[a][1], sz = kHexSign[a][2];
    const double ax = 1.0 + sx * x, ay = 1.0 + sy * y, az = 1.0 + sz * z;
    phi[a] = 0.125 * ax * ay * az;
    g[a][0] = 0.125 * sx * ay * az;
    g[a][1] = 0.125 * sy * ax * az;
    g[a][2] = 0.125 * sz * ax * ay;
  }
}

// Q1 + BF2: the bubble of face f is the Q1 factor of the face-normal
// coordinate that is 1 on f times the quadratic bubbles (1 - t^2) of the two
// tangential coordinates (value 1 at the face centre, 1/2 at the cell centre)
// (hybrid_hxt2/hxt2_main.cu:176-187, prepare_hxt1.py bf2_value)
void hex_basis(double x, double y, double z, double phi[14], double g[14][3]) {
  hex_q1(x, y, z, phi, g);
  const double bx = 1 - x * x, by = 1 - y * y, bz = 1 - z * z;
  const double dx = -2 * x, dy = -2 * y, dz = -2 * z;
  // normal coordinate n in {x, y, z}, side sgn = -1 / +1
  auto face = [&](int f, int n, double sgn) {
    const double c[3] = {x, y, z}, b[3] = {bx, by, bz}, d[3] = {dx, dy, dz};
    const int t1 = n == 0 ? 1 : 0, t2 = n == 2 ? 1 : 2;
    const double s = 0.5 * (1.0 + sgn * c[n]);
    phi[8 + f] = s * b[t1] * b[t2];
    g[8 + f][n] = 0.5 * sgn * b[t1] * b[t2];
    g[8 + f][t1] = s * d[t1] * b[t2];
    g[8 + f][t2] = s * b[t1] * d[t2];
  };
  face(0, 2, -1.0);
  face(1, 2, 1.0);
  face(2, 1, -1.0);
  face(3, 0, 1.0);
  face(4, 1, 1.0);
  face(5, 0, -1.0);
}

// J^-1 (row-major, I[3 j + d] = d xi_j / d x_d) and det J at (x, y, z)
void hex_metric(const HybridMesh& m, int c, double x, double y, double z, double I[9], double& det) {
  double phi[8], g[8][3];
  hex_q1(x, y, z, phi, g);
  double J[9] = {};
  for (int a = 0; a < 8; ++a) {
    const double* p = &m.xyz[3 * (size_t)m.hexes[(size_t)c][(size_t)a]];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) J[3 * i + j] += p[i] * g[a][j];
  }
  det = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) + J[2] * (J[3] * J[7] - J[4] * J[6]);
  if (!(det > 0)) throw std::runtime_error("hybrid mesh: non-positive hex Jacobian in cell " + std::to_string(c));
  const double q = 1.0 / det;
  I[0] = (J[4] * J[8] - J[5] * J[7]) * q;
  I[1] = (J[2] * J[7] - J[1] * J[8]) * q;
  I[2] = (J[1] * J[5] - J[2] * J[4]) * q;
  I[3] = (J[5] * J[6] - J[3] * J[8]) * q;
  I[4] = (J[0] * J[8] - J[2] * J[6]) * q;
  I[5] = (J[2] * J[3] - J[0] * J[5]) * q;
  I[6] = (J[3] * J[7] - J[4] * J[6]) * q;
  I[7] = (J[1] * J[6] - J[0] * J[7]) * q;
  I[8] = (J[0] * J[4] - J[1] * J[3]) * q;
}

template <int N>
void phys_grad(const double g[][3], const double I[9], double gp[][3]) {
  for (int a = 0; a < N; ++a)
    for (int d = 0; d < 3; ++d) gp[a][d] = g[a][0] * I[d] + g[a][1] * I[3 + d] + g[a][2] * I[6 + d];
}

struct V3 {
  double x, y, z;
};
V3 point(const HybridMesh& m, int v) { return {m.xyz[3 * (size_t)v], m.xyz[3 * (size_t)v + 1], m.xyz[3 * (size_t)v + 2]}; }
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
double tri_area(V3 a, V3 b, V3 c) { return 0.5 * std::sqrt(dot(cross(sub(b, a), sub(c, a)), cross(sub(b, a), sub(c, a)))); }
V3 hex_centroid(const HybridMesh& m, int c) {
  V3 q{0, 0, 0};
  for (int a = 0; a < 8; ++a) {
    const V3 p = point(m, m.hexes[(size_t)c][(size_t)a]);
    q = {q.x + p.x, q.y + p.y, q.z + p.z};
  }
  return {q.x / 8, q.y / 8, q.z / 8};
}
V3 tet_centroid(const HybridMesh& m, int c) {
  V3 q{0, 0, 0};
  for (int a = 0; a < 4; ++a) {
    const V3 p = point(m, m.tets[(size_t)c][(size_t)a]);
    q = {q.x + p.x, q.y + p.y, q.z + p.z};
  }
  return {q.x / 4, q.y / 4, q.z / 4};
}

// tensor-product rules: 3-point Gauss on [-1,1] for hex volumes; the
// collapsed 5 x 5 rule on interface triangles (Gauss-Legendre on [0,1] in
// both directions, weight (1 - r) folded in by the Duffy map)
struct Rules {
  double g3x[3], g3w[3];
  std::vector<double> q5x, q5w;
  Rules() {
    const double a = std::sqrt(0.6);
    g3x[0] = -a; g3x[1] = 0.0; g3x[2] = a;
    g3w[0] = 5.0 / 9.0; g3w[1] = 8.0 / 9.0; g3w[2] = 5.0 / 9.0;
    gauss_jacobi01(5, 0, q5x, q5w);
  }
};
const Rules& rules() {
  static const Rules r;
  return r;
}

// The 25 points of interface triangle s of plan p, each with the hex and
// tet basis values and physical gradients there.
template <class F>
void for_interface_points(const HybridMesh& m, const InterfacePlan& p, int s, F&& f) {
  const Rules& R = rules();
  const auto& tg = m.tet_geom[(size_t)p.tet_cell[s]];
  for (int ia = 0; ia < 5; ++ia)
    for (int ib = 0; ib < 5; ++ib) {
      const double rr = R.q5x[(size_t)ia], ss = R.q5x[(size_t)ib], om = 1.0 - rr;
      const double L[3] = {om * (1.0 - ss), rr, om * ss};
      const double w = R.q5w[(size_t)ia] * R.q5w[(size_t)ib] * om * 2.0 * p.area_tri[s];
      double xr = 0, yr = 0, zr = 0;
      for (int k = 0; k < 3; ++k) {
        const int hl = p.hex_tri_local[s][k];
        xr += L[k] * kHexSign[hl][0];
        yr += L[k] * kHexSign[hl][1];
        zr += L[k] * kHexSign[hl][2];
      }
      double ph[14], gh[14][3], gph[14][3], I[9], det;
      hex_basis(xr, yr, zr, ph, gh);
      hex_metric(m, p.hex_cell, xr, yr, zr, I, det);
      phys_grad<14>(gh, I, gph);
      std::array<double, 4> lam{0, 0, 0, 0};
      for (int k = 0; k < 3; ++k) lam[(size_t)kTetFace[p.tet_face[s]][k]] = L[k];
      double pt[8], gt[8][3], gpt[8][3];
      basis_eval(lam, pt, gt);
      phys_grad<8>(gt, tg.data() + 3, gpt);
      f(w, ph, gph, pt, gpt);
    }
}

}  // namespace

HybridMesh read_hxt1_hybrid(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw std::runtime_error("cannot open " + path);
  char magic[8];
  in.read(magic, 8);
  if (!in || std::memcmp(magic, "HXT1BIN1", 8) != 0) throw std::runtime_error("bad HXT1 magic in " + path);
  uint32_t version = 0, reserved = 0;
  in.read(reinterpret_cast<char*>(&version), 4);
  in.read(reinterpret_cast<char*>(&reserved), 4);
  if (!in || version != 1) throw std::runtime_error("unsupported HXT1 version in " + path);
  HybridMesh m;
  in.read(reinterpret_cast<char*>(m.count), sizeof(m.count));
  if (!in) throw std::runtime_error("short read: HXT1 header counts in " + path);
  for (uint64_t c : m.count)
    if (c > (uint64_t)INT32_MAX) throw std::runtime_error("HXT1 mesh too large: " + path);
  auto read = [&](auto& v, uint64_t n, const char* what) {
    v.resize((size_t)n);
    if (n) in.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(n * sizeof(v[0])));
    if (!in) throw std::runtime_error(std::string("short read: HXT1 ") + what + " in " + path);
  };
  std::vector<int32_t> hp, tp;
  m.xyz.resize(3 * (size_t)m.count[0]);
  if (m.count[0]) in.read(reinterpret_cast<char*>(m.xyz.data()), (std::streamsize)(m.xyz.size() * sizeof(double)));
  if (!in) throw std::runtime_error("short read: HXT1 points in " + path);
  read(m.hexes, m.count[1], "hexes");
  read(m.tets, m.count[2], "tets");
  read(m.hex_dofs, m.count[1], "hex velocity dofs");
  read(m.tet_dofs, m.count[2], "tet velocity dofs");
  read(hp, m.count[1], "hex pressure ids");
  read(tp, m.count[2], "tet pressure ids");
  read(m.hex_geom, m.count[1], "hex geometry");
  read(m.tet_geom, m.count[2], "tet geometry");
  read(m.interface, m.count[7], "interface");
  read(m.wall_hex, m.count[8], "wall hex");
  read(m.in_hex, m.count[9], "inlet hex");
  read(m.in_tet, m.count[10], "inlet tet");
  read(m.out_hex, m.count[11], "outlet hex");
  read(m.out_tet, m.count[12], "outlet tet");
  char extra = 0;
  in.read(&extra, 1);
  if (in.gcount() != 0) throw std::runtime_error("trailing bytes in HXT1 mesh " + path);
  for (int c = 0; c < m.nhex(); ++c)
    if (hp[(size_t)c] != c) throw std::runtime_error("HXT1 hex pressure ids are not 0..nhex-1 in " + path);
  for (int c = 0; c < m.ntet(); ++c)
    if (tp[(size_t)c] != m.nhex() + c) throw std::runtime_error("HXT1 tet pressure ids do not follow the hexes in " + path);
  const int nvel = m.nvel();
  auto dofs_ok = [&](const int32_t* g, int n) {
    for (int a = 0; a < n; ++a)
      if (g[a] < 0 || g[a] >= nvel) return false;
    return true;
  };
  for (const auto& h : m.hex_dofs)
    if (!dofs_ok(h.data(), 14)) throw std::runtime_error("HXT1 hex velocity dof out of range in " + path);
  for (const auto& t : m.tet_dofs)
    if (!dofs_ok(t.data(), 8)) throw std::runtime_error("HXT1 tet velocity dof out of range in " + path);
  return m;
}

std::vector<InterfacePlan> interface_plans(const HybridMesh& m) {
  std::vector<InterfacePlan> P;
  P.reserve(m.interface.size());
  for (const auto& r : m.interface) {
    InterfacePlan p{};
    p.hex_cell = r[0];
    p.hex_face = r[1];
    p.tet_cell[0] = r[3];
    p.tet_face[0] = r[4];
    p.tet_cell[1] = r[6];
    p.tet_face[1] = r[7];
    if (p.hex_cell < 0 || p.hex_cell >= m.nhex() || p.hex_face < 0 || p.hex_face > 5)
      throw std::runtime_error("HXT1 interface record out of range");
    const auto& hc = m.hexes[(size_t)p.hex_cell];
    V3 q[4];
    for (int k = 0; k < 4; ++k) q[k] = point(m, hc[(size_t)kHexFace[p.hex_face][k]]);
    p.area_quad = tri_area(q[0], q[1], q[2]) + tri_area(q[0], q[2], q[3]);
    V3 n = cross(sub(q[1], q[0]), sub(q[3], q[0]));
    const double nn = std::sqrt(dot(n, n));
    if (!(nn > 0)) throw std::runtime_error("hybrid mesh: zero interface quad normal");
    n = {n.x / nn, n.y / nn, n.z / nn};
    if (p.tet_cell[0] < 0 || p.tet_cell[0] >= m.ntet() || p.tet_cell[1] < 0 || p.tet_cell[1] >= m.ntet())
      throw std::runtime_error("HXT1 interface record out of range");
    if (dot(n, sub(tet_centroid(m, p.tet_cell[0]), hex_centroid(m, p.hex_cell))) < 0) n = {-n.x, -n.y, -n.z};
    p.normal[0] = n.x;
    p.normal[1] = n.y;
    p.normal[2] = n.z;
    const double vh = m.hex_geom[(size_t)p.hex_cell][0];
    if (!(vh > 0)) throw std::runtime_error("hybrid mesh: non-positive hex volume");
    p.inv_h_hex = p.area_quad / (2.0 * vh);
    for (int s = 0; s < 2; ++s) {
      const auto& tc = m.tets[(size_t)p.tet_cell[s]];
      V3 tp[3];
      for (int k = 0; k < 3; ++k) {
        const int gv = tc[(size_t)kTetFace[p.tet_face[s]][k]];
        tp[k] = point(m, gv);
        int hl = -1;
        for (int a = 0; a < 8; ++a)
          if (hc[(size_t)a] == gv) hl = a;
        bool on_face = false;
        for (int a = 0; a < 4; ++a)
          if (kHexFace[p.hex_face][a] == hl) on_face = true;
        if (!on_face) throw std::runtime_error("hybrid mesh: interface triangle vertex not on its hex face");
        p.hex_tri_local[s][k] = hl;
      }
      p.area_tri[s] = tri_area(tp[0], tp[1], tp[2]);
      const double vt = m.tet_geom[(size_t)p.tet_cell[s]][0];
      if (!(vt > 0 && p.area_tri[s] > 0)) throw std::runtime_error("hybrid mesh: bad interface tet geometry");
      p.inv_h_tet[s] = p.area_tri[s] / (2.0 * vt);
    }
    if (std::abs(p.area_tri[0] + p.area_tri[1] - p.area_quad) > 1e-12 * p.area_quad)
      throw std::runtime_error("hybrid mesh: interface quad and triangle areas differ (non-planar quad)");
    P.push_back(p);
  }
  return P;
}

namespace {
// Velocity operator of diffusion and Nitsche coupling, merged into CSR
// (columns sorted; equal positions summed in generation order: hexes,
// tets, interface triangles).  diag_rau gets the diagonal without the
// Nitsche penalty.
struct Trip {
  int32_t r, c;
  double v;
};
// Stable sort of triplets by (row, column): a counting sort by row, then a
// stable sort of each row's run by column, so duplicates keep the order in
// which the cells produced them.
void sort_trips(std::vector<Trip>& t, int nrows) {
  std::vector<int64_t> off((size_t)nrows + 1, 0);
  for (const Trip& x : t) ++off[(size_t)x.r + 1];
  for (int r = 0; r < nrows; ++r) off[(size_t)r + 1] += off[(size_t)r];
  std::vector<Trip> o(t.size());
  {
    std::vector<int64_t> next(off.begin(), off.end() - 1);
    for (const Trip& x : t) o[(size_t)next[(size_t)x.r]++] = x;
  }
#pragma omp parallel for schedule(dynamic, 512)
  for (int r = 0; r < nrows; ++r)
    std::stable_sort(o.begin() + off[(size_t)r], o.begin() + off[(size_t)r + 1],
                     [](const Trip& x, const Trip& y) { return x.c < y.c; });
  t.swap(o);
}

// The element loops run in parallel, each cell (and interface triangle)
// writing its block into its own slots in cell order; the diagonal sums and
// the merge of duplicates then follow that order, as a serial loop would.
void assemble_velocity(const HybridMesh& m, const std::vector<InterfacePlan>& plans, double nu, double gamma,
                       std::vector<int32_t>& row, std::vector<int32_t>& col, std::vector<double>& val,
                       std::vector<double>& diag_rau, bool with_interface = true) {
  const Rules& R = rules();
  const int nv = m.nvel(), nh = m.nhex(), nt = m.ntet(), np2 = with_interface ? 2 * (int)plans.size() : 0;
  diag_rau.assign((size_t)nv, 0.0);
  // union of the hex's and the tet's unknowns of each interface triangle
  std::vector<std::array<int, 22>> iu((size_t)np2);
  std::vector<std::array<int, 14>> ihu((size_t)np2);
  std::vector<std::array<int, 8>> itu((size_t)np2);
  std::vector<int> inu((size_t)np2);
  std::vector<int64_t> ioff((size_t)np2 + 1, 0), coff((size_t)np2 + 1, 0);
  for (int k = 0; k < np2; ++k) {
    const InterfacePlan& p = plans[(size_t)(k / 2)];
    const auto& hg = m.hex_dofs[(size_t)p.hex_cell];
    const auto& tgd = m.tet_dofs[(size_t)p.tet_cell[k % 2]];
    int n = 0;
    for (int a = 0; a < 14; ++a) {
      ihu[(size_t)k][(size_t)a] = n;
      iu[(size_t)k][(size_t)n++] = hg[(size_t)a];
    }
    for (int b = 0; b < 8; ++b) {
      int at = -1;
      for (int q = 0; q < n; ++q)
        if (iu[(size_t)k][(size_t)q] == tgd[(size_t)b]) at = q;
      if (at < 0) {
        at = n;
        iu[(size_t)k][(size_t)n++] = tgd[(size_t)b];
      }
      itu[(size_t)k][(size_t)b] = at;
    }
    inu[(size_t)k] = n;
    ioff[(size_t)k + 1] = ioff[(size_t)k] + (int64_t)n * n;
    coff[(size_t)k + 1] = coff[(size_t)k] + n;
  }
  const int64_t tet0 = (int64_t)nh * 196, if0 = tet0 + (int64_t)nt * 64;
  std::vector<Trip> t((size_t)(if0 + ioff[(size_t)np2]));
  std::vector<double> cons((size_t)coff[(size_t)np2]);
  int bad_hex = -1;
  // hex volumes: K_ab = sum_q nu det w grad phi_a . grad phi_b (27 points)
#pragma omp parallel for schedule(dynamic, 64)
  for (int c = 0; c < nh; ++c) {
    double K[14][14] = {};
    try {
      for (int ix = 0; ix < 3; ++ix)
        for (int iy = 0; iy < 3; ++iy)
          for (int iz = 0; iz < 3; ++iz) {
            const double x = R.g3x[ix], y = R.g3x[iy], z = R.g3x[iz], w = R.g3w[ix] * R.g3w[iy] * R.g3w[iz];
            double ph[14], g[14][3], gp[14][3], I[9], det;
            hex_basis(x, y, z, ph, g);
            hex_metric(m, c, x, y, z, I, det);
            phys_grad<14>(g, I, gp);
            const double q = nu * det * w;
            for (int a = 0; a < 14; ++a)
              for (int b = 0; b < 14; ++b) K[a][b] += q * (gp[a][0] * gp[b][0] + gp[a][1] * gp[b][1] + gp[a][2] * gp[b][2]);
          }
    } catch (...) {
#pragma omp critical(hybrid_bad_hex)
      bad_hex = bad_hex < 0 ? c : std::min(bad_hex, c);
    }
    const auto& g = m.hex_dofs[(size_t)c];
    for (int a = 0; a < 14; ++a)
      for (int b = 0; b < 14; ++b) t[(size_t)(196 * (int64_t)c + a * 14 + b)] = {g[(size_t)a], g[(size_t)b], K[a][b]};
  }
  if (bad_hex >= 0) throw std::runtime_error("hybrid mesh: non-positive hex Jacobian in cell " + std::to_string(bad_hex));
  // tet volumes: K_ab = nu det sum_jk D[a][b][j][k] (J^-T J^-1)_jk
  const auto& D = ref_tensors().D;
#pragma omp parallel for schedule(static)
  for (int c = 0; c < nt; ++c) {
    const auto& tg = m.tet_geom[(size_t)c];
    double M[3][3] = {};
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k)
        for (int d = 0; d < 3; ++d) M[j][k] += tg[3 + 3 * (size_t)j + d] * tg[3 + 3 * (size_t)k + d];
    const auto& g = m.tet_dofs[(size_t)c];
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b) {
        double kd = 0;
        for (int j = 0; j < 3; ++j)
          for (int k = 0; k < 3; ++k) kd += D[a][b][j][k] * M[j][k];
        t[(size_t)(tet0 + 64 * (int64_t)c + a * 8 + b)] = {g[(size_t)a], g[(size_t)b], nu * tg[2] * kd};
      }
  }
  // Nitsche coupling on each interface triangle.  Over the union u of the
  // hex's and the tet's unknowns, the jump coefficient J_i = phi^hex_i -
  // phi^tet_i and the averaged flux coefficient F_i = nu/2 (grad phi^hex_i +
  // grad phi^tet_i) . n give K_ij = w (-J_i F_j - F_i J_j + tau J_i J_j),
  // tau = gamma nu max(1/h_hex, 1/h_tet)  (hybrid_hxt4b/hxt4b_main.cu
  // interface_assemble; hybrid_hxt2/hxt2_main.cu interface_kernel)
#pragma omp parallel for schedule(dynamic, 16)
  for (int k = 0; k < np2; ++k) {
    const InterfacePlan& p = plans[(size_t)(k / 2)];
    const int s = k % 2, nu_ = inu[(size_t)k];
    const int* hu = ihu[(size_t)k].data();
    const int* tu = itu[(size_t)k].data();
    const double tau = gamma * nu * std::max(p.inv_h_hex, p.inv_h_tet[s]);
    const double* n = p.normal;
    double K[22][22] = {}, cn[22] = {};
    try {
    for_interface_points(m, p, s, [&](double w, const double* ph, const double (*gph)[3], const double* pt,
                                      const double (*gpt)[3]) {
      double J[22] = {}, F[22] = {};
      for (int a = 0; a < 14; ++a) {
        J[hu[a]] += ph[a];
        F[hu[a]] += 0.5 * nu * (gph[a][0] * n[0] + gph[a][1] * n[1] + gph[a][2] * n[2]);
      }
      for (int b = 0; b < 8; ++b) {
        J[tu[b]] -= pt[b];
        F[tu[b]] += 0.5 * nu * (gpt[b][0] * n[0] + gpt[b][1] * n[1] + gpt[b][2] * n[2]);
      }
      for (int i = 0; i < nu_; ++i) {
        for (int j = 0; j < nu_; ++j) K[i][j] += w * (-F[j] * J[i] - F[i] * J[j] + tau * J[i] * J[j]);
        cn[i] += w * (-2.0 * F[i] * J[i]);
      }
    });
    } catch (...) {
#pragma omp critical(hybrid_bad_hex)
      bad_hex = bad_hex < 0 ? p.hex_cell : std::min(bad_hex, p.hex_cell);
    }
    const auto& u = iu[(size_t)k];
    for (int i = 0; i < nu_; ++i) {
      cons[(size_t)(coff[(size_t)k] + i)] = cn[i];
      for (int j = 0; j < nu_; ++j) t[(size_t)(if0 + ioff[(size_t)k] + i * nu_ + j)] = {u[(size_t)i], u[(size_t)j], K[i][j]};
    }
  }
  if (bad_hex >= 0) throw std::runtime_error("hybrid mesh: non-positive hex Jacobian in cell " + std::to_string(bad_hex));
  // penalty-free diagonal, summed in cell order: hex, tet, then interface
  for (int c = 0; c < nh; ++c)
    for (int a = 0; a < 14; ++a) diag_rau[(size_t)t[(size_t)(196 * (int64_t)c + 15 * a)].r] += t[(size_t)(196 * (int64_t)c + 15 * a)].v;
  for (int c = 0; c < nt; ++c)
    for (int a = 0; a < 8; ++a) {
      const Trip& x = t[(size_t)(tet0 + 64 * (int64_t)c + 9 * a)];
      diag_rau[(size_t)x.r] += x.v;
    }
  for (int k = 0; k < np2; ++k)
    for (int i = 0; i < inu[(size_t)k]; ++i) diag_rau[(size_t)iu[(size_t)k][(size_t)i]] += cons[(size_t)(coff[(size_t)k] + i)];
  sort_trips(t, nv);
  row.assign((size_t)nv + 1, 0);
  col.clear();
  val.clear();
  for (size_t a = 0; a < t.size();) {
    size_t b = a;
    double v = 0;
    while (b < t.size() && t[b].r == t[a].r && t[b].c == t[a].c) v += t[b++].v;
    col.push_back(t[a].c);
    val.push_back(v);
    ++row[(size_t)t[a].r + 1];
    a = b;
  }
  for (int i = 0; i < nv; ++i) row[(size_t)i + 1] += row[(size_t)i];
}

int32_t csr_find(const std::vector<int32_t>& row, const std::vector<int32_t>& col, int i, int j) {
  const auto b = col.begin() + row[(size_t)i], e = col.begin() + row[(size_t)i + 1];
  const auto it = std::lower_bound(b, e, j);
  if (it == e || *it != j) throw std::runtime_error("hybrid velocity CSR: missing entry");
  return (int32_t)(it - col.begin());
}
}  // namespace

namespace {
// manufactured pressure: (z_centroid - zmin) / L, shifted to 0 at cell 0
void p_exact_of(const HybridMesh& m, HybridStokes& H) {
  double zmin = 1e300, zmax = -1e300;
  for (int v = 0; v < m.nv(); ++v) {
    zmin = std::min(zmin, m.xyz[3 * (size_t)v + 2]);
    zmax = std::max(zmax, m.xyz[3 * (size_t)v + 2]);
  }
  const double L = zmax - zmin;
  H.p_exact.resize((size_t)H.np);
  for (int c = 0; c < m.nhex(); ++c) H.p_exact[(size_t)c] = (hex_centroid(m, c).z - zmin) / L;
  for (int c = 0; c < m.ntet(); ++c) H.p_exact[(size_t)(m.nhex() + c)] = (tet_centroid(m, c).z - zmin) / L;
  const double sh = H.p_exact[0];
  for (double& q : H.p_exact) q -= sh;
}
}  // namespace

HybridStokes build_hybrid_stokes(const HybridMesh& m, const std::vector<InterfacePlan>& plans, double nu,
                                 double gamma) {
  HybridStokes H;
  H.nvel = m.nvel();
  H.np = m.np();
  const int nv = H.nvel;
  std::vector<int32_t> arow, acol;
  std::vector<double> aval;
  assemble_velocity(m, plans, nu, gamma, arow, acol, aval, H.diag_rau);
  H.diag_full.assign((size_t)nv, 0.0);
  for (int i = 0; i < nv; ++i) H.diag_full[(size_t)i] = aval[(size_t)csr_find(arow, acol, i, i)];
  // fixed unknowns: every vertex and bubble of the wall, inlet and outlet faces
  H.fixed.assign((size_t)nv, 0);
  auto fix_hex = [&](const std::array<int32_t, 3>& r) {
    H.fixed[(size_t)r[2]] = 1;
    for (int k = 0; k < 4; ++k) H.fixed[(size_t)m.hexes[(size_t)r[0]][(size_t)kHexFace[r[1]][k]]] = 1;
  };
  auto fix_tet = [&](const std::array<int32_t, 3>& r) {
    H.fixed[(size_t)r[2]] = 1;
    for (int k = 0; k < 3; ++k) H.fixed[(size_t)m.tets[(size_t)r[0]][(size_t)kTetFace[r[1]][k]]] = 1;
  };
  for (const auto& r : m.wall_hex) fix_hex(r);
  for (const auto& r : m.in_hex) fix_hex(r);
  for (const auto& r : m.out_hex) fix_hex(r);
  for (const auto& r : m.in_tet) fix_tet(r);
  for (const auto& r : m.out_tet) fix_tet(r);
  // free rows as assembled, identity rows for the fixed unknowns
  H.a_row.assign((size_t)nv + 1, 0);
  for (int i = 0; i < nv; ++i) {
    if (H.fixed[(size_t)i]) {
      H.a_col.push_back(i);
      H.a_val.push_back(1.0);
    } else {
      for (int32_t k = arow[(size_t)i]; k < arow[(size_t)i + 1]; ++k) {
        H.a_col.push_back(acol[(size_t)k]);
        H.a_val.push_back(aval[(size_t)k]);
      }
    }
    H.a_row[(size_t)i + 1] = (int32_t)H.a_col.size();
  }
  build_hybrid_divergence(m, plans, H);
  p_exact_of(m, H);
  return H;
}

void build_hybrid_divergence(const HybridMesh& m, const std::vector<InterfacePlan>& plans, HybridStokes& H) {
  const Rules& R = rules();
  H.nvel = m.nvel();
  H.np = m.np();
  const int nv = H.nvel;
  // ---- divergence rows: cell volume integrals, then the averaged traces
  // on interface triangles (hybrid_hxt3a/hxt3a_main.cu:132-246)
  std::vector<std::map<int32_t, std::array<double, 3>>> rows((size_t)H.np);
  auto add = [](std::map<int32_t, std::array<double, 3>>& r, int32_t g, double x, double y, double z) {
    auto& e = r[g];
    e[0] += x;
    e[1] += y;
    e[2] += z;
  };
  for (int c = 0; c < m.nhex(); ++c) {
    double Bv[14][3] = {};
    for (int ix = 0; ix < 3; ++ix)
      for (int iy = 0; iy < 3; ++iy)
        for (int iz = 0; iz < 3; ++iz) {
          const double x = R.g3x[ix], y = R.g3x[iy], z = R.g3x[iz], w = R.g3w[ix] * R.g3w[iy] * R.g3w[iz];
          double ph[14], g[14][3], gp[14][3], I[9], det;
          hex_basis(x, y, z, ph, g);
          hex_metric(m, c, x, y, z, I, det);
          phys_grad<14>(g, I, gp);
          for (int a = 0; a < 14; ++a)
            for (int d = 0; d < 3; ++d) Bv[a][d] += w * det * gp[a][d];
        }
    for (int a = 0; a < 14; ++a) add(rows[(size_t)c], m.hex_dofs[(size_t)c][(size_t)a], Bv[a][0], Bv[a][1], Bv[a][2]);
  }
  static const double gl[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int c = 0; c < m.ntet(); ++c) {
    const auto& tg = m.tet_geom[(size_t)c];
    double Bv[8][3];
    for (int i = 0; i < 4; ++i)
      for (int d = 0; d < 3; ++d) {
        Bv[i][d] = tg[0] * (gl[i][0] * tg[3 + d] + gl[i][1] * tg[6 + d] + gl[i][2] * tg[9 + d]);
        Bv[4 + i][d] = (-27.0 / 20.0) * Bv[i][d];
      }
    for (int a = 0; a < 8; ++a)
      add(rows[(size_t)(m.nhex() + c)], m.tet_dofs[(size_t)c][(size_t)a], Bv[a][0], Bv[a][1], Bv[a][2]);
  }
  for (const auto& p : plans)
    for (int s = 0; s < 2; ++s) {
      double TH[14] = {}, TT[8] = {};
      for_interface_points(m, p, s, [&](double w, const double* ph, const double (*)[3], const double* pt,
                                        const double (*)[3]) {
        for (int a = 0; a < 14; ++a) TH[a] += w * ph[a];
        for (int a = 0; a < 8; ++a) TT[a] += w * pt[a];
      });
      auto& rh = rows[(size_t)p.hex_cell];
      auto& rt = rows[(size_t)(m.nhex() + p.tet_cell[s])];
      const double* n = p.normal;
      for (int a = 0; a < 14; ++a) {
        const double q = 0.5 * TH[a];
        const int32_t g = m.hex_dofs[(size_t)p.hex_cell][(size_t)a];
        add(rh, g, -q * n[0], -q * n[1], -q * n[2]);
        add(rt, g, -q * n[0], -q * n[1], -q * n[2]);
      }
      for (int a = 0; a < 8; ++a) {
        const double q = 0.5 * TT[a];
        const int32_t g = m.tet_dofs[(size_t)p.tet_cell[s]][(size_t)a];
        add(rh, g, q * n[0], q * n[1], q * n[2]);
        add(rt, g, q * n[0], q * n[1], q * n[2]);
      }
    }
  H.b_row.assign((size_t)H.np + 1, 0);
  for (int i = 0; i < H.np; ++i) {
    for (const auto& [g, v] : rows[(size_t)i]) {
      if (std::max({std::abs(v[0]), std::abs(v[1]), std::abs(v[2])}) < 1e-28) continue;
      H.b_col.push_back(g);
      H.bx.push_back(v[0]);
      H.by.push_back(v[1]);
      H.bz.push_back(v[2]);
    }
    H.b_row[(size_t)i + 1] = (int32_t)H.b_col.size();
  }
  // transpose, rows ascending in pressure index
  H.bt_row.assign((size_t)nv + 1, 0);
  for (int32_t g : H.b_col) ++H.bt_row[(size_t)g + 1];
  for (int i = 0; i < nv; ++i) H.bt_row[(size_t)i + 1] += H.bt_row[(size_t)i];
  H.bt_col.resize(H.b_col.size());
  H.btx.resize(H.b_col.size());
  H.bty.resize(H.b_col.size());
  H.btz.resize(H.b_col.size());
  {
    std::vector<int32_t> next(H.bt_row.begin(), H.bt_row.end() - 1);
    for (int i = 0; i < H.np; ++i)
      for (int32_t k = H.b_row[(size_t)i]; k < H.b_row[(size_t)i + 1]; ++k) {
        const int32_t q = next[(size_t)H.b_col[(size_t)k]]++;
        H.bt_col[(size_t)q] = i;
        H.btx[(size_t)q] = H.bx[(size_t)k];
        H.bty[(size_t)q] = H.by[(size_t)k];
        H.btz[(size_t)q] = H.bz[(size_t)k];
      }
  }
}

HybridFlow build_hybrid_flow(const HybridMesh& m, const std::vector<InterfacePlan>& plans, double re, double bulk,
                             double gamma) {
  HybridFlow F;
  F.nvel = m.nvel();
  F.np = m.np();
  F.nhex = m.nhex();
  F.ntet = m.ntet();
  const int nv = F.nvel;
  // pipe geometry from the mesh (hxt4b_main.cu:233-236)
  double zmin = 1e300, zmax = -1e300, R = 0;
  for (int v = 0; v < m.nv(); ++v) {
    const double x = m.xyz[3 * (size_t)v], y = m.xyz[3 * (size_t)v + 1], z = m.xyz[3 * (size_t)v + 2];
    zmin = std::min(zmin, z);
    zmax = std::max(zmax, z);
    R = std::max(R, std::sqrt(x * x + y * y));
  }
  F.radius = R;
  F.length = zmax - zmin;
  F.diameter = 2 * R;
  F.nu = bulk * F.diameter / re;
  if (std::abs(F.length / F.diameter - 10) > 1e-6)
    throw std::runtime_error("the mixed-mesh pipe SIMPLE expects a pipe of 10 diameters");
  assemble_velocity(m, plans, F.nu, gamma, F.row, F.col, F.base, F.diag_r_base);
  F.diag_pos.resize((size_t)nv);
  for (int i = 0; i < nv; ++i) F.diag_pos[(size_t)i] = csr_find(F.row, F.col, i, i);
  // convection gather lists: the CSR entry of each local value (local value
  // q: 196 per hex, row-major, then 64 per tet), then the values of each entry
  // in cell order (a stable counting sort by entry)
  const int64_t tet0 = (int64_t)m.nhex() * 196, nloc = tet0 + (int64_t)m.ntet() * 64;
  if (nloc > INT32_MAX) throw std::runtime_error("mixed mesh too large for 32-bit convection gather lists");
  std::vector<int32_t> entry((size_t)nloc);
  auto find = [&](int i, int j) -> int32_t {
    const auto b = F.col.begin() + F.row[(size_t)i], e = F.col.begin() + F.row[(size_t)i + 1];
    const auto it = std::lower_bound(b, e, j);
    return it == e || *it != j ? -1 : (int32_t)(it - F.col.begin());
  };
#pragma omp parallel for schedule(static)
  for (int h = 0; h < m.nhex(); ++h) {
    const auto& g = m.hex_dofs[(size_t)h];
    for (int a = 0; a < 14; ++a)
      for (int b = 0; b < 14; ++b)
        entry[(size_t)(196 * (int64_t)h + a * 14 + b)] = find(g[(size_t)a], g[(size_t)b]);
  }
#pragma omp parallel for schedule(static)
  for (int t = 0; t < m.ntet(); ++t) {
    const auto& g = m.tet_dofs[(size_t)t];
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b)
        entry[(size_t)(tet0 + 64 * (int64_t)t + a * 8 + b)] = find(g[(size_t)a], g[(size_t)b]);
  }
  for (int32_t k : entry)
    if (k < 0) throw std::runtime_error("hybrid velocity CSR: missing entry");
  F.src_off.assign(F.col.size() + 1, 0);
  F.src.resize((size_t)nloc);
  for (int32_t k : entry) ++F.src_off[(size_t)k + 1];
  for (size_t k = 0; k < F.col.size(); ++k) F.src_off[k + 1] += F.src_off[k];
  {
    std::vector<int32_t> next(F.src_off.begin(), F.src_off.end() - 1);
    for (int64_t q = 0; q < nloc; ++q) F.src[(size_t)next[(size_t)entry[(size_t)q]]++] = (int32_t)q;
  }
  // Dirichlet data and initial state (hxt4b_main.cu:175-186): parabolic
  // axial velocity at every vertex; wall faces no-slip; inlet faces the
  // profile, their bubble the profile at the face centre minus the mean of
  // the vertex values; the outlet is natural
  F.fixed.assign((size_t)nv, 0);
  F.u0.assign((size_t)nv, 0.0);
  F.u1.assign((size_t)nv, 0.0);
  F.u2.assign((size_t)nv, 0.0);
  for (int v = 0; v < m.nv(); ++v) F.u2[(size_t)v] = pipe_profile(m.xyz[3 * (size_t)v], m.xyz[3 * (size_t)v + 1], R, bulk);
  for (const auto& r : m.wall_hex) {
    F.fixed[(size_t)r[2]] = 1;
    F.u2[(size_t)r[2]] = 0;
    for (int k = 0; k < 4; ++k) {
      const int g = m.hexes[(size_t)r[0]][(size_t)kHexFace[r[1]][k]];
      F.fixed[(size_t)g] = 1;
      F.u0[(size_t)g] = F.u1[(size_t)g] = F.u2[(size_t)g] = 0;
    }
  }
  auto inlet = [&](const int32_t* v, int nvert, int bubble) {
    double av = 0, cx = 0, cy = 0;
    for (int k = 0; k < nvert; ++k) {
      const double x = m.xyz[3 * (size_t)v[k]], y = m.xyz[3 * (size_t)v[k] + 1];
      const double q = pipe_profile(x, y, R, bulk);
      F.fixed[(size_t)v[k]] = 1;
      F.u2[(size_t)v[k]] = q;
      if (nvert == 4) {
        av += .25 * q;
        cx += .25 * x;
        cy += .25 * y;
      } else {
        av += q / 3;
        cx += x / 3;
        cy += y / 3;
      }
    }
    F.fixed[(size_t)bubble] = 1;
    F.u2[(size_t)bubble] = pipe_profile(cx, cy, R, bulk) - av;
  };
  for (const auto& r : m.in_hex) {
    int32_t v[4];
    for (int k = 0; k < 4; ++k) v[k] = m.hexes[(size_t)r[0]][(size_t)kHexFace[r[1]][k]];
    inlet(v, 4, r[2]);
  }
  for (const auto& r : m.in_tet) {
    int32_t v[3];
    for (int k = 0; k < 3; ++k) v[k] = m.tets[(size_t)r[0]][(size_t)kTetFace[r[1]][k]];
    inlet(v, 3, r[2]);
  }
  // greedy colouring of the free rows over their lower free neighbours
  // (hxt4b_main.cu color_free_rows)
  std::vector<int> colour((size_t)nv, -1), mark(128, -1);
  int nc = 0, nfree = 0;
  for (int i = 0; i < nv; ++i) {
    if (F.fixed[(size_t)i]) continue;
    ++nfree;
    for (int32_t q = F.row[(size_t)i]; q < F.row[(size_t)i + 1]; ++q) {
      const int j = F.col[(size_t)q];
      if (j >= i || F.fixed[(size_t)j]) continue;
      const int cj = colour[(size_t)j];
      if (cj >= 0) {
        if (cj >= (int)mark.size()) mark.resize((size_t)cj + 32, -1);
        mark[(size_t)cj] = i;
      }
    }
    int cc = 0;
    while (cc < (int)mark.size() && mark[(size_t)cc] == i) ++cc;
    if (cc >= (int)mark.size()) mark.resize((size_t)cc + 32, -1);
    colour[(size_t)i] = cc;
    nc = std::max(nc, cc + 1);
  }
  F.colour_off.assign((size_t)nc + 1, 0);
  for (int i = 0; i < nv; ++i)
    if (colour[(size_t)i] >= 0) ++F.colour_off[(size_t)colour[(size_t)i] + 1];
  for (int k = 0; k < nc; ++k) F.colour_off[(size_t)k + 1] += F.colour_off[(size_t)k];
  F.colour_rows.resize((size_t)nfree);
  {
    std::vector<int32_t> next(F.colour_off.begin(), F.colour_off.end() - 1);
    for (int i = 0; i < nv; ++i)
      if (colour[(size_t)i] >= 0) F.colour_rows[(size_t)next[(size_t)colour[(size_t)i]]++] = i;
  }
  for (int k = 0; k < nc; ++k) F.max_colour = std::max(F.max_colour, F.colour_off[(size_t)k + 1] - F.colour_off[(size_t)k]);
  F.pin = hybrid_pin(m);
  return F;
}

double hybrid_pressure_slope(const HybridMesh& m, const std::vector<double>& p) {
  long double W = 0, Wz = 0, Wp = 0, Wzz = 0, Wzp = 0;
  for (int c = 0; c < m.np(); ++c) {
    const bool h = c < m.nhex();
    const int lc = h ? c : c - m.nhex();
    const double z = h ? hex_centroid(m, lc).z : tet_centroid(m, lc).z;
    const double v = h ? m.hex_geom[(size_t)lc][0] : m.tet_geom[(size_t)lc][0];
    W += v;
    Wz += v * z;
    Wp += v * p[(size_t)c];
    Wzz += v * z * z;
    Wzp += v * z * p[(size_t)c];
  }
  return (double)((W * Wzp - Wz * Wp) / (W * Wzz - Wz * Wz));
}

double hybrid_boundary_pressure(const HybridMesh& m, const std::vector<double>& p, bool inlet) {
  long double num = 0, den = 0;
  for (const auto& r : inlet ? m.in_hex : m.out_hex) {
    V3 q[4];
    for (int k = 0; k < 4; ++k) q[k] = point(m, m.hexes[(size_t)r[0]][(size_t)kHexFace[r[1]][k]]);
    const double A = tri_area(q[0], q[1], q[2]) + tri_area(q[0], q[2], q[3]);
    num += (long double)A * p[(size_t)r[0]];
    den += A;
  }
  for (const auto& r : inlet ? m.in_tet : m.out_tet) {
    V3 q[3];
    for (int k = 0; k < 3; ++k) q[k] = point(m, m.tets[(size_t)r[0]][(size_t)kTetFace[r[1]][k]]);
    const double A = tri_area(q[0], q[1], q[2]);
    num += (long double)A * p[(size_t)(m.nhex() + r[0])];
    den += A;
  }
  return (double)(num / den);
}

HybridSchurCsr hybrid_schur_csr(const HybridStokes& B, int pin, const std::vector<double>& rau) {
  const int np = B.np;
  if ((int)rau.size() != B.nvel) throw std::runtime_error("hybrid pressure matrix: rAU size mismatch");
  auto entry = [&](int i, int j) {
    int32_t a = B.b_row[(size_t)i], b = B.b_row[(size_t)j];
    const int32_t ae = B.b_row[(size_t)i + 1], be = B.b_row[(size_t)j + 1];
    long double s = 0;
    while (a < ae && b < be) {
      const int32_t ga = B.b_col[(size_t)a], gb = B.b_col[(size_t)b];
      if (ga < gb) { ++a; continue; }
      if (gb < ga) { ++b; continue; }
      s += (long double)rau[(size_t)ga] * ((long double)B.bx[(size_t)a] * B.bx[(size_t)b] +
                                           (long double)B.by[(size_t)a] * B.by[(size_t)b] +
                                           (long double)B.bz[(size_t)a] * B.bz[(size_t)b]);
      ++a;
      ++b;
    }
    return (double)s;
  };
  HybridSchurCsr H;
  CsrHost& A = H.A;
  A.n = np;
  A.row.assign((size_t)np + 1, 0);
  // rows are independent: patterns, then values, in parallel
  std::vector<std::vector<int32_t>> nbs((size_t)np);
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < np; ++i) {
    std::vector<int32_t>& nb = nbs[(size_t)i];
    nb.assign(1, i);
    if (i != pin) {
      for (int32_t k = B.b_row[(size_t)i]; k < B.b_row[(size_t)i + 1]; ++k) {
        const int32_t g = B.b_col[(size_t)k];
        for (int32_t q = B.bt_row[(size_t)g]; q < B.bt_row[(size_t)g + 1]; ++q)
          if (B.bt_col[(size_t)q] != pin) nb.push_back(B.bt_col[(size_t)q]);
      }
      std::sort(nb.begin(), nb.end());
      nb.erase(std::unique(nb.begin(), nb.end()), nb.end());
    }
  }
  for (int i = 0; i < np; ++i) A.row[(size_t)i + 1] = A.row[(size_t)i] + (int64_t)nbs[(size_t)i].size();
  A.col.resize((size_t)A.row[(size_t)np]);
  A.val.resize(A.col.size());
  A.diag.assign((size_t)np, 0.0);
  H.entry_row.resize(A.col.size());
  H.diag_pos.assign((size_t)np, -1);
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : bad)
  for (int i = 0; i < np; ++i) {
    std::copy(nbs[(size_t)i].begin(), nbs[(size_t)i].end(), A.col.begin() + A.row[(size_t)i]);
    for (int64_t k = A.row[(size_t)i]; k < A.row[(size_t)i + 1]; ++k) {
      const int j = A.col[(size_t)k];
      H.entry_row[(size_t)k] = i;
      const double v = i == pin ? (j == pin ? 1.0 : 0.0) : entry(i, j);
      A.val[(size_t)k] = v;
      if (j == i) {
        H.diag_pos[(size_t)i] = (int32_t)k;
        A.diag[(size_t)i] = v;
      }
    }
    if (!(A.diag[(size_t)i] > 0.0) || !std::isfinite(A.diag[(size_t)i])) ++bad;
  }
  if (bad) throw std::runtime_error("hybrid pressure matrix: nonpositive diagonal");
  return H;
}

void hybrid_velocity_operator(const HybridMesh& m, const std::vector<InterfacePlan>& plans, double nu, double gamma,
                              bool with_interface, std::vector<int32_t>& row, std::vector<int32_t>& col,
                              std::vector<double>& val) {
  std::vector<double> diag;
  assemble_velocity(m, plans, nu, gamma, row, col, val, diag, with_interface);
}

int hybrid_pin(const HybridMesh& m) {
  return !m.out_hex.empty() ? m.out_hex[0][0] : (!m.out_tet.empty() ? m.nhex() + m.out_tet[0][0] : 0);
}

AmgOptions hybrid_amg_options(const nds_hybrid_flow_options& o) {
  auto bad = [](const char* what) { throw std::invalid_argument(what); };
  if (o.amg_smoother < NDS_SM_CHEB2 || o.amg_smoother > NDS_SM_MCGS) bad("unknown AMG smoother");
  if (o.cf_interp != NDS_CF_DIRECT && o.cf_interp != NDS_CF_EXTI) bad("CF interp must be direct or exti");
  if (o.amg_mcgs_order < NDS_MCGS_SYMMETRIC || o.amg_mcgs_order > NDS_MCGS_BACKWARD) bad("bad MCGS order");
  if (o.pressure_solver == 1 && o.amg_smoother == NDS_SM_MCGS && o.amg_mcgs_order != NDS_MCGS_SYMMETRIC)
    bad("PCG requires symmetric MCGS");
  if (o.amg_spectrum_policy < NDS_SPEC_AUTO || o.amg_spectrum_policy > NDS_SPEC_OFF) bad("bad AMG spectrum policy");
  if (o.amg_terminal < 1 || o.cf_pmax < 1 || !(o.cf_theta > 0) || o.amg_cheb_degree < 1 || o.amg_power_its < 0 ||
      o.amg_jacobi_fine_sweeps < 1 || o.amg_jacobi_coarse_sweeps < 1 || o.amg_mcgs_fine_sweeps < 1 ||
      o.amg_mcgs_coarse_sweeps < 1 || !(o.amg_lambda_safety > 0) || !(o.amg_lambda_low_fraction > 0))
    bad("bad AMG option value");
  AmgOptions a;
  a.hierarchy = "cf";
  a.terminal = o.amg_terminal;
  a.power_its = o.amg_spectrum_policy == NDS_SPEC_ALWAYS || (o.amg_spectrum_policy == NDS_SPEC_AUTO &&
                                                             o.amg_smoother == NDS_SM_CHEB2)
                    ? o.amg_power_its
                    : 0;
  if (o.amg_smoother == NDS_SM_CHEB2 && a.power_its <= 0) bad("Chebyshev requires spectrum estimation");
  a.lambda_safety = o.amg_lambda_safety;
  a.cf_theta = o.cf_theta;
  a.cf_pmax = o.cf_pmax;
  a.cf_interp = o.cf_interp == NDS_CF_EXTI ? "exti" : "direct";
  a.cf_aggressive_first = o.cf_aggressive_first != 0;
  return a;
}

void write_hybrid_vtu(const HybridMesh& m, const std::string& path, const double* u0, const double* u1,
                      const double* u2, const double* p) {
  const int nv = m.nv(), nh = m.nhex(), nt = m.ntet();
  // vertex pressure = sum over the cells at the vertex of (V/k) p / sum of V/k,
  // k the cell's vertex count; hexes first, then tets, in cell order
  std::vector<long double> wsum((size_t)nv, 0.0L), psum((size_t)nv, 0.0L);
  for (int c = 0; c < nh; ++c) {
    const double share = m.hex_geom[(size_t)c][0] / 8;
    for (int a = 0; a < 8; ++a) {
      const size_t v = (size_t)m.hexes[(size_t)c][(size_t)a];
      wsum[v] += share;
      psum[v] += share * p[(size_t)c];
    }
  }
  for (int c = 0; c < nt; ++c) {
    const double share = m.tet_geom[(size_t)c][0] / 4;
    for (int a = 0; a < 4; ++a) {
      const size_t v = (size_t)m.tets[(size_t)c][(size_t)a];
      wsum[v] += share;
      psum[v] += share * p[(size_t)(nh + c)];
    }
  }
  std::ofstream f(path);
  if (!f) throw std::runtime_error("cannot write " + path);
  f.precision(16);
  f << "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
    << "<UnstructuredGrid><Piece NumberOfPoints=\"" << nv << "\" NumberOfCells=\"" << nh + nt << "\">\n"
    << "<Points><DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n";
  for (int v = 0; v < nv; ++v)
    f << m.xyz[3 * (size_t)v] << ' ' << m.xyz[3 * (size_t)v + 1] << ' ' << m.xyz[3 * (size_t)v + 2] << '\n';
  f << "</DataArray></Points><Cells><DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n";
  for (const auto& h : m.hexes) {
    for (int32_t v : h) f << v << ' ';
    f << '\n';
  }
  for (const auto& t : m.tets) {
    for (int32_t v : t) f << v << ' ';
    f << '\n';
  }
  f << "</DataArray><DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\">\n";
  long long end = 0;
  for (int c = 0; c < nh + nt; ++c) f << (end += c < nh ? 8 : 4) << '\n';
  f << "</DataArray><DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n";
  for (int c = 0; c < nh + nt; ++c) f << (c < nh ? "12\n" : "10\n");
  f << "</DataArray></Cells><PointData><DataArray type=\"Float64\" Name=\"velocity_Q1P1_vertex\" "
       "NumberOfComponents=\"3\" format=\"ascii\">\n";
  for (int v = 0; v < nv; ++v) f << u0[v] << ' ' << u1[v] << ' ' << u2[v] << '\n';
  f << "</DataArray><DataArray type=\"Float64\" Name=\"pressure_Q0P0_vertex_volume_average\" format=\"ascii\">\n";
  for (int v = 0; v < nv; ++v) f << (wsum[(size_t)v] > 0 ? (double)(psum[(size_t)v] / wsum[(size_t)v]) : 0.0) << '\n';
  f << "</DataArray></PointData><CellData><DataArray type=\"Float64\" Name=\"pressure_Q0P0\" format=\"ascii\">\n";
  for (int c = 0; c < nh + nt; ++c) f << p[c] << '\n';
  f << "</DataArray><DataArray type=\"Int32\" Name=\"region\" format=\"ascii\">\n";
  for (int c = 0; c < nh + nt; ++c) f << (c < nh ? "1\n" : "2\n");
  f << "</DataArray></CellData></Piece></UnstructuredGrid></VTKFile>\n";
  if (!f) throw std::runtime_error("short write to " + path);
}

}  // namespace nds
