#include "setup.hpp"

#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>

#include "fem.hpp"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace nds {

namespace {

struct V3 {
  double x, y, z;
};
inline V3 pt(const Mesh& m, int v) { return {m.x(v), m.y(v), m.z(v)}; }
inline V3 sub(const V3& a, const V3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 cross(const V3& a, const V3& b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double norm(const V3& a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

// face area vector pointing out of the owner cell
V3 outward_area(const Mesh& m, int f) {
  const auto& F = m.faces[(size_t)f];
  const V3 a = pt(m, F[0]), b = pt(m, F[1]), c = pt(m, F[2]);
  const V3 u = sub(b, a), v = sub(c, a);
  V3 sf{0.5 * (u.y * v.z - u.z * v.y), 0.5 * (u.z * v.x - u.x * v.z), 0.5 * (u.x * v.y - u.y * v.x)};
  const int cell = m.owner[(size_t)f];
  const V3 fc{(a.x + b.x + c.x) / 3.0, (a.y + b.y + c.y) / 3.0, (a.z + b.z + c.z) / 3.0};
  V3 cc{0, 0, 0};
  for (int i = 0; i < 4; ++i) {
    const V3 x = pt(m, m.tets[(size_t)cell][(size_t)i]);
    cc.x += 0.25 * x.x;
    cc.y += 0.25 * x.y;
    cc.z += 0.25 * x.z;
  }
  if (sf.x * (fc.x - cc.x) + sf.y * (fc.y - cc.y) + sf.z * (fc.z - cc.z) < 0.0) sf = {-sf.x, -sf.y, -sf.z};
  return sf;
}

double ideal_uz(const PipeBC& P, double x, double y) {
  const double rr = (x - P.cx) * (x - P.cx) + (y - P.cy) * (y - P.cy);
  return 2.0 * P.bulk * (1.0 - rr / (P.R * P.R));
}
// exact mean of the Poiseuille profile over a triangle
double tri_avg_uz(const PipeBC& P, const V3 X[3]) {
  double xx[3], yy[3];
  for (int i = 0; i < 3; ++i) {
    xx[i] = X[i].x - P.cx;
    yy[i] = X[i].y - P.cy;
  }
  const double ax = (xx[0] * xx[0] + xx[1] * xx[1] + xx[2] * xx[2] + xx[0] * xx[1] + xx[1] * xx[2] + xx[2] * xx[0]) / 6.0;
  const double ay = (yy[0] * yy[0] + yy[1] * yy[1] + yy[2] * yy[2] + yy[0] * yy[1] + yy[1] * yy[2] + yy[2] * yy[0]) / 6.0;
  return 2.0 * P.bulk * (1.0 - (ax + ay) / (P.R * P.R));
}

PipeBC make_pipe(const Mesh& m, const SetupOptions& o) {
  PipeBC P;
  P.wall = m.patch_index(o.wall);
  P.inlet = m.patch_index(o.inlet);
  P.outlet = m.patch_index(o.outlet);
  P.re = o.re;
  P.bulk = o.bulk;
  if (P.wall < 0 || P.inlet < 0 || P.outlet < 0) throw std::runtime_error("pipe patch not found");
  double xmin = 1e300, xmax = -1e300, ymin = 1e300, ymax = -1e300, zmin = 1e300, zmax = -1e300;
  for (int v = 0; v < m.n_points(); ++v) {
    xmin = std::min(xmin, m.x(v)); xmax = std::max(xmax, m.x(v));
    ymin = std::min(ymin, m.y(v)); ymax = std::max(ymax, m.y(v));
    zmin = std::min(zmin, m.z(v)); zmax = std::max(zmax, m.z(v));
  }
  P.z_in = zmin;
  P.z_out = zmax;
  P.L = zmax - zmin;
  if (o.geom_from_inlet) {
    // the inlet disk's own extent (its rim vertices lie on the pipe wall)
    const auto& pin0 = m.patches[(size_t)P.inlet];
    xmin = ymin = 1e300;
    xmax = ymax = -1e300;
    for (int f = pin0.start; f < pin0.start + pin0.count; ++f)
      for (int v : m.faces[(size_t)f]) {
        xmin = std::min(xmin, m.x(v)); xmax = std::max(xmax, m.x(v));
        ymin = std::min(ymin, m.y(v)); ymax = std::max(ymax, m.y(v));
      }
  }
  P.cx = 0.5 * (xmin + xmax);
  P.cy = 0.5 * (ymin + ymax);
  P.R = 0.5 * std::max(xmax - xmin, ymax - ymin);
  P.D = 2 * P.R;
  if (!(P.R > 0 && P.L > 0 && o.re > 0 && o.bulk > 0)) throw std::runtime_error("invalid pipe geometry or flow parameters");
  P.nu = o.bulk * P.D / o.re;
  P.circle_area = 3.14159265358979323846 * P.R * P.R;
  const auto& pin = m.patches[(size_t)P.inlet];
  double raw = 0;
  V3 sfs{0, 0, 0};
  for (int f = pin.start; f < pin.start + pin.count; ++f) {
    const auto& F = m.faces[(size_t)f];
    const V3 X[3] = {pt(m, F[0]), pt(m, F[1]), pt(m, F[2])};
    const double a = 0.5 * norm(cross(sub(X[1], X[0]), sub(X[2], X[0])));
    P.inlet_area += a;
    raw += a * tri_avg_uz(P, X);
    const V3 sf = outward_area(m, f);
    sfs.x += sf.x;
    sfs.y += sf.y;
    sfs.z += sf.z;
  }
  P.inlet_projected_area = norm(sfs);
  if (!(P.inlet_projected_area > 0.0)) throw std::runtime_error("degenerate inlet projected area");
  P.inlet_normal[0] = sfs.x / P.inlet_projected_area;
  P.inlet_normal[1] = sfs.y / P.inlet_projected_area;
  P.inlet_normal[2] = sfs.z / P.inlet_projected_area;
  for (int d = 0; d < 3; ++d) P.inlet_velocity[d] = -o.bulk * P.inlet_normal[d];
  if (!(raw > 0)) throw std::runtime_error("non-positive inlet flux");
  P.profile_scale = o.bulk * P.inlet_area / raw;
  P.hp_gradient = 32.0 * P.nu * o.bulk / (P.D * P.D);
  P.hp_drop = P.hp_gradient * P.L;
  return P;
}

int hw_threads(int req) {
#ifdef _OPENMP
  return req > 0 ? req : omp_get_max_threads();
#else
  (void)req;
  return 1;
#endif
}

}  // namespace

StageTimer::StageTimer(const char* scope) : scope_(scope), t0_(std::chrono::steady_clock::now()), last_(t0_) {
  const char* e = std::getenv("NDS_SETUP_TIMING");
  on_ = e && *e && std::strcmp(e, "0") != 0;
}
void StageTimer::mark(const char* stage) {
  const auto t = std::chrono::steady_clock::now();
  if (on_)
    std::fprintf(stderr, "NDS_SETUP_STAGE scope=%s stage=%s seconds=%.6f total=%.6f\n", scope_, stage,
                 std::chrono::duration<double>(t - last_).count(), std::chrono::duration<double>(t - t0_).count());
  last_ = t;
}

namespace {

// Exceptions cannot leave an OpenMP region: record the first message and
// rethrow after the region ends.
struct OmpError {
  bool bad = false;
  std::string msg;
  void set(const char* m) {
#pragma omp critical(nds_omp_error)
    if (!bad) { bad = true; msg = m; }
  }
  void rethrow() const { if (bad) throw std::runtime_error(msg); }
};

inline int entity_of(const Mesh& m, int c, int a) {
  return a < 4 ? m.tets[(size_t)c][(size_t)a] : m.n_points() + m.opp[(size_t)c][(size_t)(a - 4)];
}

}  // namespace

double bcoeff(double det, const double* invJ, int a, int d) {
  const double g1 = invJ[d], g2 = invJ[3 + d], g3 = invJ[6 + d];
  const int i = a < 4 ? a : a - 4;
  const double gl = i == 0 ? -(g1 + g2 + g3) : (i == 1 ? g1 : (i == 2 ? g2 : g3));
  const double base = (det / 6.0) * gl;
  return a < 4 ? base : -(27.0 / 20.0) * base;
}

Setup build_setup(const Mesh& m, const SetupOptions& o) {
  StageTimer tm("setup");
  Setup S;
  const int nth = hw_threads(o.threads);
  (void)nth;
  S.pipe = make_pipe(m, o);
  const int np = m.n_points(), nf = m.n_faces(), ni = m.n_internal(), nc = m.n_cells();
  S.nc = nc;
  S.n_vert = np;
  S.n_face = nf;
  const size_t ne = (size_t)np + (size_t)nf;

  // --- Dirichlet mask: every boundary face except the outlet, with its vertices
  std::vector<uint8_t> fixed(ne, 0);
  for (int f = ni; f < nf; ++f) {
    if (m.face_patch[(size_t)f] == S.pipe.outlet) continue;
    fixed[(size_t)np + f] = 1;
    for (int v : m.faces[(size_t)f]) fixed[(size_t)v] = 1;
  }
  S.g2free.assign(ne, -1);
  S.fixed_slot.assign(ne, -1);
  int next = 0;
  for (int v = 0; v < np; ++v)
    if (!fixed[(size_t)v]) S.g2free[(size_t)v] = next++;
  for (int f = 0; f < nf; ++f)
    if (!fixed[(size_t)np + f]) S.g2free[(size_t)np + f] = next++;
  S.nv = next;
  int ns = 0;
  for (size_t e = 0; e < ne; ++e)
    if (fixed[e]) S.fixed_slot[e] = ns++;
  S.n_fixed = ns;
  S.fixed_value.assign(3 * (size_t)ns, 0.0);

  // --- inlet profile: vertex values, then flux-exact face-bubble values
  std::vector<uint8_t> on_wall((size_t)np, 0), on_inlet((size_t)np, 0);
  for (int f = ni; f < nf; ++f) {
    const int p = m.face_patch[(size_t)f];
    if (p == S.pipe.wall)
      for (int v : m.faces[(size_t)f]) on_wall[(size_t)v] = 1;
    if (p == S.pipe.inlet)
      for (int v : m.faces[(size_t)f]) on_inlet[(size_t)v] = 1;
  }
  for (int v = 0; v < np; ++v)
    if (on_inlet[(size_t)v] && !on_wall[(size_t)v]) {
      const int s = S.fixed_slot[(size_t)v];
      S.fixed_value[3 * (size_t)s + 2] = S.pipe.profile_scale * ideal_uz(S.pipe, m.x(v), m.y(v));
    }
  {
    const auto& pin = m.patches[(size_t)S.pipe.inlet];
    for (int f = pin.start; f < pin.start + pin.count; ++f) {
      const auto& F = m.faces[(size_t)f];
      const V3 X[3] = {pt(m, F[0]), pt(m, F[1]), pt(m, F[2])};
      const double exact = S.pipe.profile_scale * tri_avg_uz(S.pipe, X);
      double vm = 0;
      for (int j = 0; j < 3; ++j) vm += S.fixed_value[3 * (size_t)S.fixed_slot[(size_t)F[(size_t)j]] + 2] / 3.0;
      const int fs = S.fixed_slot[(size_t)np + f];
      S.fixed_value[3 * (size_t)fs + 2] = (20.0 / 9.0) * (exact - vm);
    }
  }

  tm.mark("numbering");
  // --- cell refs, geometry
  S.ref.assign(8 * (size_t)nc, 0);
  S.det.assign((size_t)nc, 0);
  S.h2.assign((size_t)nc, 0);
  S.invJ.assign(9 * (size_t)nc, 0);
  OmpError oerr;
#pragma omp parallel for schedule(static)
  for (int c = 0; c < nc; ++c) {
    try {
    for (int a = 0; a < 8; ++a) {
      const int e = entity_of(m, c, a);
      const int g = S.g2free[(size_t)e];
      S.ref[8 * (size_t)c + a] = g >= 0 ? g : -(S.fixed_slot[(size_t)e] + 1);
    }
    double J[3][3], I[3][3];
    tet_jacobian(m, m.tets[(size_t)c], J);
    const double d = det3(J);
    if (!(d > 0.0)) throw std::runtime_error("non-positive tetrahedron");
    inv3(J, I);
    S.det[(size_t)c] = d;
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) S.invJ[9 * (size_t)c + 3 * j + k] = I[j][k];
    double h2 = 0;
    for (int a = 0; a < 4; ++a)
      for (int b = a + 1; b < 4; ++b) {
        const V3 xa = pt(m, m.tets[(size_t)c][(size_t)a]), xb = pt(m, m.tets[(size_t)c][(size_t)b]);
        const double dx = xa.x - xb.x, dy = xa.y - xb.y, dz = xa.z - xb.z;
        h2 = std::max(h2, dx * dx + dy * dy + dz * dz);
      }
    S.h2[(size_t)c] = h2;
    } catch (const std::exception& e) { oerr.set(e.what()); }
  }
  oerr.rethrow();

  // --- row -> (cell, local) incidence in ascending cell order
  const int nv = S.nv;
  std::vector<int64_t> iptr((size_t)nv + 1, 0);
  for (int c = 0; c < nc; ++c)
    for (int a = 0; a < 8; ++a) {
      const int g = S.ref[8 * (size_t)c + a];
      if (g >= 0) ++iptr[(size_t)g + 1];
    }
  for (int r = 0; r < nv; ++r) iptr[(size_t)r + 1] += iptr[(size_t)r];
  std::vector<int32_t> inc_cell((size_t)iptr[(size_t)nv]);
  std::vector<uint8_t> inc_a((size_t)iptr[(size_t)nv]);
  {
    std::vector<int64_t> cur(iptr.begin(), iptr.end() - 1);
    for (int c = 0; c < nc; ++c)
      for (int a = 0; a < 8; ++a) {
        const int g = S.ref[8 * (size_t)c + a];
        if (g < 0) continue;
        const int64_t z = cur[(size_t)g]++;
        inc_cell[(size_t)z] = c;
        inc_a[(size_t)z] = (uint8_t)a;
      }
  }

  tm.mark("geometry+incidence");
  // --- momentum topology: sorted unique free neighbours of every row
  S.mom.n = nv;
  S.mom.row.assign((size_t)nv + 1, 0);
  std::vector<std::vector<int32_t>> rows((size_t)nv);
#pragma omp parallel for schedule(dynamic, 256)
  for (int r = 0; r < nv; ++r) {
    auto& rr = rows[(size_t)r];
    for (int64_t z = iptr[(size_t)r]; z < iptr[(size_t)r + 1]; ++z) {
      const int c = inc_cell[(size_t)z];
      for (int b = 0; b < 8; ++b) {
        const int g = S.ref[8 * (size_t)c + b];
        if (g >= 0) rr.push_back(g);
      }
    }
    std::sort(rr.begin(), rr.end());
    rr.erase(std::unique(rr.begin(), rr.end()), rr.end());
  }
  for (int r = 0; r < nv; ++r) {
    if (!std::binary_search(rows[(size_t)r].begin(), rows[(size_t)r].end(), r))
      throw std::runtime_error("momentum CSR row missing its diagonal");
    S.mom.row[(size_t)r + 1] = S.mom.row[(size_t)r] + (int64_t)rows[(size_t)r].size();
  }
  S.mom.col.resize((size_t)S.mom.row[(size_t)nv]);
  for (int r = 0; r < nv; ++r) std::copy(rows[(size_t)r].begin(), rows[(size_t)r].end(), S.mom.col.begin() + S.mom.row[(size_t)r]);
  std::vector<std::vector<int32_t>>().swap(rows);
  S.mom_diag_pos.assign((size_t)nv, -1);
  for (int r = 0; r < nv; ++r) {
    auto b = S.mom.col.begin() + S.mom.row[(size_t)r], e = S.mom.col.begin() + S.mom.row[(size_t)r + 1];
    auto it = std::lower_bound(b, e, r);
    const int64_t k = it - S.mom.col.begin();
    if (k > INT32_MAX) throw std::runtime_error("momentum diagonal position exceeds int32");
    S.mom_diag_pos[(size_t)r] = (int32_t)k;
  }

  // --- cell row slots
  S.row_slot.assign(64 * (size_t)nc, 255);
#pragma omp parallel for schedule(static)
  for (int c = 0; c < nc; ++c) {
    const int32_t* rf = &S.ref[8 * (size_t)c];
    for (int a = 0; a < 8 && !oerr.bad; ++a) {
      if (rf[a] < 0) continue;
      const int r = rf[a];
      auto b0 = S.mom.col.begin() + S.mom.row[(size_t)r], e0 = S.mom.col.begin() + S.mom.row[(size_t)r + 1];
      for (int b = 0; b < 8; ++b) {
        if (rf[b] < 0) continue;
        auto it = std::lower_bound(b0, e0, rf[b]);
        if (it == e0 || *it != rf[b]) { oerr.set("cell row slot missing"); break; }
        const auto slot = it - b0;
        if (slot >= 255) { oerr.set("momentum row slot overflow (>= 255)"); break; }
        S.row_slot[64 * (size_t)c + 8 * a + b] = (uint8_t)slot;
      }
    }
  }
  oerr.rethrow();

  // --- diffusion numerics, accumulated per row in ascending cell order
  const RefTensors& T = ref_tensors();
  S.mom.val.assign(S.mom.col.size(), 0.0);
  const double nu = S.pipe.nu;
#pragma omp parallel for schedule(dynamic, 64)
  for (int r = 0; r < nv; ++r) {
    const int64_t rb = S.mom.row[(size_t)r];
    for (int64_t z = iptr[(size_t)r]; z < iptr[(size_t)r + 1]; ++z) {
      const int c = inc_cell[(size_t)z];
      const int a = inc_a[(size_t)z];
      const double* I = &S.invJ[9 * (size_t)c];
      for (int b = 0; b < 8; ++b) {
        if (S.ref[8 * (size_t)c + b] < 0) continue;
        double v = 0.0;
        for (int j = 0; j < 3; ++j)
          for (int k = 0; k < 3; ++k)
            for (int d = 0; d < 3; ++d) v += T.D[a][b][j][k] * I[3 * j + d] * I[3 * k + d];
        v *= nu * S.det[(size_t)c];
        S.mom.val[(size_t)(rb + S.row_slot[64 * (size_t)c + 8 * a + b])] += v;
      }
    }
  }
  S.mom.diag.assign((size_t)nv, 0.0);
  for (int r = 0; r < nv; ++r) {
    const double d = S.mom.val[(size_t)S.mom_diag_pos[(size_t)r]];
    if (!(d > 0.0) || !std::isfinite(d)) throw std::runtime_error("non-positive diffusion diagonal");
    S.mom.diag[(size_t)r] = d;
  }

  tm.mark("momentum_csr");
  // --- greedy colouring in row order: lowest colour unused by lower neighbours
  S.color.assign((size_t)nv, -1);
  {
    std::vector<int> mark(64, -1);
    int maxc = -1;
    for (int i = 0; i < nv; ++i) {
      for (int64_t k = S.mom.row[(size_t)i]; k < S.mom.row[(size_t)i + 1]; ++k) {
        const int j = S.mom.col[(size_t)k];
        if (j >= i) continue;
        const int cj = S.color[(size_t)j];
        if (cj >= (int)mark.size()) mark.resize((size_t)cj + 32, -1);
        mark[(size_t)cj] = i;
      }
      int c = 0;
      while (c < (int)mark.size() && mark[(size_t)c] == i) ++c;
      if (c == (int)mark.size()) mark.resize(mark.size() + 32, -1);
      S.color[(size_t)i] = c;
      maxc = std::max(maxc, c);
    }
    S.ncolors = maxc + 1;
    S.color_off.assign((size_t)S.ncolors + 1, 0);
    for (int i = 0; i < nv; ++i) ++S.color_off[(size_t)S.color[(size_t)i] + 1];
    for (int c = 0; c < S.ncolors; ++c) S.color_off[(size_t)c + 1] += S.color_off[(size_t)c];
    S.color_rows.resize((size_t)nv);
    std::vector<int32_t> pos(S.color_off.begin(), S.color_off.end() - 1);
    for (int i = 0; i < nv; ++i) S.color_rows[(size_t)pos[(size_t)S.color[(size_t)i]]++] = i;
    for (int i = 0; i < nv; ++i)
      for (int64_t k = S.mom.row[(size_t)i]; k < S.mom.row[(size_t)i + 1]; ++k) {
        const int j = S.mom.col[(size_t)k];
        if (j != i && S.color[(size_t)j] == S.color[(size_t)i]) throw std::runtime_error("colouring conflict");
      }
  }

  tm.mark("colouring");
  // --- static Dirichlet diffusion RHS (cell order)
  for (auto& r : S.static_rhs) r.assign((size_t)nv, 0.0);
  for (int c = 0; c < nc; ++c) {
    const int32_t* rf = &S.ref[8 * (size_t)c];
    bool any_fixed = false, any_free = false;
    for (int a = 0; a < 8; ++a) (rf[a] < 0 ? any_fixed : any_free) = true;
    if (!any_fixed || !any_free) continue;
    const double* I = &S.invJ[9 * (size_t)c];
    double metric[3][3] = {{0}};
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k)
        for (int d = 0; d < 3; ++d) metric[j][k] += I[3 * j + d] * I[3 * k + d];
    for (int a = 0; a < 8; ++a) {
      if (rf[a] < 0) continue;
      for (int b = 0; b < 8; ++b) {
        if (rf[b] >= 0) continue;
        double v = 0;
        for (int j = 0; j < 3; ++j)
          for (int k = 0; k < 3; ++k) v += T.D[a][b][j][k] * metric[j][k];
        const double K = nu * S.det[(size_t)c] * v;
        const double* fv = &S.fixed_value[3 * (size_t)(-rf[b] - 1)];
        for (int d = 0; d < 3; ++d) S.static_rhs[(size_t)d][(size_t)rf[a]] -= K * fv[d];
      }
    }
  }

  // --- divergence coefficients, fixedDiv, volumes
  S.bco.assign(24 * (size_t)nc, 0.0);
  S.fixed_div.assign((size_t)nc, 0.0);
  S.volume.assign((size_t)nc, 0.0);
#pragma omp parallel for schedule(static)
  for (int c = 0; c < nc; ++c) {
    const double* I = &S.invJ[9 * (size_t)c];
    for (int a = 0; a < 8; ++a)
      for (int d = 0; d < 3; ++d) S.bco[24 * (size_t)c + 3 * a + d] = bcoeff(S.det[(size_t)c], I, a, d);
    S.volume[(size_t)c] = S.det[(size_t)c] / 6.0;
    double q = 0;
    for (int a = 0; a < 8; ++a) {
      const int r = S.ref[8 * (size_t)c + a];
      if (r >= 0) continue;
      const double* fv = &S.fixed_value[3 * (size_t)(-r - 1)];
      for (int d = 0; d < 3; ++d) q += S.bco[24 * (size_t)c + 3 * a + d] * fv[d];
    }
    S.fixed_div[(size_t)c] = q;
  }

  tm.mark("rhs+bcoeff");
  // --- fine Schur topology (velocity incidence, sorted unique pressure columns)
  {
    FineTopo& F = S.fine;
    F.n = nc;
    F.nv = nv;
    if ((uint64_t)nc >= (1ull << 29)) throw std::runtime_error("cell index exceeds 29 bits of the packed incidence");
    F.inc_off.assign((size_t)nv + 1, 0);
    for (int r = 0; r < nv; ++r) {
      const int64_t t = iptr[(size_t)r + 1];
      if (t > INT32_MAX) throw std::runtime_error("velocity incidence exceeds int32");
      F.inc_off[(size_t)r + 1] = (int32_t)t;
    }
    F.packed.resize(inc_cell.size());
    for (size_t z = 0; z < inc_cell.size(); ++z) F.packed[z] = ((uint32_t)inc_cell[z] << 3) | inc_a[z];
    // two passes: counts, then fill
    std::vector<int64_t> ncol((size_t)nc + 1, 0), ncon((size_t)nc + 1, 0);
#pragma omp parallel
    {
      std::vector<int32_t> tgt;
      tgt.reserve(256);
#pragma omp for schedule(dynamic, 256)
      for (int c = 0; c < nc; ++c) {
        tgt.clear();
        for (int a = 0; a < 8; ++a) {
          const int g = S.ref[8 * (size_t)c + a];
          if (g < 0) continue;
          for (int k = F.inc_off[(size_t)g]; k < F.inc_off[(size_t)g + 1]; ++k) tgt.push_back((int32_t)(F.packed[(size_t)k] >> 3));
        }
        ncon[(size_t)c + 1] = (int64_t)tgt.size();
        std::sort(tgt.begin(), tgt.end());
        ncol[(size_t)c + 1] = std::unique(tgt.begin(), tgt.end()) - tgt.begin();
      }
    }
    for (int c = 0; c < nc; ++c) {
      if (ncol[(size_t)c + 1] > 255) throw std::runtime_error("pressure row width exceeds uint8 slot capacity");
      if (ncol[(size_t)c + 1] == 0) throw std::runtime_error("empty pressure row");
      ncol[(size_t)c + 1] += ncol[(size_t)c];
      ncon[(size_t)c + 1] += ncon[(size_t)c];
    }
    if (ncol[(size_t)nc] > INT32_MAX || ncon[(size_t)nc] > INT32_MAX) throw std::runtime_error("fine pressure CSR exceeds int32");
    F.row.assign((size_t)nc + 1, 0);
    F.contrib_off.assign((size_t)nc + 1, 0);
    for (int c = 0; c <= nc; ++c) {
      F.row[(size_t)c] = (int32_t)ncol[(size_t)c];
      F.contrib_off[(size_t)c] = (int32_t)ncon[(size_t)c];
    }
    F.col.resize((size_t)ncol[(size_t)nc]);
    F.slot.resize((size_t)ncon[(size_t)nc]);
    F.diag_pos.assign((size_t)nc, -1);
    uint32_t rmax = 0;
#pragma omp parallel
    {
      std::vector<int32_t> tgt, uq;
      tgt.reserve(256);
      uq.reserve(256);
#pragma omp for schedule(dynamic, 256) reduction(max : rmax)
      for (int c = 0; c < nc; ++c) {
        tgt.clear();
        for (int a = 0; a < 8; ++a) {
          const int g = S.ref[8 * (size_t)c + a];
          if (g < 0) continue;
          for (int k = F.inc_off[(size_t)g]; k < F.inc_off[(size_t)g + 1]; ++k) tgt.push_back((int32_t)(F.packed[(size_t)k] >> 3));
        }
        uq = tgt;
        std::sort(uq.begin(), uq.end());
        uq.erase(std::unique(uq.begin(), uq.end()), uq.end());
        std::copy(uq.begin(), uq.end(), F.col.begin() + F.row[(size_t)c]);
        auto dit = std::lower_bound(uq.begin(), uq.end(), c);
        if (dit == uq.end() || *dit != c) { oerr.set("fine pressure diagonal absent"); continue; }
        F.diag_pos[(size_t)c] = F.row[(size_t)c] + (int32_t)(dit - uq.begin());
        size_t q = (size_t)F.contrib_off[(size_t)c];
        for (int32_t t : tgt) F.slot[q++] = (uint8_t)(std::lower_bound(uq.begin(), uq.end(), t) - uq.begin());
        rmax = std::max(rmax, (uint32_t)uq.size());
      }
    }
    oerr.rethrow();
    F.row_max = rmax;
  }
  tm.mark("fine_topology");
  // --- initial rAU: assemble at U = 0 (Dirichlet values still convect) and relax
  {
    std::array<std::vector<double>, 3> U0, conv;
    for (auto& u : U0) u.assign((size_t)nv, 0.0);
    std::vector<double> a;
    host_assemble_central(S, U0, a, conv);
    // the SUPG entry's snapshot includes the SUPG terms (h8_supg_main_setup.inc:6-7):
    // the Dirichlet inlet values convect even at U = 0
    if (o.supg) host_add_supg(S, U0, o.supg_tau_scale, o.supg_magic, a, conv);
    S.init_rau = host_finalize_relax(S, a, o.alpha_u, &S.init_delta);
    if (o.rau_scale != 1.0)
      for (double& q : S.init_rau) q *= o.rau_scale;
  }

  tm.mark("initial_rau");
  return S;
}

void host_assemble_central(const Setup& S, const std::array<std::vector<double>, 3>& U, std::vector<double>& aval,
                           std::array<std::vector<double>, 3>& conv) {
  // Row-owned gather over the incident cells of each row in ascending cell
  // order: every entry is summed in the order of the reference's cell-major
  // loop (g4_host.hpp:326-340), so the result is identical to it.
  aval = S.mom.val;
  for (auto& r : conv) r.assign((size_t)S.nv, 0.0);
  const RefTensors& T = ref_tensors();
  const FineTopo& F = S.fine;
#pragma omp parallel for schedule(dynamic, 256)
  for (int r = 0; r < S.nv; ++r) {
    const int64_t rb = S.mom.row[(size_t)r];
    for (int z = F.inc_off[(size_t)r]; z < F.inc_off[(size_t)r + 1]; ++z) {
      const int c = (int)(F.packed[(size_t)z] >> 3), a = (int)(F.packed[(size_t)z] & 7u);
      const int32_t* rf = &S.ref[8 * (size_t)c];
      const double* I = &S.invJ[9 * (size_t)c];
      double cf[3][8];
      for (int m = 0; m < 8; ++m)
        for (int d = 0; d < 3; ++d)
          cf[d][m] = rf[m] >= 0 ? U[(size_t)d][(size_t)rf[m]] : S.fixed_value[3 * (size_t)(-rf[m] - 1) + d];
      double ur[8][3] = {{0}};
      for (int m = 0; m < 8; ++m)
        for (int j = 0; j < 3; ++j)
          for (int d = 0; d < 3; ++d) ur[m][j] += cf[d][m] * I[3 * j + d];
      for (int b = 0; b < 8; ++b) {
        double v = 0;
        for (int m = 0; m < 8; ++m)
          for (int j = 0; j < 3; ++j) v += ur[m][j] * T.T[a][m][b][j];
        const double C = S.det[(size_t)c] * v;
        if (rf[b] >= 0) {
          aval[(size_t)(rb + S.row_slot[64 * (size_t)c + 8 * a + b])] += C;
        } else {
          const double* fv = &S.fixed_value[3 * (size_t)(-rf[b] - 1)];
          for (int d = 0; d < 3; ++d) conv[(size_t)d][(size_t)r] -= C * fv[d];
        }
      }
    }
  }
}

void supg_cell_block(const Setup& S, int c, const std::array<std::vector<double>, 3>& U, double tau_scale, double magic,
                     double out[64]) {
  const int32_t* rf = &S.ref[8 * (size_t)c];
  double coeff[3][8];
  for (int m = 0; m < 8; ++m)
    for (int d = 0; d < 3; ++d)
      coeff[d][m] = rf[m] >= 0 ? U[(size_t)d][(size_t)rf[m]] : S.fixed_value[3 * (size_t)(-rf[m] - 1) + d];
  const double* I = &S.invJ[9 * (size_t)c];
  double gl[4][3], gd[4][4];
  for (int d = 0; d < 3; ++d) {
    gl[0][d] = -(I[d] + I[3 + d] + I[6 + d]);
    gl[1][d] = I[d];
    gl[2][d] = I[3 + d];
    gl[3][d] = I[6 + d];
  }
  for (int i = 0; i < 4; ++i)
    for (int j = i; j < 4; ++j) {
      double q = 0.0;
      for (int d = 0; d < 3; ++d) q += gl[i][d] * gl[j][d];
      gd[i][j] = gd[j][i] = q;
    }
  for (int k = 0; k < 64; ++k) out[k] = 0.0;
  const double nu = S.pipe.nu, h2 = S.h2[(size_t)c], diff = 4.0 * nu / h2;
  for (const QuadPoint& qp : tet_rule_64()) {
    const auto& lam = qp.lam;
    int js[4][3];
    double phi[8];
    for (int i = 0; i < 4; ++i) {
      int kk = 0;
      for (int j = 0; j < 4; ++j)
        if (j != i) js[i][kk++] = j;
      phi[i] = lam[(size_t)i];
      phi[4 + i] = 27.0 * lam[(size_t)js[i][0]] * lam[(size_t)js[i][1]] * lam[(size_t)js[i][2]];
    }
    double adv[3] = {0, 0, 0};
    for (int d = 0; d < 3; ++d)
      for (int m = 0; m < 8; ++m) adv[d] += coeff[d][m] * phi[m];
    const double speed2 = adv[0] * adv[0] + adv[1] * adv[1] + adv[2] * adv[2];
    double stream[8], strong[8];
    for (int a = 0; a < 4; ++a) stream[a] = strong[a] = adv[0] * gl[a][0] + adv[1] * gl[a][1] + adv[2] * gl[a][2];
    for (int i = 0; i < 4; ++i) {
      const int* j = js[i];
      const double l0 = lam[(size_t)j[0]], l1 = lam[(size_t)j[1]], l2 = lam[(size_t)j[2]];
      double gb[3];
      for (int d = 0; d < 3; ++d) gb[d] = 27.0 * (l1 * l2 * gl[j[0]][d] + l0 * l2 * gl[j[1]][d] + l0 * l1 * gl[j[2]][d]);
      stream[4 + i] = adv[0] * gb[0] + adv[1] * gb[1] + adv[2] * gb[2];
      const double lap = 54.0 * (l2 * gd[j[0]][j[1]] + l1 * gd[j[0]][j[2]] + l0 * gd[j[1]][j[2]]);
      strong[4 + i] = -nu * lap + stream[4 + i];
    }
    const double den = std::max(4.0 * speed2 / h2 + magic * diff * diff, 1.0e-30);
    const double w = tau_scale / std::sqrt(den) * qp.w * S.det[(size_t)c];
    for (int a = 0; a < 8; ++a) {
      const double ta = w * stream[a];
      for (int b = 0; b < 8; ++b) out[8 * a + b] += ta * strong[b];
    }
  }
}

void host_add_supg(const Setup& S, const std::array<std::vector<double>, 3>& U, double tau_scale, double magic,
                   std::vector<double>& aval, std::array<std::vector<double>, 3>& conv) {
  std::vector<double> blk(64 * (size_t)S.nc);
#pragma omp parallel for schedule(static)
  for (int c = 0; c < S.nc; ++c) supg_cell_block(S, c, U, tau_scale, magic, &blk[64 * (size_t)c]);
  // row gather in ascending cell order: the order of the cell loop of the
  // reference's host twin
  const FineTopo& F = S.fine;
#pragma omp parallel for schedule(dynamic, 256)
  for (int r = 0; r < S.nv; ++r) {
    const int64_t rb = S.mom.row[(size_t)r];
    for (int z = F.inc_off[(size_t)r]; z < F.inc_off[(size_t)r + 1]; ++z) {
      const int c = (int)(F.packed[(size_t)z] >> 3), a = (int)(F.packed[(size_t)z] & 7u);
      const int32_t* rf = &S.ref[8 * (size_t)c];
      for (int b = 0; b < 8; ++b) {
        const double v = blk[64 * (size_t)c + 8 * a + b];
        if (rf[b] >= 0) {
          aval[(size_t)(rb + S.row_slot[64 * (size_t)c + 8 * a + b])] += v;
        } else {
          const double* fv = &S.fixed_value[3 * (size_t)(-rf[b] - 1)];
          for (int d = 0; d < 3; ++d) conv[(size_t)d][(size_t)r] -= v * fv[d];
        }
      }
    }
  }
}

std::vector<double> host_finalize_relax(const Setup& S, std::vector<double>& a, double alpha_u, std::vector<double>* delta) {
  std::vector<double> rau((size_t)S.nv), dl((size_t)S.nv);
  const double fac = 1.0 / alpha_u - 1.0;
  for (int i = 0; i < S.nv; ++i) {
    double m = 0;
    for (int64_t k = S.mom.row[(size_t)i]; k < S.mom.row[(size_t)i + 1]; ++k) m += std::abs(a[(size_t)k]);
    const double de = fac * m;
    dl[(size_t)i] = de;
    const size_t dp = (size_t)S.mom_diag_pos[(size_t)i];
    a[dp] += de;
    if (!(a[dp] > 0)) throw std::runtime_error("relaxed momentum diagonal invalid");
    rau[(size_t)i] = 1.0 / a[dp];
  }
  if (delta) *delta = std::move(dl);
  return rau;
}

CsrHost host_fine_csr(const Setup& S, const std::vector<double>& rau) {
  const FineTopo& F = S.fine;
  CsrHost A;
  A.n = F.n;
  A.row.assign(F.row.begin(), F.row.end());
  A.col = F.col;
  A.val.assign(F.col.size(), 0.0);
  A.diag.assign((size_t)F.n, 0.0);
  OmpError oerr;
#pragma omp parallel for schedule(dynamic, 256)
  for (int c = 0; c < F.n; ++c) {
    const int rb = F.row[(size_t)c];
    int q = F.contrib_off[(size_t)c];
    for (int a = 0; a < 8; ++a) {
      const int g = S.ref[8 * (size_t)c + a];
      if (g < 0) continue;
      const double rv = rau[(size_t)g];
      const double* ba = &S.bco[24 * (size_t)c + 3 * a];
      for (int k = F.inc_off[(size_t)g]; k < F.inc_off[(size_t)g + 1]; ++k, ++q) {
        const uint32_t pk = F.packed[(size_t)k];
        const double* bb = &S.bco[24 * (size_t)(pk >> 3) + 3 * (pk & 7u)];
        const double dot = ba[0] * bb[0] + ba[1] * bb[1] + ba[2] * bb[2];
        A.val[(size_t)(rb + F.slot[(size_t)q])] += rv * dot;
      }
    }
    const double d = A.val[(size_t)F.diag_pos[(size_t)c]];
    if (!(d > 0.0) || !std::isfinite(d)) oerr.set("fine pressure CSR non-positive diagonal");
    A.diag[(size_t)c] = d;
  }
  oerr.rethrow();
  return A;
}

}  // namespace nds
