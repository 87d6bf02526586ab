// Output surface of the solver: VTU file, Hagen-Poiseuille errors and the
// pressure-drop fit, following
//   h12_vtu_output.hpp:26-94          (ASCII VTU, 17 significant digits)
//   h8_hp_diagnostics.inc:18-100      (U and shifted-P L2 errors, Duffy 125-point rule)
//   g4_host.hpp:424                    (least-squares dp/dz over cell centroids)
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "diagnostics.hpp"
#include "fem.hpp"

namespace nds {

namespace {
inline double coeff_value(const Setup& S, int c, int a, int d, const double* const U[3]) {
  const int r = S.ref[8 * (size_t)c + a];
  if (r >= 0) return U[d][r];
  return S.fixed_value[3 * (size_t)(-r - 1) + d];
}
}  // namespace

double pressure_drop_fit(const Mesh& m, const double* p) {
  long double sz = 0, sp = 0, szz = 0, szp = 0;
  const long double n = (long double)m.n_cells();
  for (int c = 0; c < m.n_cells(); ++c) {
    double z = 0;
    for (int i = 0; i < 4; ++i) z += m.z(m.tets[(size_t)c][(size_t)i]) * .25;
    sz += z;
    sp += p[c];
    szz += (long double)z * z;
    szp += (long double)z * p[c];
  }
  const long double den = n * szz - sz * sz;
  if (std::abs((double)den) < 1e-300) return 0;
  const long double slope = (n * szp - sz * sp) / den;
  double zmin = 1e300, zmax = -1e300;
  for (int v = 0; v < m.n_points(); ++v) {
    zmin = std::min(zmin, m.z(v));
    zmax = std::max(zmax, m.z(v));
  }
  return (double)(-slope * (zmax - zmin));
}

HpErrors hp_errors(const Mesh& m, const Setup& S, const double* u0, const double* u1, const double* u2, const double* p) {
  const double* U[3] = {u0, u1, u2};
  const auto& Q = tet_rule_125();
  const PipeBC& P = S.pipe;
  long double total = 0, shift_int = 0;
  for (int c = 0; c < S.nc; ++c) {
    const auto& t = m.tets[(size_t)c];
    const double det = S.det[(size_t)c];
    for (const auto& q : Q) {
      double z = 0;
      for (int i = 0; i < 4; ++i) z += q.lam[(size_t)i] * m.z(t[(size_t)i]);
      const double pe = P.hp_gradient * (P.z_out - z);
      const double w = q.w * det;
      total += w;
      shift_int += (long double)(p[c] - pe) * w;
    }
  }
  const double shift = (double)(shift_int / std::max(total, (long double)1e-300L));
  long double ue2 = 0, un2 = 0, pe2 = 0, pn2 = 0;
  for (int c = 0; c < S.nc; ++c) {
    const auto& t = m.tets[(size_t)c];
    double coeff[3][8];
    for (int a = 0; a < 8; ++a)
      for (int d = 0; d < 3; ++d) coeff[d][a] = coeff_value(S, c, a, d, U);
    for (const auto& q : Q) {
      double phi[8], g[8][3];
      basis_eval(q.lam, phi, g);
      double x = 0, y = 0, z = 0;
      for (int i = 0; i < 4; ++i) {
        x += q.lam[(size_t)i] * m.x(t[(size_t)i]);
        y += q.lam[(size_t)i] * m.y(t[(size_t)i]);
        z += q.lam[(size_t)i] * m.z(t[(size_t)i]);
      }
      double uh[3] = {0, 0, 0};
      for (int d = 0; d < 3; ++d)
        for (int a = 0; a < 8; ++a) uh[d] += coeff[d][a] * phi[a];
      const double rr = (x - P.cx) * (x - P.cx) + (y - P.cy) * (y - P.cy);
      const double uz = 2.0 * P.bulk * (1.0 - rr / (P.R * P.R));
      const double pe = P.hp_gradient * (P.z_out - z);
      const double w = q.w * S.det[(size_t)c];
      const double d0 = uh[0], d1 = uh[1], d2 = uh[2] - uz;
      ue2 += (long double)(d0 * d0 + d1 * d1 + d2 * d2) * w;
      un2 += (long double)(uz * uz) * w;
      const double dp = p[c] - shift - pe;
      pe2 += (long double)(dp * dp) * w;
      pn2 += (long double)(pe * pe) * w;
    }
  }
  HpErrors E;
  const double ideal = 3.141592653589793238462643383279502884 * P.R * P.R * P.L;
  E.h_eff = std::cbrt(ideal / (double)std::max(1, S.nc));
  E.u_l2 = std::sqrt((double)ue2);
  E.u_rel_l2 = std::sqrt((double)(ue2 / std::max(un2, (long double)1e-300L)));
  E.p_shifted_l2 = std::sqrt((double)pe2);
  E.p_shifted_rel_l2 = std::sqrt((double)(pe2 / std::max(pn2, (long double)1e-300L)));
  E.pressure_shift = shift;
  E.dp_fit = pressure_drop_fit(m, p);
  E.dp_exact = P.hp_drop;
  E.dp_rel_err = std::abs(E.dp_fit - E.dp_exact) / std::max(std::abs(E.dp_exact), 1e-300);
  return E;
}

void cell_average_velocity(const Setup& S, const double* u0, const double* u1, const double* u2, std::vector<double>& out) {
  const double* U[3] = {u0, u1, u2};
  out.assign(3 * (size_t)S.nc, 0.0);
  for (int c = 0; c < S.nc; ++c)
    for (int d = 0; d < 3; ++d) {
      double v = 0;
      for (int a = 0; a < 4; ++a) v += 0.25 * coeff_value(S, c, a, d, U);
      for (int a = 4; a < 8; ++a) v += (9.0 / 40.0) * coeff_value(S, c, a, d, U);
      out[3 * (size_t)c + d] = v;
    }
}

void write_vtu(const std::string& path, const Mesh& m, const Setup& S, const double* u0, const double* u1, const double* u2,
               const double* p, bool converged, int outer) {
  std::vector<double> uc;
  cell_average_velocity(S, u0, u1, u2, uc);
  std::vector<double> us(3 * (size_t)m.n_points(), 0.0), w((size_t)m.n_points(), 0.0);
  for (int c = 0; c < S.nc; ++c) {
    const double vol = S.det[(size_t)c] / 6.0;
    for (int i = 0; i < 4; ++i) {
      const int v = m.tets[(size_t)c][(size_t)i];
      for (int d = 0; d < 3; ++d) us[3 * (size_t)v + d] += vol * uc[3 * (size_t)c + d];
      w[(size_t)v] += vol;
    }
  }
  for (int v = 0; v < m.n_points(); ++v)
    if (w[(size_t)v] > 0.0)
      for (int d = 0; d < 3; ++d) us[3 * (size_t)v + d] /= w[(size_t)v];
  std::ofstream out(path);
  if (!out) throw std::runtime_error("cannot open VTU output: " + path);
  out << std::setprecision(17) << std::scientific;
  out << "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
      << "<UnstructuredGrid>\n<Piece NumberOfPoints=\"" << m.n_points() << "\" NumberOfCells=\"" << m.n_cells() << "\">\n";
  out << "<Points><DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n";
  for (int v = 0; v < m.n_points(); ++v) out << m.x(v) << ' ' << m.y(v) << ' ' << m.z(v) << '\n';
  out << "</DataArray></Points>\n<Cells>\n<DataArray type=\"Int64\" Name=\"connectivity\" format=\"ascii\">\n";
  for (const auto& t : m.tets) out << t[0] << ' ' << t[1] << ' ' << t[2] << ' ' << t[3] << '\n';
  out << "</DataArray>\n<DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\">\n";
  for (int c = 0; c < m.n_cells(); ++c) out << 4 * (c + 1) << '\n';
  out << "</DataArray>\n<DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n";
  for (int c = 0; c < m.n_cells(); ++c) out << 10 << '\n';
  out << "</DataArray>\n</Cells>\n<PointData Vectors=\"U0_stream\">\n"
      << "<DataArray type=\"Float64\" Name=\"U0_stream\" NumberOfComponents=\"3\" format=\"ascii\">\n";
  for (int v = 0; v < m.n_points(); ++v) out << us[3 * (size_t)v] << ' ' << us[3 * (size_t)v + 1] << ' ' << us[3 * (size_t)v + 2] << '\n';
  out << "</DataArray>\n</PointData>\n<CellData Scalars=\"p_P0\" Vectors=\"U0\">\n"
      << "<DataArray type=\"Float64\" Name=\"p_P0\" NumberOfComponents=\"1\" format=\"ascii\">\n";
  for (int c = 0; c < S.nc; ++c) out << p[c] << '\n';
  out << "</DataArray>\n<DataArray type=\"Float64\" Name=\"U0\" NumberOfComponents=\"3\" format=\"ascii\">\n";
  for (int c = 0; c < S.nc; ++c) out << uc[3 * (size_t)c] << ' ' << uc[3 * (size_t)c + 1] << ' ' << uc[3 * (size_t)c + 2] << '\n';
  out << "</DataArray>\n<DataArray type=\"Int32\" Name=\"solve_converged\" NumberOfComponents=\"1\" format=\"ascii\">\n";
  for (int c = 0; c < S.nc; ++c) out << (converged ? 1 : 0) << '\n';
  out << "</DataArray>\n<DataArray type=\"Int32\" Name=\"outer_iterations\" NumberOfComponents=\"1\" format=\"ascii\">\n";
  for (int c = 0; c < S.nc; ++c) out << outer << '\n';
  out << "</DataArray>\n</CellData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n";
  out.close();
  if (!out) throw std::runtime_error("VTU write failed: " + path);
}

}  // namespace nds
