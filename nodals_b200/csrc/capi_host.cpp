// Host half of the C ABI: meshes, options and the host setup ("problem").
// No CUDA call is made here, so these entry points work on CPU-only hosts.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/nodals_b200.h"
#include "capi_internal.hpp"
#include "host/hybrid.hpp"
#include "host/amg.hpp"
#include "host/diagnostics.hpp"
#include "host/fem.hpp"
#include "host/mesh.hpp"
#include "host/setup.hpp"

namespace {
thread_local std::string g_err;
}

namespace nds {
void set_error(const std::string& e) { g_err = e; }
}  // namespace nds

using nds::set_error;

namespace {
struct HybridAmgHandle {
  nds::HybridSchurCsr fine;
  nds::Hierarchy H;
  nds::HybridFlow flow;
  nds::HybridStokes div;
  std::vector<double> scalars[4];
  std::vector<int64_t> ncoarse;
  std::map<std::string, nds_array> arrays;
};
template <class T> nds_array view_of(const std::vector<T>& v, int dtype) { return nds_array{v.data(), (int64_t)v.size(), dtype}; }
}  // namespace

extern "C" {

const char* nds_last_error(void) { return g_err.c_str(); }
const char* nds_version(void) { return "nodals_b200 0.1 (sm_100a)"; }

void nds_options_default(nds_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  // the H8 binary's own defaults (h8_main_base.cu:1749-1785)
  o->re = 20;
  o->bulk = 1;
  o->simple_tol = 1e-6;
  o->alpha_u = 0.5;
  o->alpha_p = 0.5;
  o->rau_scale = 1.0;
  o->max_outer = 2500;
  o->run_mode = NDS_RUN_FIXED10;
  o->momentum_work = NDS_MOM_FGS1;
  o->mom_omega = 1.0;
  o->mom_rtol = 1e-6;
  o->mom_atol = 1e-12;
  o->mom_drop = 0.1;
  o->mom_max = 20000;
  o->pressure_solver = NDS_P_PCG;
  o->p_rtol = 0.5;
  o->p_atol = 1e-12;
  o->p_max = 20;
  o->snapshot_tol = 5e-6;
  o->fine_csr_refresh_every = 1;
  o->p_richardson_omega = 1.0;
  o->p_cheb_degree = 3;
  o->p_power_its = 6;
  o->p_cheb_low_fraction = 0.05;
  o->p_power_safety = 1.15;
  o->amg_hierarchy = NDS_AMG_SA;
  o->amg_smoother = NDS_SM_CHEB2;
  o->amg_terminal = 1000;
  o->amg_spectrum_policy = NDS_SPEC_AUTO;
  o->amg_power_its = 16;
  o->amg_cheb_degree = 2;
  o->amg_lambda_safety = 1.5;
  o->amg_lambda_low_fraction = 0.05;
  o->amg_jacobi_omega = 0.7;
  o->amg_jacobi_fine_sweeps = 1;
  o->amg_jacobi_coarse_sweeps = 1;
  o->amg_mcgs_omega = 1.0;
  o->amg_mcgs_fine_sweeps = 1;
  o->amg_mcgs_coarse_sweeps = 1;
  o->amg_mcgs_order = NDS_MCGS_SYMMETRIC;
  o->cf_theta = 0.25;
  o->cf_pmax = 4;
  o->cf_interp = NDS_CF_DIRECT;
  o->cf_aggressive_first = 0;
  std::strcpy(o->wall, "patch_0_0");
  std::strcpy(o->inlet, "patch_2_0");
  std::strcpy(o->outlet, "patch_1_0");
  o->precision = NDS_FP64;
  o->threads = 0;
  o->device = 0;
  o->verbose = 0;
  o->supg = 0;
  o->supg_tau_scale = 0.05;
  o->supg_magic = 9.0;
  o->p_krylov = NDS_KRYLOV_PCG;
  o->p_restart = 30;
  o->p_inner_rtol = 1e-3;
  o->p_refine_max = 8;
  o->p_guess = 0;
  o->learned = 0;
  o->geom_from_inlet = 0;
  o->p_guess_fresh = 0;
  o->amg_half = 0;
}

int nds_mesh_read_polymesh(const char* dir, nds_mesh** out) {
  if (!dir || !out) { set_error("null argument"); return NDS_E_INVALID; }
  try {
    *out = reinterpret_cast<nds_mesh*>(new nds::Mesh(nds::read_polymesh(dir)));
    return NDS_OK;
  } catch (const std::exception& e) {
    set_error(e.what());
    return NDS_E_SETUP;
  }
}

int nds_mesh_read_msh2(const char* path, nds_mesh** out) {
  if (!path || !out) { set_error("null argument"); return NDS_E_INVALID; }
  try {
    *out = reinterpret_cast<nds_mesh*>(new nds::Mesh(nds::read_msh2(path)));
    return NDS_OK;
  } catch (const std::exception& e) {
    set_error(e.what());
    return NDS_E_SETUP;
  }
}
int nds_hybrid_operator_audit(const char* path, double nu, double gamma, double rau_scale, double norms[3]) {
  if (!path || !norms || !(nu > 0) || !(gamma > 0) || !(rau_scale > 0)) {
    set_error("nds_hybrid_operator_audit: bad argument");
    return NDS_E_INVALID;
  }
  try {
    const nds::HybridMesh m = nds::read_hxt1_hybrid(path);
    const nds::HybridStokes H = nds::build_hybrid_stokes(m, nds::interface_plans(m), nu, gamma);
    const int nv = H.nvel, np = H.np;
    std::vector<double> a((size_t)nv), b0((size_t)nv), b1((size_t)nv), b2((size_t)nv), p((size_t)np);
    for (int g = 0; g < nv; ++g) {
      const double q = g + 1;
      a[(size_t)g] = std::sin(0.00113 * q);
      b0[(size_t)g] = std::cos(.00131 * q);
      b1[(size_t)g] = std::sin(.00091 * q + .2);
      b2[(size_t)g] = std::cos(.00157 * q - .1);
    }
    for (int i = 0; i < np; ++i) p[(size_t)i] = std::sin(.00107 * (i + 1));
    auto norm = [](const std::vector<double>& x) {
      long double s = 0;
      for (double v : x) s += (long double)v * v;
      return (double)std::sqrt(s);
    };
    std::vector<double> y((size_t)nv, 0.0), c((size_t)np, 0.0), v[3];
    for (int i = 0; i < nv; ++i)
      for (int32_t k = H.a_row[(size_t)i]; k < H.a_row[(size_t)i + 1]; ++k) y[(size_t)i] += H.a_val[(size_t)k] * a[(size_t)H.a_col[(size_t)k]];
    norms[0] = norm(y);
    for (int i = 0; i < np; ++i)
      for (int32_t k = H.b_row[(size_t)i]; k < H.b_row[(size_t)i + 1]; ++k) {
        const size_t g = (size_t)H.b_col[(size_t)k];
        c[(size_t)i] += H.bx[(size_t)k] * b0[g] + H.by[(size_t)k] * b1[g] + H.bz[(size_t)k] * b2[g];
      }
    norms[1] = norm(c);
    for (auto& q : v) q.assign((size_t)nv, 0.0);
    for (int g = 0; g < nv; ++g) {
      const double r = H.fixed[(size_t)g] ? 0.0 : rau_scale / H.diag_rau[(size_t)g];
      for (int32_t k = H.bt_row[(size_t)g]; k < H.bt_row[(size_t)g + 1]; ++k) {
        const double q = p[(size_t)H.bt_col[(size_t)k]];
        v[0][(size_t)g] += H.btx[(size_t)k] * q;
        v[1][(size_t)g] += H.bty[(size_t)k] * q;
        v[2][(size_t)g] += H.btz[(size_t)k] * q;
      }
      for (auto& q : v) q[(size_t)g] *= r;
    }
    std::fill(c.begin(), c.end(), 0.0);
    for (int i = 1; i < np; ++i)  // row 0 is the pressure pin
      for (int32_t k = H.b_row[(size_t)i]; k < H.b_row[(size_t)i + 1]; ++k) {
        const size_t g = (size_t)H.b_col[(size_t)k];
        c[(size_t)i] += H.bx[(size_t)k] * v[0][g] + H.by[(size_t)k] * v[1][g] + H.bz[(size_t)k] * v[2][g];
      }
    norms[2] = norm(c);
    return NDS_OK;
  } catch (const std::exception& e) {
    set_error(e.what());
    return NDS_E_SETUP;
  }
}

int nds_hybrid_operator_patch(const char* path, double nu, double gamma, double out[12]) {
  if (!path || !out || !(nu > 0) || !(gamma > 0)) { set_error("nds_hybrid_operator_patch: bad argument"); return NDS_E_INVALID; }
  try {
    const nds::HybridMesh m = nds::read_hxt1_hybrid(path);
    const auto P = nds::interface_plans(m);
    std::vector<int32_t> fr, fc, vr, vc;
    std::vector<double> fv, vv;
    nds::hybrid_velocity_operator(m, P, nu, gamma, true, fr, fc, fv);
    nds::hybrid_velocity_operator(m, P, nu, gamma, false, vr, vc, vv);
    const int nv = m.nvel();
    auto apply = [&](const std::vector<int32_t>& r, const std::vector<int32_t>& c, const std::vector<double>& v,
                     const std::vector<double>& x) {
      std::vector<double> y((size_t)nv, 0.0);
      for (int i = 0; i < nv; ++i)
        for (int32_t k = r[(size_t)i]; k < r[(size_t)i + 1]; ++k) y[(size_t)i] += v[(size_t)k] * x[(size_t)c[(size_t)k]];
      return y;
    };
    // vertex values c + a . x, bubbles zero (the field is in both spaces)
    auto affine = [&](double c0, double ax, double ay, double az) {
      std::vector<double> u((size_t)nv, 0.0);
      for (int i = 0; i < m.nv(); ++i)
        u[(size_t)i] = c0 + ax * m.xyz[3 * (size_t)i] + ay * m.xyz[3 * (size_t)i + 1] + az * m.xyz[3 * (size_t)i + 2];
      return u;
    };
    std::vector<int32_t> ids;
    for (const auto& r : m.interface) {
      ids.push_back(r[2]);
      ids.push_back(r[5]);
      ids.push_back(r[8]);
    }
    std::sort(ids.begin(), ids.end());
    ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
    auto bubble_max = [&](const std::vector<double>& y) {
      double q = 0;
      for (int32_t g : ids) q = std::max(q, std::abs(y[(size_t)g]));
      return q;
    };
    double cmax = 0;
    for (double v : apply(fr, fc, fv, affine(1.0, 0, 0, 0))) cmax = std::max(cmax, std::abs(v));
    out[0] = cmax;
    const double coeff[3][4] = {{0.7, 1.0, 0.20, -0.10}, {-0.4, 0.30, 1.10, 0.15}, {0.2, -0.25, 0.35, 0.90}};
    for (int k = 0; k < 3; ++k) {
      const auto u = affine(coeff[k][0], coeff[k][1], coeff[k][2], coeff[k][3]);
      out[1 + k] = bubble_max(apply(vr, vc, vv, u));
      out[4 + k] = bubble_max(apply(fr, fc, fv, u));
    }
    std::vector<double> x((size_t)nv, 0.0), y((size_t)nv, 0.0);
    for (int32_t g : ids) {
      x[(size_t)g] = std::sin(0.001731 * (g + 1));
      y[(size_t)g] = std::cos(0.002117 * (g + 3));
    }
    const auto Ax = apply(fr, fc, fv, x), Ay = apply(fr, fc, fv, y);
    auto dot = [&](const std::vector<double>& a, const std::vector<double>& b) {
      long double q = 0;
      for (int i = 0; i < nv; ++i) q += (long double)a[(size_t)i] * b[(size_t)i];
      return (double)q;
    };
    out[7] = dot(x, Ax);
    out[8] = dot(y, Ay);
    out[9] = dot(x, Ay);
    out[10] = dot(y, Ax);
    out[11] = (double)ids.size();
    return NDS_OK;
  } catch (const std::exception& e) {
    set_error(e.what());
    return NDS_E_SETUP;
  }
}

int nds_hybrid_divergence_audit(const char* path, double out[16]) {
  if (!path || !out) { set_error("nds_hybrid_divergence_audit: null argument"); return NDS_E_INVALID; }
  try {
    const nds::HybridMesh m = nds::read_hxt1_hybrid(path);
    const auto P = nds::interface_plans(m);
    nds::HybridStokes B;
    nds::build_hybrid_divergence(m, P, B);
    const int nv = B.nvel, np = B.np, nh = m.nhex();
    std::vector<double> rau((size_t)nv);
    for (int g = 0; g < nv; ++g) rau[(size_t)g] = 0.8 + 0.2 * (0.5 + 0.5 * std::sin(0.000731 * (g + 1)));
    auto Bu = [&](const std::vector<double>& u0, const std::vector<double>& u1, const std::vector<double>& u2) {
      std::vector<double> y((size_t)np, 0.0);
      for (int i = 0; i < np; ++i)
        for (int32_t k = B.b_row[(size_t)i]; k < B.b_row[(size_t)i + 1]; ++k) {
          const size_t g = (size_t)B.b_col[(size_t)k];
          y[(size_t)i] += B.bx[(size_t)k] * u0[g] + B.by[(size_t)k] * u1[g] + B.bz[(size_t)k] * u2[g];
        }
      return y;
    };
    auto BTp = [&](const std::vector<double>& p, std::vector<double> v[3]) {
      for (int d = 0; d < 3; ++d) v[d].assign((size_t)nv, 0.0);
      for (int g = 0; g < nv; ++g)
        for (int32_t k = B.bt_row[(size_t)g]; k < B.bt_row[(size_t)g + 1]; ++k) {
          const double q = p[(size_t)B.bt_col[(size_t)k]];
          v[0][(size_t)g] += B.btx[(size_t)k] * q;
          v[1][(size_t)g] += B.bty[(size_t)k] * q;
          v[2][(size_t)g] += B.btz[(size_t)k] * q;
        }
    };
    auto dot = [](const std::vector<double>& a, const std::vector<double>& b) {
      long double q = 0;
      for (size_t i = 0; i < a.size(); ++i) q += (long double)a[i] * b[i];
      return (double)q;
    };
    out[0] = (double)B.b_col.size();
    double cmax = 0;
    for (int d = 0; d < 3; ++d) {
      std::vector<double> u[3] = {std::vector<double>((size_t)nv, 0.0), std::vector<double>((size_t)nv, 0.0),
                                  std::vector<double>((size_t)nv, 0.0)};
      for (int v = 0; v < m.nv(); ++v) u[d][(size_t)v] = 1.0;
      for (double y : Bu(u[0], u[1], u[2])) cmax = std::max(cmax, std::abs(y));
    }
    out[1] = cmax;
    {
      std::vector<double> u[3] = {std::vector<double>((size_t)nv, 0.0), std::vector<double>((size_t)nv, 0.0),
                                  std::vector<double>((size_t)nv, 0.0)};
      for (int v = 0; v < m.nv(); ++v)
        for (int d = 0; d < 3; ++d) u[d][(size_t)v] = m.xyz[3 * (size_t)v + d];
      const auto dv = Bu(u[0], u[1], u[2]);
      double ma = 0, mr = 0;
      for (int c = 0; c < np; ++c) {
        const double V = c < nh ? m.hex_geom[(size_t)c][0] : m.tet_geom[(size_t)(c - nh)][0];
        const double e = std::abs(dv[(size_t)c] - 3.0 * V);
        ma = std::max(ma, e);
        mr = std::max(mr, e / std::max(std::abs(3.0 * V), 1e-300));
      }
      out[2] = ma;
      out[3] = mr;
    }
    {
      std::vector<double> r[3] = {std::vector<double>((size_t)nv), std::vector<double>((size_t)nv),
                                  std::vector<double>((size_t)nv)};
      std::vector<double> pp((size_t)np), bt[3];
      for (int g = 0; g < nv; ++g) {
        const double q = g + 1;
        r[0][(size_t)g] = std::sin(.00113 * q);
        r[1][(size_t)g] = std::cos(.00171 * q);
        r[2][(size_t)g] = std::sin(.00091 * q + .3);
      }
      for (int i = 0; i < np; ++i) pp[(size_t)i] = std::cos(.00137 * (i + 1) + .2);
      BTp(pp, bt);
      out[4] = dot(pp, Bu(r[0], r[1], r[2]));
      out[5] = dot(r[0], bt[0]) + dot(r[1], bt[1]) + dot(r[2], bt[2]);
    }
    {
      std::vector<double> px((size_t)np), py((size_t)np);
      for (int i = 0; i < np; ++i) {
        const double q = i + 1;
        px[(size_t)i] = std::sin(.00073 * q);
        py[(size_t)i] = std::cos(.00109 * q + .17);
      }
      auto S = [&](const std::vector<double>& x) {
        std::vector<double> v[3];
        BTp(x, v);
        for (int d = 0; d < 3; ++d)
          for (int g = 0; g < nv; ++g) v[d][(size_t)g] *= rau[(size_t)g];
        return Bu(v[0], v[1], v[2]);
      };
      const auto Sx = S(px), Sy = S(py);
      out[6] = dot(px, Sx);
      out[7] = dot(py, Sy);
      out[8] = dot(px, Sy);
      out[9] = dot(py, Sx);
    }
    // interface sensitivity: each hex row carries the tet's traces and the
    // other way round, and the direct Schur entry of the pair is nonzero
    auto coeff = [&](int row, int g, double b[3]) {
      const auto bg = B.b_col.begin() + B.b_row[(size_t)row], en = B.b_col.begin() + B.b_row[(size_t)row + 1];
      const auto it = std::lower_bound(bg, en, g);
      if (it == en || *it != g) return false;
      const size_t k = (size_t)(it - B.b_col.begin());
      b[0] = B.bx[k];
      b[1] = B.by[k];
      b[2] = B.bz[k];
      return true;
    };
    double cmin = 1e300, cmx = 0, smin = 1e300, smx = 0;
    int missing = 0;
    for (const auto& p : P)
      for (int s2 = 0; s2 < 2; ++s2) {
        const int rh = p.hex_cell, rt = nh + p.tet_cell[s2];
        const auto& tv = m.tet_dofs[(size_t)p.tet_cell[s2]];
        const auto& hv = m.hex_dofs[(size_t)p.hex_cell];
        bool h_has_t = false, t_has_h = false;
        double cm = 0, b[3];
        for (int a = 0; a < 8; ++a)
          if (coeff(rh, tv[(size_t)a], b)) {
            h_has_t = true;
            cm = std::max(cm, std::sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]));
          }
        for (int a = 0; a < 14; ++a)
          if (coeff(rt, hv[(size_t)a], b)) {
            t_has_h = true;
            cm = std::max(cm, std::sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]));
          }
        long double ss = 0;
        for (int32_t k = B.b_row[(size_t)rh]; k < B.b_row[(size_t)rh + 1]; ++k) {
          double bt[3];
          if (coeff(rt, B.b_col[(size_t)k], bt))
            ss += (long double)rau[(size_t)B.b_col[(size_t)k]] *
                  (B.bx[(size_t)k] * bt[0] + B.by[(size_t)k] * bt[1] + B.bz[(size_t)k] * bt[2]);
        }
        const double sa = std::abs((double)ss);
        if (!(h_has_t && t_has_h) || !(sa > 0)) ++missing;
        if (sa > 0) {
          smin = std::min(smin, sa);
          smx = std::max(smx, sa);
        }
        if (cm > 0) {
          cmin = std::min(cmin, cm);
          cmx = std::max(cmx, cm);
        }
      }
    out[10] = cmin;
    out[11] = cmx;
    out[12] = smin;
    out[13] = smx;
    out[14] = 2.0 * (double)P.size();
    out[15] = missing;
    return NDS_OK;
  } catch (const std::exception& e) {
    set_error(e.what());
    return NDS_E_SETUP;
  }
}

int nds_hybrid_counts(const char* path, uint64_t counts[13]) {
  if (!path || !counts) { set_error("null argument"); return NDS_E_INVALID; }
  try {
    const nds::HybridMesh m = nds::read_hxt1_hybrid(path);
    std::copy(m.count, m.count + 13, counts);
    return NDS_OK;
  } catch (const std::exception& e) {
    set_error(e.what());
    return NDS_E_SETUP;
  }
}

int nds_hybrid_amg_create(const char* path, const double* rau, const nds_hybrid_flow_options* o, nds_hybrid_amg** out) {
  if (!path || !rau || !o || !out) { set_error("null argument"); return NDS_E_INVALID; }
  try {
    const nds::AmgOptions ao = nds::hybrid_amg_options(*o);
    const nds::HybridMesh m = nds::read_hxt1_hybrid(path);
    nds::HybridStokes B;
    nds::build_hybrid_divergence(m, nds::interface_plans(m), B);
    auto h = std::make_unique<HybridAmgHandle>();
    const int pin = nds::hybrid_pin(m);
    h->fine = nds::hybrid_schur_csr(B, pin, std::vector<double>(rau, rau + B.nvel));
    h->H = nds::build_cf_hierarchy(h->fine.A, ao);
    auto& A = h->arrays;
    h->scalars[0] = {(double)pin};
    h->scalars[1] = {(double)h->H.A.size()};
    h->scalars[2] = {h->H.fine_lambda};
    A["pin"] = view_of(h->scalars[0], 0);
    A["amg.levels"] = view_of(h->scalars[1], 0);
    A["amg.fineLambda"] = view_of(h->scalars[2], 0);
    A["fine.row"] = view_of(h->fine.A.row, 2);
    A["fine.col"] = view_of(h->fine.A.col, 1);
    A["fine.val"] = view_of(h->fine.A.val, 0);
    A["fine.diag"] = view_of(h->fine.A.diag, 0);
    A["fine.entryRow"] = view_of(h->fine.entry_row, 1);
    A["fine.diagPos"] = view_of(h->fine.diag_pos, 1);
    A["amg.levelLambda"] = view_of(h->H.level_lambda, 0);
    A["amg.terminal_inv"] = view_of(h->H.terminal_inv, 0);
    h->ncoarse.resize(h->H.P.size());
    for (size_t l = 0; l < h->H.P.size(); ++l) {
      const std::string p = "amg.P" + std::to_string(l) + ".";
      h->ncoarse[l] = h->H.P[l].nc;
      A[p + "nCoarse"] = nds_array{&h->ncoarse[l], 1, 2};
      A[p + "row"] = view_of(h->H.P[l].row, 2);
      A[p + "col"] = view_of(h->H.P[l].col, 1);
      A[p + "val"] = view_of(h->H.P[l].val, 0);
    }
    for (size_t l = 0; l < h->H.A.size(); ++l) {
      const std::string p = "amg.A" + std::to_string(l) + ".";
      A[p + "row"] = view_of(h->H.A[l].row, 2);
      A[p + "col"] = view_of(h->H.A[l].col, 1);
      A[p + "val"] = view_of(h->H.A[l].val, 0);
      A[p + "diag"] = view_of(h->H.A[l].diag, 0);
    }
    *out = reinterpret_cast<nds_hybrid_amg*>(h.release());
    return NDS_OK;
  } catch (const std::invalid_argument& e) {
    set_error(e.what());
    return NDS_E_INVALID;
  } catch (const std::exception& e) {
    set_error(e.what());
    return NDS_E_SETUP;
  }
}

int nds_hybrid_flow_setup(const char* path, const nds_hybrid_flow_options* o, nds_hybrid_amg** out) {
  if (!path || !o || !out) { set_error("null argument"); return NDS_E_INVALID; }
  try {
    auto h = std::make_unique<HybridAmgHandle>();
    const nds::HybridMesh m = nds::read_hxt1_hybrid(path);
    const auto P = nds::interface_plans(m);
    nds::HybridFlow& F = h->flow;
    F = nds::build_hybrid_flow(m, P, o->re, o->bulk, o->gamma);
    nds::build_hybrid_divergence(m, P, h->div);
    auto& A = h->arrays;
    h->scalars[0] = {(double)F.pin, F.radius, F.length, F.diameter, F.nu, (double)F.nhex, (double)F.ntet};
    A["flow.scalars"] = view_of(h->scalars[0], 0);  // pin, R, L, D, nu, nhex, ntet
    A["flow.row"] = view_of(F.row, 1);
    A["flow.col"] = view_of(F.col, 1);
    A["flow.diagPos"] = view_of(F.diag_pos, 1);
    A["flow.base"] = view_of(F.base, 0);
    A["flow.diagRBase"] = view_of(F.diag_r_base, 0);
    A["flow.srcOff"] = view_of(F.src_off, 1);
    A["flow.src"] = view_of(F.src, 1);
    A["flow.fixed"] = view_of(F.fixed, 3);
    A["flow.u0"] = view_of(F.u0, 0);
    A["flow.u1"] = view_of(F.u1, 0);
    A["flow.u2"] = view_of(F.u2, 0);
    A["flow.colourOff"] = view_of(F.colour_off, 1);
    A["flow.colourRows"] = view_of(F.colour_rows, 1);
    A["b.row"] = view_of(h->div.b_row, 1);
    A["b.col"] = view_of(h->div.b_col, 1);
    A["b.bx"] = view_of(h->div.bx, 0);
    A["b.by"] = view_of(h->div.by, 0);
    A["b.bz"] = view_of(h->div.bz, 0);
    {
      const auto& T = nds::ref_tensors().T;
      h->scalars[1].assign(&T[0][0][0][0], &T[0][0][0][0] + 8 * 8 * 8 * 3);
      A["centT"] = view_of(h->scalars[1], 0);  // T[a][m][b][j] = int phi_a phi_m dphi_b/dxi_j on the reference tet
    }
    *out = reinterpret_cast<nds_hybrid_amg*>(h.release());
    return NDS_OK;
  } catch (const std::exception& e) {
    set_error(e.what());
    return NDS_E_SETUP;
  }
}

int nds_hybrid_amg_array(const nds_hybrid_amg* hh, const char* name, nds_array* out) {
  if (!hh || !name || !out) { set_error("null argument"); return NDS_E_INVALID; }
  const auto* h = reinterpret_cast<const HybridAmgHandle*>(hh);
  auto it = h->arrays.find(name);
  if (it == h->arrays.end()) {
    set_error(std::string("unknown hybrid AMG array ") + name);
    return NDS_E_INVALID;
  }
  *out = it->second;
  return NDS_OK;
}

void nds_hybrid_amg_destroy(nds_hybrid_amg* h) { delete reinterpret_cast<HybridAmgHandle*>(h); }

int nds_hybrid_write_vtu(const char* hxt1_path, const char* vtu_path, const double* u0, const double* u1,
                         const double* u2, const double* pressure) {
  if (!hxt1_path || !vtu_path || !u0 || !u1 || !u2 || !pressure) { set_error("null argument"); return NDS_E_INVALID; }
  try {
    nds::write_hybrid_vtu(nds::read_hxt1_hybrid(hxt1_path), vtu_path, u0, u1, u2, pressure);
    return NDS_OK;
  } catch (const std::exception& e) {
    set_error(e.what());
    return NDS_E_SETUP;
  }
}

int nds_mesh_read_hxt1(const char* path, nds_mesh** out) {
  if (!path || !out) { set_error("null argument"); return NDS_E_INVALID; }
  try {
    *out = reinterpret_cast<nds_mesh*>(new nds::Mesh(nds::read_hxt1(path)));
    return NDS_OK;
  } catch (const std::exception& e) {
    set_error(e.what());
    return NDS_E_SETUP;
  }
}

int nds_mesh_from_arrays(int n_points, const double* xyz, int n_cells, const int32_t* tets, int n_bfaces,
                         const int32_t* btri, const int32_t* bpatch, int n_patches, const char* const* patch_names,
                         nds_mesh** out) {
  if (!xyz || !tets || !btri || !bpatch || !patch_names || !out || n_patches <= 0) {
    set_error("null or empty mesh arrays");
    return NDS_E_INVALID;
  }
  try {
    std::vector<std::string> names;
    for (int i = 0; i < n_patches; ++i) names.emplace_back(patch_names[i] ? patch_names[i] : "");
    *out = reinterpret_cast<nds_mesh*>(
        new nds::Mesh(nds::mesh_from_arrays(n_points, xyz, n_cells, tets, n_bfaces, btri, bpatch, names)));
    return NDS_OK;
  } catch (const std::exception& e) {
    set_error(e.what());
    return NDS_E_SETUP;
  }
}

int nds_mesh_counts(const nds_mesh* mm, int* np, int* nc, int* nf, int* ni) {
  if (!mm) { set_error("null mesh"); return NDS_E_INVALID; }
  const auto* m = reinterpret_cast<const nds::Mesh*>(mm);
  if (np) *np = m->n_points();
  if (nc) *nc = m->n_cells();
  if (nf) *nf = m->n_faces();
  if (ni) *ni = m->n_internal();
  return NDS_OK;
}

void nds_mesh_destroy(nds_mesh* m) { delete reinterpret_cast<nds::Mesh*>(m); }

int nds_problem_create(const nds_mesh* mm, const nds_options* o, nds_problem** out) {
  if (!mm || !o || !out) { set_error("null argument"); return NDS_E_INVALID; }
  try {
    std::string why;
    if (!nds::validate_options(*o, why)) {
      set_error(why);
      return NDS_E_INVALID;
    }
    auto P = std::make_unique<nds::Problem>();
    P->opt = *o;
    P->mesh = *reinterpret_cast<const nds::Mesh*>(mm);
    nds::SetupOptions so;
    so.re = o->re;
    so.bulk = o->bulk;
    so.alpha_u = o->alpha_u;
    so.rau_scale = o->rau_scale;
    so.wall = o->wall;
    so.inlet = o->inlet;
    so.outlet = o->outlet;
    so.threads = o->threads;
    so.supg = o->supg != 0;
    so.supg_tau_scale = o->supg_tau_scale;
    so.supg_magic = o->supg_magic;
    so.geom_from_inlet = o->geom_from_inlet != 0;
    P->setup = nds::build_setup(P->mesh, so);
    P->power_its = nds::effective_amg_power_its(*o);
    nds::AmgOptions ao;
    ao.hierarchy = o->amg_hierarchy == NDS_AMG_SA ? "sa" : "cf";
    ao.terminal = o->amg_terminal;
    ao.power_its = P->power_its;
    ao.lambda_safety = o->amg_lambda_safety;
    ao.cf_theta = o->cf_theta;
    ao.cf_pmax = o->cf_pmax;
    ao.cf_interp = o->cf_interp == NDS_CF_EXTI ? "exti" : "direct";
    ao.cf_aggressive_first = o->cf_aggressive_first != 0;
    P->hier = nds::build_hierarchy(P->mesh, P->setup, P->setup.init_rau, ao);
    P->index_arrays();
    *out = reinterpret_cast<nds_problem*>(P.release());
    return NDS_OK;
  } catch (const std::exception& e) {
    set_error(e.what());
    return NDS_E_SETUP;
  }
}

int nds_problem_array(const nds_problem* pp, const char* name, nds_array* out) {
  if (!pp || !name || !out) { set_error("null argument"); return NDS_E_INVALID; }
  const auto* P = reinterpret_cast<const nds::Problem*>(pp);
  auto it = P->arrays.find(name);
  if (it == P->arrays.end()) {
    set_error(std::string("unknown problem array ") + name);
    return NDS_E_INVALID;
  }
  *out = it->second;
  return NDS_OK;
}

int nds_problem_counts(const nds_problem* pp, int* nc, int* nv, int* ncolors, int* levels) {
  if (!pp) { set_error("null problem"); return NDS_E_INVALID; }
  const auto* P = reinterpret_cast<const nds::Problem*>(pp);
  if (nc) *nc = P->setup.nc;
  if (nv) *nv = P->setup.nv;
  if (ncolors) *ncolors = P->setup.ncolors;
  if (levels) *levels = (int)P->hier.A.size();
  return NDS_OK;
}

void nds_problem_destroy(nds_problem* p) { delete reinterpret_cast<nds::Problem*>(p); }

int nds_write_vtu(const nds_problem* pp, const char* path, const double* u0, const double* u1, const double* u2,
                  const double* pr, int converged, int outer_its) {
  if (!pp || !path || !u0 || !u1 || !u2 || !pr) { set_error("null argument"); return NDS_E_INVALID; }
  const auto* P = reinterpret_cast<const nds::Problem*>(pp);
  try {
    nds::write_vtu(path, P->mesh, P->setup, u0, u1, u2, pr, converged != 0, outer_its);
    return NDS_OK;
  } catch (const std::exception& e) {
    set_error(e.what());
    return NDS_E_SETUP;
  }
}

int nds_compute_hp_errors(const nds_problem* pp, const double* u0, const double* u1, const double* u2, const double* pr,
                          nds_hp_errors* out) {
  if (!pp || !u0 || !u1 || !u2 || !pr || !out) { set_error("null argument"); return NDS_E_INVALID; }
  const auto* P = reinterpret_cast<const nds::Problem*>(pp);
  const nds::HpErrors E = nds::hp_errors(P->mesh, P->setup, u0, u1, u2, pr);
  out->h_eff = E.h_eff;
  out->u_l2 = E.u_l2;
  out->u_rel_l2 = E.u_rel_l2;
  out->p_shifted_l2 = E.p_shifted_l2;
  out->p_shifted_rel_l2 = E.p_shifted_rel_l2;
  out->pressure_shift = E.pressure_shift;
  out->dp_fit = E.dp_fit;
  out->dp_exact = E.dp_exact;
  out->dp_rel_err = E.dp_rel_err;
  return NDS_OK;
}

int nds_cell_average_velocity(const nds_problem* pp, const double* u0, const double* u1, const double* u2,
                              double* out_xyz) {
  if (!pp || !u0 || !u1 || !u2 || !out_xyz) { set_error("null argument"); return NDS_E_INVALID; }
  const auto* P = reinterpret_cast<const nds::Problem*>(pp);
  std::vector<double> v;
  nds::cell_average_velocity(P->setup, u0, u1, u2, v);
  std::copy(v.begin(), v.end(), out_xyz);
  return NDS_OK;
}

}  // extern "C"

namespace nds {

int effective_amg_power_its(const nds_options& o) {
  if (o.amg_spectrum_policy == NDS_SPEC_ALWAYS) return o.amg_power_its;
  // the SUPG entry also estimates the spectrum for smoothed aggregation
  // (h8_supg_main_setup.inc:10-14)
  const bool need = o.amg_smoother == NDS_SM_CHEB2 || (o.supg && o.amg_hierarchy == NDS_AMG_SA);
  if (o.amg_spectrum_policy == NDS_SPEC_AUTO && need) return o.amg_power_its;
  return 0;
}

bool validate_options(const nds_options& o, std::string& why) {
  auto bad = [&](const char* m) { why = m; return false; };
  // ranges of h8_main_base.cu:1851-1911 (laminar subset)
  if (!(o.simple_tol > 0.0) || o.max_outer < 1) return bad("H8 invalid SIMPLE controls");
  if (!(o.alpha_u > 0.0 && o.alpha_u <= 1.0) || !(o.alpha_p > 0.0 && o.alpha_p <= 1.0)) return bad("H8 alpha-u/alpha-p must be in (0,1]");
  if (!(o.rau_scale > 0.0)) return bad("H8 rau-scale must be finite and > 0");
  if (o.mom_rtol < 0.0 || o.mom_atol < 0.0 || o.mom_drop < 0.0 || o.mom_max < 1 || !(o.mom_omega > 0.0)) return bad("H8 invalid momentum controls");
  if (o.p_rtol < 0.0 || o.p_atol < 0.0 || o.p_max < 1) return bad("H8 invalid pressure controls");
  if (o.amg_hierarchy != NDS_AMG_SA && o.amg_hierarchy != NDS_AMG_CF) return bad("H8 amg-hierarchy must be sa or cf");
  if (!(o.cf_theta > 0.0 && o.cf_theta <= 1.0)) return bad("H8 cf-theta must be in (0,1]");
  if (o.cf_pmax < 1 || o.cf_pmax > 16) return bad("H8 cf-pmax must be in [1,16]");
  if (o.cf_interp != NDS_CF_DIRECT && o.cf_interp != NDS_CF_EXTI) return bad("H8 cf-interp must be direct or exti");
  if (o.cf_aggressive_first != 0 && o.cf_aggressive_first != 1) return bad("H8 cf-aggressive-first must be 0 or 1");
  if (o.amg_terminal < 16) return bad("H8 amg-terminal must be >=16");
  if (o.amg_spectrum_policy < 0 || o.amg_spectrum_policy > 2) return bad("H8 amg-spectrum-policy must be auto, always or off");
  if (o.amg_power_its < 1 || o.amg_power_its > 64) return bad("H8 amg-power-its must be in [1,64]");
  if (o.amg_cheb_degree < 1 || o.amg_cheb_degree > 16) return bad("H8 amg-cheb-degree must be in [1,16]");
  if (!(o.amg_lambda_safety > 1.0 && o.amg_lambda_safety <= 3.0)) return bad("H8 amg-lambda-safety must be in (1,3]");
  if (!(o.amg_lambda_low_fraction > 0.0 && o.amg_lambda_low_fraction < 1.0)) return bad("H8 amg-lambda-low-fraction must be in (0,1)");
  if (o.pressure_solver < 0 || o.pressure_solver > 2) return bad("G12 pressure-solver must be pcg, richardson or cheb");
  if (!(o.p_richardson_omega > 0.0 && o.p_richardson_omega < 2.0)) return bad("G12 Richardson omega must be in (0,2)");
  if (o.p_cheb_degree < 1 || o.p_cheb_degree > 16) return bad("G12 Cheb degree must be in [1,16]");
  if (o.p_power_its < 1 || o.p_power_its > 64) return bad("G12 pressure power its must be in [1,64]");
  if (!(o.p_cheb_low_fraction > 0.0 && o.p_cheb_low_fraction < 1.0)) return bad("G12 Cheb low fraction must be in (0,1)");
  if (!(o.p_power_safety > 1.0 && o.p_power_safety <= 2.0)) return bad("G12 pressure power safety must be in (1,2]");
  if (o.amg_smoother < 0 || o.amg_smoother > 3) return bad("H8 amg-smoother must be cheb2, jacobi, l1jacobi or mcgs");
  if (!(o.amg_jacobi_omega > 0.0 && o.amg_jacobi_omega <= 2.0)) return bad("H8 amg-jacobi-omega must be in (0,2]");
  if (o.amg_jacobi_fine_sweeps < 1 || o.amg_jacobi_fine_sweeps > 16 || o.amg_jacobi_coarse_sweeps < 1 || o.amg_jacobi_coarse_sweeps > 16)
    return bad("H8 Jacobi sweeps must be in [1,16]");
  if (!(o.amg_mcgs_omega > 0.0 && o.amg_mcgs_omega < 2.0)) return bad("H8 amg-mcgs-omega must be in (0,2)");
  if (o.amg_mcgs_fine_sweeps < 1 || o.amg_mcgs_fine_sweeps > 16 || o.amg_mcgs_coarse_sweeps < 1 || o.amg_mcgs_coarse_sweeps > 16)
    return bad("H8 MCGS sweeps must be in [1,16]");
  if (o.amg_mcgs_order < 0 || o.amg_mcgs_order > 2) return bad("H8 amg-mcgs-order must be symmetric, forward or backward");
  if (o.pressure_solver == NDS_P_PCG && o.amg_smoother == NDS_SM_MCGS && o.amg_mcgs_order != NDS_MCGS_SYMMETRIC)
    return bad("H8 PCG requires symmetric MCGS");
  if (!(o.snapshot_tol > 0.0)) return bad("H8 snapshot tolerance must be positive");
  if (o.fine_csr_refresh_every != 1) return bad("H8 requires fine CSR refreshEvery=1");
  if (o.momentum_work < 0 || o.momentum_work > 2) return bad("H8 momentum-work must be fgs1, altgs1 or sgs1");
  if (o.run_mode != NDS_RUN_FIXED10 && o.run_mode != NDS_RUN_CONVERGE) return bad("H8 run-mode must be fixed10 or converge");
  if (o.run_mode == NDS_RUN_FIXED10 && o.max_outer != 10) return bad("H8 fixed10 requires maxOuter=10");
  if (o.amg_smoother == NDS_SM_CHEB2 && effective_amg_power_its(o) <= 0) return bad("H8 Chebyshev AMG smoother requires spectrum estimation");
  if (o.precision < 0 || o.precision > 3) return bad("precision must be fp64, fp32, amg_fp32 or mixed");
  if (o.p_krylov < 0 || o.p_krylov > 1) return bad("p_krylov must be pcg or fgmres");
  if (o.p_restart < 1 || o.p_restart > 64) return bad("p_restart must be in 1..64");
  if (!(o.p_inner_rtol > 0.0 && o.p_inner_rtol < 1.0)) return bad("p_inner_rtol must be in (0, 1)");
  if (o.p_refine_max < 1) return bad("p_refine_max must be >= 1");
  if (o.p_guess < 0 || o.p_guess > 8) return bad("p_guess must be in 0..8");
  if (o.learned && (o.precision != NDS_MIXED || o.p_krylov != NDS_KRYLOV_FGMRES))
    return bad("the learned stage needs precision mixed and p_krylov fgmres (a varying preconditioner)");
  if (o.precision == NDS_MIXED && o.pressure_solver != NDS_P_PCG)
    return bad("precision mixed runs its own Krylov solve: pressure_solver must be pcg (the default)");
  if (o.amg_half && o.precision != NDS_MIXED) return bad("amg_half needs precision mixed");
  if (o.precision == NDS_MIXED && o.amg_smoother == NDS_SM_MCGS)
    return bad("precision mixed supports the polynomial smoothers (cheb2, jacobi, l1jacobi)");
  if (o.supg != 0 && o.supg != 1) return bad("H8 supg must be 0 or 1");
  if (o.supg) {  // h8_supg_main_cli.inc:92-124
    if (!(o.supg_tau_scale > 0.0)) return bad("H8 SUPG tau scale must be positive");
    if (!(o.supg_magic > 0.0)) return bad("H8 SUPG magic must be positive");
    if (o.amg_hierarchy == NDS_AMG_SA && effective_amg_power_its(o) <= 0)
      return bad("P7D smoothed aggregation requires spectrum estimation to smooth interpolation");
    if (o.momentum_work != NDS_MOM_FGS1) return bad("H8 requires momentum-work=fgs1");
  }
  return true;
}

namespace {
template <class T>
nds_array view(const std::vector<T>& v, int dt) {
  nds_array a;
  a.data = v.data();
  a.count = (int64_t)v.size();
  a.dtype = dt;
  return a;
}
}  // namespace

void Problem::index_arrays() {
  auto& A = arrays;
  auto& S = setup;
  auto& H = hier;
  auto scal = [&](const std::string& n, double x) {
    scalars[n] = {x};
    A[n] = view(scalars[n], 0);
  };
  mesh_tets.clear();
  mesh_opp.clear();
  for (auto& t : mesh.tets) for (int k = 0; k < 4; ++k) mesh_tets.push_back(t[(size_t)k]);
  for (auto& t : mesh.opp) for (int k = 0; k < 4; ++k) mesh_opp.push_back(t[(size_t)k]);
  A["mesh.tets"] = view(mesh_tets, 1);
  A["mesh.opp_face"] = view(mesh_opp, 1);
  A["mesh.face_patch"] = view(mesh.face_patch, 1);
  A["mesh.xyz"] = view(mesh.xyz, 0);
  {
    const RefTensors& RT = ref_tensors();
    auto& t = scalars["centT"];
    t.assign(&RT.T[0][0][0][0], &RT.T[0][0][0][0] + 8 * 8 * 8 * 3);
    A["centT"] = view(t, 0);
    auto& dd = scalars["diffT"];
    dd.assign(&RT.D[0][0][0][0], &RT.D[0][0][0][0] + 8 * 8 * 3 * 3);
    A["diffT"] = view(dd, 0);
  }
  scal("pipe.nu", S.pipe.nu);
  scal("pipe.R", S.pipe.R);
  scal("pipe.L", S.pipe.L);
  scal("pipe.profileScale", S.pipe.profile_scale);
  scal("pipe.hpDrop", S.pipe.hp_drop);
  scal("pipe.hpGradient", S.pipe.hp_gradient);
  scal("pipe.zOut", S.pipe.z_out);
  scal("pipe.cx", S.pipe.cx);
  scal("pipe.cy", S.pipe.cy);
  scal("pipe.bulk", S.pipe.bulk);
  A["g2free"] = view(S.g2free, 1);
  A["fixedSlot"] = view(S.fixed_slot, 1);
  A["fixedValue"] = view(S.fixed_value, 0);
  A["mom.row"] = view(S.mom.row, 2);
  A["mom.col"] = view(S.mom.col, 1);
  A["mom.val"] = view(S.mom.val, 0);
  A["mom.diagPos"] = view(S.mom_diag_pos, 1);
  A["color"] = view(S.color, 1);
  A["color.offset"] = view(S.color_off, 1);
  A["color.rows"] = view(S.color_rows, 1);
  A["cell.ref"] = view(S.ref, 1);
  A["cell.rowSlot"] = view(S.row_slot, 3);
  A["cell.det"] = view(S.det, 0);
  A["cell.invJ"] = view(S.invJ, 0);
  A["cell.bcoeff"] = view(S.bco, 0);
  for (int d = 0; d < 3; ++d) A["staticRhs" + std::to_string(d)] = view(S.static_rhs[(size_t)d], 0);
  A["fixedDiv"] = view(S.fixed_div, 0);
  A["volume"] = view(S.volume, 0);
  A["cell.h2"] = view(S.h2, 0);
  {
    const auto& q = tet_rule_64();
    supg_rule.clear();
    for (const auto& x : q) {
      for (int k = 0; k < 4; ++k) supg_rule.push_back(x.lam[(size_t)k]);
      supg_rule.push_back(x.w);
    }
    A["supg.rule"] = view(supg_rule, 0);  // 64 x (lambda0..3, weight)
  }
  A["initRau"] = view(S.init_rau, 0);
  A["initDelta"] = view(S.init_delta, 0);
  A["fine.row"] = view(S.fine.row, 1);
  A["fine.col"] = view(S.fine.col, 1);
  A["fine.diagPos"] = view(S.fine.diag_pos, 1);
  A["fine.incOff"] = view(S.fine.inc_off, 1);
  A["fine.packed"] = view(S.fine.packed, 4);
  A["fine.contribOff"] = view(S.fine.contrib_off, 1);
  A["fine.slot"] = view(S.fine.slot, 3);
  scal("amg.levels", (double)H.A.size());
  scal("amg.fineLambda", H.fine_lambda);
  scal("amg.powerIts", (double)power_its);
  A["amg.fineDiag"] = view(H.fine_diag, 0);
  A["amg.levelLambda"] = view(H.level_lambda, 0);
  A["amg.terminal_inv"] = view(H.terminal_inv, 0);
  for (size_t l = 0; l < H.agg.size(); ++l) A["amg.agg" + std::to_string(l)] = view(H.agg[l], 1);
  for (size_t l = 0; l < H.P.size(); ++l) {
    const std::string p = "amg.P" + std::to_string(l) + ".";
    scal(p + "nCoarse", (double)H.P[l].nc);
    A[p + "row"] = view(H.P[l].row, 2);
    A[p + "col"] = view(H.P[l].col, 1);
    A[p + "val"] = view(H.P[l].val, 0);
  }
  for (size_t l = 0; l < H.A.size(); ++l) {
    const std::string p = "amg.A" + std::to_string(l) + ".";
    A[p + "row"] = view(H.A[l].row, 2);
    A[p + "col"] = view(H.A[l].col, 1);
    A[p + "val"] = view(H.A[l].val, 0);
    A[p + "diag"] = view(H.A[l].diag, 0);
  }
}

}  // namespace nds
