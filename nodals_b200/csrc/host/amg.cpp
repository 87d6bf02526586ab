#include "amg.hpp"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <unordered_map>
#include <utility>

namespace nds {

namespace {

using Entry = std::pair<int, double>;

// SA transfer row: merge duplicates, keep own + largest |w|, normalise to sum 1
void normalize_prune(std::vector<Entry>& row, int own, int max_nnz) {
  if (row.empty()) row.push_back({own, 1.0});
  std::sort(row.begin(), row.end(), [](const Entry& a, const Entry& b) { return a.first < b.first; });
  size_t w = 0;
  for (size_t k = 0; k < row.size();) {
    const int c = row[k].first;
    double v = 0.0;
    size_t j = k;
    for (; j < row.size() && row[j].first == c; ++j) v += row[j].second;
    row[w++] = {c, v};
    k = j;
  }
  row.resize(w);
  if (max_nnz > 0 && (int)row.size() > max_nnz) {
    std::vector<Entry> keep;
    keep.reserve((size_t)max_nnz);
    auto it = std::find_if(row.begin(), row.end(), [&](const Entry& e) { return e.first == own; });
    keep.push_back(it != row.end() ? *it : Entry{own, 0.0});
    std::vector<Entry> others;
    for (const auto& e : row)
      if (e.first != own) others.push_back(e);
    std::sort(others.begin(), others.end(), [](const Entry& a, const Entry& b) {
      const double aa = std::abs(a.second), bb = std::abs(b.second);
      return aa > bb || (aa == bb && a.first < b.first);
    });
    for (const auto& e : others)
      if ((int)keep.size() < max_nnz) keep.push_back(e);
    std::sort(keep.begin(), keep.end(), [](const Entry& a, const Entry& b) { return a.first < b.first; });
    row.swap(keep);
  }
  double sum = 0.0;
  for (const auto& e : row) sum += e.second;
  if (!std::isfinite(sum) || std::abs(sum) < 1e-14) {
    row.clear();
    row.push_back({own, 1.0});
    return;
  }
  for (auto& e : row) e.second /= sum;
}

void csr_apply(const CsrHost& A, const std::vector<double>& x, std::vector<double>& y) {
  y.assign((size_t)A.n, 0.0);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < A.n; ++i) {
    double s = 0.0;
    for (int64_t k = A.row[(size_t)i]; k < A.row[(size_t)i + 1]; ++k) s += A.val[(size_t)k] * x[(size_t)A.col[(size_t)k]];
    y[(size_t)i] = s;
  }
}

// deterministic power-iteration start vector
inline double power_seed(int i) {
  const double g = (double)(i + 1);
  return std::sin(.731 * g) + .27 * std::cos(1.117 * g);
}

// lambda_max(D^-1/2 A D^-1/2) by power iteration, with a generic apply
template <class Apply>
double power_generic(int n, const std::vector<double>& diag, int its, double safety, Apply apply) {
  std::vector<double> v((size_t)n), u((size_t)n), au, w((size_t)n);
  long double ss = 0;
  for (int i = 0; i < n; ++i) {
    v[(size_t)i] = power_seed(i);
    ss += (long double)v[(size_t)i] * v[(size_t)i];
  }
  const double vn = std::sqrt((double)ss);
  for (auto& q : v) q /= vn;
  double ray = 0.0;
  for (int it = 0; it < its; ++it) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) u[(size_t)i] = v[(size_t)i] / std::sqrt(diag[(size_t)i]);
    apply(u, au);
    long double num = 0, den = 0, nw = 0;
    for (int i = 0; i < n; ++i) {
      w[(size_t)i] = au[(size_t)i] / std::sqrt(diag[(size_t)i]);
      num += (long double)v[(size_t)i] * w[(size_t)i];
      den += (long double)v[(size_t)i] * v[(size_t)i];
      nw += (long double)w[(size_t)i] * w[(size_t)i];
    }
    ray = (double)(num / std::max(den, (long double)1e-300));
    const double nrm = std::sqrt((double)nw);
    if (!(nrm > 0.0) || !std::isfinite(nrm) || !(ray > 0.0) || !std::isfinite(ray))
      throw std::runtime_error("AMG power iteration failed");
    for (int i = 0; i < n; ++i) v[(size_t)i] = w[(size_t)i] / nrm;
  }
  return safety * ray;
}

// matrix-free fine Schur action y = B diag(rau) B^T x; B^T x gathered per
// velocity dof over its incident cells in ascending cell order (the order of
// the reference's cell-major scatter)
struct FineApply {
  const Setup& S;
  const std::vector<double>& rau;
  std::vector<double> v0, v1, v2;
  FineApply(const Setup& s, const std::vector<double>& r) : S(s), rau(r), v0((size_t)s.nv), v1((size_t)s.nv), v2((size_t)s.nv) {}
  void operator()(const std::vector<double>& x, std::vector<double>& y) {
    const FineTopo& F = S.fine;
#pragma omp parallel for schedule(static)
    for (int g = 0; g < S.nv; ++g) {
      double s0 = 0.0, s1 = 0.0, s2 = 0.0;
      for (int k = F.inc_off[(size_t)g]; k < F.inc_off[(size_t)g + 1]; ++k) {
        const uint32_t pk = F.packed[(size_t)k];
        const int c = (int)(pk >> 3);
        const double* b = &S.bco[24 * (size_t)c + 3 * (pk & 7u)];
        const double p = x[(size_t)c];
        s0 += b[0] * p;
        s1 += b[1] * p;
        s2 += b[2] * p;
      }
      const double r = rau[(size_t)g];
      v0[(size_t)g] = s0 * r;
      v1[(size_t)g] = s1 * r;
      v2[(size_t)g] = s2 * r;
    }
    y.assign((size_t)S.nc, 0.0);
#pragma omp parallel for schedule(static)
    for (int c = 0; c < S.nc; ++c) {
      double s = 0.0;
      for (int a = 0; a < 8; ++a) {
        const int g = S.ref[8 * (size_t)c + a];
        if (g < 0) continue;
        const double* b = &S.bco[24 * (size_t)c + 3 * a];
        s += b[0] * v0[(size_t)g] + b[1] * v1[(size_t)g] + b[2] * v2[(size_t)g];
      }
      y[(size_t)c] = s;
    }
  }
};

// Row-owned accumulation of a sparse matrix: fill(I, add) calls add(J, v) for
// every non-zero contribution to row I in the order that defines the sum;
// entries whose final sum is exactly zero are dropped (as the reference
// packer does, g5_sa_host.hpp:504-521).  Rows are independent -> parallel.
template <class Fill>
CsrHost accumulate_rows(int nrows, int ncols, Fill fill) {
  std::vector<std::vector<int32_t>> cols((size_t)nrows);
  std::vector<std::vector<double>> vals((size_t)nrows);
#pragma omp parallel
  {
    std::vector<double> acc((size_t)ncols, 0.0);
    std::vector<char> mark((size_t)ncols, 0);
    std::vector<int32_t> touched;
#pragma omp for schedule(dynamic, 32)
    for (int I = 0; I < nrows; ++I) {
      touched.clear();
      fill(I, [&](int J, double v) {
        if (!mark[(size_t)J]) {
          mark[(size_t)J] = 1;
          touched.push_back(J);
        }
        acc[(size_t)J] += v;
      });
      std::sort(touched.begin(), touched.end());
      auto& c = cols[(size_t)I];
      auto& w = vals[(size_t)I];
      for (int32_t J : touched) {
        if (acc[(size_t)J] != 0.0) {
          c.push_back(J);
          w.push_back(acc[(size_t)J]);
        }
        acc[(size_t)J] = 0.0;
        mark[(size_t)J] = 0;
      }
    }
  }
  CsrHost A;
  A.n = nrows;
  A.row.assign((size_t)nrows + 1, 0);
  for (int I = 0; I < nrows; ++I) A.row[(size_t)I + 1] = A.row[(size_t)I] + (int64_t)cols[(size_t)I].size();
  A.col.resize((size_t)A.row.back());
  A.val.resize((size_t)A.row.back());
  A.diag.assign((size_t)nrows, 0.0);
#pragma omp parallel for schedule(static)
  for (int I = 0; I < nrows; ++I) {
    std::copy(cols[(size_t)I].begin(), cols[(size_t)I].end(), A.col.begin() + A.row[(size_t)I]);
    std::copy(vals[(size_t)I].begin(), vals[(size_t)I].end(), A.val.begin() + A.row[(size_t)I]);
    for (size_t k = 0; k < cols[(size_t)I].size(); ++k)
      if (cols[(size_t)I][k] == I) A.diag[(size_t)I] = vals[(size_t)I][k];
  }
  for (int i = 0; i < A.n; ++i)
    if (!(A.diag[(size_t)i] > 0.0) || !std::isfinite(A.diag[(size_t)i]))
      throw std::runtime_error("coarse AMG matrix has a non-positive diagonal");
  return A;
}

// coarse row -> (fine row, weight) incidence of a transfer, ascending fine row
struct RevTransfer {
  std::vector<int64_t> off;
  std::vector<int32_t> fine;
  std::vector<double> w;
};
RevTransfer reverse(const Transfer& P) {
  RevTransfer R;
  R.off.assign((size_t)P.nc + 1, 0);
  for (int32_t c : P.col) ++R.off[(size_t)c + 1];
  for (int c = 0; c < P.nc; ++c) R.off[(size_t)c + 1] += R.off[(size_t)c];
  R.fine.resize(P.col.size());
  R.w.resize(P.col.size());
  std::vector<int64_t> pos(R.off.begin(), R.off.end() - 1);
  for (int i = 0; i < P.nf; ++i)
    for (int64_t k = P.row[(size_t)i]; k < P.row[(size_t)i + 1]; ++k) {
      const int c = P.col[(size_t)k];
      R.fine[(size_t)pos[(size_t)c]] = i;
      R.w[(size_t)pos[(size_t)c]++] = P.val[(size_t)k];
    }
  return R;
}

// Galerkin P^T A P (g5_sa_host.hpp:940-971): q_i = A_i P merged per coarse
// column, then coarse entry (I,K) = sum over fine rows i (ascending) of
// P_iI q_i(K) -- the reference's accumulation order.
CsrHost galerkin(const CsrHost& A, const Transfer& P) {
  if (P.nf != A.n) throw std::runtime_error("Galerkin transfer size mismatch");
  std::vector<std::vector<Entry>> q((size_t)A.n);
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < A.n; ++i) {
    auto& qi = q[(size_t)i];
    for (int64_t k = A.row[(size_t)i]; k < A.row[(size_t)i + 1]; ++k) {
      const int j = A.col[(size_t)k];
      const double a = A.val[(size_t)k];
      for (int64_t kp = P.row[(size_t)j]; kp < P.row[(size_t)j + 1]; ++kp) qi.push_back({P.col[(size_t)kp], a * P.val[(size_t)kp]});
    }
    std::sort(qi.begin(), qi.end(), [](const Entry& x, const Entry& y) { return x.first < y.first; });
    size_t w = 0;
    for (size_t k = 0; k < qi.size();) {
      const int c = qi[k].first;
      double v = 0.0;
      size_t j = k;
      for (; j < qi.size() && qi[j].first == c; ++j) v += qi[j].second;
      qi[w++] = {c, v};
      k = j;
    }
    qi.resize(w);
    qi.shrink_to_fit();
  }
  const RevTransfer R = reverse(P);
  return accumulate_rows(P.nc, P.nc, [&](int I, auto&& add) {
    for (int64_t z = R.off[(size_t)I]; z < R.off[(size_t)I + 1]; ++z) {
      const double pi = R.w[(size_t)z];
      for (const auto& e : q[(size_t)R.fine[(size_t)z]]) {
        const double v = pi * e.second;
        if (v != 0.0) add(e.first, v);
      }
    }
  });
}

// ----------------------------------------------------------------------------
// SA pieces
// ----------------------------------------------------------------------------
std::vector<std::vector<int32_t>> face_graph(const Mesh& m) {
  std::vector<std::vector<int32_t>> g((size_t)m.n_cells());
  for (int f = 0; f < m.n_internal(); ++f) {
    const int a = m.owner[(size_t)f], b = m.neighbour[(size_t)f];
    g[(size_t)a].push_back(b);
    g[(size_t)b].push_back(a);
  }
  for (auto& v : g) {
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
  }
  return g;
}

std::vector<std::vector<int32_t>> csr_graph(const CsrHost& A) {
  std::vector<std::vector<int32_t>> g((size_t)A.n);
  for (int i = 0; i < A.n; ++i)
    for (int64_t k = A.row[(size_t)i]; k < A.row[(size_t)i + 1]; ++k) {
      const int j = A.col[(size_t)k];
      if (j != i) g[(size_t)i].push_back(j);
    }
  return g;
}

Transfer pack_transfer(int nf, int nc, std::vector<std::vector<Entry>>& rows) {
  Transfer P;
  P.nf = nf;
  P.nc = nc;
  P.row.assign((size_t)nf + 1, 0);
  for (int i = 0; i < nf; ++i) P.row[(size_t)i + 1] = P.row[(size_t)i] + (int64_t)rows[(size_t)i].size();
  P.col.resize((size_t)P.row.back());
  P.val.resize((size_t)P.row.back());
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nf; ++i) {
    int64_t k = P.row[(size_t)i];
    for (const auto& e : rows[(size_t)i]) {
      P.col[(size_t)k] = e.first;
      P.val[(size_t)k++] = e.second;
    }
  }
  return P;
}

// fine -> first aggregate level, smoothed with damping / lambda (g5_sa_host.hpp:173-203)
Transfer sa_fine_transfer(const Setup& S, const std::vector<double>& rau, const std::vector<int32_t>& id, int nagg,
                          const std::vector<double>& diag, double lambda, double damping, int max_nnz) {
  const double omega = damping / lambda;
  const FineTopo& F = S.fine;
  std::vector<std::vector<Entry>> rows((size_t)S.nc);
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < S.nc; ++i) {
    auto& row = rows[(size_t)i];
    const int own = id[(size_t)i];
    row.push_back({own, 1.0});
    const double invd = 1.0 / diag[(size_t)i];
    for (int a = 0; a < 8; ++a) {
      const int g = S.ref[8 * (size_t)i + a];
      if (g < 0) continue;
      const double* bi = &S.bco[24 * (size_t)i + 3 * a];
      for (int k = F.inc_off[(size_t)g]; k < F.inc_off[(size_t)g + 1]; ++k) {
        const uint32_t pk = F.packed[(size_t)k];
        const int j = (int)(pk >> 3);
        const double* bj = &S.bco[24 * (size_t)j + 3 * (pk & 7u)];
        double dot = 0.0;
        for (int d = 0; d < 3; ++d) dot += bi[d] * bj[d];
        row.push_back({id[(size_t)j], -omega * invd * rau[(size_t)g] * dot});
      }
    }
    normalize_prune(row, own, max_nnz);
  }
  return pack_transfer(S.nc, nagg, rows);
}

// A1 = P^T B diag(rau) B^T P (g5_sa_host.hpp:525-546): per velocity dof g the
// merged list q_g of (coarse, P-weighted B row); coarse entry (I,J) sums
// rau_g q_g(I).q_g(J) over ascending g, the reference's order.
CsrHost sa_first_coarse(const Setup& S, const std::vector<double>& rau, const Transfer& P) {
  const FineTopo& F = S.fine;
  struct QE {
    int coarse;
    double b[3];
  };
  std::vector<std::vector<QE>> qs((size_t)S.nv);
#pragma omp parallel for schedule(dynamic, 512)
  for (int g = 0; g < S.nv; ++g) {
    auto& q = qs[(size_t)g];
    for (int k = F.inc_off[(size_t)g]; k < F.inc_off[(size_t)g + 1]; ++k) {
      const uint32_t pk = F.packed[(size_t)k];
      const int c = (int)(pk >> 3);
      const double* bb = &S.bco[24 * (size_t)c + 3 * (pk & 7u)];
      for (int64_t kp = P.row[(size_t)c]; kp < P.row[(size_t)c + 1]; ++kp) {
        const double pv = P.val[(size_t)kp];
        QE e;
        e.coarse = P.col[(size_t)kp];
        for (int d = 0; d < 3; ++d) e.b[d] = pv * bb[d];
        q.push_back(e);
      }
    }
    std::sort(q.begin(), q.end(), [](const QE& a, const QE& b) { return a.coarse < b.coarse; });
    size_t w = 0;
    for (size_t k = 0; k < q.size();) {
      const int c = q[k].coarse;
      double s[3] = {0, 0, 0};
      size_t j = k;
      for (; j < q.size() && q[j].coarse == c; ++j)
        for (int d = 0; d < 3; ++d) s[d] += q[j].b[d];
      q[w].coarse = c;
      for (int d = 0; d < 3; ++d) q[w].b[d] = s[d];
      ++w;
      k = j;
    }
    q.resize(w);
    q.shrink_to_fit();
  }
  // coarse row -> (g, position in q_g), ascending g
  std::vector<int64_t> off((size_t)P.nc + 1, 0);
  for (int g = 0; g < S.nv; ++g)
    for (const auto& e : qs[(size_t)g]) ++off[(size_t)e.coarse + 1];
  for (int c = 0; c < P.nc; ++c) off[(size_t)c + 1] += off[(size_t)c];
  std::vector<int32_t> rg((size_t)off.back());
  std::vector<int32_t> ra((size_t)off.back());
  {
    std::vector<int64_t> pos(off.begin(), off.end() - 1);
    for (int g = 0; g < S.nv; ++g)
      for (size_t a = 0; a < qs[(size_t)g].size(); ++a) {
        const int c = qs[(size_t)g][a].coarse;
        rg[(size_t)pos[(size_t)c]] = g;
        ra[(size_t)pos[(size_t)c]++] = (int32_t)a;
      }
  }
  return accumulate_rows(P.nc, P.nc, [&](int I, auto&& add) {
    for (int64_t z = off[(size_t)I]; z < off[(size_t)I + 1]; ++z) {
      const int g = rg[(size_t)z];
      const auto& q = qs[(size_t)g];
      const QE& qa = q[(size_t)ra[(size_t)z]];
      const double r = rau[(size_t)g];
      for (const auto& qb : q) {
        const double v = r * (qa.b[0] * qb.b[0] + qa.b[1] * qb.b[1] + qa.b[2] * qb.b[2]);
        if (v != 0.0) add(qb.coarse, v);
      }
    }
  });
}

Transfer sa_explicit_transfer(const CsrHost& A, const std::vector<int32_t>& id, int nagg, double lambda, double damping,
                              int max_nnz) {
  const double omega = damping / lambda;
  std::vector<std::vector<Entry>> rows((size_t)A.n);
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < A.n; ++i) {
    auto& row = rows[(size_t)i];
    const int own = id[(size_t)i];
    row.push_back({own, 1.0});
    const double invd = 1.0 / A.diag[(size_t)i];
    for (int64_t k = A.row[(size_t)i]; k < A.row[(size_t)i + 1]; ++k)
      row.push_back({id[(size_t)A.col[(size_t)k]], -omega * invd * A.val[(size_t)k]});
    normalize_prune(row, own, max_nnz);
  }
  return pack_transfer(A.n, nagg, rows);
}

// ----------------------------------------------------------------------------
// CF pieces
// ----------------------------------------------------------------------------
inline uint64_t mix64(uint64_t x) {  // splitmix64 output function (Steele, Lea, Flood 2014)
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

struct Split {
  int n = 0, nC = 0;
  std::vector<uint8_t> state;  // 1 = C, 2 = F
  std::vector<int32_t> cid;
  std::vector<std::vector<int32_t>> strong, graph;
};

double csr_entry(const CsrHost& A, int i, int j) {
  auto b = A.col.begin() + A.row[(size_t)i], e = A.col.begin() + A.row[(size_t)i + 1];
  auto it = std::lower_bound(b, e, j);
  return (it == e || *it != j) ? 0.0 : A.val[(size_t)(it - A.col.begin())];
}

Split pmis_split(const CsrHost& A, double theta) {
  Split R;
  R.n = A.n;
  R.strong.resize((size_t)A.n);
  R.graph.resize((size_t)A.n);
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < A.n; ++i) {
    double maxneg = 0.0;
    for (int64_t k = A.row[(size_t)i]; k < A.row[(size_t)i + 1]; ++k) {
      const int j = A.col[(size_t)k];
      const double a = A.val[(size_t)k];
      if (j != i && a < 0.0) maxneg = std::max(maxneg, -a);
    }
    const double thr = theta * maxneg;
    auto& s = R.strong[(size_t)i];
    if (thr > 0.0)
      for (int64_t k = A.row[(size_t)i]; k < A.row[(size_t)i + 1]; ++k) {
        const int j = A.col[(size_t)k];
        const double a = A.val[(size_t)k];
        if (j != i && a < 0.0 && -a >= thr) s.push_back(j);
      }
    std::sort(s.begin(), s.end());
    s.erase(std::unique(s.begin(), s.end()), s.end());
  }
  for (int i = 0; i < A.n; ++i) {
    for (int j : R.strong[(size_t)i]) {
      R.graph[(size_t)i].push_back(j);
      R.graph[(size_t)j].push_back(i);
    }
  }
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < A.n; ++i) {
    auto& g = R.graph[(size_t)i];
    std::sort(g.begin(), g.end());
    g.erase(std::unique(g.begin(), g.end()), g.end());
  }
  std::vector<uint64_t> h((size_t)A.n);
  for (int i = 0; i < A.n; ++i) h[(size_t)i] = mix64((uint64_t)i + 0x63021ull);
  auto higher = [&](int a, int b) {
    const size_t da = R.graph[(size_t)a].size(), db = R.graph[(size_t)b].size();
    if (da != db) return da > db;
    if (h[(size_t)a] != h[(size_t)b]) return h[(size_t)a] > h[(size_t)b];
    return a > b;
  };
  R.state.assign((size_t)A.n, 0);
  int undecided = A.n, rounds = 0;
  std::vector<int32_t> win;
  while (undecided > 0) {
    win.clear();
    for (int i = 0; i < A.n; ++i) {
      if (R.state[(size_t)i]) continue;
      bool w = true;
      for (int j : R.graph[(size_t)i])
        if (R.state[(size_t)j] == 0 && higher(j, i)) { w = false; break; }
      if (w) win.push_back(i);
    }
    if (win.empty()) throw std::runtime_error("PMIS made no progress");
    for (int i : win)
      if (R.state[(size_t)i] == 0) { R.state[(size_t)i] = 1; --undecided; }
    for (int i : win)
      for (int j : R.graph[(size_t)i])
        if (R.state[(size_t)j] == 0) { R.state[(size_t)j] = 2; --undecided; }
    if (++rounds > A.n) throw std::runtime_error("PMIS excessive rounds");
  }
  R.cid.assign((size_t)A.n, -1);
  for (int i = 0; i < A.n; ++i)
    if (R.state[(size_t)i] == 1) R.cid[(size_t)i] = R.nC++;
  return R;
}

Transfer cf_transfer(const CsrHost& A, const Split& S, int pmax, const std::string& interp) {
  if (interp != "direct" && interp != "exti") throw std::runtime_error("CF interpolation must be direct or exti");
  const bool ext = interp == "exti";
  std::vector<std::vector<Entry>> rows((size_t)A.n);
  bool bad_target = false, bad_sum = false;
#pragma omp parallel
  {
    std::unordered_map<int, double> acc;
#pragma omp for schedule(dynamic, 256)
    for (int i = 0; i < A.n; ++i) {
      auto& cand = rows[(size_t)i];
      if (S.state[(size_t)i] == 1) {
        cand.push_back({S.cid[(size_t)i], 1.0});
        continue;
      }
      acc.clear();
      // direct strong C neighbours, weight |a_ij|
      for (int j : S.strong[(size_t)i]) {
        if (S.state[(size_t)j] != 1) continue;
        const double a = csr_entry(A, i, j);
        const double w = a < 0.0 ? -a : std::abs(a);
        if (w > 0.0) acc[S.cid[(size_t)j]] += w;
      }
      // extended+i: i -> strong F k -> strong C j, |a_ik| split by k's negative couplings
      if (ext) {
        for (int k : S.strong[(size_t)i]) {
          if (S.state[(size_t)k] != 2) continue;
          const double aik = csr_entry(A, i, k);
          const double path = aik < 0.0 ? -aik : 0.0;
          if (!(path > 0.0)) continue;
          double denom = 0.0;
          for (int j : S.strong[(size_t)k]) {
            if (S.state[(size_t)j] != 1) continue;
            const double akj = csr_entry(A, k, j);
            if (akj < 0.0) denom += -akj;
          }
          if (!(denom > 0.0)) continue;
          for (int j : S.strong[(size_t)k]) {
            if (S.state[(size_t)j] != 1) continue;
            const double akj = csr_entry(A, k, j);
            if (akj < 0.0) acc[S.cid[(size_t)j]] += path * ((-akj) / denom);
          }
        }
      }
      // fallback: C neighbours in the symmetric strength graph
      if (acc.empty()) {
        for (int j : S.graph[(size_t)i]) {
          if (S.state[(size_t)j] != 1) continue;
          const double w = std::abs(csr_entry(A, i, j));
          if (w > 0.0) acc[S.cid[(size_t)j]] += w;
        }
      }
      for (const auto& kv : acc)
        if (kv.second > 0.0) cand.push_back(kv);
      if (cand.empty()) {
#pragma omp atomic write
        bad_target = true;
        continue;
      }
      // keep the pmax largest weights (ties: lower coarse id), normalise to sum 1
      std::sort(cand.begin(), cand.end(), [](const Entry& x, const Entry& y) {
        if (x.second != y.second) return x.second > y.second;
        return x.first < y.first;
      });
      if (pmax > 0 && (int)cand.size() > pmax) cand.resize((size_t)pmax);
      double sum = 0.0;
      for (const auto& e : cand) sum += e.second;
      if (!(sum > 0.0) || !std::isfinite(sum)) {
#pragma omp atomic write
        bad_sum = true;
        continue;
      }
      for (auto& e : cand) e.second /= sum;
      std::sort(cand.begin(), cand.end(), [](const Entry& x, const Entry& y) { return x.first < y.first; });
    }
  }
  if (bad_target) throw std::runtime_error("CF interpolation row has no C target");
  if (bad_sum) throw std::runtime_error("CF interpolation invalid weight sum");
  return pack_transfer(A.n, S.nC, rows);
}

// exact product P01 * P12 (no pruning)
Transfer compose(const Transfer& A, const Transfer& B) {
  if (A.nc != B.nf) throw std::runtime_error("transfer composition size mismatch");
  Transfer P;
  P.nf = A.nf;
  P.nc = B.nc;
  P.row.assign((size_t)A.nf + 1, 0);
  std::vector<Entry> q;
  for (int i = 0; i < A.nf; ++i) {
    q.clear();
    for (int64_t k = A.row[(size_t)i]; k < A.row[(size_t)i + 1]; ++k) {
      const int j = A.col[(size_t)k];
      const double a = A.val[(size_t)k];
      for (int64_t kb = B.row[(size_t)j]; kb < B.row[(size_t)j + 1]; ++kb) q.push_back({B.col[(size_t)kb], a * B.val[(size_t)kb]});
    }
    std::stable_sort(q.begin(), q.end(), [](const Entry& a, const Entry& b) { return a.first < b.first; });
    for (size_t k = 0; k < q.size();) {
      const int c = q[k].first;
      double v = 0.0;
      size_t j = k;
      for (; j < q.size() && q[j].first == c; ++j) v += q[j].second;
      if (v != 0.0) {
        P.col.push_back(c);
        P.val.push_back(v);
      }
      k = j;
    }
    P.row[(size_t)i + 1] = (int64_t)P.col.size();
  }
  return P;
}

}  // namespace

std::vector<int32_t> aggregate_graph(const std::vector<std::vector<int32_t>>& g, int target, int minsz, int softmax,
                                     int* nagg_out) {
  const int n = (int)g.size();
  std::vector<int> id((size_t)n, -1);
  std::vector<std::vector<int>> m;
  std::vector<int> q;
  for (int seed = 0; seed < n; ++seed) {
    if (id[(size_t)seed] >= 0) continue;
    const int a = (int)m.size();
    q.clear();
    q.push_back(seed);
    id[(size_t)seed] = a;
    for (size_t h = 0; h < q.size() && (int)q.size() < target; ++h) {
      const int i = q[h];
      for (int j : g[(size_t)i])
        if (id[(size_t)j] < 0 && (int)q.size() < target) {
          id[(size_t)j] = a;
          q.push_back(j);
        }
    }
    m.push_back(q);
  }
  for (int a = 0; a < (int)m.size(); ++a) {
    if (m[(size_t)a].empty() || (int)m[(size_t)a].size() >= minsz) continue;
    int best = -1, bestsize = INT_MAX;
    bool bestfit = false;
    for (int i : m[(size_t)a])
      for (int j : g[(size_t)i]) {
        const int b = id[(size_t)j];
        if (b < 0 || b == a || m[(size_t)b].empty()) continue;
        const int combined = (int)m[(size_t)a].size() + (int)m[(size_t)b].size();
        const bool fit = combined <= softmax;
        if (best < 0 || (fit && !bestfit) || (fit == bestfit && (int)m[(size_t)b].size() < bestsize)) {
          best = b;
          bestsize = (int)m[(size_t)b].size();
          bestfit = fit;
        }
      }
    if (best >= 0) {
      for (int i : m[(size_t)a]) {
        id[(size_t)i] = best;
        m[(size_t)best].push_back(i);
      }
      m[(size_t)a].clear();
    }
  }
  std::vector<int> compact(m.size(), -1);
  int na = 0;
  for (size_t a = 0; a < m.size(); ++a)
    if (!m[a].empty()) compact[a] = na++;
  std::vector<int32_t> out((size_t)n);
  for (int i = 0; i < n; ++i) {
    out[(size_t)i] = compact[(size_t)id[(size_t)i]];
    if (out[(size_t)i] < 0) throw std::runtime_error("aggregation lost a row");
  }
  if (nagg_out) *nagg_out = na;
  return out;
}

double power_csr(const CsrHost& A, int its, double safety) {
  return power_generic(A.n, A.diag, its, safety, [&](const std::vector<double>& x, std::vector<double>& y) { csr_apply(A, x, y); });
}

std::vector<double> dense_inverse_cholesky(const CsrHost& A) {
  const int n = A.n;
  std::vector<double> M((size_t)n * n, 0.0), L((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int64_t k = A.row[(size_t)i]; k < A.row[(size_t)i + 1]; ++k) M[(size_t)i * n + A.col[(size_t)k]] = A.val[(size_t)k];
  double md = 0;
  for (int i = 0; i < n; ++i) md = std::max(md, std::abs(M[(size_t)i * n + i]));
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      double s = M[(size_t)i * n + j];
      for (int k = 0; k < j; ++k) s -= L[(size_t)i * n + k] * L[(size_t)j * n + k];
      if (i == j) {
        if (!(s > std::max(1e-30, md * 1e-20)) || !std::isfinite(s))
          throw std::runtime_error("terminal Cholesky pivot failure at row " + std::to_string(i));
        L[(size_t)i * n + j] = std::sqrt(s);
      } else {
        L[(size_t)i * n + j] = s / L[(size_t)j * n + j];
      }
    }
  std::vector<double> inv((size_t)n * n, 0.0);
#pragma omp parallel
  {
    std::vector<double> y((size_t)n), x((size_t)n);
#pragma omp for schedule(dynamic, 8)
    for (int col = 0; col < n; ++col) {
      for (int i = 0; i < n; ++i) {
        double s = (i == col) ? 1.0 : 0.0;
        for (int k = 0; k < i; ++k) s -= L[(size_t)i * n + k] * y[(size_t)k];
        y[(size_t)i] = s / L[(size_t)i * n + i];
      }
      for (int i = n - 1; i >= 0; --i) {
        double s = y[(size_t)i];
        for (int k = i + 1; k < n; ++k) s -= L[(size_t)k * n + i] * x[(size_t)k];
        x[(size_t)i] = s / L[(size_t)i * n + i];
      }
      for (int i = 0; i < n; ++i) inv[(size_t)i * n + col] = x[(size_t)i];
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      const double v = 0.5 * (inv[(size_t)i * n + j] + inv[(size_t)j * n + i]);
      inv[(size_t)i * n + j] = inv[(size_t)j * n + i] = v;
    }
  return inv;
}

Hierarchy build_cf_hierarchy(CsrHost A, const AmgOptions& o) {
  StageTimer tm("amg");
  Hierarchy H;
  H.fine_diag = A.diag;
  H.fine_lambda = o.power_its > 0 ? power_csr(A, o.power_its, o.lambda_safety) : 1.0;
  int logical = 0;
  if (o.cf_aggressive_first && A.n > o.terminal) {
    Split s0 = pmis_split(A, o.cf_theta);
    Transfer P01 = cf_transfer(A, s0, o.cf_pmax, o.cf_interp);
    CsrHost A1 = galerkin(A, P01);
    if (A1.n <= o.terminal) {
      H.P.push_back(std::move(P01));
      H.A.push_back(std::move(A1));
    } else {
      Split s1 = pmis_split(A1, o.cf_theta);
      Transfer P12 = cf_transfer(A1, s1, o.cf_pmax, o.cf_interp);
      CsrHost A2 = galerkin(A1, P12);
      H.P.push_back(compose(P01, P12));
      H.A.push_back(std::move(A2));
    }
    if (H.A.back().n > o.terminal) {
      H.level_lambda.resize(H.A.size(), 0.0);
      H.level_lambda[0] = o.power_its > 0 ? power_csr(H.A.back(), o.power_its, o.lambda_safety) : 1.0;
    }
    A = H.A.back();
    logical = 1;
  }
  while (H.A.empty() || H.A.back().n > o.terminal) {
    Split s = pmis_split(A, o.cf_theta);
    tm.mark("pmis");
    H.P.push_back(cf_transfer(A, s, o.cf_pmax, o.cf_interp));
    tm.mark("interpolation");
    H.A.push_back(galerkin(A, H.P.back()));
    tm.mark("galerkin");
    if (H.A.back().n <= o.terminal) break;
    const size_t idx = H.A.size() - 1;
    if (H.level_lambda.size() < H.A.size()) H.level_lambda.resize(H.A.size(), 0.0);
    H.level_lambda[idx] = o.power_its > 0 ? power_csr(H.A.back(), o.power_its, o.lambda_safety) : 1.0;
    A = H.A.back();
    if (++logical > 20) throw std::runtime_error("CF hierarchy excessive levels");
  }
  if (H.level_lambda.size() < H.A.size()) H.level_lambda.resize(H.A.size(), 1.0);
  H.terminal_n = H.A.back().n;
  H.terminal_inv = dense_inverse_cholesky(H.A.back());
  tm.mark("terminal_inverse");
  return H;
}

Hierarchy build_hierarchy(const Mesh& m, const Setup& S, const std::vector<double>& rau, const AmgOptions& o) {
  StageTimer tm("amg");
  Hierarchy H;
  if (o.hierarchy == "sa") {
    int na = 0;
    auto id0 = aggregate_graph(face_graph(m), o.agg_target, o.agg_min, o.agg_softmax, &na);
    H.agg.push_back(id0);
    tm.mark("aggregate0");
    // fine diagonal of B diag(rau) B^T
    H.fine_diag.assign((size_t)S.nc, 0.0);
    for (int c = 0; c < S.nc; ++c) {
      double s = 0;
      for (int a = 0; a < 8; ++a) {
        const int g = S.ref[8 * (size_t)c + a];
        if (g < 0) continue;
        for (int k = 0; k < 3; ++k) {
          const double b = S.bco[24 * (size_t)c + 3 * a + k];
          s += rau[(size_t)g] * b * b;
        }
      }
      H.fine_diag[(size_t)c] = s;
    }
    FineApply fa(S, rau);
    H.fine_lambda = power_generic(S.nc, H.fine_diag, o.power_its, o.lambda_safety,
                                  [&](const std::vector<double>& x, std::vector<double>& y) { fa(x, y); });
    tm.mark("fine_power");
    H.P.push_back(sa_fine_transfer(S, rau, id0, na, H.fine_diag, H.fine_lambda, o.sa_damping, o.interp_max_nnz));
    tm.mark("P0");
    H.A.push_back(sa_first_coarse(S, rau, H.P[0]));
    tm.mark("A1");
    while (H.A.back().n > o.terminal) {
      const CsrHost& A = H.A.back();
      const double lam = power_csr(A, o.power_its, o.lambda_safety);
      if (H.level_lambda.size() < H.A.size()) H.level_lambda.resize(H.A.size(), 0.0);
      H.level_lambda[H.A.size() - 1] = lam;
      int nb = 0;
      auto id = aggregate_graph(csr_graph(A), o.agg_target, o.agg_min, o.agg_softmax, &nb);
      H.agg.push_back(id);
      H.P.push_back(sa_explicit_transfer(A, id, nb, lam, o.sa_damping, o.interp_max_nnz));
      CsrHost C = galerkin(A, H.P.back());
      H.A.push_back(std::move(C));
      tm.mark("level");
    }
    if (H.level_lambda.size() < H.A.size()) H.level_lambda.resize(H.A.size(), 0.0);
  } else if (o.hierarchy == "cf") {
    return build_cf_hierarchy(host_fine_csr(S, rau), o);
  } else {
    throw std::runtime_error("amg hierarchy must be sa or cf");
  }
  H.terminal_n = H.A.back().n;
  H.terminal_inv = dense_inverse_cholesky(H.A.back());
  tm.mark("terminal_inverse");
  return H;
}

}  // namespace nds
