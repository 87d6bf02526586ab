#include "fem.hpp"

#include <cmath>
#include <stdexcept>

namespace nds {

namespace {
// P_n^{(a,b)}(x) and its derivative by the standard three-term recurrence.
void jacobi_p(int n, long double a, long double b, long double x, long double& p, long double& dp) {
  long double p0 = 1.0L, p1 = 0.5L * (a - b + (a + b + 2.0L) * x);
  if (n == 0) { p = p0; dp = 0; return; }
  for (int k = 2; k <= n; ++k) {
    const long double kk = k, s = 2.0L * kk + a + b;
    const long double c1 = 2.0L * kk * (kk + a + b) * (s - 2.0L);
    const long double c2 = (s - 1.0L) * (s * (s - 2.0L) * x + a * a - b * b);
    const long double c3 = 2.0L * (kk + a - 1.0L) * (kk + b - 1.0L) * s;
    const long double p2 = (c2 * p1 - c3 * p0) / c1;
    p0 = p1;
    p1 = p2;
  }
  p = p1;
  // derivative from (1-x^2) P_n' = n[(a-b) - (2n+a+b)x] P_n / (2n+a+b) + 2(n+a)(n+b) P_{n-1} / (2n+a+b)
  const long double nn = n, s = 2.0L * nn + a + b;
  dp = (nn * ((a - b) - s * x) * p1 + 2.0L * (nn + a) * (nn + b) * p0) / (s * (1.0L - x * x));
}
}  // namespace

void gauss_jacobi01(int n, int alpha, std::vector<double>& xo, std::vector<double>& wo) {
  if (n < 1 || alpha < 0) throw std::runtime_error("invalid Gauss-Jacobi rule");
  const long double a = alpha, b = 0.0L;
  const long double pi = 3.141592653589793238462643383279502884L;
  std::vector<long double> x((size_t)n), w((size_t)n);
  for (int i = 0; i < n; ++i) {
    // initial guess (Chebyshev-like), refined by Newton with deflation
    long double z = -std::cos(pi * (i + 0.75L) / (n + 0.5L));
    for (int it = 0; it < 100; ++it) {
      long double p, dp;
      jacobi_p(n, a, b, z, p, dp);
      long double defl = 0;
      for (int j = 0; j < i; ++j) defl += 1.0L / (z - x[(size_t)j]);
      const long double dz = p / (dp - p * defl);
      z -= dz;
      if (std::fabs(dz) < 1e-19L) break;
    }
    x[(size_t)i] = z;
  }
  // Gauss-Jacobi weights on [-1,1]:
  //   w_i = Gamma(n+a+1) Gamma(n+b+1) / (Gamma(n+a+b+1) n!) * 2^(a+b+1) / ((1-x_i^2) P_n'(x_i)^2)
  const long double g = std::exp(std::lgamma(n + a + 1.0L) + std::lgamma(n + b + 1.0L) -
                                 std::lgamma(n + a + b + 1.0L) - std::lgamma(n + 1.0L));
  for (int i = 0; i < n; ++i) {
    long double p, dp;
    jacobi_p(n, a, b, x[(size_t)i], p, dp);
    w[(size_t)i] = g * std::pow(2.0L, a + b + 1.0L) / ((1.0L - x[(size_t)i] * x[(size_t)i]) * dp * dp);
  }
  // sort ascending and map to [0,1]: x -> (x+1)/2, weight (1-x)^a dx -> 2^(a+1) (1-r)^a dr
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j)
      if (x[(size_t)j] < x[(size_t)i]) { std::swap(x[(size_t)i], x[(size_t)j]); std::swap(w[(size_t)i], w[(size_t)j]); }
  xo.resize((size_t)n);
  wo.resize((size_t)n);
  const long double scale = std::pow(2.0L, -(a + 1.0L));
  for (int i = 0; i < n; ++i) {
    xo[(size_t)i] = (double)(0.5L * (x[(size_t)i] + 1.0L));
    wo[(size_t)i] = (double)(w[(size_t)i] * scale);
  }
}

namespace {
// n^3-point collapsed rule: Gauss-Jacobi (1-r)^2, (1-s)^1, Gauss-Legendre t
std::vector<QuadPoint> collapsed_rule(int n) {
  std::vector<double> rn, rw, sn, sw, tn, tw;
  gauss_jacobi01(n, 2, rn, rw);
  gauss_jacobi01(n, 1, sn, sw);
  gauss_jacobi01(n, 0, tn, tw);
  std::vector<QuadPoint> out;
  out.reserve((size_t)n * n * n);
  for (int ir = 0; ir < n; ++ir)
    for (int is = 0; is < n; ++is)
      for (int it = 0; it < n; ++it) {
        const double r = rn[(size_t)ir], s = sn[(size_t)is], t = tn[(size_t)it];
        const double omr = 1 - r, oms = 1 - s;
        out.push_back({{omr * oms * (1 - t), r, omr * s, omr * oms * t}, rw[(size_t)ir] * sw[(size_t)is] * tw[(size_t)it]});
      }
  return out;
}
}  // namespace

const std::vector<QuadPoint>& tet_rule_125() {
  static const std::vector<QuadPoint> q = collapsed_rule(5);
  return q;
}

const std::vector<QuadPoint>& tet_rule_64() {
  static const std::vector<QuadPoint> q = collapsed_rule(4);
  return q;
}

void basis_eval(const std::array<double, 4>& l, double phi[8], double grad[8][3]) {
  static const double gl[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int i = 0; i < 4; ++i) {
    phi[i] = l[(size_t)i];
    for (int d = 0; d < 3; ++d) grad[i][d] = gl[i][d];
  }
  for (int i = 0; i < 4; ++i) {
    int o[3], k = 0;
    for (int j = 0; j < 4; ++j)
      if (j != i) o[k++] = j;
    phi[4 + i] = 27.0 * l[(size_t)o[0]] * l[(size_t)o[1]] * l[(size_t)o[2]];
    // d(27 l0 l1 l2) = 27 (l1 l2 dl0 + l2 l0 dl1 + l0 l1 dl2)
    for (int d = 0; d < 3; ++d) grad[4 + i][d] = 0.0;
    for (int m = 0; m < 3; ++m) {
      const int j = o[m], p = o[(m + 1) % 3], q = o[(m + 2) % 3];
      for (int d = 0; d < 3; ++d) grad[4 + i][d] += 27.0 * l[(size_t)p] * l[(size_t)q] * gl[j][d];
    }
  }
}

const RefTensors& ref_tensors() {
  static const RefTensors T = [] {
    RefTensors o{};
    for (const auto& q : tet_rule_125()) {
      double phi[8], g[8][3];
      basis_eval(q.lam, phi, g);
      for (int a = 0; a < 8; ++a)
        for (int b = 0; b < 8; ++b)
          for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) o.D[a][b][j][k] += g[a][j] * g[b][k] * q.w;
      for (int a = 0; a < 8; ++a)
        for (int m = 0; m < 8; ++m)
          for (int b = 0; b < 8; ++b)
            for (int j = 0; j < 3; ++j) o.T[a][m][b][j] += phi[a] * phi[m] * g[b][j] * q.w;
    }
    return o;
  }();
  return T;
}

}  // namespace nds
