// Host-side 1D nodal basis on Legendre-Gauss-Lobatto (LGL) nodes and the interpolation
// helpers the setup needs.  The operators are the ones the reference builds in
// src/interpolation/basis.f90 and src/dg/dg.f90:181-252 (InitDGbasis):
//   D        polynomial derivative matrix on the nodes,
//   D_hat    = -M^{-1} D^T M            (weak-form volume operator),
//   Dvolsurf = 2 D - M^{-1} B           (split-form operator, B = diag(-1,0..0,1) on LGL),
//   L_HatMinus0 = 1/w_0                 (surface lift of the first node, LGL).
#pragma once
#include <cmath>
#include <vector>

namespace fluxo {
namespace host {

// Legendre polynomial P_n and its derivative at x by the three-term recurrence.
inline void legendre(int n, double x, double& P, double& dP) {
  double p0 = 1., p1 = x, d0 = 0., d1 = 1.;
  if (n == 0) { P = 1.; dP = 0.; return; }
  for (int k = 2; k <= n; ++k) {
    double p2 = ((2. * k - 1.) * x * p1 - (k - 1.) * p0) / k;
    double d2 = d0 + (2. * k - 1.) * p1;
    p0 = p1; p1 = p2; d0 = d1; d1 = d2;
  }
  P = p1; dP = d1;
}

// LGL nodes: x_0=-1, x_N=1 and the roots of P'_N, found by Newton's method on
// q(x) = P_{N+1}(x) - P_{N-1}(x) (a multiple of (1-x^2) P'_N) from Chebyshev-Lobatto guesses.
// Weights w_i = 2 / (N (N+1) P_N(x_i)^2).
inline void lgl(int N, std::vector<double>& x, std::vector<double>& w) {
  x.assign(N + 1, 0.); w.assign(N + 1, 0.);
  x[0] = -1.; x[N] = 1.;
  for (int i = 1; i < N; ++i) {
    double xi = -std::cos(M_PI * i / N);
    for (int it = 0; it < 100; ++it) {
      double a, da, b, db;
      legendre(N + 1, xi, a, da);
      legendre(N - 1, xi, b, db);
      double dx = (a - b) / (da - db);
      xi -= dx;
      if (std::fabs(dx) < 1e-16 * std::max(1., std::fabs(xi))) break;
    }
    x[i] = xi;
  }
  for (int i = 0; i <= N / 2; ++i) {  // enforce exact symmetry
    double s = 0.5 * (x[N - i] - x[i]);
    x[i] = -s; x[N - i] = s;
  }
  if (N % 2 == 0) x[N / 2] = 0.;
  for (int i = 0; i <= N; ++i) {
    double P, dP;
    legendre(N, x[i], P, dP);
    w[i] = 2. / (N * (N + 1.) * P * P);
  }
}

inline void gauss(int N, std::vector<double>& x, std::vector<double>& w) {
  x.assign(N + 1, 0.); w.assign(N + 1, 0.);
  for (int i = 0; i <= N; ++i) {
    double xi = -std::cos(M_PI * (i + 0.75) / (N + 1.5));
    for (int it = 0; it < 100; ++it) {
      double P, dP;
      legendre(N + 1, xi, P, dP);
      double dx = P / dP;
      xi -= dx;
      if (std::fabs(dx) < 1e-16) break;
    }
    double P, dP;
    legendre(N + 1, xi, P, dP);
    x[i] = xi;
    w[i] = 2. / ((1. - xi * xi) * dP * dP);
  }
}

inline std::vector<double> bary(const std::vector<double>& x) {
  const int n = (int)x.size();
  std::vector<double> wb(n, 1.);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      if (j != i) wb[i] *= (x[i] - x[j]);
  for (int i = 0; i < n; ++i) wb[i] = 1. / wb[i];
  return wb;
}

// Lagrange basis of nodes x evaluated at y (exact 0/1 when y hits a node).
inline void lagrange_at(const std::vector<double>& x, const std::vector<double>& wb, double y, double* L) {
  const int n = (int)x.size();
  for (int i = 0; i < n; ++i)
    if (std::fabs(y - x[i]) <= 2.220446049250313e-16 * std::max(std::fabs(y), std::fabs(x[i])) ||
        (y == 0. && std::fabs(x[i]) <= 4.4e-16) || (x[i] == 0. && std::fabs(y) <= 4.4e-16)) {
      for (int k = 0; k < n; ++k) L[k] = (k == i) ? 1. : 0.;
      return;
    }
  double s = 0.;
  for (int i = 0; i < n; ++i) { L[i] = wb[i] / (y - x[i]); s += L[i]; }
  for (int i = 0; i < n; ++i) L[i] /= s;
}

// Interpolation matrix V[o][i] from nodes xin to xout (row-major, out x in).
inline std::vector<double> interp_matrix(const std::vector<double>& xin, const std::vector<double>& xout) {
  const int ni = (int)xin.size(), no = (int)xout.size();
  std::vector<double> V((size_t)no * ni);
  std::vector<double> wb = bary(xin);
  for (int o = 0; o < no; ++o) lagrange_at(xin, wb, xout[o], &V[(size_t)o * ni]);
  return V;
}

// Derivative matrix D[i][j] = l_j'(x_i) on nodes x, diagonal by the negative row sum.
inline std::vector<double> deriv_matrix(const std::vector<double>& x) {
  const int n = (int)x.size();
  std::vector<double> wb = bary(x), D((size_t)n * n, 0.);
  for (int i = 0; i < n; ++i) {
    double diag = 0.;
    for (int j = 0; j < n; ++j)
      if (j != i) {
        D[(size_t)i * n + j] = wb[j] / (wb[i] * (x[i] - x[j]));
        diag -= D[(size_t)i * n + j];
      }
    D[(size_t)i * n + i] = diag;
  }
  return D;
}

// L2 projection (modal truncation in the orthonormal Legendre basis) from nodes xin of degree
// Nin to nodes xout of degree Nout < Nin; quadrature of the modes with 3*Nin/2+2 Gauss points.
inline std::vector<double> modal_projection(const std::vector<double>& xin, const std::vector<double>& xout) {
  const int Nin = (int)xin.size() - 1, Nout = (int)xout.size() - 1;
  std::vector<double> xg, wg;
  gauss(3 * Nin / 2 + 1, xg, wg);
  std::vector<double> Vg = interp_matrix(xin, xg);  // nodal(in) -> gauss
  std::vector<double> V((size_t)(Nout + 1) * (Nin + 1), 0.);
  // coefficient c_m = sum_g w_g phi_m(x_g) u(x_g);  u_out(x_o) = sum_m c_m phi_m(x_o)
  for (int o = 0; o <= Nout; ++o)
    for (int m = 0; m <= Nout; ++m) {
      double Po, dPo;
      legendre(m, xout[o], Po, dPo);
      double nm = std::sqrt(m + 0.5);
      for (size_t g = 0; g < xg.size(); ++g) {
        double Pg, dPg;
        legendre(m, xg[g], Pg, dPg);
        double f = nm * Po * nm * Pg * wg[g];
        for (int i = 0; i <= Nin; ++i) V[(size_t)o * (Nin + 1) + i] += f * Vg[g * (Nin + 1) + i];
      }
    }
  return V;
}

// Nodal -> modal transform onto the orthonormal Legendre polynomials sqrt(m+1/2) P_m on the LGL
// nodes of degree N (sVdm_Leg of BuildLegendreVdm, basis.f90:196-251): c_m = sum_i S[m*(N+1)+i] u_i,
// the L2 projection with 3N/2+2 Gauss points.
inline std::vector<double> legendre_modal(int N) {
  std::vector<double> x, w, xg, wg;
  lgl(N, x, w);
  gauss(3 * N / 2 + 1, xg, wg);
  std::vector<double> Vg = interp_matrix(x, xg);  // L_i(x_g) at [g*(N+1)+i]
  const int n = N + 1;
  std::vector<double> S((size_t)n * n, 0.);
  for (int m = 0; m < n; ++m)
    for (size_t g = 0; g < xg.size(); ++g) {
      double P, dP;
      legendre(m, xg[g], P, dP);
      const double f = std::sqrt(m + 0.5) * P * wg[g];
      for (int i = 0; i < n; ++i) S[(size_t)m * n + i] += f * Vg[g * n + i];
    }
  return S;
}

struct LGLBasis {
  int N;
  std::vector<double> x, w, D, Dhat, Dvs;
  double LhatM0;
  explicit LGLBasis(int N_) : N(N_) {
    lgl(N, x, w);
    D = deriv_matrix(x);
    const int n = N + 1;
    Dhat.assign((size_t)n * n, 0.);
    Dvs.assign((size_t)n * n, 0.);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        Dhat[(size_t)i * n + j] = -D[(size_t)j * n + i] * w[j] / w[i];
        double b = 0.;
        if (i == j && i == 0) b = -1.;
        if (i == j && i == N) b = 1.;
        Dvs[(size_t)i * n + j] = 2. * D[(size_t)i * n + j] - b / w[i];
      }
    LhatM0 = 1. / w[0];
  }
};

// Gauss-Legendre basis of degree N (InitDGbasis dg.f90:181-252 with NodeType 'GAUSS'): D, D_hat, the
// interpolation to the element faces L_Minus / L_Plus, L_HatMinus = L_Minus / w and the split-form
// operator Dvolsurf = 2 D - M^-1 Vf^T B Vf (Vf rows L_Minus, L_Plus; B = diag(-1, 1)), skew-symmetric
// in the M inner product, so its diagonal is zero.
struct GaussBasis {
  int N;
  std::vector<double> x, w, D, Dhat, Dvs, Lminus, Lplus, LhatMinus;
  explicit GaussBasis(int N_) : N(N_) {
    gauss(N, x, w);
    D = deriv_matrix(x);
    const int n = N + 1;
    std::vector<double> wb = bary(x);
    Lminus.assign(n, 0.); Lplus.assign(n, 0.); LhatMinus.assign(n, 0.);
    lagrange_at(x, wb, -1., Lminus.data());
    lagrange_at(x, wb, 1., Lplus.data());
    for (int i = 0; i < n; ++i) LhatMinus[i] = Lminus[i] / w[i];
    Dhat.assign((size_t)n * n, 0.);
    Dvs.assign((size_t)n * n, 0.);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        Dhat[(size_t)i * n + j] = -D[(size_t)j * n + i] * w[j] / w[i];
        const double vbv = -Lminus[i] * Lminus[j] + Lplus[i] * Lplus[j];
        Dvs[(size_t)i * n + j] = 2. * D[(size_t)i * n + j] - vbv / w[i];
      }
  }
};

}  // namespace host
}  // namespace fluxo
