// ORACLE — test infrastructure only.  CPU restatement, in C++17 and FP64, of
// the reference's (FLUXO, Fortran 2003) DGSEM split-form right-hand side and
// LSERK time step on conforming periodic hexahedral meshes.  Only tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it, and
// only as the checker; the product path (fluxo_b200/) never touches it.
//
// Each routine below names the reference file:line it restates.  Loops keep
// the reference's order of summation where it matters for roundoff.
// The reference cannot be compiled here (no Fortran compiler, MPI or HDF5):
// parity of this restatement is pinned on the reference's own regression
// criteria (freestream preservation, discrete entropy conservation and
// stability, convergence order) rather than on value-level golden arrays,
// which the reference does not ship.
#include "fluxo_oracle.h"
#include "fluxo_oracle_timedisc.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

extern "C" { uint64_t g_oracle_flops = 0; }

#ifdef FLUXO_COUNT
#include "counted.h"
typedef Counted real;
#else
typedef double real;
static inline double val(double a) { return a; }
#endif

namespace {

const double PI = 3.14159265358979323846264338327950288;
const double REALTOL = 2.220446049250313e-16;  // EPSILON(1.0D0), globals/preprocessing.f90:25

// local side ids, defines.h:67-72
enum { ZETA_MINUS = 1, ETA_MINUS = 2, XI_PLUS = 3, ETA_PLUS = 4, XI_MINUS = 5, ZETA_PLUS = 6 };
// mesh/mesh_vars.f90:91-93
const int NormalDirs[7] = {0, 3, 2, 1, 2, 1, 3};
const int TangDirs[7] = {0, 1, 3, 2, 3, 2, 1};
const double NormalSigns[7] = {0, -1., -1., 1., 1., -1., 1.};

// ----------------------------------------------------------------------------------------------
// 1D basis, interpolation/basis.f90
// ----------------------------------------------------------------------------------------------
// LegendrePolynomialAndDerivative, basis.f90:286-324 (orthonormal scaling)
void LegendrePolyAndDer(int N, double x, double& L, double& Lder) {
  if (N == 0) { L = 1.; Lder = 0.; }
  else if (N == 1) { L = x; Lder = 1.; }
  else {
    double Lm2 = 1., Lm1 = x, Dm2 = 0., Dm1 = 1.;
    for (int i = 2; i <= N; ++i) {
      L = ((double)(2 * i - 1) * x * Lm1 - (double)(i - 1) * Lm2) / (double)i;
      Lder = Dm2 + (double)(2 * i - 1) * Lm1;
      Lm2 = Lm1; Lm1 = L; Dm2 = Dm1; Dm1 = Lder;
    }
  }
  L *= std::sqrt((double)N + 0.5);
  Lder *= std::sqrt((double)N + 0.5);
}

// qAndLEvaluation, basis.f90:500-537
void qAndL(int N, double x, double& q, double& qder, double& L) {
  double Lm2 = 1., Lm1 = x, Dm2 = 0., Dm1 = 1., Lder = 0.;
  L = x;
  for (int i = 2; i <= N; ++i) {
    L = ((double)(2 * i - 1) * x * Lm1 - (double)(i - 1) * Lm2) / (double)i;
    Lder = Dm2 + (double)(2 * i - 1) * Lm1;
    Lm2 = Lm1; Lm1 = L; Dm2 = Dm1; Dm1 = Lder;
  }
  q = (double)(2 * N + 1) / (double)(N + 1) * (x * L - Lm2);
  qder = (double)(2 * N + 1) * L;
}

// LegGaussLobNodesAndWeights, basis.f90:544-608
void LGLNodesWeights(int N, double* x, double* w) {
  x[0] = -1.; x[N] = 1.;
  if (w) { w[0] = 2. / (double)(N * (N + 1)); w[N] = w[0]; }
  if (N > 1) {
    double c1 = PI / (double)N, c2 = 3. / ((double)(8 * N) * PI);
    for (int i = 1; i <= (N + 1) / 2 - 1; ++i) {
      x[i] = -std::cos(c1 * ((double)i + 0.25) - c2 / ((double)i + 0.25));
      double q, qd, L;
      for (int it = 0; it <= 10; ++it) {
        qAndL(N, x[i], q, qd, L);
        double dx = -q / qd;
        x[i] += dx;
        if (std::fabs(dx) < 1.e-15 * std::fabs(x[i])) break;
      }
      qAndL(N, x[i], q, qd, L);
      x[N - i] = -x[i];
      if (w) { w[i] = w[0] / (L * L); w[N - i] = w[i]; }
    }
  }
  if (N % 2 == 0) {
    x[N / 2] = 0.;
    double q, qd, L;
    qAndL(N, x[N / 2], q, qd, L);
    if (w) w[N / 2] = w[0] / (L * L);
  }
}

// LegendreGaussNodesAndWeights, basis.f90:430-496
void GaussNodesWeights(int N, double* x, double* w) {
  if (N == 0) { x[0] = 0.; if (w) w[0] = 2.; return; }
  if (N == 1) { x[0] = -std::sqrt(1. / 3.); x[1] = -x[0]; if (w) { w[0] = w[1] = 1.; } return; }
  double ct = 2. * std::atan(1.) / (double)(N + 1);
  for (int i = 0; i <= (N + 1) / 2 - 1; ++i) {
    x[i] = -std::cos(ct * (double)(2 * i + 1));
    double L, Ld;
    for (int it = 0; it <= 10; ++it) {
      LegendrePolyAndDer(N + 1, x[i], L, Ld);
      double dx = -L / Ld;
      x[i] += dx;
      if (std::fabs(dx) < 1.e-15 * std::fabs(x[i])) break;
    }
    LegendrePolyAndDer(N + 1, x[i], L, Ld);
    x[N - i] = -x[i];
    if (w) { w[i] = (2. * N + 3) / ((1. - x[i] * x[i]) * Ld * Ld); w[N - i] = w[i]; }
  }
  if (N % 2 == 0) {
    x[N / 2] = 0.;
    double L, Ld;
    LegendrePolyAndDer(N + 1, x[N / 2], L, Ld);
    if (w) w[N / 2] = (2. * N + 3) / (Ld * Ld);
  }
}

// BarycentricWeights, basis.f90:615-634
void BaryWeights(int N, const double* x, double* wb) {
  for (int i = 0; i <= N; ++i) wb[i] = 1.;
  for (int i = 1; i <= N; ++i)
    for (int j = 0; j <= i - 1; ++j) {
      wb[j] *= (x[j] - x[i]);
      wb[i] *= (x[i] - x[j]);
    }
  for (int i = 0; i <= N; ++i) wb[i] = 1. / wb[i];
}

// PolynomialDerivativeMatrix, basis.f90:641-664;  D[i + (N+1)*j] = D(i,j)
void DerivMatrix(int N, const double* x, double* D) {
  std::vector<double> wb(N + 1);
  BaryWeights(N, x, wb.data());
  int n = N + 1;
  for (int k = 0; k < n * n; ++k) D[k] = 0.;
  for (int lag = 0; lag <= N; ++lag)
    for (int i = 0; i <= N; ++i)
      if (lag != i) {
        D[i + n * lag] = wb[lag] / (wb[i] * (x[i] - x[lag]));
        D[i + n * i] -= D[i + n * lag];
      }
}

// ALMOSTEQUAL, basis.f90:673-690
bool AlmostEqual(double x, double y) {
  if (x == 0. || y == 0.) return std::fabs(x - y) <= 2. * REALTOL;
  return std::fabs(x - y) <= REALTOL * std::fabs(x) && std::fabs(x - y) <= REALTOL * std::fabs(y);
}

// LagrangeInterpolationPolys, basis.f90:732-770
void LagrangePolys(double x, int N, const double* xGP, const double* wb, double* L) {
  bool eq = false;
  for (int i = 0; i <= N; ++i) {
    L[i] = 0.;
    if (AlmostEqual(x, xGP[i])) { L[i] = 1.; eq = true; }
  }
  if (eq) return;
  double s = 0.;
  for (int i = 0; i <= N; ++i) { L[i] = wb[i] / (x - xGP[i]); s += L[i]; }
  for (int i = 0; i <= N; ++i) L[i] /= s;
}

enum NodeType { NT_GAUSS = 0, NT_GL = 1, NT_EQUI = 2 };

void Nodes(int N, NodeType t, double* x, double* w = nullptr) {
  if (t == NT_GL) LGLNodesWeights(N, x, w);
  else if (t == NT_GAUSS) GaussNodesWeights(N, x, w);
  else {  // interpolation/interpolation.f90:210-218
    for (int i = 0; i <= N; ++i) x[i] = 2. * (double)i / (double)N - 1.;
    if (w) { for (int i = 0; i <= N; ++i) w[i] = 2. / (double)N; w[0] *= 0.5; w[N] *= 0.5; }
  }
}

// InitializeVandermonde, basis.f90:259-277; V[o + (Nout+1)*i] = Vdm(o,i)
void InitVdm(int Nin, int Nout, const double* wb, const double* xin, const double* xout, double* V) {
  std::vector<double> L(Nin + 1);
  for (int o = 0; o <= Nout; ++o) {
    LagrangePolys(xout[o], Nin, xin, wb, L.data());
    for (int i = 0; i <= Nin; ++i) V[o + (Nout + 1) * i] = L[i];
  }
}

// BuildLegendreVdm, basis.f90:196-251 (Vdm_Leg(i,j): nodal i <- mode j; sVdm_Leg its inverse by projection)
void LegendreVdm(int N, const double* xi, double* Vdm, double* sVdm) {
  int n = N + 1, Ng = 3 * N / 2 + 1;
  std::vector<double> xg(Ng + 1), wg(Ng + 1), wb(n), VT(n * (Ng + 1)), Vgp((Ng + 1) * n);
  BaryWeights(N, xi, wb.data());
  GaussNodesWeights(Ng, xg.data(), wg.data());
  double dummy;
  for (int i = 0; i <= Ng; ++i)
    for (int j = 0; j <= N; ++j) LegendrePolyAndDer(j, xg[i], VT[j + n * i], dummy);
  for (int i = 0; i <= Ng; ++i)
    for (int j = 0; j <= N; ++j) VT[j + n * i] *= wg[i];
  InitVdm(N, Ng, wb.data(), xi, xg.data(), Vgp.data());
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) {
      double s = 0.;
      for (int k = 0; k <= Ng; ++k) s += VT[a + n * k] * Vgp[k + (Ng + 1) * b];
      sVdm[a + n * b] = s;
    }
  for (int i = 0; i <= N; ++i)
    for (int j = 0; j <= N; ++j) LegendrePolyAndDer(j, xi[i], Vdm[i + n * j], dummy);
}

// GetVandermonde, interpolation/interpolation.f90:258-320
std::vector<double> GetVdm(int Nin, NodeType tin, int Nout, NodeType tout, bool modal) {
  std::vector<double> V((Nout + 1) * (Nin + 1), 0.);
  if (tin == tout && Nin == Nout) {
    for (int i = 0; i <= Nin; ++i) V[i + (Nout + 1) * i] = 1.;
    return V;
  }
  std::vector<double> xin(Nin + 1), xout(Nout + 1), wb(Nin + 1);
  Nodes(Nin, tin, xin.data());
  BaryWeights(Nin, xin.data(), wb.data());
  Nodes(Nout, tout, xout.data());
  if (Nout < Nin && modal) {
    std::vector<double> Vli((Nin + 1) * (Nin + 1)), sVli((Nin + 1) * (Nin + 1));
    std::vector<double> Vlo((Nout + 1) * (Nout + 1)), sVlo((Nout + 1) * (Nout + 1));
    LegendreVdm(Nin, xin.data(), Vli.data(), sVli.data());
    LegendreVdm(Nout, xout.data(), Vlo.data(), sVlo.data());
    // Vdm_In_Out = MATMUL(Vdm_Leg_Out(0:Nout,0:Nout), sVdm_Leg_In(0:Nout,0:Nin))
    for (int o = 0; o <= Nout; ++o)
      for (int i = 0; i <= Nin; ++i) {
        double s = 0.;
        for (int m = 0; m <= Nout; ++m) s += Vlo[o + (Nout + 1) * m] * sVli[m + (Nin + 1) * i];
        V[o + (Nout + 1) * i] = s;
      }
  } else {
    InitVdm(Nin, Nout, wb.data(), xin.data(), xout.data(), V.data());
  }
  return V;
}

// ChangeBasis3D_Single, interpolation/changeBasis.f90:225-275 (dim1 interleaved fastest)
void ChangeBasis3D(int dim1, int Nin, int Nout, const double* V, const double* Xin, double* Xout) {
  int ni = Nin + 1, no = Nout + 1;
  std::vector<double> b1((size_t)dim1 * no * ni * ni, 0.), b2((size_t)dim1 * no * no * ni, 0.);
  for (int k = 0; k < ni; ++k)
    for (int j = 0; j < ni; ++j)
      for (int i = 0; i < ni; ++i)
        for (int io = 0; io < no; ++io)
          for (int d = 0; d < dim1; ++d)
            b1[d + dim1 * (io + no * (j + ni * k))] += V[io + no * i] * Xin[d + dim1 * (i + ni * (j + ni * k))];
  for (int k = 0; k < ni; ++k)
    for (int j = 0; j < ni; ++j)
      for (int jo = 0; jo < no; ++jo)
        for (int io = 0; io < no; ++io)
          for (int d = 0; d < dim1; ++d)
            b2[d + dim1 * (io + no * (jo + no * k))] += V[jo + no * j] * b1[d + dim1 * (io + no * (j + ni * k))];
  for (size_t z = 0; z < (size_t)dim1 * no * no * no; ++z) Xout[z] = 0.;
  for (int k = 0; k < ni; ++k)
    for (int ko = 0; ko < no; ++ko)
      for (int jo = 0; jo < no; ++jo)
        for (int io = 0; io < no; ++io)
          for (int d = 0; d < dim1; ++d)
            Xout[d + dim1 * (io + no * (jo + no * ko))] += V[ko + no * k] * b2[d + dim1 * (io + no * (jo + no * k))];
}

// ChangeBasis2D, interpolation/changeBasis.f90:346-381
void ChangeBasis2D(int dim1, int Nin, int Nout, const double* V, const double* Xin, double* Xout) {
  int ni = Nin + 1, no = Nout + 1;
  std::vector<double> b1((size_t)dim1 * no * ni, 0.);
  for (int j = 0; j < ni; ++j)
    for (int i = 0; i < ni; ++i)
      for (int io = 0; io < no; ++io)
        for (int d = 0; d < dim1; ++d) b1[d + dim1 * (io + no * j)] += V[io + no * i] * Xin[d + dim1 * (i + ni * j)];
  for (int z = 0; z < dim1 * no * no; ++z) Xout[z] = 0.;
  for (int j = 0; j < ni; ++j)
    for (int jo = 0; jo < no; ++jo)
      for (int io = 0; io < no; ++io)
        for (int d = 0; d < dim1; ++d) Xout[d + dim1 * (io + no * jo)] += V[jo + no * j] * b1[d + dim1 * (io + no * j)];
}

// ----------------------------------------------------------------------------------------------
// Side <-> volume mappings, mesh/mappings.f90:262-520
// ----------------------------------------------------------------------------------------------
void Flip_S2M(int N, int p, int q, int flip, int& a, int& b) {  // mappings.f90:262-283
  switch (flip) {
    case 0: a = p; b = q; break;
    case 1: a = q; b = p; break;
    case 2: a = N - p; b = q; break;
    case 3: a = N - q; b = N - p; break;
    default: a = p; b = N - q; break;
  }
}
void CGNS_SideToVol(int N, int l, int p, int q, int s, int* ijk) {  // mappings.f90:343-366
  switch (s) {
    case XI_MINUS: ijk[0] = l; ijk[1] = q; ijk[2] = p; break;
    case XI_PLUS: ijk[0] = N - l; ijk[1] = p; ijk[2] = q; break;
    case ETA_MINUS: ijk[0] = p; ijk[1] = l; ijk[2] = q; break;
    case ETA_PLUS: ijk[0] = N - p; ijk[1] = N - l; ijk[2] = q; break;
    case ZETA_MINUS: ijk[0] = q; ijk[1] = p; ijk[2] = l; break;
    default: ijk[0] = p; ijk[1] = q; ijk[2] = N - l; break;
  }
}
void CGNS_SideToVol2(int N, int p, int q, int s, int& a, int& b) {  // mappings.f90:375-398
  switch (s) {
    case XI_MINUS: a = q; b = p; break;
    case XI_PLUS: a = p; b = q; break;
    case ETA_MINUS: a = p; b = q; break;
    case ETA_PLUS: a = N - p; b = q; break;
    case ZETA_MINUS: a = q; b = p; break;
    default: a = p; b = q; break;
  }
}
void SideToVol(int N, int l, int p, int q, int flip, int s, int* ijk) {  // mappings.f90:448-464
  int a, b;
  Flip_S2M(N, p, q, flip, a, b);  // Flip_M2S == Flip_S2M
  CGNS_SideToVol(N, l, a, b, s, ijk);
}

// ----------------------------------------------------------------------------------------------
// Case data
// ----------------------------------------------------------------------------------------------
const int NVMAX = 9;  // nVar: 5 (Navier-Stokes), 9 (MHD with GLM)

struct Case {
  orc_params P;
  int N, np, nVar, nElems, nSides, nDOFElem;
  bool parabolic;
  // MHD (equation/mhd/equation.f90:134-285): eqn 2 ideal, eqn 3 with resistivity/viscosity
  bool mhd = false;
  int nAux = 6;                 // auxiliary variables of the split form (NS 6, MHD 8)
  int noncons = 0;              // NONCONS: 0 off, 1 Powell, 2 Brackbill, 3 Janhunen
  bool ncGLM = false;           // PP_NC_GLM
  double mu_0 = 1., smu_0 = 1., s2mu_0 = 0.5, kappaM2 = 0., eta = 0., etasmu_0 = 0., muMHD = 0.;
  double GLM_scale = 0.5, GLM_scr = 0., GLM_ch = 0., GLM_dtch1 = 0.;
  bool GLM_init = false;
  // NFVSE shock capturing (shockcapturing/nfvse_vars.f90): blending coefficients, sub-cell metrics
  std::vector<double> alpha, alphaMaster, alphaSlave, scNv, scT1, scT2, scNorm;
  std::vector<real> FFVmFDG;    // NFVSE_CORR: (F_FV - Ut_DG) (-sJ) of the last RHS, nfvse_vars.f90
  int corrErr = 0;              // element + 1 whose safe state was not admissible (the reference stops)
  // basis (double), dg/dg.f90:181-252
  std::vector<double> xGP, wGP, wBary, D, D_T, Dhat, Dhat_T, Dvolsurf, Dvolsurf_T, Lminus, Lplus;
  double L_HatMinus0, L_HatPlus0;
  // Gauss nodes (PP_NodeType = 1): L_HatMinus(0:N), the surface metrics of every element side
  // SurfMetrics(3,0:N,0:N,6,nElems) in the master side's point order (mesh_vars.f90:67-70), and the
  // entropy variables of the entropy-projected ProlongToFace (dg_vars.f90:54-61)
  bool gauss = false;
  std::vector<double> LhatMinus, SurfMetrics;
  std::vector<real> Vent;
  // mesh
  std::vector<int> SideToElem, ElemToSide;   // 1-based ids, reference layout
  std::vector<int> S2V;                      // [((((s-1)*5+f)*np+q)*np+p)*np+l]*3
  std::vector<double> NodeCoords, Elem_xGP, Mf, Mg, Mh, sJ, NormVec, TangVec1, TangVec2, SurfElem;
  bool meshNodesGL = false;                  // NodeCoords on Gauss-Lobatto (else equidistant) points
  // state
  std::vector<real> U, Ut, Umaster, Uslave, Fmaster, Fslave, UtTmp;
  std::vector<real> gx, gy, gz, gxm, gym, gzm, gxs, gys, gzs, FX, FY, FZ;
  // equation constants, equation/navierstokes/equation.f90:162-260
  double kappa, sKappa, kappaM1, sKappaM1, kappaP1, sKappaP1, R, s23, Pr, KappasPr, mu0, Ts, sTref,
      ExpoSuth, cSuth, ExpoPow, etaBR2;
  // time disc
  int nRKStages;
  std::vector<double> RKA, RKb, RKc;  // index 1..nStages (RKA[0], RKc[0] unused)
  const OrcRKTable* rk = nullptr;     // the TimeDiscMethod's table (type and all its coefficients)
  double CFLScale, DFLScale;
  bool doCalcSource;

  int s2v(int l, int p, int q, int f, int s, int c) const {
    return S2V[((((((s - 1) * 5 + f) * np + q) * np + p) * np + l) * 3) + c];
  }
  size_t vol(int v, int i, int j, int k, int e) const {
    return (size_t)v + nVar * ((size_t)i + np * ((size_t)j + np * ((size_t)k + (size_t)np * e)));
  }
  size_t nod(int i, int j, int k, int e) const {
    return (size_t)i + np * ((size_t)j + np * ((size_t)k + (size_t)np * e));
  }
  size_t fac(int v, int p, int q, int s) const {  // s = SideID-1
    return (size_t)v + nVar * ((size_t)p + np * ((size_t)q + (size_t)np * s));
  }
};

// ----------------------------------------------------------------------------------------------
// Equation system: compressible Euler / Navier-Stokes, equation/navierstokes/*
// ----------------------------------------------------------------------------------------------
// LN_MEAN, flux_average.f90:1945-1965
inline real LN_MEAN(real aL, real aR) {
  real Xi = aR / aL;
  real u = (Xi * (Xi - 2.) + 1.) / (Xi * (Xi + 2.) + 1.);
  if (u < 1.0E-4) return (aL + aR) * 52.5 / (105. + u * (35. + u * (21. + u * 15.)));
  return (aR - aL) / log(Xi);
}

// EvalUaux, flux_average.f90:305-332  (srho, v1, v2, v3, p, |v|^2)
inline void EvalUaux(const Case& C, const real* U, real* a) {
  real srho = 1. / U[0];
  real v1 = U[1] * srho, v2 = U[2] * srho, v3 = U[3] * srho;
  real v2s = v1 * v1 + v2 * v2 + v3 * v3;
  a[0] = srho; a[1] = v1; a[2] = v2; a[3] = v3; a[5] = v2s;
  a[4] = C.kappaM1 * (U[4] - 0.5 * U[0] * v2s);
}

// Vec two-point fluxes with metric averaging: flux_average.f90
void VolumeFluxVec(const Case& C, const real* UL, const real* UR, const real* aL, const real* aR,
                   const real* mL, const real* mR, real* F) {
  real m1, m2, m3;
  switch (C.P.volume_flux) {
    case 0: {  // StandardDGFluxVec :394-439
      real qL = aL[1] * mL[0] + aL[2] * mL[1] + aL[3] * mL[2];
      real qR = aR[1] * mR[0] + aR[2] * mR[1] + aR[3] * mR[2];
      F[0] = 0.5 * (UL[0] * qL + UR[0] * qR);
      F[1] = 0.5 * (UL[1] * qL + UR[1] * qR + mL[0] * aL[4] + mR[0] * aR[4]);
      F[2] = 0.5 * (UL[2] * qL + UR[2] * qR + mL[1] * aL[4] + mR[1] * aR[4]);
      F[3] = 0.5 * (UL[3] * qL + UR[3] * qR + mL[2] * aL[4] + mR[2] * aR[4]);
      F[4] = 0.5 * ((UL[4] + aL[4]) * qL + (UR[4] + aR[4]) * qR);
      return;
    }
    default: break;
  }
  m1 = 0.5 * (mL[0] + mR[0]);
  m2 = 0.5 * (mL[1] + mR[1]);
  m3 = 0.5 * (mL[2] + mR[2]);
  switch (C.P.volume_flux) {
    case 1: {  // StandardDGFluxDealiasedMetricVec :446-494
      real qL = aL[1] * m1 + aL[2] * m2 + aL[3] * m3;
      real qR = aR[1] * m1 + aR[2] * m2 + aR[3] * m3;
      F[0] = 0.5 * (UL[0] * qL + UR[0] * qR);
      F[1] = 0.5 * (UL[1] * qL + UR[1] * qR + m1 * (aL[4] + aR[4]));
      F[2] = 0.5 * (UL[2] * qL + UR[2] * qR + m2 * (aL[4] + aR[4]));
      F[3] = 0.5 * (UL[3] * qL + UR[3] * qR + m3 * (aL[4] + aR[4]));
      F[4] = 0.5 * ((UL[4] + aL[4]) * qL + (UR[4] + aR[4]) * qR);
      return;
    }
    case 2: {  // KennedyAndGruberFluxVec1 :731-803
      real rhoHat = 0.5 * (UL[0] + UR[0]);
      real uHat = 0.5 * (aL[1] + aR[1]), vHat = 0.5 * (aL[2] + aR[2]), wHat = 0.5 * (aL[3] + aR[3]);
      real p1Hat = 0.5 * (aL[4] + aR[4]);
      real eHat = 0.5 * (aL[0] * UL[4] + aR[0] * UR[4]);
      real qHat = uHat * m1 + vHat * m2 + wHat * m3;
      F[0] = rhoHat * qHat;
      F[1] = F[0] * uHat + m1 * p1Hat;
      F[2] = F[0] * vHat + m2 * p1Hat;
      F[3] = F[0] * wHat + m3 * p1Hat;
      F[4] = F[0] * eHat + p1Hat * qHat;
      return;
    }
    case 5: {  // EntropyAndEnergyConservingFluxVec :1277-1356
      real betaL = 0.5 * UL[0] / aL[4], betaR = 0.5 * UR[0] / aR[4];
      real rhoM = 0.5 * (UL[0] + UR[0]);
      real rhoHat = LN_MEAN(UL[0], UR[0]);
      real betaM = 0.5 * (betaL + betaR);
      real betaHat = LN_MEAN(betaL, betaR);
      real uHat = 0.5 * (aL[1] + aR[1]), vHat = 0.5 * (aL[2] + aR[2]), wHat = 0.5 * (aL[3] + aR[3]);
      real p1Hat = 0.5 * rhoM / betaM;
      real qHat = uHat * m1 + vHat * m2 + wHat * m3;
      F[0] = rhoHat * qHat;
      F[1] = F[0] * uHat + m1 * p1Hat;
      F[2] = F[0] * vHat + m2 * p1Hat;
      F[3] = F[0] * wHat + m3 * p1Hat;
      F[4] = F[0] * 0.5 * (C.sKappaM1 / betaHat - 0.5 * (aL[5] + aR[5])) + uHat * F[1] + vHat * F[2] +
             wHat * F[3];
      return;
    }
    case 10: {  // TwoPointEntropyConservingFluxVec :574-673 (Ismail-Roe)
      real z1L = sqrt(UL[0] / aL[4]), z1R = sqrt(UR[0] / aR[4]);
      real z1Mean = 0.5 * (z1L + z1R);
      real z1LN = LN_MEAN(z1L, z1R);
      real z2Mean = 0.5 * (z1L * aL[1] + z1R * aR[1]);
      real z3Mean = 0.5 * (z1L * aL[2] + z1R * aR[2]);
      real z4Mean = 0.5 * (z1L * aL[3] + z1R * aR[3]);
      real z5L = z1L * aL[4], z5R = z1R * aR[4];
      real z5Mean = 0.5 * (z5L + z5R);
      real z5LN = LN_MEAN(z5L, z5R);
      real rhoHat = z1Mean * z5LN;
      real sz1Mean = 1. / z1Mean;
      real uHat = z2Mean * sz1Mean, vHat = z3Mean * sz1Mean, wHat = z4Mean * sz1Mean;
      real p1Hat = z5Mean * sz1Mean;
      real qHat = uHat * m1 + vHat * m2 + wHat * m3;
      F[0] = rhoHat * qHat;
      F[1] = F[0] * uHat + m1 * p1Hat;
      F[2] = F[0] * vHat + m2 * p1Hat;
      F[3] = F[0] * wHat + m3 * p1Hat;
      F[4] = 0.5 * (qHat * C.kappaP1 * C.sKappaM1 * (z5LN / z1LN) + uHat * F[1] + vHat * F[2] + wHat * F[3]);
      return;
    }
    case 32: {  // RanochaFluxVec :1876-1929
      real rhoLN = LN_MEAN(UL[0], UR[0]);
      real va1 = 0.5 * (aL[1] + aR[1]), va2 = 0.5 * (aL[2] + aR[2]), va3 = 0.5 * (aL[3] + aR[3]);
      real v2ZIP = 0.5 * (aL[1] * aR[1] + aL[2] * aR[2] + aL[3] * aR[3]);
      real pavg = 0.5 * (aL[4] + aR[4]);
      real vmL = aL[1] * m1 + aL[2] * m2 + aL[3] * m3;
      real vmR = aR[1] * m1 + aR[2] * m2 + aR[3] * m3;
      real rspL = UL[0] / aL[4], rspR = UR[0] / aR[4];
      real rspM = LN_MEAN(rspL, rspR);
      F[0] = rhoLN * 0.5 * (vmL + vmR);
      F[1] = F[0] * va1 + m1 * pavg;
      F[2] = F[0] * va2 + m2 * pavg;
      F[3] = F[0] * va3 + m3 * pavg;
      F[4] = F[0] * (v2ZIP + 1. / rspM * C.sKappaM1) + 0.5 * (aL[4] * vmR + aR[4] * vmL);
      return;
    }
    case 3: {  // DucrosFluxVec :986-1059
      real rhoHat = 0.5 * (UL[0] + UR[0]);
      real uHat = 0.5 * (aL[1] + aR[1]), vHat = 0.5 * (aL[2] + aR[2]), wHat = 0.5 * (aL[3] + aR[3]);
      real rhouHat = 0.5 * (UL[1] + UR[1]), rhovHat = 0.5 * (UL[2] + UR[2]), rhowHat = 0.5 * (UL[3] + UR[3]);
      real rhoeHat = 0.5 * (UL[4] + UR[4]);
      real p1Hat = 0.5 * (aL[4] + aR[4]);
      real qHat = uHat * m1 + vHat * m2 + wHat * m3;
      F[0] = rhoHat * qHat;
      F[1] = rhouHat * qHat + m1 * p1Hat;
      F[2] = rhovHat * qHat + m2 * p1Hat;
      F[3] = rhowHat * qHat + m3 * p1Hat;
      F[4] = (rhoeHat + p1Hat) * qHat;
      return;
    }
    case 4: {  // MorinishiFluxVec :1121-1205
      real uHat = 0.5 * (aL[1] + aR[1]), vHat = 0.5 * (aL[2] + aR[2]), wHat = 0.5 * (aL[3] + aR[3]);
      real p1Hat = 0.5 * (aL[4] + aR[4]);
      real qL = aL[1] * m1 + aL[2] * m2 + aL[3] * m3;
      real qR = aR[1] * m1 + aR[2] * m2 + aR[3] * m3;
      real rq2L = 0.5 * UL[0] * qL, rq2R = 0.5 * UR[0] * qR;
      F[0] = rq2L + rq2R;
      F[1] = F[0] * uHat + m1 * p1Hat;
      F[2] = F[0] * vHat + m2 * p1Hat;
      F[3] = F[0] * wHat + m3 * p1Hat;
      F[4] = 0.5 * (C.kappa * C.sKappaM1 * (aL[4] * qL + aR[4] * qR) - (rq2L * aL[5] + rq2R * aR[5])) +
             rq2L * (aL[1] * uHat + aL[2] * vHat + aL[3] * wHat) + rq2R * (aR[1] * uHat + aR[2] * vHat + aR[3] * wHat);
      return;
    }
    case 6: {  // EntropyAndEnergyConservingFluxVec2 :1427-1504
      real betaL = 0.5 * UL[0] / aL[4], betaR = 0.5 * UR[0] / aR[4];
      real rhoM = 0.5 * (UL[0] + UR[0]);
      real sbetaM = 2. / (betaL + betaR);
      real uHat = 0.5 * (aL[1] + aR[1]), vHat = 0.5 * (aL[2] + aR[2]), wHat = 0.5 * (aL[3] + aR[3]);
      real p1Hat = 0.5 * rhoM * sbetaM;
      real qHat = uHat * m1 + vHat * m2 + wHat * m3;
      F[0] = rhoM * qHat;
      F[1] = F[0] * uHat + m1 * p1Hat;
      F[2] = F[0] * vHat + m2 * p1Hat;
      F[3] = F[0] * wHat + m3 * p1Hat;
      F[4] = F[0] * 0.5 * (C.sKappaM1 * sbetaM - 0.5 * (aL[5] + aR[5])) + uHat * F[1] + vHat * F[2] + wHat * F[3];
      return;
    }
    case 7: {  // ggFluxVec :1575-1653 (its log mean of rho is computed but unused there; left out)
      real betaL = 0.5 * UL[0] / aL[4], betaR = 0.5 * UR[0] / aR[4];
      real rhoM = 0.5 * (UL[0] + UR[0]);
      real betaHat = LN_MEAN(betaL, betaR);
      real uHat = 0.5 * (aL[1] + aR[1]), vHat = 0.5 * (aL[2] + aR[2]), wHat = 0.5 * (aL[3] + aR[3]);
      real p1Hat = 0.5 * (aL[4] + aR[4]);
      real qHat = uHat * m1 + vHat * m2 + wHat * m3;
      F[0] = rhoM * qHat;
      F[1] = F[0] * uHat + m1 * p1Hat;
      F[2] = F[0] * vHat + m2 * p1Hat;
      F[3] = F[0] * wHat + m3 * p1Hat;
      F[4] = F[0] * 0.5 * (C.sKappaM1 / betaHat - 0.5 * (aL[5] + aR[5])) + uHat * F[1] + vHat * F[2] + wHat * F[3];
      return;
    }
    case 8: {  // KennedyAndGruberFluxVec2 :857-929
      real rhoHat = 0.5 * (UL[0] + UR[0]);
      real uHat = 0.5 * (aL[1] + aR[1]), vHat = 0.5 * (aL[2] + aR[2]), wHat = 0.5 * (aL[3] + aR[3]);
      real p1Hat = 0.5 * (aL[4] + aR[4]);
      real HHat = 0.5 * ((UL[4] + aL[4]) * aL[0] + (UR[4] + aR[4]) * aR[0]);
      real qHat = uHat * m1 + vHat * m2 + wHat * m3;
      F[0] = rhoHat * qHat;
      F[1] = F[0] * uHat + m1 * p1Hat;
      F[2] = F[0] * vHat + m2 * p1Hat;
      F[3] = F[0] * wHat + m3 * p1Hat;
      F[4] = F[0] * HHat;
      return;
    }
    case 9: {  // GassnerWintersWalchFluxVec :1724-1799
      real sqL = sqrt(UL[0]), sqR = sqrt(UR[0]);
      real rhoHat = 0.5 * (sqL + sqR);
      real uHat = 0.5 * (sqL * aL[1] + sqR * aR[1]);
      real vHat = 0.5 * (sqL * aL[2] + sqR * aR[2]);
      real wHat = 0.5 * (sqL * aL[3] + sqR * aR[3]);
      real HHat = 0.5 * (sqL * aL[0] * (UL[4] + aL[4]) + sqR * aR[0] * (UR[4] + aR[4]));
      real p1Hat = C.kappaM1 * C.sKappa * (rhoHat * HHat - 0.5 * (uHat * uHat + vHat * vHat + wHat * wHat));
      real qHat = uHat * m1 + vHat * m2 + wHat * m3;
      F[0] = rhoHat * qHat;
      F[1] = qHat * uHat + m1 * p1Hat;
      F[2] = qHat * vHat + m2 * p1Hat;
      F[3] = qHat * wHat + m3 * p1Hat;
      F[4] = qHat * HHat;
      return;
    }
    default: throw std::runtime_error("volume flux not implemented");
  }
}

// 1D two-point fluxes in the rotated frame (VolumeFluxAverage pointer), flux_average.f90
struct Hat { real u, v, w, a, H, p1, rho; };
void VolumeFluxAverage(const Case& C, int which, const real* UL, const real* UR, real* F, Hat& h) {
  real sRL = 1. / UL[0], sRR = 1. / UR[0];
  real uL = sRL * UL[1], vL = sRL * UL[2], wL = sRL * UL[3];
  real uR = sRR * UR[1], vR = sRR * UR[2], wR = sRR * UR[3];
  switch (which) {
    case 10: {  // TwoPointEntropyConservingFlux :500-568
      real pL = C.kappaM1 * (UL[4] - 0.5 * (UL[1] * uL + UL[2] * vL + UL[3] * wL));
      real pR = C.kappaM1 * (UR[4] - 0.5 * (UR[1] * uR + UR[2] * vR + UR[3] * wR));
      real z1L = sqrt(UL[0] / pL), z1R = sqrt(UR[0] / pR);
      real z1Mean = 0.5 * (z1L + z1R);
      real z1LN = LN_MEAN(z1L, z1R);
      real z2Mean = 0.5 * (z1L * uL + z1R * uR);
      real z3Mean = 0.5 * (z1L * vL + z1R * vR);
      real z4Mean = 0.5 * (z1L * wL + z1R * wR);
      real z5L = pL * z1L, z5R = pR * z1R;
      real z5Mean = 0.5 * (z5L + z5R);
      real z5LN = LN_MEAN(z5L, z5R);
      h.rho = z1Mean * z5LN;
      real sz1Mean = 1. / z1Mean;
      h.u = z2Mean * sz1Mean; h.v = z3Mean * sz1Mean; h.w = z4Mean * sz1Mean;
      h.p1 = z5Mean * sz1Mean;
      real kp2 = 0.5 * (C.kappaP1 * (z5LN / z1LN) + C.kappaM1 * h.p1);
      h.a = sqrt(kp2 / h.rho);
      h.H = kp2 / (h.rho * C.kappaM1) + 0.5 * (h.u * h.u + h.v * h.v + h.w * h.w);
      F[0] = h.rho * h.u;
      F[1] = F[0] * h.u + h.p1;
      F[2] = F[0] * h.v;
      F[3] = F[0] * h.w;
      F[4] = F[0] * h.H;
      return;
    }
    case 5: {  // EntropyAndEnergyConservingFlux :1214-1269
      real v2s2L = 0.5 * (uL * uL + vL * vL + wL * wL), v2s2R = 0.5 * (uR * uR + vR * vR + wR * wR);
      real pL = C.kappaM1 * (UL[4] - UL[0] * v2s2L), pR = C.kappaM1 * (UR[4] - UR[0] * v2s2R);
      real betaL = 0.5 * UL[0] / pL, betaR = 0.5 * UR[0] / pR;
      real rhoM = 0.5 * (UL[0] + UR[0]);
      h.rho = LN_MEAN(UL[0], UR[0]);
      real betaM = 0.5 * (betaL + betaR);
      real betaHat = LN_MEAN(betaL, betaR);
      h.u = 0.5 * (uL + uR); h.v = 0.5 * (vL + vR); h.w = 0.5 * (wL + wR);
      h.a = sqrt(C.kappa * 0.5 * (pL + pR) / h.rho);
      h.H = C.kappa / (2. * C.kappaM1 * betaHat) + 0.5 * (uL * uR + vL * vR + wL * wR);
      h.p1 = 0.5 * rhoM / betaM;
      real v2M = v2s2L + v2s2R;
      F[0] = h.rho * h.u;
      F[1] = F[0] * h.u + h.p1;
      F[2] = F[0] * h.v;
      F[3] = F[0] * h.w;
      F[4] = F[0] * 0.5 * (C.sKappaM1 / betaHat - v2M) + h.u * F[1] + h.v * F[2] + h.w * F[3];
      return;
    }
    case 32: {  // RanochaFlux :1806-1860
      real v2L = uL * uL + vL * vL + wL * wL, v2R = uR * uR + vR * vR + wR * wR;
      real pL = C.kappaM1 * (UL[4] - 0.5 * UL[0] * v2L), pR = C.kappaM1 * (UR[4] - 0.5 * UR[0] * v2R);
      h.rho = LN_MEAN(UL[0], UR[0]);
      h.u = 0.5 * (uL + uR); h.v = 0.5 * (vL + vR); h.w = 0.5 * (wL + wR);
      real v2ZIP = 0.5 * (uL * uR + vL * vR + wL * wR);
      h.p1 = 0.5 * (pL + pR);
      h.a = sqrt(C.kappa * h.p1 / h.rho);
      h.H = C.kappa * h.p1 * C.sKappaM1 / h.rho + 0.5 * (h.u * h.u + h.v * h.v + h.w * h.w);
      real rspL = UL[0] / pL, rspR = UR[0] / pR;
      real rspM = LN_MEAN(rspL, rspR);
      F[0] = h.rho * h.u;
      F[1] = F[0] * h.u + h.p1;
      F[2] = F[0] * h.v;
      F[3] = F[0] * h.w;
      F[4] = F[0] * (v2ZIP + 1. / rspM * C.sKappaM1) + 0.5 * (pL * uR + pR * uL);
      return;
    }
    case 2: {  // KennedyAndGruberFlux1 :680-721
      h.rho = 0.5 * (UL[0] + UR[0]);
      h.u = 0.5 * (uL + uR); h.v = 0.5 * (vL + vR); h.w = 0.5 * (wL + wR);
      h.p1 = 0.5 * C.kappaM1 *
             (UL[4] + UR[4] - 0.5 * (UL[1] * uL + UL[2] * vL + UL[3] * wL + UR[1] * uR + UR[2] * vR + UR[3] * wR));
      real eHat = 0.5 * (sRL * UL[4] + sRR * UR[4]);
      h.a = sqrt(C.kappa * h.p1 / h.rho);
      h.H = C.kappa * h.p1 / (h.rho * C.kappaM1) + 0.5 * (h.u * h.u + h.v * h.v + h.w * h.w);
      F[0] = h.rho * h.u;
      F[1] = F[0] * h.u + h.p1;
      F[2] = F[0] * h.v;
      F[3] = F[0] * h.w;
      F[4] = F[0] * eHat + h.p1 * h.u;
      return;
    }
    case 3: {  // DucrosFlux :937-979
      h.rho = 0.5 * (UL[0] + UR[0]);
      h.u = 0.5 * (uL + uR); h.v = 0.5 * (vL + vR); h.w = 0.5 * (wL + wR);
      h.p1 = 0.5 * C.kappaM1 *
             (UL[4] + UR[4] - 0.5 * (UL[1] * uL + UL[2] * vL + UL[3] * wL + UR[1] * uR + UR[2] * vR + UR[3] * wR));
      h.a = sqrt(C.kappa * h.p1 / h.rho);
      h.H = C.kappa * h.p1 / (h.rho * C.kappaM1) + 0.5 * (h.u * h.u + h.v * h.v + h.w * h.w);
      real qLR = 0.5 * h.u;
      F[0] = h.rho * (qLR + qLR);
      F[1] = qLR * (UL[1] + UR[1]) + h.p1;
      F[2] = qLR * (UL[2] + UR[2]);
      F[3] = qLR * (UL[3] + UR[3]);
      F[4] = qLR * ((UL[4] + UR[4]) + (h.p1 + h.p1));
      return;
    }
    case 4: {  // MorinishiFlux :1066-1113
      real vel2L = uL * uL + vL * vL + wL * wL, vel2R = uR * uR + vR * vR + wR * wR;
      real pL = C.kappaM1 * (UL[4] - 0.5 * UL[0] * vel2L), pR = C.kappaM1 * (UR[4] - 0.5 * UR[0] * vel2R);
      h.rho = 0.5 * (UL[0] + UR[0]);
      h.u = 0.5 * (uL + uR); h.v = 0.5 * (vL + vR); h.w = 0.5 * (wL + wR);
      h.p1 = 0.5 * (pL + pR);
      h.a = sqrt(C.kappa * h.p1 / h.rho);
      h.H = C.kappa * h.p1 / (h.rho * C.kappaM1) + 0.5 * (h.u * h.u + h.v * h.v + h.w * h.w);
      real rq2L = 0.5 * UL[0] * uL, rq2R = 0.5 * UR[0] * uR;
      F[0] = rq2L + rq2R;
      F[1] = F[0] * h.u + h.p1;
      F[2] = F[0] * h.v;
      F[3] = F[0] * h.w;
      F[4] = 0.5 * (C.kappa * C.sKappaM1 * (pL * uL + pR * uR) - (rq2L * vel2L + rq2R * vel2R)) +
             rq2L * (uL * h.u + vL * h.v + wL * h.w) + rq2R * (uR * h.u + vR * h.v + wR * h.w);
      return;
    }
    case 6: {  // EntropyAndEnergyConservingFlux2 :1365-1419 (a, H = 0)
      real v2s2L = 0.5 * (uL * uL + vL * vL + wL * wL), v2s2R = 0.5 * (uR * uR + vR * vR + wR * wR);
      real pL = C.kappaM1 * (UL[4] - UL[0] * v2s2L), pR = C.kappaM1 * (UR[4] - UR[0] * v2s2R);
      real betaL = 0.5 * UL[0] / pL, betaR = 0.5 * UR[0] / pR;
      real rhoM = 0.5 * (UL[0] + UR[0]);
      real sbetaM = 2. / (betaL + betaR);
      h.a = 0.; h.H = 0.;
      h.rho = LN_MEAN(UL[0], UR[0]);
      h.u = 0.5 * (uL + uR); h.v = 0.5 * (vL + vR); h.w = 0.5 * (wL + wR);
      h.p1 = 0.5 * rhoM * sbetaM;
      F[0] = rhoM * h.u;
      F[1] = F[0] * h.u + h.p1;
      F[2] = F[0] * h.v;
      F[3] = F[0] * h.w;
      F[4] = F[0] * 0.5 * (C.sKappaM1 * sbetaM - (v2s2L + v2s2R)) + h.u * F[1] + h.v * F[2] + h.w * F[3];
      return;
    }
    case 7: {  // ggFlux :1513-1567 (a, H = 0)
      real v2s2L = 0.5 * (uL * uL + vL * vL + wL * wL), v2s2R = 0.5 * (uR * uR + vR * vR + wR * wR);
      real pL = C.kappaM1 * (UL[4] - UL[0] * v2s2L), pR = C.kappaM1 * (UR[4] - UR[0] * v2s2R);
      real betaL = 0.5 * UL[0] / pL, betaR = 0.5 * UR[0] / pR;
      h.a = 0.; h.H = 0.;
      h.rho = LN_MEAN(UL[0], UR[0]);
      real betaHat = LN_MEAN(betaL, betaR);
      h.u = 0.5 * (uL + uR); h.v = 0.5 * (vL + vR); h.w = 0.5 * (wL + wR);
      h.p1 = 0.5 * (pL + pR);
      F[0] = h.rho * h.u;
      F[1] = F[0] * h.u + h.p1;
      F[2] = F[0] * h.v;
      F[3] = F[0] * h.w;
      F[4] = F[0] * 0.5 * (C.sKappaM1 / betaHat - (v2s2L + v2s2R)) + h.u * F[1] + h.v * F[2] + h.w * F[3];
      return;
    }
    case 8: {  // KennedyAndGruberFlux2 :810-850
      real pL = C.kappaM1 * (UL[4] - 0.5 * (UL[1] * uL + UL[2] * vL + UL[3] * wL));
      real pR = C.kappaM1 * (UR[4] - 0.5 * (UR[1] * uR + UR[2] * vR + UR[3] * wR));
      h.rho = 0.5 * (UL[0] + UR[0]);
      h.u = 0.5 * (uL + uR); h.v = 0.5 * (vL + vR); h.w = 0.5 * (wL + wR);
      h.p1 = 0.5 * (pL + pR);
      h.a = sqrt(C.kappa * h.p1 / h.rho);
      h.H = 0.5 * ((UL[4] + pL) * sRL + (UR[4] + pR) * sRR);
      F[0] = h.rho * h.u;
      F[1] = F[0] * h.u + h.p1;
      F[2] = F[0] * h.v;
      F[3] = F[0] * h.w;
      F[4] = F[0] * h.H;
      return;
    }
    case 9: {  // GassnerWintersWalchFlux :1661-1716 (a = 0; Hat values are the averaged Roe variables)
      real pL = C.kappaM1 * (UL[4] - 0.5 * (UL[1] * uL + UL[2] * vL + UL[3] * wL));
      real pR = C.kappaM1 * (UR[4] - 0.5 * (UR[1] * uR + UR[2] * vR + UR[3] * wR));
      real hL = sRL * (UL[4] + pL), hR = sRR * (UR[4] + pR);
      real w1L = sqrt(UL[0]), w1R = sqrt(UR[0]);
      h.rho = 0.5 * (w1L + w1R);
      h.u = 0.5 * (w1L * uL + w1R * uR);
      h.v = 0.5 * (w1L * vL + w1R * vR);
      h.w = 0.5 * (w1L * wL + w1R * wR);
      h.H = 0.5 * (w1L * hL + w1R * hR);
      h.p1 = C.kappaM1 * C.sKappa * (h.rho * h.H - 0.5 * (h.u * h.u + h.v * h.v + h.w * h.w));
      h.a = 0.;
      F[0] = h.u * h.rho;
      F[1] = h.u * h.u + h.p1;
      F[2] = h.u * h.v;
      F[3] = h.u * h.w;
      F[4] = h.u * h.H;
      return;
    }
    default: throw std::runtime_error("two-point flux for Riemann solver not implemented");
  }
}

// EvalEulerFlux1D, navierstokes/flux.f90:298-329
inline void EulerFlux1D(const Case& C, const real* U, real* F) {
  real srho = 1. / U[0];
  real v1 = U[1] * srho, v2 = U[2] * srho, v3 = U[3] * srho;
  real p = C.kappaM1 * (U[4] - 0.5 * (U[1] * v1 + U[2] * v2 + U[3] * v3));
  F[0] = U[1];
  F[1] = U[1] * v1 + p;
  F[2] = U[1] * v2;
  F[3] = U[1] * v3;
  F[4] = (U[4] + p) * v1;
}

// SoundSpeed2, navierstokes/equation_vars.f90:342-356
inline real SoundSpeed2(const Case& C, const real* U) {
  return C.kappa * C.kappaM1 * (U[4] * U[0] - 0.5 * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3])) / (U[0] * U[0]);
}

inline real lambdaMaxPair(const Case& C, const real* LL, const real* RR) {
  return fmax(fabs(LL[1] / LL[0]), fabs(RR[1] / RR[0])) + sqrt(fmax(SoundSpeed2(C, LL), SoundSpeed2(C, RR)));
}

// SolveRiemannProblem on one side (all (N+1)^2 points), rotated states.  navierstokes/riemann.f90
// RiemannSolver_EntropyStable_VolFluxAndDissipMatrices, navierstokes/riemann.f90:936-975: the EC
// two-point flux of the solver (4: Ismail-Roe, 44: EC-KEP, 33: Ranocha; equation.f90:381-404), the
// diagonal scaling DHat = |Lambda| S and the right eigenvectors RHat[row][col] at the flux's mean state
void ES_VolFluxAndDissipMatrices(const Case& C, int rs, const real* L, const real* R, real* Fc, real* Dh,
                                 real Rh[5][5]) {
  const int which = (rs == 4) ? 10 : (rs == 44 ? 5 : 32);
  Hat h;
  VolumeFluxAverage(C, which, L, R, Fc, h);
  const real rows[5][5] = {{1., 1., 0., 0., 1.},
                           {h.u - h.a, h.u, 0., 0., h.u + h.a},
                           {h.v, h.v, 1., 0., h.v},
                           {h.w, h.w, 0., 1., h.w},
                           {h.H - h.u * h.a, 0.5 * (h.u * h.u + h.v * h.v + h.w * h.w), h.v, h.w, h.H + h.u * h.a}};
  for (int r = 0; r < 5; ++r)
    for (int c = 0; c < 5; ++c) Rh[r][c] = rows[r][c];
  Dh[0] = 0.5 * fabs(h.u - h.a) * h.rho / C.kappa;
  Dh[1] = fabs(h.u) * (C.kappaM1 / C.kappa) * h.rho;
  Dh[2] = fabs(h.u) * h.p1;
  Dh[3] = Dh[2];
  Dh[4] = 0.5 * fabs(h.u + h.a) * h.rho / C.kappa;
}

void SolveRiemann(const Case& C, int npts, const real* ULL, const real* URR, real* F) {
  const int rs = C.P.riemann;
  const int nv = 5;
  switch (rs) {
    case 0:  // RiemannSolverCentral :250-272
      for (int i = 0; i < npts; ++i) {
        real FL[5], FR[5];
        EulerFlux1D(C, ULL + nv * i, FL);
        EulerFlux1D(C, URR + nv * i, FR);
        for (int v = 0; v < 5; ++v) F[nv * i + v] = 0.5 * (FL[v] + FR[v]);
      }
      return;
    case 1:  // RiemannSolverByRusanov :279-313
      for (int i = 0; i < npts; ++i) {
        const real* L = ULL + nv * i;
        const real* R = URR + nv * i;
        real lmax = lambdaMaxPair(C, L, R);
        real FL[5], FR[5];
        EulerFlux1D(C, L, FL);
        EulerFlux1D(C, R, FR);
        for (int v = 0; v < 5; ++v) F[nv * i + v] = 0.5 * ((FL[v] + FR[v]) - lmax * (R[v] - L[v]));
      }
      return;
    case 22:  // RiemannSolverByHLL :320-388
      for (int i = 0; i < npts; ++i) {
        const real* L = ULL + nv * i;
        const real* R = URR + nv * i;
        real FL[5], FR[5];
        EulerFlux1D(C, L, FL);
        EulerFlux1D(C, R, FR);
        real sRL = 1. / L[0], sRR = 1. / R[0];
        real vL[3] = {L[1] * sRL, L[2] * sRL, L[3] * sRL};
        real vR[3] = {R[1] * sRR, R[2] * sRR, R[3] * sRR};
        real pL = C.kappaM1 * (L[4] - 0.5 * (L[1] * vL[0] + L[2] * vL[1] + L[3] * vL[2]));
        real pR = C.kappaM1 * (R[4] - 0.5 * (R[1] * vR[0] + R[2] * vR[1] + R[3] * vR[2]));
        real HL = (L[4] + pL) / L[0], HR = (R[4] + pR) / R[0];
        real sqL = sqrt(L[0]), sqR = sqrt(R[0]);
        real HT = (sqL * HL + sqR * HR) / (sqL + sqR);
        real vT = (sqL * vL[0] + sqR * vR[0]) / (sqL + sqR);
        real aT = sqrt((C.kappa - 1.) * (HT - 0.5 * (vT * vT)));
        real ssl = vT - aT, ssr = vT + aT;
        if (ssl >= 0. && ssr > 0.) {
          for (int v = 0; v < 5; ++v) F[nv * i + v] = FL[v];
        } else if (ssr <= 0. && ssl < 0.) {
          for (int v = 0; v < 5; ++v) F[nv * i + v] = FR[v];
        } else {
          for (int v = 0; v < 5; ++v)
            F[nv * i + v] = (ssr * FL[v] - ssl * FR[v] + ssl * ssr * (R[v] - L[v])) / (ssr - ssl);
        }
      }
      return;
    case 4: case 44: case 33: {  // RiemannSolver_EntropyStable :874-931, matrices :936-975
      for (int i = 0; i < npts; ++i) {
        const real* L = ULL + nv * i;
        const real* R = URR + nv * i;
        real Fc[5], Dh[5], Rh[5][5];
        ES_VolFluxAndDissipMatrices(C, rs, L, R, Fc, Dh, Rh);
        real sRL = 1. / L[0], sRR = 1. / R[0];
        real vL[3] = {L[1] * sRL, L[2] * sRL, L[3] * sRL};
        real vR[3] = {R[1] * sRR, R[2] * sRR, R[3] * sRR};
        real pL = C.kappaM1 * (L[4] - 0.5 * (L[1] * vL[0] + L[2] * vL[1] + L[3] * vL[2]));
        real pR = C.kappaM1 * (R[4] - 0.5 * (R[1] * vR[0] + R[2] * vR[1] + R[3] * vR[2]));
        real sR = log(pR) - C.kappa * log(R[0]);
        real sL = log(pL) - C.kappa * log(L[0]);
        real rpR = R[0] / pR, rpL = L[0] / pL;
        real wL[5], wR[5];
        wL[0] = (C.kappa - sL) / C.kappaM1 - 0.5 * rpL * (vL[0] * vL[0] + vL[1] * vL[1] + vL[2] * vL[2]);
        wR[0] = (C.kappa - sR) / C.kappaM1 - 0.5 * rpR * (vR[0] * vR[0] + vR[1] * vR[1] + vR[2] * vR[2]);
        for (int d = 0; d < 3; ++d) { wL[1 + d] = rpL * vL[d]; wR[1 + d] = rpR * vR[d]; }
        wR[4] = -rpR;
        wL[4] = -rpL;
        real jump[5], diss[5];
        for (int v = 0; v < 5; ++v) jump[v] = wR[v] - wL[v];
        // diss = RHat(1,:)*vJump(1) + ... : diss(c) = sum_r RHat(r,c)*jump(r)
        for (int c = 0; c < 5; ++c)
          diss[c] = Rh[0][c] * jump[0] + Rh[1][c] * jump[1] + Rh[2][c] * jump[2] + Rh[3][c] * jump[3] +
                    Rh[4][c] * jump[4];
        for (int v = 0; v < 5; ++v) diss[v] = Dh[v] * diss[v];
        real d2[5];
        for (int r = 0; r < 5; ++r)
          d2[r] = Rh[r][0] * diss[0] + Rh[r][1] * diss[1] + Rh[r][2] * diss[2] + Rh[r][3] * diss[3] +
                  Rh[r][4] * diss[4];
        for (int v = 0; v < 5; ++v) F[nv * i + v] = Fc[v] - 0.5 * d2[v];
      }
      return;
    }
    case 2:  // RiemannSolverByHLLC :552-615
      for (int i = 0; i < npts; ++i) {
        const real* L = ULL + nv * i;
        const real* R = URR + nv * i;
        real FL[5], FR[5];
        EulerFlux1D(C, L, FL);
        EulerFlux1D(C, R, FR);
        real sRL = 1. / L[0], sRR = 1. / R[0];
        real vL[3] = {L[1] * sRL, L[2] * sRL, L[3] * sRL};
        real vR[3] = {R[1] * sRR, R[2] * sRR, R[3] * sRR};
        real pL = C.kappaM1 * (L[4] - 0.5 * (L[1] * vL[0] + L[2] * vL[1] + L[3] * vL[2]));
        real pR = C.kappaM1 * (R[4] - 0.5 * (R[1] * vR[0] + R[2] * vR[1] + R[3] * vR[2]));
        real ssl = vL[0] - sqrt(C.kappa * pL * sRL);
        real ssr = vR[0] + sqrt(C.kappa * pR * sRR);
        real* Fo = F + nv * i;
        if (ssl >= 0.) {
          for (int v = 0; v < 5; ++v) Fo[v] = FL[v];
        } else if (ssr <= 0.) {
          for (int v = 0; v < 5; ++v) Fo[v] = FR[v];
        } else {
          real smuL = ssl - vL[0], smuR = ssr - vR[0];
          real sStar = (pR - pL + L[1] * smuL - R[1] * smuR) / (L[0] * smuL - R[0] * smuR);
          const bool left = (ssl <= 0.) && (sStar >= 0.);
          const real* U = left ? L : R;
          const real* FF = left ? FL : FR;
          real ss = left ? ssl : ssr, smu = left ? smuL : smuR, sr = left ? sRL : sRR, p = left ? pL : pR;
          real vn = left ? vL[0] : vR[0];
          real fac = U[0] * smu / (ss - sStar);
          real Ustar[5] = {fac * 1., fac * sStar, fac * (U[2] * sr), fac * (U[3] * sr),
                           fac * (U[4] * sr + (sStar - vn) * (sStar + p * sr / smu))};
          for (int v = 0; v < 5; ++v) Fo[v] = FF[v] + ss * (Ustar[v] - U[v]);
        }
      }
      return;
    case 23: case 24:  // RiemannSolverByHLLE :393-462, RiemannSolverByHLLEM :466-547
      for (int i = 0; i < npts; ++i) {
        const real* L = ULL + nv * i;
        const real* R = URR + nv * i;
        real FL[5], FR[5];
        EulerFlux1D(C, L, FL);
        EulerFlux1D(C, R, FR);
        real beta = sqrt(0.5 * C.kappaM1 / C.kappa);
        real sRL = 1. / L[0], sRR = 1. / R[0];
        real vL[3] = {L[1] * sRL, L[2] * sRL, L[3] * sRL};
        real vR[3] = {R[1] * sRR, R[2] * sRR, R[3] * sRR};
        real pL = C.kappaM1 * (L[4] - 0.5 * (L[1] * vL[0] + L[2] * vL[1] + L[3] * vL[2]));
        real pR = C.kappaM1 * (R[4] - 0.5 * (R[1] * vR[0] + R[2] * vR[1] + R[3] * vR[2]));
        real aL = sqrt(C.kappa * pL * sRL), aR = sqrt(C.kappa * pR * sRR);
        real HL = (L[4] + pL) * sRL, HR = (R[4] + pR) * sRR;
        real sqL = sqrt(L[0]), sqR = sqrt(R[0]);
        real ssq = 1. / (sqL + sqR);
        real rv[3];
        for (int d = 0; d < 3; ++d) rv[d] = (sqR * vR[d] + sqL * vL[d]) * ssq;
        real rH = (sqR * HR + sqL * HL) * ssq;
        real absVel = rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2];
        real rc = sqrt(C.kappaM1 * (rH - 0.5 * absVel));
        real ssl = fmin(fmin(rv[0] - rc, vL[0] - beta * aL), real(0.));
        real ssr = fmax(fmax(rv[0] + rc, vR[0] + beta * aR), real(0.));
        real* Fo = F + nv * i;
        if (ssl >= 0. && ssr > 0.) {
          for (int v = 0; v < 5; ++v) Fo[v] = FL[v];
        } else if (ssr <= 0. && ssl < 0.) {
          for (int v = 0; v < 5; ++v) Fo[v] = FR[v];
        } else if (rs == 23) {
          for (int v = 0; v < 5; ++v) Fo[v] = (ssr * FL[v] - ssl * FR[v] + ssl * ssr * (R[v] - L[v])) / (ssr - ssl);
        } else {  // HLLEM: anti-diffusion along the Roe-mean entropy and shear waves
          real rd = sqrt(L[0] * R[0]);
          real delta = rc / (rc + fabs(0.5 * (ssl + ssr)));
          real al2 = (R[0] - L[0]) - (pR - pL) / (rc * rc);
          real al3 = rd * (vR[1] - vL[1]), al4 = rd * (vR[2] - vL[2]);
          real r2[5] = {1., rv[0], rv[1], rv[2], 0.5 * absVel};
          real r3[5] = {0., 0., 1., 0., rv[1]};
          real r4[5] = {0., 0., 0., 1., rv[2]};
          for (int v = 0; v < 5; ++v)
            Fo[v] = (ssr * FL[v] - ssl * FR[v] +
                     ssl * ssr * (R[v] - L[v] - delta * (r2[v] * al2 + r3[v] * al3 + r4[v] * al4))) /
                    (ssr - ssl);
        }
      }
      return;
    case 3:  // RiemannSolverByRoe :742-869 (baseline flux chosen by the volume flux id)
      for (int i = 0; i < npts; ++i) {
        const real* L = ULL + nv * i;
        const real* R = URR + nv * i;
        real FL[5], FR[5];
        EulerFlux1D(C, L, FL);
        EulerFlux1D(C, R, FR);
        real sRL = 1. / L[0], sRR = 1. / R[0];
        real vL[3] = {L[1] * sRL, L[2] * sRL, L[3] * sRL};
        real vR[3] = {R[1] * sRR, R[2] * sRR, R[3] * sRR};
        real HL = (L[4] + C.kappaM1 * (L[4] - 0.5 * (L[1] * vL[0] + L[2] * vL[1] + L[3] * vL[2]))) * sRL;
        real HR = (R[4] + C.kappaM1 * (R[4] - 0.5 * (R[1] * vR[0] + R[2] * vR[1] + R[3] * vR[2]))) * sRR;
        real sqL = sqrt(L[0]), sqR = sqrt(R[0]);
        real ssq = 1. / (sqL + sqR);
        real rv[3];
        for (int d = 0; d < 3; ++d) rv[d] = (sqR * vR[d] + sqL * vL[d]) * ssq;
        real rH = (sqR * HR + sqL * HL) * ssq;
        real rc = sqrt(C.kappaM1 * (rH - 0.5 * (rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2])));
        real a1 = rv[0] - rc, a2 = rv[0], a5 = rv[0] + rc;
        real r1[5] = {1., a1, rv[1], rv[2], rH - rv[0] * rc};
        real r2[5] = {1., rv[0], rv[1], rv[2], 0.5 * (rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2])};
        real r3[5] = {0., 0., 1., 0., rv[1]};
        real r4[5] = {0., 0., 0., 1., rv[2]};
        real r5[5] = {1., a5, rv[1], rv[2], rH + rv[0] * rc};
        real dU[6];
        for (int v = 0; v < 5; ++v) dU[v] = R[v] - L[v];
        dU[5] = dU[4] - (dU[2] - rv[1] * dU[0]) * rv[1] - (dU[3] - rv[2] * dU[0]) * rv[2];
        real al3 = dU[2] - rv[1] * dU[0];
        real al4 = dU[3] - rv[2] * dU[0];
        real al2 = C.kappaM1 / (rc * rc) * (dU[0] * (rH - rv[0] * rv[0]) - dU[5] + rv[0] * dU[1]);
        real al1 = 0.5 / rc * (dU[0] * (rv[0] + rc) - dU[1] - rc * al2);
        real al5 = dU[0] - al1 - al2;
        real Fc[5];
        Hat h;
        switch (C.P.volume_flux) {
          case 2:
            VolumeFluxAverage(C, 2, L, R, Fc, h);
            a1 = fmax(fabs(rv[0] - rc), fabs(rv[0] + rc));
            a5 = fmax(fabs(rv[0] - rc), fabs(rv[0] + rc));
            break;
          case 3: VolumeFluxAverage(C, 3, L, R, Fc, h); break;
          case 4:  // the reference pairs volume flux 4 with the Pirozzoli Kennedy-Gruber flux here
            VolumeFluxAverage(C, 8, L, R, Fc, h);
            a1 = fmax(fabs(rv[0] - rc), fabs(rv[0] + rc));
            a5 = fmax(fabs(rv[0] - rc), fabs(rv[0] + rc));
            break;
          default:
            for (int v = 0; v < 5; ++v) Fc[v] = 0.5 * (FL[v] + FR[v]);
        }
        real g1 = al1 * fabs(a1), g2 = al2 * fabs(a2), g3 = al3 * fabs(a2), g4 = al4 * fabs(a2), g5 = al5 * fabs(a5);
        for (int v = 0; v < 5; ++v)
          F[nv * i + v] = Fc[v] - 0.5 * (g1 * r1[v] + g2 * r2[v] + g3 * r3[v] + g4 * r4[v] + g5 * r5[v]);
      }
      return;
    case 5: case 9: case 32: case 6: case 7: case 8: case 10: case 11: case 12: case 20: {
      // RiemannSolver_VolumeFluxAverage :980-1005 with the point flux of equation.f90:291-406
      int which = 0;
      switch (rs) {
        case 5: which = 10; break;
        case 9: which = 5; break;
        case 32: which = 32; break;
        case 6: which = 2; break;
        case 7: which = 3; break;
        case 8: which = 4; break;
        case 10: which = 6; break;
        case 11: which = 7; break;
        case 12: which = 8; break;
        default: which = 9; break;  // 20
      }
      for (int i = 0; i < npts; ++i) {
        Hat h;
        VolumeFluxAverage(C, which, ULL + nv * i, URR + nv * i, F + nv * i, h);
      }
      return;
    }
    case 13: case 14: case 16: case 15: case 17: case 18: case 19: case 21: {
      // LLF-dissipation variants :1011-1209 (lambda max over the side)
      real lmm = 0.;
      for (int i = 0; i < npts; ++i) lmm = fmax(lmm, lambdaMaxPair(C, ULL + nv * i, URR + nv * i));
      for (int i = 0; i < npts; ++i) {
        const real* L = ULL + nv * i;
        const real* R = URR + nv * i;
        real Fc[5];
        Hat h;
        if (rs != 13 && rs != 16) {  // RiemannSolver_VolumeFluxAverage_LLF :1117-1151
          const int which = rs == 14 ? 2 : rs == 15 ? 3 : rs == 17 ? 7 : rs == 18 ? 8 : rs == 19 ? 4 : 9;
          VolumeFluxAverage(C, which, L, R, Fc, h);
          for (int v = 0; v < 5; ++v) F[nv * i + v] = Fc[v] - 0.5 * lmm * (R[v] - L[v]);
        } else if (rs == 13) {  // RiemannSolver_EC_LLF :1011-1110
          VolumeFluxAverage(C, 10, L, R, Fc, h);
          real sRL = 1. / L[0], sRR = 1. / R[0];
          real vL[3] = {L[1] * sRL, L[2] * sRL, L[3] * sRL};
          real vR[3] = {R[1] * sRR, R[2] * sRR, R[3] * sRR};
          real pL = C.kappaM1 * (L[4] - 0.5 * (L[1] * vL[0] + L[2] * vL[1] + L[3] * vL[2]));
          real pR = C.kappaM1 * (R[4] - 0.5 * (R[1] * vR[0] + R[2] * vR[1] + R[3] * vR[2]));
          real sL = log(pL) - C.kappa * log(L[0]);
          real jump[5];
          jump[0] = -((C.kappa - sL) / C.kappaM1 - 0.5 * L[0] * (vL[0] * vL[0] + vL[1] * vL[1] + vL[2] * vL[2]) / pL);
          for (int d = 0; d < 3; ++d) jump[1 + d] = -L[0] * vL[d] / pL;
          jump[4] = L[0] / pL;
          real sR = log(pR) - C.kappa * log(R[0]);
          jump[0] = jump[0] + ((C.kappa - sR) / C.kappaM1 - 0.5 * R[0] * (vR[0] * vR[0] + vR[1] * vR[1] + vR[2] * vR[2]) / pR);
          for (int d = 0; d < 3; ++d) jump[1 + d] = jump[1 + d] + R[0] * vR[d] / pR;
          jump[4] = jump[4] - R[0] / pR;
          real ra = h.rho, v1 = h.u, v2 = h.v, v3 = h.w, pa = h.p1, aa = h.a, Ha = h.H;
          real rhoea = pa / C.kappaM1 + 0.5 * ra * (v1 * v1 + v2 * v2 + v3 * v3);
          real H[5][5];
          H[0][0] = ra; H[1][1] = ra * v1 * v1 + pa; H[2][2] = ra * v2 * v2 + pa; H[3][3] = ra * v3 * v3 + pa;
          H[4][4] = ra * Ha * Ha - aa * aa * pa / C.kappaM1;
          H[0][1] = H[1][0] = ra * v1; H[0][2] = H[2][0] = ra * v2; H[0][3] = H[3][0] = ra * v3;
          H[0][4] = H[4][0] = rhoea;
          H[1][2] = H[2][1] = ra * v1 * v2; H[1][3] = H[3][1] = ra * v1 * v3; H[1][4] = H[4][1] = ra * v1 * Ha;
          H[2][3] = H[3][2] = ra * v2 * v3; H[2][4] = H[4][2] = ra * v2 * Ha; H[3][4] = H[4][3] = ra * v3 * Ha;
          for (int r = 0; r < 5; ++r) {
            real d = H[r][0] * jump[0] + H[r][1] * jump[1] + H[r][2] * jump[2] + H[r][3] * jump[3] + H[r][4] * jump[4];
            F[nv * i + r] = Fc[r] - 0.5 * lmm * d;
          }
        } else {  // 16: RiemannSolver_ECKEP_LLF :1153-1209
          VolumeFluxAverage(C, 5, L, R, Fc, h);
          real sRL = 1. / L[0], sRR = 1. / R[0];
          real vL[3] = {L[1] * sRL, L[2] * sRL, L[3] * sRL};
          real vR[3] = {R[1] * sRR, R[2] * sRR, R[3] * sRR};
          real pL = C.kappaM1 * (L[4] - 0.5 * (L[1] * vL[0] + L[2] * vL[1] + L[3] * vL[2]));
          real pR = C.kappaM1 * (R[4] - 0.5 * (R[1] * vR[0] + R[2] * vR[1] + R[3] * vR[2]));
          real bL = 0.5 * L[0] / pL, bR = 0.5 * R[0] / pR;
          real ra = 0.5 * (R[0] + L[0]);
          real bLN = LN_MEAN(bL, bR);
          for (int v = 0; v < 4; ++v) F[nv * i + v] = Fc[v] - 0.5 * lmm * (R[v] - L[v]);
          F[nv * i + 4] = Fc[4] - 0.5 * lmm *
                                      ((0.5 / (C.kappaM1 * bLN) + 0.5 * (vL[0] * vR[0] + vL[1] * vR[1] + vL[2] * vR[2])) *
                                           (R[0] - L[0]) +
                                       ra * (h.u * (vR[0] - vL[0]) + h.v * (vR[1] - vL[1]) + h.w * (vR[2] - vL[2]) +
                                             0.5 / C.kappaM1 * (1. / bR - 1. / bL)));
        }
      }
      return;
    }
    default: throw std::runtime_error("Riemann solver not implemented");
  }
}

// ConsToEntropy, navierstokes/equation_vars.f90:362-391 (and the Vec form :397-429)
inline void ConsToEntropy(const Case& C, const real* U, real* W) {
  real srho = 1. / U[0];
  real u = U[1] * srho, v = U[2] * srho, w = U[3] * srho;
  real v2s2 = 0.5 * (u * u + v * v + w * w);
  real rho_sp = U[0] / (C.kappaM1 * (U[4] - U[0] * v2s2));
  real s = -log(rho_sp * pow(U[0], C.kappaM1));
  W[0] = (C.kappa - s) * C.sKappaM1 - rho_sp * v2s2;
  W[1] = rho_sp * u;
  W[2] = rho_sp * v;
  W[3] = rho_sp * w;
  W[4] = -rho_sp;
}

// EntropyToCons, navierstokes/equation_vars.f90:434-469
inline void EntropyToCons(const Case& C, const real* W, real* U) {
  real rho_sp = -W[4];
  real p_srho = 1. / rho_sp;
  real u = W[1] * p_srho, v = W[2] * p_srho, w = W[3] * p_srho;
  real v2s2 = 0.5 * (u * u + v * v + w * w);
  real s = C.kappa - ((W[0] + rho_sp * v2s2) * C.kappaM1);
  U[0] = pow(exp(-s) * p_srho, C.sKappaM1);
  U[1] = u * U[0];
  U[2] = v * U[0];
  U[3] = w * U[0];
  U[4] = U[0] * (p_srho * C.sKappaM1 + v2s2);
}

inline void ConsToPrim(const Case& C, const real* U, real* P) {  // equation_vars.f90:243-264
  real sRho = 1. / U[0];
  P[0] = U[0];
  P[1] = U[1] * sRho; P[2] = U[2] * sRho; P[3] = U[3] * sRho;
  P[4] = C.kappaM1 * (U[4] - 0.5 * (U[1] * P[1] + U[2] * P[2] + U[3] * P[3]));
}

// EvalLiftingVolumeFlux / EvalLiftingSurfFlux variable, navierstokes/flux.f90:641-716
inline void LiftingVar(const Case& C, const real* U, real* V) {
  if (C.P.lifting_var == 1) { for (int v = 0; v < 5; ++v) V[v] = U[v]; }
  else if (C.P.lifting_var == 2) ConsToPrim(C, U, V);
  else ConsToEntropy(C, U, V);
}

// ConvertToGradPrimVec, equation_vars.f90:571-647 (one point)
inline void ConvertToGradPrim(const Case& C, const real* U, real* g) {
  if (C.P.lifting_var == 1) {
    real sRho = 1. / U[0];
    real u = U[1] * sRho, v = U[2] * sRho, w = U[3] * sRho;
    real gi1 = g[0];
    real gu = sRho * (g[1] - g[0] * u);
    real gv = sRho * (g[2] - g[0] * v);
    real gw = sRho * (g[3] - g[0] * w);
    real gi5 = g[4];
    g[1] = gu; g[2] = gv; g[3] = gw;
    g[4] = C.kappaM1 * (gi5 - (0.5 * gi1 * (u * u + v * v + w * w) + (U[1] * gu + U[2] * gv + U[3] * gw)));
  } else if (C.P.lifting_var == 2) {
    return;
  } else {
    real sRho = 1. / U[0];
    real u = U[1] * sRho, v = U[2] * sRho, w = U[3] * sRho;
    real Ekin = 0.5 * (U[1] * u + U[2] * v + U[3] * w);
    real p = C.kappaM1 * (U[4] - Ekin);
    real rho_sp = U[0] / p;
    real p_srho = p * sRho;
    real gi1 = g[0];
    real gu = p_srho * (g[1] + u * g[4]);
    real gv = p_srho * (g[2] + v * g[4]);
    real gw = p_srho * (g[3] + w * g[4]);
    real gi5 = g[4];
    g[0] = U[0] * gi1 - gi5 * (Ekin - p * C.sKappaM1) + rho_sp * (U[1] * gu + U[2] * gv + U[3] * gw);
    g[1] = gu; g[2] = gv; g[3] = gw;
    g[4] = p_srho * (g[0] + p * gi5);
  }
}

// viscosity law, equation_vars.f90:672-692 and flux.f90:470-480
inline real ViscMu(const Case& C, real p, real srho) {
  if (C.P.visc == 0) return real(C.mu0);
  real T = p * srho / C.R;
  if (C.P.visc == 1) {
    real Tn = T * C.sTref;
    if (Tn >= C.Ts) return C.mu0 * pow(Tn, C.ExpoSuth) * (1 + C.Ts) / (Tn + C.Ts);
    return C.mu0 * Tn * C.cSuth;
  }
  return C.mu0 * pow(T, C.ExpoPow);
}

// EvalDiffFlux3D (one point), navierstokes/flux.f90:407-517; gradients are primitive
void DiffFlux3D(const Case& C, const real* U, const real* gX, const real* gY, const real* gZ, real* f, real* g,
                real* h) {
  real srho = 1. / U[0];
  real v1 = U[1] * srho, v2 = U[2] * srho, v3 = U[3] * srho;
  real p = C.kappaM1 * (U[4] - 0.5 * (U[1] * v1 + U[2] * v2 + U[3] * v3));
  real muS = ViscMu(C, p, srho);
  real lambda = muS * C.KappasPr;
  real divv = gX[1] + gY[2] + gZ[3];
  real cvTx = C.sKappaM1 * srho * (gX[4] - srho * p * gX[0]);
  real cvTy = C.sKappaM1 * srho * (gY[4] - srho * p * gY[0]);
  real cvTz = C.sKappaM1 * srho * (gZ[4] - srho * p * gZ[0]);
  f[0] = 0.;
  f[1] = -muS * (2 * gX[1] - C.s23 * divv);
  f[2] = -muS * (gX[2] + gY[1]);
  f[3] = -muS * (gX[3] + gZ[1]);
  f[4] = v1 * f[1] + v2 * f[2] + v3 * f[3] - lambda * cvTx;
  g[0] = 0.;
  g[1] = f[2];
  g[2] = -muS * (2 * gY[2] - C.s23 * divv);
  g[3] = -muS * (gY[3] + gZ[2]);
  g[4] = v1 * g[1] + v2 * g[2] + v3 * g[3] - lambda * cvTy;
  h[0] = 0.;
  h[1] = f[3];
  h[2] = g[3];
  h[3] = -muS * (2 * gZ[3] - C.s23 * divv);
  h[4] = v1 * h[1] + v2 * h[2] + v3 * h[3] - lambda * cvTz;
}

#include "fluxo_oracle_mhd.h"

// Equation-system dispatch (the reference selects the module at compile time).
inline void Uaux(const Case& C, const real* U, real* a) {
  if (C.mhd) MHD_Uaux(C, U, a);
  else EvalUaux(C, U, a);
}
inline void LiftVar(const Case& C, const real* U, real* V) {
  if (!C.mhd) { LiftingVar(C, U, V); return; }
  if (C.P.lifting_var == 1) { for (int v = 0; v < 9; ++v) V[v] = U[v]; }
  else if (C.P.lifting_var == 2) MHD_ConsToPrim(C, U, V);
  else MHD_ConsToEntropy(C, U, V);
}
inline void GradPrim(const Case& C, const real* U, real* g) {
  if (C.mhd) MHD_ConvertToGradPrim(C, U, g);
  else ConvertToGradPrim(C, U, g);
}
inline void DiffFlux(const Case& C, const real* U, const real* gX, const real* gY, const real* gZ, real* f, real* g,
                     real* h) {
  if (C.mhd) MHD_DiffFlux3D(C, U, gX, gY, gZ, f, g, h);
  else DiffFlux3D(C, U, gX, gY, gZ, f, g, h);
}

// ----------------------------------------------------------------------------------------------
// Exact functions, navierstokes/equation.f90:575-950
// ----------------------------------------------------------------------------------------------
void PrimToCons(const Case& C, const double* prim, double* cons) {  // equation_vars.f90:271-290
  cons[0] = prim[0];
  cons[1] = prim[1] * prim[0]; cons[2] = prim[2] * prim[0]; cons[3] = prim[3] * prim[0];
  cons[4] = C.sKappaM1 * prim[4] + 0.5 * (cons[1] * prim[1] + cons[2] * prim[2] + cons[3] * prim[3]);
}

void ExactFunc(const Case& C, int func, double t, const double* x, double* resu) {
  if (C.mhd) { MHD_ExactFunc(C, func, t, x, resu); return; }
  const orc_params& P = C.P;
  double prim[5];
  switch (func) {
    case 1:  // constant refstate
      PrimToCons(C, P.ref_state, resu);
      return;
    case 2: {  // equation.f90:632-651
      prim[0] = 1.;
      for (int d = 0; d < 3; ++d) prim[1 + d] = P.adv_vel[d];
      prim[4] = 1.;
      double cent[3], s = 0.;
      for (int d = 0; d < 3; ++d) { cent[d] = x[d] - P.adv_vel[d] * t; s += P.ini_wavenumber[d] * cent[d]; }
      prim[0] = prim[0] * (1. + P.ini_amplitude * std::sin(PI * s));
      resu[0] = prim[0];
      for (int d = 0; d < 3; ++d) resu[1 + d] = prim[0] * prim[1 + d];
      resu[4] = prim[4] * C.sKappaM1 + 0.5 * prim[0] * (prim[1] * prim[1] + prim[2] * prim[2] + prim[3] * prim[3]);
      return;
    }
    case 4: {  // manufactured solution, equation.f90:698-702
      double Omega = PI * P.ini_frequency;
      double v = 2. + P.ini_amplitude * std::sin(Omega * ((x[0] + x[1] + x[2]) - t));
      resu[0] = v; resu[1] = v; resu[2] = v; resu[3] = v;
      resu[4] = resu[0] * resu[0];
      return;
    }
    case 7: {  // Taylor-Green vortex, equation.f90:802-811
      double A = 1., Ms = 0.1;
      prim[0] = 1.;
      prim[1] = A * std::sin(x[0]) * std::cos(x[1]) * std::cos(x[2]);
      prim[2] = -A * std::cos(x[0]) * std::sin(x[1]) * std::cos(x[2]);
      prim[3] = 0.;
      prim[4] = (A / Ms * A / Ms / C.kappa * prim[0]);
      prim[4] = prim[4] + 1. / 16. * A * A * prim[0] *
                              (std::cos(2 * x[0]) * std::cos(2. * x[2]) + 2. * std::cos(2. * x[1]) +
                               2. * std::cos(2. * x[0]) + std::cos(2 * x[1]) * std::cos(2. * x[2]));
      PrimToCons(C, prim, resu);
      return;
    }
    case 14: {  // soft Sedov-Taylor blast, equation.f90:906-922 (dim_ = 3)
      double nx[3], r2 = 0.;
      for (int d = 0; d < 3; ++d) { nx[d] = x[d] - P.ini_center[d]; r2 += nx[d] * nx[d]; }
      r2 = std::sqrt(r2);
      prim[0] = 1.; prim[1] = prim[2] = prim[3] = 0.; prim[4] = 1.;
      if (r2 <= 0.5 && r2 != 0.) {
        prim[0] = 1.3416149068323;
        for (int d = 0; d < 3; ++d) prim[1 + d] = 0.361538208967199 * nx[d] / r2;
        prim[4] = 1.51333333333333;
      }
      PrimToCons(C, prim, resu);
      return;
    }
    default: throw std::runtime_error("ExactFunc not implemented in oracle");
  }
}

// CalcSource, navierstokes/equation.f90:992-1071 (CASE 4 only; other cases disable the source)
void CalcSource(Case& C, double t) {
  if (C.mhd) {  // GLM damping, mhd/equation.f90:1698-1706 (the default case has no other source)
    if (AlmostEqual(C.GLM_scr, 0.)) return;
    size_t nd = (size_t)C.np * C.np * C.np * C.nElems;
    for (size_t z = 0; z < nd; ++z) C.Ut[9 * z + 8] = C.Ut[9 * z + 8] - C.GLM_scr * C.GLM_ch * C.U[9 * z + 8];
    return;
  }
  if (!C.doCalcSource) return;
  const orc_params& P = C.P;
  double Omega = PI * P.ini_frequency;
  double tmp[6];
  tmp[0] = 2.;
  tmp[1] = 2. + 2.5 * C.kappaM1;
  tmp[2] = P.ini_amplitude * C.kappaM1;
  tmp[3] = 0.5 * (9. + C.kappa * 15.) - 4.;
  tmp[4] = P.ini_amplitude * (3. * C.kappa - 1.);
  tmp[5] = C.parabolic ? 3. * C.mu0 * C.kappa * Omega / C.Pr : 0.;
  for (int z = 0; z < 6; ++z) tmp[z] = tmp[z] * P.ini_amplitude * Omega;
  for (int e = 0; e < C.nElems; ++e)
    for (int k = 0; k < C.np; ++k)
      for (int j = 0; j < C.np; ++j)
        for (int i = 0; i < C.np; ++i) {
          const double* xg = &C.Elem_xGP[3 * C.nod(i, j, k, e)];
          double cosX = std::cos(Omega * (xg[0] + xg[1] + xg[2] - t));
          double sinX = std::sin(Omega * (xg[0] + xg[1] + xg[2] - t));
          double sin2 = 2. * sinX * cosX;
          real src[5];
          src[0] = tmp[0] * cosX;
          src[1] = src[2] = src[3] = tmp[1] * cosX + tmp[2] * sin2;
          src[4] = tmp[3] * cosX + tmp[4] * sin2 + tmp[5] * sinX;
          for (int v = 0; v < 5; ++v) C.Ut[C.vol(v, i, j, k, e)] += src[v];
        }
}

// ----------------------------------------------------------------------------------------------
// Setup: basis (dg/dg.f90:181-252), mesh, metrics (mesh/metrics.f90)
// ----------------------------------------------------------------------------------------------
void InitBasis(Case& C) {
  int N = C.N, n = C.np;
  C.xGP.resize(n); C.wGP.resize(n); C.wBary.resize(n);
  if (C.gauss) GaussNodesWeights(N, C.xGP.data(), C.wGP.data());  // InitInterpolation, NodeType 'GAUSS'
  else LGLNodesWeights(N, C.xGP.data(), C.wGP.data());
  BaryWeights(N, C.xGP.data(), C.wBary.data());
  C.D.resize(n * n); C.D_T.resize(n * n); C.Dhat.resize(n * n); C.Dhat_T.resize(n * n);
  C.Dvolsurf.resize(n * n); C.Dvolsurf_T.resize(n * n);
  DerivMatrix(N, C.xGP.data(), C.D.data());
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) C.D_T[i + n * j] = C.D[j + n * i];
  // D_Hat = -MATMUL(Minv, MATMUL(TRANSPOSE(D), M)) => Dhat(i,j) = -(1/w_i) D(j,i) w_j
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) C.Dhat[i + n * j] = -((1. / C.wGP[i]) * (C.D[j + n * i] * C.wGP[j]));
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) C.Dhat_T[i + n * j] = C.Dhat[j + n * i];
  C.Lminus.resize(n); C.Lplus.resize(n);
  LagrangePolys(1., N, C.xGP.data(), C.wBary.data(), C.Lplus.data());
  LagrangePolys(-1., N, C.xGP.data(), C.wBary.data(), C.Lminus.data());
  C.L_HatMinus0 = (1. / C.wGP[0]) * C.Lminus[0];
  C.L_HatPlus0 = (1. / C.wGP[N]) * C.Lplus[N];
  C.LhatMinus.resize(n);  // L_HatMinus = MATMUL(Minv, L_Minus), dg.f90:222-226
  for (int i = 0; i < n; ++i) C.LhatMinus[i] = (1. / C.wGP[i]) * C.Lminus[i];
  // Dvolsurf = 2*D - Minv*Vf^T*B*Vf, Vf rows (L_Minus, L_Plus), B = diag(-1,1)
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double vbv = -C.Lminus[i] * C.Lminus[j] + C.Lplus[i] * C.Lplus[j];
      C.Dvolsurf[i + n * j] = 2.0 * C.D[i + n * j] - (1. / C.wGP[i]) * vbv;
    }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) C.Dvolsurf_T[i + n * j] = C.Dvolsurf[j + n * i];
}

// Periodic box connectivity with the reference's side numbering rule (mesh/prepare_mesh.f90:59-260,
// :662-715): side ids are assigned in element / local-side order, the first element that meets a
// side owns it as master (flip 0) and the slave's flip is found from the node lattice.
void BuildS2V(Case& C) {
  const int N = C.N, n = C.np;
  // S2V, mappings.f90:93-255
  C.S2V.assign((size_t)6 * 5 * n * n * n * 3, 0);
  for (int s = 1; s <= 6; ++s)
    for (int f = 0; f <= 4; ++f)
      for (int q = 0; q < n; ++q)
        for (int p = 0; p < n; ++p)
          for (int l = 0; l < n; ++l) {
            int ijk[3];
            SideToVol(N, l, p, q, f, s, ijk);
            for (int c = 0; c < 3; ++c) C.S2V[((((((s - 1) * 5 + f) * n + q) * n + p) * n + l) * 3) + c] = ijk[c];
          }
}

void BuildMesh(Case& C) {
  const orc_params& P = C.P;
  int nx = P.nElems[0], ny = P.nElems[1], nz = P.nElems[2], N = C.N, n = C.np;
  C.nElems = nx * ny * nz;
  C.nSides = 3 * C.nElems;
  BuildS2V(C);
  auto eid = [&](int ix, int iy, int iz) { return ((iz + nz) % nz) * nx * ny + ((iy + ny) % ny) * nx + ((ix + nx) % nx); };
  auto neighbor = [&](int e, int s, int& nbE, int& nbS) {
    int ix = e % nx, iy = (e / nx) % ny, iz = e / (nx * ny);
    switch (s) {
      case XI_MINUS: nbE = eid(ix - 1, iy, iz); nbS = XI_PLUS; break;
      case XI_PLUS: nbE = eid(ix + 1, iy, iz); nbS = XI_MINUS; break;
      case ETA_MINUS: nbE = eid(ix, iy - 1, iz); nbS = ETA_PLUS; break;
      case ETA_PLUS: nbE = eid(ix, iy + 1, iz); nbS = ETA_MINUS; break;
      case ZETA_MINUS: nbE = eid(ix, iy, iz - 1); nbS = ZETA_PLUS; break;
      default: nbE = eid(ix, iy, iz + 1); nbS = ZETA_MINUS; break;
    }
  };
  // global lattice coordinate of volume node (i,j,k) of element e
  auto lattice = [&](int e, const int* ijk, long* g) {
    int ix = e % nx, iy = (e / nx) % ny, iz = e / (nx * ny);
    g[0] = ((long)ix * N + ijk[0]) % ((long)nx * N);
    g[1] = ((long)iy * N + ijk[1]) % ((long)ny * N);
    g[2] = ((long)iz * N + ijk[2]) % ((long)nz * N);
  };
  C.ElemToSide.assign((size_t)2 * 6 * C.nElems, 0);
  C.SideToElem.assign((size_t)5 * C.nSides, -1);
  std::vector<int> sideOf((size_t)6 * C.nElems, -1);
  int nextSide = 0;
  for (int e = 0; e < C.nElems; ++e)
    for (int s = 1; s <= 6; ++s) {
      if (sideOf[(size_t)6 * e + s - 1] >= 0) continue;
      int nbE, nbS;
      neighbor(e, s, nbE, nbS);
      int sid = ++nextSide;  // 1-based
      sideOf[(size_t)6 * e + s - 1] = sid;
      sideOf[(size_t)6 * nbE + nbS - 1] = sid;
      // master
      C.ElemToSide[0 + 2 * ((s - 1) + 6 * (size_t)e)] = sid;
      C.ElemToSide[1 + 2 * ((s - 1) + 6 * (size_t)e)] = 0;
      C.SideToElem[0 + 5 * (size_t)(sid - 1)] = e + 1;
      C.SideToElem[2 + 5 * (size_t)(sid - 1)] = s;
      // slave flip from the node lattice
      int flip = -1;
      for (int f = 1; f <= 4 && flip < 0; ++f) {
        bool ok = true;
        for (int q = 0; q < n && ok; ++q)
          for (int p = 0; p < n && ok; ++p) {
            int a[3], b[3];
            long ga[3], gb[3];
            SideToVol(N, 0, p, q, 0, s, a);
            SideToVol(N, 0, p, q, f, nbS, b);
            lattice(e, a, ga);
            lattice(nbE, b, gb);
            ok = (ga[0] == gb[0] && ga[1] == gb[1] && ga[2] == gb[2]);
          }
        if (ok) flip = f;
      }
      if (flip < 0) throw std::runtime_error("no flip found");
      C.ElemToSide[0 + 2 * ((nbS - 1) + 6 * (size_t)nbE)] = sid;
      C.ElemToSide[1 + 2 * ((nbS - 1) + 6 * (size_t)nbE)] = flip;
      C.SideToElem[1 + 5 * (size_t)(sid - 1)] = nbE + 1;
      C.SideToElem[3 + 5 * (size_t)(sid - 1)] = nbS;
      C.SideToElem[4 + 5 * (size_t)(sid - 1)] = flip;
    }
  if (nextSide != C.nSides) throw std::runtime_error("side count mismatch");
  // node coordinates on equidistant NGeo points, deformed like mesh/mesh.f90:238-245
  int NG = P.NGeo, ng = NG + 1;
  C.NodeCoords.assign((size_t)3 * ng * ng * ng * C.nElems, 0.);
  double L[3], h[3], cen[3];
  for (int d = 0; d < 3; ++d) {
    L[d] = P.xmax[d] - P.xmin[d];
    cen[d] = 0.5 * (P.xmax[d] + P.xmin[d]);
  }
  h[0] = L[0] / nx; h[1] = L[1] / ny; h[2] = L[2] / nz;
  for (int e = 0; e < C.nElems; ++e) {
    int ix = e % nx, iy = (e / nx) % ny, iz = e / (nx * ny);
    for (int k = 0; k < ng; ++k)
      for (int j = 0; j < ng; ++j)
        for (int i = 0; i < ng; ++i) {
          double x[3];
          x[0] = P.xmin[0] + h[0] * (ix + (double)i / NG);
          x[1] = P.xmin[1] + h[1] * (iy + (double)j / NG);
          x[2] = P.xmin[2] + h[2] * (iz + (double)k / NG);
          double fac = P.deform_amp;
          if (fac != 0.) {
            for (int d = 0; d < 3; ++d) fac *= std::sin(2. * PI * (x[d] - cen[d]) / L[d]);
          }
          double* X = &C.NodeCoords[3 * ((size_t)i + ng * ((size_t)j + ng * ((size_t)k + (size_t)ng * e)))];
          for (int d = 0; d < 3; ++d) X[d] = x[d] + fac;
        }
  }
}

// A HOPR mesh given by the arrays of its file (ElemInfo, SideInfo, BCType, NodeCoords), restating
// ReadMesh (mesh/mesh_readin.f90:295-511), setLocalSideIDs (mesh/prepare_mesh.f90:59-215) and
// fillMeshInfo (mesh/prepare_mesh.f90:662-710) for a single process.  Sides are records
// (element, local side) indexed 6*e + (locSide-1); mortar sides and sides of non-periodic
// boundaries have no counterpart in the product and are refused.
struct HoprMesh {
  int nElems, nSideInfo, nBCs, NGeo, nodesGL, useCurveds;
  const int *ElemInfo, *SideInfo, *BCType;
  const double* NodeCoords;
  double meshScale;
};

void BuildMeshHOPR(Case& C, const HoprMesh& M) {
  const int nE = M.nElems;
  C.nElems = nE;
  BuildS2V(C);
  std::vector<int> ind(6 * (size_t)nE), flip(6 * (size_t)nE), conn(6 * (size_t)nE, -1), sideID(6 * (size_t)nE, -1);
  auto SI = [&](int row, int f) { return M.SideInfo[5 * (size_t)row + (f - 1)]; };  // SideInfo(f, row+1)
  for (int e = 0; e < nE; ++e) {
    const int first = M.ElemInfo[6 * (size_t)e + 2];  // ELEM_FirstSideInd (0-based offset)
    for (int ls = 1; ls <= 6; ++ls) {
      const int row = first + ls - 1;
      if (row < 0 || row >= M.nSideInfo) throw std::runtime_error("HOPR mesh: SideInfo index out of range");
      if (SI(row, 3) < 0 || SI(row, 1) < 0) throw std::runtime_error("HOPR mesh: mortar sides are not supported");
      const size_t a = 6 * (size_t)e + ls - 1;
      ind[a] = std::abs(SI(row, 2));
      if (SI(row, 2) > 0) flip[a] = 0;
      else {
        flip[a] = SI(row, 4) % 10;
        if (flip[a] < 0 || flip[a] > 4) throw std::runtime_error("HOPR mesh: NodeID doesnt belong to side");
      }
    }
  }
  for (int e = 0; e < nE; ++e) {
    const int first = M.ElemInfo[6 * (size_t)e + 2];
    for (int ls = 1; ls <= 6; ++ls) {
      const int row = first + ls - 1;
      const size_t a = 6 * (size_t)e + ls - 1;
      const int elemID = SI(row, 3), bc = SI(row, 5);
      if (bc != 0) {
        if (bc < 1 || bc > M.nBCs) throw std::runtime_error("HOPR mesh: BC index out of range");
        const int type = M.BCType[4 * (size_t)(bc - 1)];
        if (type != 1 && type != 100) throw std::runtime_error("HOPR mesh: non-periodic boundary sides are not supported");
      }
      if (conn[a] >= 0) continue;
      if (elemID == 0) throw std::runtime_error("HOPR mesh: boundary sides are not supported");
      if (elemID < 1 || elemID > nE) throw std::runtime_error("HOPR mesh: neighbour element out of range");
      for (int nls = 1; nls <= 6; ++nls) {
        const size_t b = 6 * (size_t)(elemID - 1) + nls - 1;
        if (ind[b] == ind[a]) {
          conn[a] = (int)b;
          conn[b] = (int)a;
          break;
        }
      }
      if (conn[a] < 0) throw std::runtime_error("HOPR mesh: side connection not found");
    }
  }
  int iInner = 0;
  for (size_t a = 0; a < 6 * (size_t)nE; ++a)
    if (sideID[a] == -1) {
      sideID[a] = ++iInner;
      sideID[conn[a]] = iInner;
    }
  C.nSides = iInner;
  C.ElemToSide.assign((size_t)2 * 6 * nE, 0);
  C.SideToElem.assign((size_t)5 * C.nSides, -1);
  for (int e = 0; e < nE; ++e)
    for (int ls = 1; ls <= 6; ++ls) {
      const size_t a = 6 * (size_t)e + ls - 1;
      const int sid = sideID[a];
      C.ElemToSide[0 + 2 * a] = sid;
      C.ElemToSide[1 + 2 * a] = flip[a];
      int* se = &C.SideToElem[5 * (size_t)(sid - 1)];
      if (flip[a] == 0) { se[0] = e + 1; se[2] = ls; }
      else { se[1] = e + 1; se[3] = ls; se[4] = flip[a]; }
    }
  for (int s = 0; s < C.nSides; ++s)
    for (int f = 0; f < 5; ++f)
      if (C.SideToElem[5 * (size_t)s + f] < 0) throw std::runtime_error("HOPR mesh: a side without master or slave");
  // NodeCoords(3,0:NGeo,0:NGeo,0:NGeo,nElems); useCurveds=F keeps the corners (NGeo=1), mesh.f90:233-236 scales
  const int NG = M.NGeo, ng = NG + 1;
  if (M.useCurveds) {
    C.NodeCoords.assign(M.NodeCoords, M.NodeCoords + (size_t)3 * ng * ng * ng * nE);
    C.P.NGeo = NG;
  } else {
    C.NodeCoords.assign((size_t)24 * nE, 0.);
    for (int e = 0; e < nE; ++e)
      for (int k = 0; k < 2; ++k)
        for (int j = 0; j < 2; ++j)
          for (int i = 0; i < 2; ++i)
            for (int d = 0; d < 3; ++d)
              C.NodeCoords[3 * (i + 2 * (j + 2 * (k + 2 * (size_t)e))) + d] =
                  M.NodeCoords[3 * (i * NG + ng * (j * NG + ng * (k * NG + (size_t)ng * e))) + d];
    C.P.NGeo = 1;
  }
  if (std::fabs(M.meshScale - 1.) > 1e-14)
    for (double& x : C.NodeCoords) x *= M.meshScale;
  C.meshNodesGL = M.nodesGL && M.useCurveds;
}

// CalcMetrics (curl form), mesh/metrics.f90:78-333, and CalcSurfMetrics :334-484 (LGL nodes)
void CalcMetrics(Case& C) {
  int N = C.N, n = C.np, NG = C.P.NGeo, ng = NG + 1, NR = 3 * NG, nr = NR + 1;
  size_t nv = (size_t)n * n * n;
  C.Elem_xGP.assign(3 * nv * C.nElems, 0.);
  C.Mf.assign(3 * nv * C.nElems, 0.); C.Mg.assign(3 * nv * C.nElems, 0.); C.Mh.assign(3 * nv * C.nElems, 0.);
  C.sJ.assign(nv * C.nElems, 0.);
  C.NormVec.assign((size_t)3 * n * n * C.nSides, 0.);
  C.TangVec1.assign((size_t)3 * n * n * C.nSides, 0.);
  C.TangVec2.assign((size_t)3 * n * n * C.nSides, 0.);
  C.SurfElem.assign((size_t)n * n * C.nSides, 0.);
  // Vdm_EQNgeo_GLNgeo from the mesh file's OutputNodeType (metrics.f90:147)
  std::vector<double> V_EQ_GL = GetVdm(NG, C.meshNodesGL ? NT_GL : NT_EQUI, NG, NT_GL, false);
  std::vector<double> xGLg(ng), DGLg(ng * ng);
  Nodes(NG, NT_GL, xGLg.data());
  DerivMatrix(NG, xGLg.data(), DGLg.data());
  // solution nodes NodeType (metrics.f90:150-160): the Jacobian goes through NgeoRef points of NodeType
  const NodeType NTS = C.gauss ? NT_GAUSS : NT_GL;
  std::vector<double> V_GLg_Ref = GetVdm(NG, NT_GL, NR, NTS, false);
  std::vector<double> V_Ref_N = GetVdm(NR, NTS, N, NTS, true);
  std::vector<double> V_GLg_GLN = GetVdm(NG, NT_GL, N, NT_GL, false);
  // GetDerivativeMatrix(PP_N, GL): the solution's D for LGL nodes; Gauss nodes keep the metric terms
  // on the LGL points of degree N and interpolate them with Vdm_GLN_N (metrics.f90:325-330)
  std::vector<double> DGLNg, V_GLN_N;
  if (C.gauss) {
    std::vector<double> xGLN(n);
    Nodes(N, NT_GL, xGLN.data());
    DGLNg.resize(n * n);
    DerivMatrix(N, xGLN.data(), DGLNg.data());
    V_GLN_N = GetVdm(N, NT_GL, N, NT_GAUSS, false);
  }
  const std::vector<double>& DGLN = C.gauss ? DGLNg : C.D;
  if (C.gauss) C.SurfMetrics.assign((size_t)3 * n * n * 6 * C.nElems, 0.);
  std::vector<double> XGLg(3 * ng * ng * ng), XGLN(3 * nv), dXg(9 * ng * ng * ng), tmpd(3 * ng * ng * ng),
      tmpo(3 * nr * nr * nr), dXR(9 * nr * nr * nr), detR(nr * nr * nr), detN(nv), dXN(9 * nv), tmpN(3 * nv),
      Rm(9 * nv), Ja(9 * nv);
  for (int e = 0; e < C.nElems; ++e) {
    ChangeBasis3D(3, NG, NG, V_EQ_GL.data(), &C.NodeCoords[3 * (size_t)ng * ng * ng * e], XGLg.data());
    ChangeBasis3D(3, NG, N, V_GLg_GLN.data(), XGLg.data(), XGLN.data());
    if (C.gauss) ChangeBasis3D(3, N, N, V_GLN_N.data(), XGLN.data(), &C.Elem_xGP[3 * nv * e]);
    else
      for (size_t z = 0; z < 3 * nv; ++z) C.Elem_xGP[3 * nv * e + z] = XGLN[z];
    // dXGL_Ngeo(dd,nn,i,j,k): index dd + 3*nn + 9*node
    std::fill(dXg.begin(), dXg.end(), 0.);
    for (int k = 0; k < ng; ++k)
      for (int j = 0; j < ng; ++j)
        for (int i = 0; i < ng; ++i) {
          double* d = &dXg[9 * (i + ng * (j + ng * k))];
          for (int ll = 0; ll < ng; ++ll)
            for (int nn = 0; nn < 3; ++nn) {
              d[0 + 3 * nn] += DGLg[i + ng * ll] * XGLg[nn + 3 * (ll + ng * (j + ng * k))];
              d[1 + 3 * nn] += DGLg[j + ng * ll] * XGLg[nn + 3 * (i + ng * (ll + ng * k))];
              d[2 + 3 * nn] += DGLg[k + ng * ll] * XGLg[nn + 3 * (i + ng * (j + ng * ll))];
            }
        }
    // dX_NgeoRef(:,nn) = ChangeBasis3D(dXGL_NGeo(:,nn))
    for (int nn = 0; nn < 3; ++nn) {
      for (int z = 0; z < ng * ng * ng; ++z)
        for (int dd = 0; dd < 3; ++dd) tmpd[dd + 3 * z] = dXg[dd + 3 * nn + 9 * z];
      ChangeBasis3D(3, NG, NR, V_GLg_Ref.data(), tmpd.data(), tmpo.data());
      for (int z = 0; z < nr * nr * nr; ++z)
        for (int dd = 0; dd < 3; ++dd) dXR[dd + 3 * nn + 9 * z] = tmpo[dd + 3 * z];
    }
    for (int z = 0; z < nr * nr * nr; ++z) {
      const double* X = &dXR[9 * z];
#define DX(a, b) X[((a)-1) + 3 * ((b)-1)]
      detR[z] = 0. + DX(1, 1) * (DX(2, 2) * DX(3, 3) - DX(3, 2) * DX(2, 3)) +
                DX(2, 1) * (DX(3, 2) * DX(1, 3) - DX(1, 2) * DX(3, 3)) +
                DX(3, 1) * (DX(1, 2) * DX(2, 3) - DX(2, 2) * DX(1, 3));
#undef DX
    }
    ChangeBasis3D(1, NR, N, V_Ref_N.data(), detR.data(), detN.data());
    for (size_t z = 0; z < nv; ++z) C.sJ[nv * e + z] = 1. / detN[z];
    // dXGL_N
    if (N >= NG) {
      for (int nn = 0; nn < 3; ++nn) {
        for (int z = 0; z < ng * ng * ng; ++z)
          for (int dd = 0; dd < 3; ++dd) tmpd[dd + 3 * z] = dXg[dd + 3 * nn + 9 * z];
        ChangeBasis3D(3, NG, N, V_GLg_GLN.data(), tmpd.data(), tmpN.data());
        for (size_t z = 0; z < nv; ++z)
          for (int dd = 0; dd < 3; ++dd) dXN[dd + 3 * nn + 9 * z] = tmpN[dd + 3 * z];
      }
    } else {
      std::fill(dXN.begin(), dXN.end(), 0.);
      for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
          for (int i = 0; i < n; ++i) {
            double* d = &dXN[9 * (i + n * (j + n * k))];
            for (int ll = 0; ll < n; ++ll)
              for (int nn = 0; nn < 3; ++nn) {
                d[0 + 3 * nn] += DGLN[i + n * ll] * XGLN[nn + 3 * (ll + n * (j + n * k))];
                d[1 + 3 * nn] += DGLN[j + n * ll] * XGLN[nn + 3 * (i + n * (ll + n * k))];
                d[2 + 3 * nn] += DGLN[k + n * ll] * XGLN[nn + 3 * (i + n * (j + n * ll))];
              }
          }
    }
    // curl form: R_GL_N(dd,nn): index dd + 3*nn + 9*node
    for (size_t z = 0; z < nv; ++z) {
      const double* X = &XGLN[3 * z];
      const double* d = &dXN[9 * z];
      for (int dd = 0; dd < 3; ++dd) {
        Rm[dd + 0 + 9 * z] = 0.5 * (X[2] * d[dd + 3 * 1] - X[1] * d[dd + 3 * 2]);
        Rm[dd + 3 + 9 * z] = 0.5 * (X[0] * d[dd + 3 * 2] - X[2] * d[dd + 3 * 0]);
        Rm[dd + 6 + 9 * z] = 0.5 * (X[1] * d[dd + 3 * 0] - X[0] * d[dd + 3 * 1]);
      }
    }
    std::fill(Ja.begin(), Ja.end(), 0.);
    auto RR = [&](int dd, int nn, int i, int j, int k) { return Rm[dd + 3 * nn + 9 * (i + n * (j + n * k))]; };
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          double* J = &Ja[9 * (i + n * (j + n * k))];  // J[dd + 3*nn]
          for (int q = 0; q < n; ++q)
            for (int nn = 0; nn < 3; ++nn) {
              J[0 + 3 * nn] = J[0 + 3 * nn] - DGLN[j + n * q] * RR(2, nn, i, q, k);
              J[1 + 3 * nn] = J[1 + 3 * nn] - DGLN[k + n * q] * RR(0, nn, i, j, q);
              J[2 + 3 * nn] = J[2 + 3 * nn] - DGLN[i + n * q] * RR(1, nn, q, j, k);
            }
          for (int q = 0; q < n; ++q)
            for (int nn = 0; nn < 3; ++nn) {
              J[0 + 3 * nn] = J[0 + 3 * nn] + DGLN[k + n * q] * RR(1, nn, i, j, q);
              J[1 + 3 * nn] = J[1 + 3 * nn] + DGLN[i + n * q] * RR(2, nn, q, j, k);
              J[2 + 3 * nn] = J[2 + 3 * nn] + DGLN[j + n * q] * RR(0, nn, i, q, k);
            }
        }
    if (C.gauss) {  // ChangeBasis3D(Vdm_GLN_N) of each metric vector, metrics.f90:325-327
      std::vector<double> tin(3 * nv), tout(3 * nv);
      double* M[3] = {&C.Mf[3 * nv * e], &C.Mg[3 * nv * e], &C.Mh[3 * nv * e]};
      for (int dd = 0; dd < 3; ++dd) {
        for (size_t z = 0; z < nv; ++z)
          for (int nn = 0; nn < 3; ++nn) tin[nn + 3 * z] = Ja[dd + 3 * nn + 9 * z];
        ChangeBasis3D(3, N, N, V_GLN_N.data(), tin.data(), M[dd]);
      }
    } else {
      for (size_t z = 0; z < nv; ++z)
        for (int nn = 0; nn < 3; ++nn) {
          C.Mf[3 * (nv * e + z) + nn] = Ja[0 + 3 * nn + 9 * z];
          C.Mg[3 * (nv * e + z) + nn] = Ja[1 + 3 * nn + 9 * z];
          C.Mh[3 * (nv * e + z) + nn] = Ja[2 + 3 * nn + 9 * z];
        }
    }
    // CalcSurfMetrics (metrics.f90:334-440): Ja of the LGL points on the side, interpolated to the side's
    // solution points (ChangeBasis2D with Vdm_GLN_N; identity for LGL).  LGL: master sides only; Gauss:
    // SurfMetrics of every side in the master's point order (FS2M), face vectors of the master sides.
    std::vector<double> JaF(9 * n * n);  // JaF[dd + 3*nn + 9*(a + n*b)]: face slice in volume index order
    for (int s = 1; s <= 6; ++s) {
      int SideID = C.ElemToSide[0 + 2 * ((s - 1) + 6 * (size_t)e)];
      int flip = C.ElemToSide[1 + 2 * ((s - 1) + 6 * (size_t)e)];
      if (flip != 0 && !C.gauss) continue;
      int nd = NormalDirs[s] - 1, td = TangDirs[s] - 1;
      double sign = NormalSigns[s];
      if (C.gauss) {
        std::vector<double> sl(9 * n * n, 0.), b1(9 * n * n, 0.);
        for (int b = 0; b < n; ++b)
          for (int a = 0; a < n; ++a) {
            int i, j, k;
            switch (s) {
              case XI_MINUS: i = 0; j = a; k = b; break;
              case XI_PLUS: i = N; j = a; k = b; break;
              case ETA_MINUS: i = a; j = 0; k = b; break;
              case ETA_PLUS: i = a; j = N; k = b; break;
              case ZETA_MINUS: i = a; j = b; k = 0; break;
              default: i = a; j = b; k = N; break;
            }
            for (int c = 0; c < 9; ++c) sl[c + 9 * (a + n * b)] = Ja[c + 9 * (i + n * (j + n * k))];
          }
        for (int b = 0; b < n; ++b)  // ChangeBasis2D: first index, then second
          for (int ao = 0; ao < n; ++ao)
            for (int a = 0; a < n; ++a)
              for (int c = 0; c < 9; ++c) b1[c + 9 * (ao + n * b)] += V_GLN_N[ao + n * a] * sl[c + 9 * (a + n * b)];
        std::fill(JaF.begin(), JaF.end(), 0.);
        for (int bo = 0; bo < n; ++bo)
          for (int b = 0; b < n; ++b)
            for (int a = 0; a < n; ++a)
              for (int c = 0; c < 9; ++c) JaF[c + 9 * (a + n * bo)] += V_GLN_N[bo + n * b] * b1[c + 9 * (a + n * b)];
        for (int q = 0; q < n; ++q)
          for (int p = 0; p < n; ++p) {
            int a, b, pm, qm;
            CGNS_SideToVol2(N, p, q, s, a, b);
            Flip_S2M(N, p, q, flip, pm, qm);
            const double* J = &JaF[9 * (a + n * b)];
            double* SM = &C.SurfMetrics[3 * ((size_t)pm + n * ((size_t)qm + n * ((size_t)(s - 1) + 6 * (size_t)e)))];
            for (int c = 0; c < 3; ++c) SM[c] = J[nd + 3 * c];
          }
        if (flip != 0) continue;
      }
      for (int q = 0; q < n; ++q)
        for (int p = 0; p < n; ++p) {
          int a, b;
          CGNS_SideToVol2(N, p, q, s, a, b);
          int i, j, k;
          switch (s) {
            case XI_MINUS: i = 0; j = a; k = b; break;
            case XI_PLUS: i = N; j = a; k = b; break;
            case ETA_MINUS: i = a; j = 0; k = b; break;
            case ETA_PLUS: i = a; j = N; k = b; break;
            case ZETA_MINUS: i = a; j = b; k = 0; break;
            default: i = a; j = b; k = N; break;
          }
          const double* J = C.gauss ? &JaF[9 * (a + n * b)] : &Ja[9 * (i + n * (j + n * k))];
          double jn[3] = {J[nd + 0], J[nd + 3], J[nd + 6]};
          double jt[3] = {J[td + 0], J[td + 3], J[td + 6]};
          size_t fi = (size_t)p + n * ((size_t)q + (size_t)n * (SideID - 1));
          double se = std::sqrt(jn[0] * jn[0] + jn[1] * jn[1] + jn[2] * jn[2]);
          double nvv[3], t1[3], t2[3];
          for (int d = 0; d < 3; ++d) nvv[d] = sign * jn[d] / se;
          double dot = jt[0] * nvv[0] + jt[1] * nvv[1] + jt[2] * nvv[2];
          for (int d = 0; d < 3; ++d) t1[d] = jt[d] - dot * nvv[d];
          double tn = std::sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
          for (int d = 0; d < 3; ++d) t1[d] = t1[d] / tn;
          t2[0] = nvv[1] * t1[2] - nvv[2] * t1[1];  // CROSS, globals.f90
          t2[1] = nvv[2] * t1[0] - nvv[0] * t1[2];
          t2[2] = nvv[0] * t1[1] - nvv[1] * t1[0];
          C.SurfElem[fi] = se;
          for (int d = 0; d < 3; ++d) {
            C.NormVec[3 * fi + d] = nvv[d];
            C.TangVec1[3 * fi + d] = t1[d];
            C.TangVec2[3 * fi + d] = t2[d];
          }
        }
    }
  }
}

void InitEquationAndTime(Case& C) {
  const orc_params& P = C.P;
  C.kappa = P.kappa; C.sKappa = 1. / C.kappa; C.kappaM1 = C.kappa - 1.; C.sKappaM1 = 1. / C.kappaM1;
  C.kappaP1 = C.kappa + 1.; C.sKappaP1 = 1. / C.kappaP1; C.R = P.R; C.s23 = 2. / 3.;
  C.Pr = P.Pr; C.KappasPr = C.kappa / C.Pr;
  C.mu0 = P.mu0; C.etaBR2 = P.etaBR2;
  if (C.mhd) {  // mhd/equation.f90:178-209 (mu is the constant MHD viscosity, PP_VISC unused)
    C.kappaM2 = C.kappa - 2.;
    C.mu_0 = P.mu_0; C.smu_0 = 1. / C.mu_0; C.s2mu_0 = 0.5 * C.smu_0;
    C.eta = C.parabolic ? P.eta : 0.; C.etasmu_0 = C.eta * C.smu_0;
    C.muMHD = C.parabolic ? P.mu0 : 0.;
    C.GLM_scale = P.glm_scale; C.GLM_scr = P.glm_scr; C.GLM_ch = P.glm_ch;
    C.noncons = P.noncons; C.ncGLM = (P.noncons != 0 && P.nc_glm != 0);
    if (P.riemann == 5 && std::fabs(C.mu_0 - 1.) > 1.0e-12)  // mhd/equation.f90:343-346
      throw std::runtime_error("HLLD solver only for mu_0=1 implemented");
  } else if (P.visc == 1) {  // equation.f90:226-233
    C.Ts = P.Ts; C.sTref = 1. / P.Tref; C.ExpoSuth = P.ExpoSuth;
    C.Ts = C.Ts * C.sTref;
    C.cSuth = std::pow(C.Ts, C.ExpoSuth) * (1 + C.Ts) / (2 * C.Ts * C.Ts);
  } else if (P.visc == 2) {
    C.ExpoPow = P.ExpoPow;
    C.mu0 = P.mu0 / std::pow(P.Tref, C.ExpoPow);
  }
  C.doCalcSource = (P.ini_exact_func == 4);
  // timedisc_vars.f90:94-726
  double cflAlpha[15];
  double relDFL = 1.;
  if (P.time_disc < 0 || P.time_disc > 9) throw std::runtime_error("time disc not implemented in oracle");
  C.rk = &kOrcRKTables[P.time_disc];  // SetTimeDiscCoefs, timedisc_vars.f90:94-726
  C.nRKStages = C.rk->nStages;
  if (C.gauss) std::copy(kOrcGaussCflAlpha[P.time_disc], kOrcGaussCflAlpha[P.time_disc] + 15, cflAlpha);
  else std::copy(C.rk->cflAlpha, C.rk->cflAlpha + 15, cflAlpha);
  relDFL = C.rk->relativeDFL;
  C.RKA.assign(C.rk->A, C.rk->A + C.nRKStages + 1);
  C.RKb.assign(C.rk->b, C.rk->b + C.nRKStages + 1);
  C.RKc.assign(C.rk->c, C.rk->c + C.nRKStages + 1);
  // FillCFL_DFL, timedisc.f90:697-741
  int N = C.N;
  double alpha = cflAlpha[std::min(15, N) - 1];
  C.CFLScale = P.cfl_scale * alpha / (2. * N + 1.);
  double dflAlpha[10] = {4.50, 1.95, 1.18, 0.79, 0.56, 0.42, 0.32, 0.25, 0.20, 0.17};
  if (C.gauss) std::copy(kOrcGaussDflAlpha, kOrcGaussDflAlpha + 10, dflAlpha);
  double alphaD = dflAlpha[std::min(10, N) - 1] * relDFL;
  C.DFLScale = P.dfl_scale * alphaD / ((2. * N + 1.) * (2. * N + 1.));
}

// ----------------------------------------------------------------------------------------------
// DG operator, dg/dg.f90:282-452
// ----------------------------------------------------------------------------------------------
// ProlongToFace, interpolation/prolongtoface.f90:43-132: LGL copies the side's node, Gauss interpolates
// along the line with L_Minus (Uface = U(l=0) L_Minus(0) + sum_{l>=1} U(l) L_Minus(l), l counted from the side)
void ProlongToFace(Case& C, const std::vector<real>& Uvol, std::vector<real>& Um, std::vector<real>& Us) {
  int n = C.np;
  if (C.gauss) {
    const int NV = C.nVar;
    for (int sid = 0; sid < C.nSides; ++sid)
      for (int side = 0; side < 2; ++side) {
        const int e = C.SideToElem[side + 5 * sid];
        if (e == -1) continue;
        const int ls = C.SideToElem[2 + side + 5 * sid], fl = side ? C.SideToElem[4 + 5 * sid] : 0;
        std::vector<real>& F = side ? Us : Um;
        for (int q = 0; q < n; ++q)
          for (int p = 0; p < n; ++p)
            for (int v = 0; v < NV; ++v) {
              auto at = [&](int l) {
                return Uvol[C.vol(v, C.s2v(l, p, q, fl, ls, 0), C.s2v(l, p, q, fl, ls, 1), C.s2v(l, p, q, fl, ls, 2), e - 1)];
              };
              real acc = at(0) * C.Lminus[0];
              for (int l = 1; l < n; ++l) acc = acc + at(l) * C.Lminus[l];
              F[C.fac(v, p, q, sid)] = acc;
            }
      }
    return;
  }
  for (int sid = 0; sid < C.nSides; ++sid) {
    int e = C.SideToElem[0 + 5 * sid];
    if (e != -1) {
      int ls = C.SideToElem[2 + 5 * sid];
      for (int q = 0; q < n; ++q)
        for (int p = 0; p < n; ++p)
          for (int v = 0; v < C.nVar; ++v)
            Um[C.fac(v, p, q, sid)] =
                Uvol[C.vol(v, C.s2v(0, p, q, 0, ls, 0), C.s2v(0, p, q, 0, ls, 1), C.s2v(0, p, q, 0, ls, 2), e - 1)];
    }
    int nb = C.SideToElem[1 + 5 * sid];
    if (nb != -1) {
      int nls = C.SideToElem[3 + 5 * sid], fl = C.SideToElem[4 + 5 * sid];
      for (int q = 0; q < n; ++q)
        for (int p = 0; p < n; ++p)
          for (int v = 0; v < C.nVar; ++v)
            Us[C.fac(v, p, q, sid)] = Uvol[C.vol(v, C.s2v(0, p, q, fl, nls, 0), C.s2v(0, p, q, fl, nls, 1),
                                                 C.s2v(0, p, q, fl, nls, 2), nb - 1)];
    }
  }
}

// VolInt_SplitForm + EvalAdvFluxAverage3D, dg/volint.f90:173-218, flux_average.f90:198-269
void VolIntSplitForm(Case& C) {
  int n = C.np, N = C.N;
  size_t nv = (size_t)n * n * n;
#pragma omp parallel
  {
  const int NV = C.nVar, NA = C.nAux;
  std::vector<real> aux(NA * nv), ft((size_t)NV * n * nv), gt((size_t)NV * n * nv), ht((size_t)NV * n * nv);
  std::vector<real> mf(3 * nv), mg(3 * nv), mh(3 * nv);  // the element's metrics (copies)
  auto F4 = [&](std::vector<real>& A, int v, int l, int i, int j, int k) -> real& {
    return A[v + NV * ((size_t)l + n * ((size_t)i + n * ((size_t)j + (size_t)n * k)))];
  };
#pragma omp for schedule(static)
  for (int e = 0; e < C.nElems; ++e) {
    for (size_t z = 0; z < nv; ++z) Uaux(C, &C.U[NV * (nv * e + z)], &aux[NA * z]);
    for (size_t z = 0; z < 3 * nv; ++z) {
      mf[z] = C.Mf[3 * nv * e + z]; mg[z] = C.Mg[3 * nv * e + z]; mh[z] = C.Mh[3 * nv * e + z];
    }
    auto Up = [&](int i, int j, int k) { return &C.U[C.vol(0, i, j, k, e)]; };
    auto Ap = [&](int i, int j, int k) { return &aux[NA * (i + n * (j + n * k))]; };
    auto Mfp = [&](int i, int j, int k) { return &mf[3 * (i + n * (j + n * k))]; };
    auto Mgp = [&](int i, int j, int k) { return &mg[3 * (i + n * (j + n * k))]; };
    auto Mhp = [&](int i, int j, int k) { return &mh[3 * (i + n * (j + n * k))]; };
    auto Flux = [&](const real* UL, const real* UR, const real* aL, const real* aR, const real* mL, const real* mR,
                    real* F) {
      if (C.mhd) MHD_VolumeFluxVec(C, C.P.volume_flux, UL, UR, aL, aR, mL, mR, F);
      else VolumeFluxVec(C, UL, UR, aL, aR, mL, mR, F);
    };
    real F[NVMAX];
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          for (int v = 0; v < NV; ++v) F4(ft, v, i, i, j, k) = 0.;
          for (int l = i + 1; l <= N; ++l) {
            Flux(Up(i, j, k), Up(l, j, k), Ap(i, j, k), Ap(l, j, k), Mfp(i, j, k), Mfp(l, j, k), F);
            for (int v = 0; v < NV; ++v) { F4(ft, v, l, i, j, k) = F[v]; F4(ft, v, i, l, j, k) = F[v]; }
          }
        }
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          for (int v = 0; v < NV; ++v) F4(gt, v, j, i, j, k) = 0.;
          for (int l = j + 1; l <= N; ++l) {
            Flux(Up(i, j, k), Up(i, l, k), Ap(i, j, k), Ap(i, l, k), Mgp(i, j, k), Mgp(i, l, k), F);
            for (int v = 0; v < NV; ++v) { F4(gt, v, l, i, j, k) = F[v]; F4(gt, v, j, i, l, k) = F[v]; }
          }
        }
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          for (int v = 0; v < NV; ++v) F4(ht, v, k, i, j, k) = 0.;
          for (int l = k + 1; l <= N; ++l) {
            Flux(Up(i, j, k), Up(i, j, l), Ap(i, j, k), Ap(i, j, l), Mhp(i, j, k), Mhp(i, j, l), F);
            for (int v = 0; v < NV; ++v) { F4(ht, v, l, i, j, k) = F[v]; F4(ht, v, k, i, j, l) = F[v]; }
          }
        }
    if (C.mhd && C.noncons) {  // AddNonConsFluxTilde3D, mhd/flux_average.f90:268-366
      for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
          for (int i = 0; i < n; ++i) {
            const real* Ui = Up(i, j, k);
            const real* ai = Ap(i, j, k);
            for (int l = 0; l < n; ++l) MHD_NonConsPair(C, Ui, ai, Up(l, j, k), Mfp(i, j, k), Mfp(l, j, k), &F4(ft, 0, l, i, j, k));
            for (int l = 0; l < n; ++l) MHD_NonConsPair(C, Ui, ai, Up(i, l, k), Mgp(i, j, k), Mgp(i, l, k), &F4(gt, 0, l, i, j, k));
            for (int l = 0; l < n; ++l) MHD_NonConsPair(C, Ui, ai, Up(i, j, l), Mhp(i, j, k), Mhp(i, j, l), &F4(ht, 0, l, i, j, k));
          }
    }
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
          for (int l = 0; l < n; ++l)
            for (int v = 0; v < NV; ++v)
              C.Ut[C.vol(v, i, j, k, e)] = C.Ut[C.vol(v, i, j, k, e)] + C.Dvolsurf_T[l + n * i] * F4(ft, v, l, i, j, k) +
                                           C.Dvolsurf_T[l + n * j] * F4(gt, v, l, i, j, k) +
                                           C.Dvolsurf_T[l + n * k] * F4(ht, v, l, i, j, k);
  }
  }
}

// VolInt_visc + EvalDiffFluxTilde3D, dg/volint.f90:228-271, navierstokes/flux.f90:523-635
void VolIntVisc(Case& C) {
  int n = C.np;
  size_t nv = (size_t)n * n * n;
#pragma omp parallel
  {
  const int NV = C.nVar;
  std::vector<real> ft(NV * nv), gt(NV * nv), ht(NV * nv);
#pragma omp for schedule(static)
  for (int e = 0; e < C.nElems; ++e) {
    for (size_t z = 0; z < nv; ++z) {
      size_t o = nv * e + z;
      real f[NVMAX], g[NVMAX], h[NVMAX];
      DiffFlux(C, &C.U[NV * o], &C.gx[NV * o], &C.gy[NV * o], &C.gz[NV * o], f, g, h);
      const double* mf = &C.Mf[3 * o];
      const double* mg = &C.Mg[3 * o];
      const double* mh = &C.Mh[3 * o];
      for (int v = 0; v < NV; ++v) {
        ft[NV * z + v] = f[v] * mf[0] + g[v] * mf[1] + h[v] * mf[2];
        gt[NV * z + v] = f[v] * mg[0] + g[v] * mg[1] + h[v] * mg[2];
        ht[NV * z + v] = f[v] * mh[0] + g[v] * mh[1] + h[v] * mh[2];
      }
    }
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
          for (int l = 0; l < n; ++l)
            for (int v = 0; v < NV; ++v)
              C.Ut[C.vol(v, i, j, k, e)] = C.Ut[C.vol(v, i, j, k, e)] +
                                           C.Dhat_T[l + n * i] * ft[NV * (l + n * (j + n * k)) + v] +
                                           C.Dhat_T[l + n * j] * gt[NV * (i + n * (l + n * k)) + v] +
                                           C.Dhat_T[l + n * k] * ht[NV * (i + n * (j + n * l)) + v];
  }
  }
}

// Lifting (BR1 br1.f90:154-364, BR2 br2.f90:167-308) for LGL nodes
void Lifting(Case& C) {
  int n = C.np;
  size_t nv = (size_t)n * n * n;
  size_t nt = (size_t)C.nVar * nv * C.nElems;
  std::fill(C.gx.begin(), C.gx.end(), 0.);
  std::fill(C.gy.begin(), C.gy.end(), 0.);
  std::fill(C.gz.begin(), C.gz.end(), 0.);
  bool br2 = (C.P.lifting == 2);
  const int NV = C.nVar;
  // Lifting_FillFlux (br1_fillflux.f90:49-91) with EvalLiftingSurfFlux (flux.f90:677-716)
  for (int sid = 0; sid < C.nSides; ++sid)
    for (int q = 0; q < n; ++q)
      for (int p = 0; p < n; ++p) {
        real Fm[NVMAX], Fs[NVMAX];
        LiftVar(C, &C.Umaster[C.fac(0, p, q, sid)], Fm);
        LiftVar(C, &C.Uslave[C.fac(0, p, q, sid)], Fs);
        size_t fi = (size_t)p + n * ((size_t)q + (size_t)n * sid);
        for (int v = 0; v < NV; ++v) {
          real Fl = 0.5 * (Fs[v] - Fm[v]) * C.SurfElem[fi];
          C.FX[C.fac(v, p, q, sid)] = Fl * C.NormVec[3 * fi + 0];
          C.FY[C.fac(v, p, q, sid)] = Fl * C.NormVec[3 * fi + 1];
          C.FZ[C.fac(v, p, q, sid)] = Fl * C.NormVec[3 * fi + 2];
        }
      }
  // Lifting_VolInt: br1_volint.f90:45-98 (BR1) / br2_volint.f90:45-103 (BR2 includes sJ)
#pragma omp parallel
  {
  std::vector<real> Fl(NV * nv);
#pragma omp for schedule(static)
  for (int e = 0; e < C.nElems; ++e) {
    for (size_t z = 0; z < nv; ++z) LiftVar(C, &C.U[NV * (nv * e + z)], &Fl[NV * z]);
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          real gxi[NVMAX], geta[NVMAX], gzeta[NVMAX];
          for (int v = 0; v < NV; ++v) {
            gxi[v] = C.D_T[0 + n * i] * Fl[NV * (0 + n * (j + n * k)) + v];
            geta[v] = C.D_T[0 + n * j] * Fl[NV * (i + n * (0 + n * k)) + v];
            gzeta[v] = C.D_T[0 + n * k] * Fl[NV * (i + n * (j + n * 0)) + v];
          }
          for (int l = 1; l < n; ++l)
            for (int v = 0; v < NV; ++v) {
              gxi[v] = gxi[v] + C.D_T[l + n * i] * Fl[NV * (l + n * (j + n * k)) + v];
              geta[v] = geta[v] + C.D_T[l + n * j] * Fl[NV * (i + n * (l + n * k)) + v];
              gzeta[v] = gzeta[v] + C.D_T[l + n * k] * Fl[NV * (i + n * (j + n * l)) + v];
            }
          size_t o = C.nod(i, j, k, e);
          const double* mf = &C.Mf[3 * o];
          const double* mg = &C.Mg[3 * o];
          const double* mh = &C.Mh[3 * o];
          for (int v = 0; v < NV; ++v) {
            real ax = mf[0] * gxi[v] + mg[0] * geta[v] + mh[0] * gzeta[v];
            real ay = mf[1] * gxi[v] + mg[1] * geta[v] + mh[1] * gzeta[v];
            real az = mf[2] * gxi[v] + mg[2] * geta[v] + mh[2] * gzeta[v];
            if (br2) { ax = ax * C.sJ[o]; ay = ay * C.sJ[o]; az = az * C.sJ[o]; }
            C.gx[NV * o + v] = C.gx[NV * o + v] + ax;
            C.gy[NV * o + v] = C.gy[NV * o + v] + ay;
            C.gz[NV * o + v] = C.gz[NV * o + v] + az;
          }
        }
  }
  }
  if (!br2) {
    // BR1_SurfInt (br1_surfint.f90:52-131), then Jacobian, ConvertToGradPrim, prolong
    std::vector<real>* G[3] = {&C.gx, &C.gy, &C.gz};
    std::vector<real>* FF[3] = {&C.FX, &C.FY, &C.FZ};
    std::vector<real>* GM[3] = {&C.gxm, &C.gym, &C.gzm};
    std::vector<real>* GS[3] = {&C.gxs, &C.gys, &C.gzs};
    for (int d = 0; d < 3; ++d) {
      std::vector<real>& g = *G[d];
      std::vector<real>& F = *FF[d];
      // LGL: the side's node with L_HatMinus0; Gauss: every node of the line with L_HatMinus(l)
      const int nl = C.gauss ? n : 1;
      for (int sid = 0; sid < C.nSides; ++sid) {
        int e = C.SideToElem[0 + 5 * sid];
        if (e != -1) {
          int ls = C.SideToElem[2 + 5 * sid];
          for (int q = 0; q < n; ++q)
            for (int p = 0; p < n; ++p)
              for (int l = 0; l < nl; ++l)
                for (int v = 0; v < NV; ++v) {
                  size_t idx = C.vol(v, C.s2v(l, p, q, 0, ls, 0), C.s2v(l, p, q, 0, ls, 1), C.s2v(l, p, q, 0, ls, 2), e - 1);
                  g[idx] = g[idx] + F[C.fac(v, p, q, sid)] * (C.gauss ? C.LhatMinus[l] : C.L_HatMinus0);
                }
        }
        int nb = C.SideToElem[1 + 5 * sid];
        if (nb != -1) {
          int nls = C.SideToElem[3 + 5 * sid], fl = C.SideToElem[4 + 5 * sid];
          for (int q = 0; q < n; ++q)
            for (int p = 0; p < n; ++p)
              for (int l = 0; l < nl; ++l)
                for (int v = 0; v < NV; ++v) {
                  size_t idx = C.vol(v, C.s2v(l, p, q, fl, nls, 0), C.s2v(l, p, q, fl, nls, 1),
                                     C.s2v(l, p, q, fl, nls, 2), nb - 1);
                  g[idx] = g[idx] + F[C.fac(v, p, q, sid)] * (C.gauss ? C.LhatMinus[l] : C.L_HatMinus0);
                }
        }
      }
      for (size_t z = 0; z < nt / NV; ++z)
        for (int v = 0; v < NV; ++v) g[NV * z + v] = g[NV * z + v] * C.sJ[z];
      if (C.gauss) {  // br1.f90:318-350: prolong the lifting-variable gradient, then convert with U and the face U
        ProlongToFace(C, g, *GM[d], *GS[d]);
        for (size_t z = 0; z < nt / NV; ++z) GradPrim(C, &C.U[NV * z], &g[NV * z]);
        size_t nf = (size_t)n * n * C.nSides;
        for (size_t z = 0; z < nf; ++z) {
          GradPrim(C, &C.Umaster[NV * z], &(*GM[d])[NV * z]);
          GradPrim(C, &C.Uslave[NV * z], &(*GS[d])[NV * z]);
        }
      } else {
        for (size_t z = 0; z < nt / NV; ++z) GradPrim(C, &C.U[NV * z], &g[NV * z]);
        ProlongToFace(C, g, *GM[d], *GS[d]);
      }
    }
  } else {
    // BR2: prolong the volume gradient, then BR2_SurfInt (br2_surfint.f90:53-148) adds the
    // surface part to the volume (with sJ) and eta_BR2 times it to the face gradients
    std::vector<real>* G[3] = {&C.gx, &C.gy, &C.gz};
    std::vector<real>* FF[3] = {&C.FX, &C.FY, &C.FZ};
    std::vector<real>* GM[3] = {&C.gxm, &C.gym, &C.gzm};
    std::vector<real>* GS[3] = {&C.gxs, &C.gys, &C.gzs};
    for (int d = 0; d < 3; ++d) ProlongToFace(C, *G[d], *GM[d], *GS[d]);
    for (int d = 0; d < 3; ++d) {
      std::vector<real>& g = *G[d];
      std::vector<real>& F = *FF[d];
      std::vector<real>& gm = *GM[d];
      std::vector<real>& gs = *GS[d];
      // LGL: the side's node; Gauss: every node of the line (br2_surfint.f90:109-115, 131-137), the face
      // gradient taking etaBR2 L_Minus(l) F_loc
      const int nl = C.gauss ? n : 1;
      for (int sid = 0; sid < C.nSides; ++sid) {
        int e = C.SideToElem[0 + 5 * sid];
        if (e != -1) {
          int ls = C.SideToElem[2 + 5 * sid];
          for (int q = 0; q < n; ++q)
            for (int p = 0; p < n; ++p)
              for (int l = 0; l < nl; ++l) {
                size_t o = C.nod(C.s2v(l, p, q, 0, ls, 0), C.s2v(l, p, q, 0, ls, 1), C.s2v(l, p, q, 0, ls, 2), e - 1);
                for (int v = 0; v < NV; ++v) {
                  real Floc = C.sJ[o] * (C.gauss ? C.LhatMinus[l] : C.L_HatMinus0) * F[C.fac(v, p, q, sid)];
                  g[NV * o + v] = g[NV * o + v] + Floc;
                  if (C.gauss) gm[C.fac(v, p, q, sid)] = gm[C.fac(v, p, q, sid)] + C.etaBR2 * C.Lminus[l] * Floc;
                  else gm[C.fac(v, p, q, sid)] = gm[C.fac(v, p, q, sid)] + C.etaBR2 * Floc;
                }
              }
        }
        int nb = C.SideToElem[1 + 5 * sid];
        if (nb != -1) {
          int nls = C.SideToElem[3 + 5 * sid], fl = C.SideToElem[4 + 5 * sid];
          for (int q = 0; q < n; ++q)
            for (int p = 0; p < n; ++p)
              for (int l = 0; l < nl; ++l) {
                size_t o = C.nod(C.s2v(l, p, q, fl, nls, 0), C.s2v(l, p, q, fl, nls, 1), C.s2v(l, p, q, fl, nls, 2), nb - 1);
                for (int v = 0; v < NV; ++v) {
                  real Floc = C.sJ[o] * (C.gauss ? C.LhatMinus[l] : C.L_HatMinus0) * F[C.fac(v, p, q, sid)];
                  g[NV * o + v] = g[NV * o + v] + Floc;
                  if (C.gauss) gs[C.fac(v, p, q, sid)] = gs[C.fac(v, p, q, sid)] + C.etaBR2 * C.Lminus[l] * Floc;
                  else gs[C.fac(v, p, q, sid)] = gs[C.fac(v, p, q, sid)] + C.etaBR2 * Floc;
                }
              }
        }
      }
      for (size_t z = 0; z < nt / NV; ++z) GradPrim(C, &C.U[NV * z], &g[NV * z]);
      size_t nf = (size_t)n * n * C.nSides;
      for (size_t z = 0; z < nf; ++z) {
        GradPrim(C, &C.Umaster[NV * z], &gm[NV * z]);
        GradPrim(C, &C.Uslave[NV * z], &gs[NV * z]);
      }
    }
  }
}

// FillFlux, dg/fillflux.f90:41-110 with Riemann (riemann.f90:104-169)
void FillFlux(Case& C) {
  int n = C.np, npts = n * n;
#pragma omp parallel
  {
  const int NV = C.nVar;
  std::vector<real> ULL(NV * npts), URR(NV * npts), F(NV * npts), FS(NV * npts);
  // RotateState (navierstokes/riemann.f90:218-231, mhd/riemann.f90:185-200: also B)
  auto rotate = [&](const real* U, const double* nv, const double* t1, const double* t2, real* R) {
    for (int v = 0; v < NV; ++v) R[v] = U[v];
    R[1] = U[1] * nv[0] + U[2] * nv[1] + U[3] * nv[2];
    R[2] = U[1] * t1[0] + U[2] * t1[1] + U[3] * t1[2];
    R[3] = U[1] * t2[0] + U[2] * t2[1] + U[3] * t2[2];
    if (C.mhd) {
      R[5] = U[5] * nv[0] + U[6] * nv[1] + U[7] * nv[2];
      R[6] = U[5] * t1[0] + U[6] * t1[1] + U[7] * t1[2];
      R[7] = U[5] * t2[0] + U[6] * t2[1] + U[7] * t2[2];
    }
  };
#pragma omp for schedule(static)
  for (int sid = 0; sid < C.nSides; ++sid) {
    for (int z = 0; z < npts; ++z) {
      size_t fi = (size_t)npts * sid + z;
      const double* nv = &C.NormVec[3 * fi];
      const double* t1 = &C.TangVec1[3 * fi];
      const double* t2 = &C.TangVec2[3 * fi];
      rotate(&C.Umaster[NV * fi], nv, t1, t2, &ULL[NV * z]);
      rotate(&C.Uslave[NV * fi], nv, t1, t2, &URR[NV * z]);
    }
    if (C.mhd) {
      for (int z = 0; z < npts; ++z) MHD_Riemann(C, &ULL[NV * z], &URR[NV * z], &F[NV * z]);
    } else {
      SolveRiemann(C, npts, ULL.data(), URR.data(), F.data());
    }
    for (int z = 0; z < npts; ++z) {  // RotateFluxBack :235-246 (mhd/riemann.f90:204-217: also B)
      size_t fi = (size_t)npts * sid + z;
      const double* nv = &C.NormVec[3 * fi];
      const double* t1 = &C.TangVec1[3 * fi];
      const double* t2 = &C.TangVec2[3 * fi];
      real f2 = F[NV * z + 1], f3 = F[NV * z + 2], f4 = F[NV * z + 3];
      F[NV * z + 1] = nv[0] * f2 + t1[0] * f3 + t2[0] * f4;
      F[NV * z + 2] = nv[1] * f2 + t1[1] * f3 + t2[1] * f4;
      F[NV * z + 3] = nv[2] * f2 + t1[2] * f3 + t2[2] * f4;
      if (C.mhd) {
        real f6 = F[NV * z + 5], f7 = F[NV * z + 6], f8 = F[NV * z + 7];
        F[NV * z + 5] = nv[0] * f6 + t1[0] * f7 + t2[0] * f8;
        F[NV * z + 6] = nv[1] * f6 + t1[1] * f7 + t2[1] * f8;
        F[NV * z + 7] = nv[2] * f6 + t1[2] * f7 + t2[2] * f8;
      }
    }
    if (C.parabolic) {  // riemann.f90:155-168 (mhd/riemann.f90:120-141)
      for (int z = 0; z < npts; ++z) {
        size_t fi = (size_t)npts * sid + z;
        real kL[NVMAX], gL[NVMAX], jL[NVMAX], kR[NVMAX], gR[NVMAX], jR[NVMAX];
        DiffFlux(C, &C.Umaster[NV * fi], &C.gxm[NV * fi], &C.gym[NV * fi], &C.gzm[NV * fi], kL, gL, jL);
        DiffFlux(C, &C.Uslave[NV * fi], &C.gxs[NV * fi], &C.gys[NV * fi], &C.gzs[NV * fi], kR, gR, jR);
        const double* nv = &C.NormVec[3 * fi];
        for (int v = 1; v < NV; ++v)
          F[NV * z + v] = F[NV * z + v] + 0.5 * (nv[0] * (kL[v] + kR[v]) + nv[1] * (gL[v] + gR[v]) + nv[2] * (jL[v] + jR[v]));
      }
    }
    for (size_t z = 0; z < F.size(); ++z) FS[z] = F[z];  // Flux_slave = Flux_master (fillflux.f90:91)
    if (C.mhd && C.noncons) {  // AddNonConsFlux on both sides, fillflux.f90:92-100
      for (int z = 0; z < npts; ++z) {
        size_t fi = (size_t)npts * sid + z;
        const double* nv = &C.NormVec[3 * fi];
        MHD_NonConsSurf(C, &C.Umaster[NV * fi], &C.Uslave[NV * fi], nv, &F[NV * z]);
        MHD_NonConsSurf(C, &C.Uslave[NV * fi], &C.Umaster[NV * fi], nv, &FS[NV * z]);
      }
    }
    for (int z = 0; z < npts; ++z) {
      size_t fi = (size_t)npts * sid + z;
      for (int v = 0; v < NV; ++v) {
        C.Fmaster[NV * fi + v] = F[NV * z + v] * C.SurfElem[fi];
        C.Fslave[NV * fi + v] = FS[NV * z + v] * C.SurfElem[fi];
      }
    }
  }
  }
}

// SurfInt (LGL), dg/surfint.f90:48-264
void SurfInt(Case& C) {
  int n = C.np;
  if (C.gauss) {
    // Gauss nodes (surfint.f90:118-175, 196-253): every node of the line takes the surface flux times
    // L_HatMinus(l); the split form adds the correction -(FluxB_sum - FluxB(l)) NormalSign with
    // FluxB(l) = the two-point volume flux between node l and the side's state (metric average of the
    // node's metric and SurfMetrics) and FluxB_sum = sum_l FluxB(l) L_Minus(l).  MHD with NONCONS: the
    // sum takes FluxB(l) plus the non-conservative flux from the side state to node l, and FluxB(l)
    // itself gains the one from node l to the side state (AddNonConsFluxVec, mhd/flux_average.f90:378-418)
    const int NV = C.nVar;
    const size_t nv = (size_t)n * n * n;
    std::vector<real> FB((size_t)NV * n);
    for (int sid = 0; sid < C.nSides; ++sid)
      for (int side = 0; side < 2; ++side) {
        const int e1 = C.SideToElem[side + 5 * sid];
        if (e1 == -1) continue;
        const int e = e1 - 1;
        const int ls = C.SideToElem[2 + side + 5 * sid], fl = side ? C.SideToElem[4 + 5 * sid] : 0;
        const std::vector<double>& Mx = (ls == 3 || ls == 5) ? C.Mf : ((ls == 2 || ls == 4) ? C.Mg : C.Mh);
        const std::vector<real>& Uf = side ? C.Uslave : C.Umaster;
        const std::vector<real>& Ff = side ? C.Fslave : C.Fmaster;
        const double sg = NormalSigns[ls];
        for (int q = 0; q < n; ++q)
          for (int p = 0; p < n; ++p) {
            const real* UB = &Uf[C.fac(0, p, q, sid)];
            real aB[NVMAX + 4], aN[NVMAX + 4], sum[NVMAX];
            Uaux(C, UB, aB);
            const double* SM = &C.SurfMetrics[3 * ((size_t)p + n * ((size_t)q + n * ((size_t)(ls - 1) + 6 * (size_t)e)))];
            for (int v = 0; v < NV; ++v) sum[v] = 0.;
            for (int l = 0; l < n; ++l) {
              const size_t o = C.nod(C.s2v(l, p, q, fl, ls, 0), C.s2v(l, p, q, fl, ls, 1), C.s2v(l, p, q, fl, ls, 2), e);
              Uaux(C, &C.U[NV * o], aN);
              const real mL[3] = {Mx[3 * o], Mx[3 * o + 1], Mx[3 * o + 2]}, mR[3] = {SM[0], SM[1], SM[2]};
              real* F = &FB[(size_t)NV * l];
              if (C.mhd) MHD_VolumeFluxVec(C, C.P.volume_flux, &C.U[NV * o], UB, aN, aB, mL, mR, F);
              else VolumeFluxVec(C, &C.U[NV * o], UB, aN, aB, mL, mR, F);
              if (C.mhd && C.noncons) {
                real Fc[NVMAX];
                for (int v = 0; v < NV; ++v) Fc[v] = F[v];
                MHD_NonConsPair(C, UB, aB, &C.U[NV * o], mR, mL, Fc);  // side state -> node l
                for (int v = 0; v < NV; ++v) sum[v] = sum[v] + Fc[v] * C.Lminus[l];
                MHD_NonConsPair(C, &C.U[NV * o], aN, UB, mL, mR, F);   // node l -> side state
              } else {
                for (int v = 0; v < NV; ++v) sum[v] = sum[v] + F[v] * C.Lminus[l];
              }
            }
            for (int l = 0; l < n; ++l) {
              const size_t o = C.nod(C.s2v(l, p, q, fl, ls, 0), C.s2v(l, p, q, fl, ls, 1), C.s2v(l, p, q, fl, ls, 2), e);
              for (int v = 0; v < NV; ++v) {
                const real fv = Ff[C.fac(v, p, q, sid)];
                const real corr = (sum[v] - FB[(size_t)NV * l + v]) * sg;
                if (side == 0) C.Ut[NV * o + v] = C.Ut[NV * o + v] + (fv - corr) * C.LhatMinus[l];
                else C.Ut[NV * o + v] = C.Ut[NV * o + v] - (fv + corr) * C.LhatMinus[l];
              }
            }
          }
      }
    (void)nv;
    return;
  }
  for (int sid = 0; sid < C.nSides; ++sid) {
    int e = C.SideToElem[0 + 5 * sid];
    if (e != -1) {
      int ls = C.SideToElem[2 + 5 * sid];
      for (int q = 0; q < n; ++q)
        for (int p = 0; p < n; ++p)
          for (int v = 0; v < C.nVar; ++v) {
            size_t idx = C.vol(v, C.s2v(0, p, q, 0, ls, 0), C.s2v(0, p, q, 0, ls, 1), C.s2v(0, p, q, 0, ls, 2), e - 1);
            C.Ut[idx] = C.Ut[idx] + C.Fmaster[C.fac(v, p, q, sid)] * C.L_HatMinus0;
          }
    }
    int nb = C.SideToElem[1 + 5 * sid];
    if (nb != -1) {
      int nls = C.SideToElem[3 + 5 * sid], fl = C.SideToElem[4 + 5 * sid];
      for (int q = 0; q < n; ++q)
        for (int p = 0; p < n; ++p)
          for (int v = 0; v < C.nVar; ++v) {
            size_t idx = C.vol(v, C.s2v(0, p, q, fl, nls, 0), C.s2v(0, p, q, fl, nls, 1), C.s2v(0, p, q, fl, nls, 2), nb - 1);
            C.Ut[idx] = C.Ut[idx] - C.Fslave[C.fac(v, p, q, sid)] * C.L_HatMinus0;
          }
    }
  }
}

#include "fluxo_oracle_nfvse.h"

uint64_t g_phase[8] = {0, 0, 0, 0, 0, 0, 0, 0};
struct PhaseCount {  // operation count of one phase of the RHS (counting build)
  int k;
  uint64_t start;
  explicit PhaseCount(int k_) : k(k_), start(g_oracle_flops) {}
  ~PhaseCount() { g_phase[k] += g_oracle_flops - start; }
};

// useEntropyProlongToFace: the EC / EC-KEP volume fluxes (navierstokes/equation.f90:413-455; MHD:
// Derigs 10 and FloGor 12, mhd/equation.f90:411-427)
inline bool UseEntropyProlong(const Case& C) {
  const int vf = C.P.volume_flux;
  if (C.mhd) return vf == 10 || vf == 12;
  return vf == 5 || vf == 6 || vf == 7 || vf == 10 || vf == 32;
}

// ProlongToFace_U, dg.f90:458-511: Gauss nodes with an entropy-conservative volume flux prolong the
// entropy variables V = ConsToEntropyVec(U) (dg.f90:338-340) and convert the face values back
void ProlongToFaceU(Case& C) {
  if (!(C.gauss && UseEntropyProlong(C))) {
    ProlongToFace(C, C.U, C.Umaster, C.Uslave);
    return;
  }
  const int NV = C.nVar;
  C.Vent.resize(C.U.size());
  for (size_t z = 0; z < C.U.size() / NV; ++z) {
    if (C.mhd) MHD_ConsToEntropy(C, &C.U[NV * z], &C.Vent[NV * z]);
    else ConsToEntropy(C, &C.U[NV * z], &C.Vent[NV * z]);
  }
  std::vector<real> Vm(C.Umaster.size()), Vs(C.Uslave.size());
  ProlongToFace(C, C.Vent, Vm, Vs);
  for (size_t z = 0; z < Vm.size() / NV; ++z) {
    if (C.mhd) {
      MHD_EntropyToCons(C, &Vm[NV * z], &C.Umaster[NV * z]);
      MHD_EntropyToCons(C, &Vs[NV * z], &C.Uslave[NV * z]);
    } else {
      EntropyToCons(C, &Vm[NV * z], &C.Umaster[NV * z]);
      EntropyToCons(C, &Vs[NV * z], &C.Uslave[NV * z]);
    }
  }
}

// Phases: 0 volume split form, 1 lifting, 2 viscous volume integral, 3 face fluxes,
//         4 surface integral, 5 Jacobian + source
void DGTimeDerivative(Case& C, double t) {
  std::fill(C.Ut.begin(), C.Ut.end(), real(0.));  // VNullify
  ProlongToFaceU(C);
  if (C.P.nfvse) CalcBlendingCoefficient(C);  // dg.f90:358-361
  { PhaseCount pc(0); VolIntSplitForm(C); }
  if (C.P.nfvse) { PhaseCount pc(6); VolIntNFVSE(C); }  // dg.f90:380-383
  if (C.parabolic) {
    { PhaseCount pc(1); Lifting(C); }
    { PhaseCount pc(2); VolIntVisc(C); }
  }
  { PhaseCount pc(3); FillFlux(C); }
  { PhaseCount pc(4); SurfInt(C); }
  PhaseCount pc(5);
  size_t nd = (size_t)C.np * C.np * C.np * C.nElems;
  for (size_t z = 0; z < nd; ++z)  // V2D_M_V1D(Ut,-sJ), vector.f90:144-166
    for (int v = 0; v < C.nVar; ++v) C.Ut[C.nVar * z + v] = C.Ut[C.nVar * z + v] * (-C.sJ[z]);
  CalcSource(C, t);
}

// CALCTIMESTEP, navierstokes/calctimestep.f90:39-170
double CalcTimeStep(Case& C, int* errType) {
  if (C.mhd) return MHD_CalcTimeStep(C, errType);
  *errType = 0;
  int n = C.np;
  double KappasPr_max = std::max(4. / 3., C.KappasPr);
  double dtConv = 1.7976931348623157e308, dtVisc = 1.7976931348623157e308;
  for (int e = 0; e < C.nElems; ++e) {
    double ml1 = 1e-12, ml2 = 1e-12, ml3 = 1e-12, mv1 = 1e-12, mv2 = 1e-12, mv3 = 1e-12;
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          size_t o = C.nod(i, j, k, e);
          const real* U = &C.U[5 * o];
          if (std::isnan(val(U[0]))) *errType = 1;
          double sRho = 1. / val(U[0]);
          double v[3] = {val(U[1]) * sRho, val(U[2]) * sRho, val(U[3]) * sRho};
          double p = C.kappaM1 * (val(U[4]) - 0.5 * val(U[0]) * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
          if (p <= 0.) *errType = 2;
          double c = std::sqrt(C.kappa * p * sRho);
          const double* mf = &C.Mf[3 * o];
          const double* mg = &C.Mg[3 * o];
          const double* mh = &C.Mh[3 * o];
          double sj = C.sJ[o];
          ml1 = std::max(ml1, sj * (std::fabs(mf[0] * v[0] + mf[1] * v[1] + mf[2] * v[2]) +
                                    c * std::sqrt(mf[0] * mf[0] + mf[1] * mf[1] + mf[2] * mf[2])));
          ml2 = std::max(ml2, sj * (std::fabs(mg[0] * v[0] + mg[1] * v[1] + mg[2] * v[2]) +
                                    c * std::sqrt(mg[0] * mg[0] + mg[1] * mg[1] + mg[2] * mg[2])));
          ml3 = std::max(ml3, sj * (std::fabs(mh[0] * v[0] + mh[1] * v[1] + mh[2] * v[2]) +
                                    c * std::sqrt(mh[0] * mh[0] + mh[1] * mh[1] + mh[2] * mh[2])));
          if (C.parabolic) {
            double mu = val(ViscMu(C, real(p), real(sRho)));
            double muX = sRho * KappasPr_max * mu;
            auto sq = [&](const double* m) {
              double a = m[0] * sj, b = m[1] * sj, cc = m[2] * sj;
              return a * a + b * b + cc * cc;
            };
            mv1 = std::max(mv1, muX * sq(mf));
            mv2 = std::max(mv2, muX * sq(mg));
            mv3 = std::max(mv3, muX * sq(mh));
          }
        }
    double dtE = C.CFLScale * 2. / (ml1 + ml2 + ml3);
    dtConv = std::min(dtConv, dtE);
    if (std::isnan(dtConv)) *errType = 3;
    if (C.parabolic) {
      double dtV = C.DFLScale * 4. / (mv1 + mv2 + mv3);
      dtVisc = std::min(dtVisc, dtV);
      if (std::isnan(dtVisc)) *errType = 4;
    }
    if (*errType != 0) break;
  }
  return std::min(dtConv, dtVisc);
}

// Get_Pressure / Get_dpdU (navierstokes/equation_vars.f90:752-760, 792-809; mhd/equation_vars.f90:803-812, 844-862)
inline real CorrPressure(const Case& C, const real* U) {
  const real m2 = U[1] * U[1] + U[2] * U[2] + U[3] * U[3];
  if (C.mhd)
    return C.kappaM1 * (U[4] - 0.5 * (m2 / U[0]) - C.s2mu_0 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7] + U[8] * U[8]));
  return C.kappaM1 * (U[4] - 0.5 * (m2 / U[0]));
}
inline void CorrDpdU(const Case& C, const real* U, real* d) {
  const real vel[3] = {U[1] / U[0], U[2] / U[0], U[3] / U[0]};
  d[0] = 0.5 * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
  for (int c = 0; c < 3; ++c) d[1 + c] = -vel[c];
  d[4] = 1.0;
  if (C.mhd)
    for (int z = 5; z < 9; ++z) d[z] = -C.smu_0 * U[z];
  for (int v = 0; v < C.nVar; ++v) d[v] = d[v] * C.kappaM1;
}

// Apply_NFVSE_Correction (nfvse.f90:1688-1883) after the update of an RK stage with step dt = b_dt(stage):
// per element the smallest increase of alpha (as a correction of U along FFV_m_FDG) that keeps the density,
// then the pressure, at PositCorrFactor of the values of the 'safe' state U + dt (1-alpha) FFV_m_FDG
// (Newton iterations for the pressure); alpha <= 1.  Ut gets the matching change.  A safe state with
// negative density or pressure sets corrErr (the reference stops the run).
void ApplyNFVSECorrection(Case& C, double dt) {
  const double eps = 1.e-14, NEWTON_ABSTOL = 1.e-8, alpha_maxPosit = 1.0;
  const double sdt = 1. / dt;
  const int NV = C.nVar, nd = C.nDOFElem;
  std::vector<real> p_safe(nd);
  for (int e = 0; e < C.nElems; ++e) {
    const double alphadiff = C.alpha[e] - alpha_maxPosit;
    if (std::fabs(alphadiff) < eps) continue;
    real* U = &C.U[(size_t)NV * nd * e];
    real* Ut = &C.Ut[(size_t)NV * nd * e];
    const real* FF = &C.FFVmFDG[(size_t)NV * nd * e];
    for (int z = 0; z < nd; ++z) {
      real us[NVMAX];
      for (int v = 0; v < NV; ++v) us[v] = U[NV * z + v] + dt * FF[NV * z + v] * (1. - C.alpha[e]);
      p_safe[z] = CorrPressure(C, us);
      if (p_safe[z] < 0. || us[0] < 0.) { if (!C.corrErr) C.corrErr = e + 1; }
    }
    auto correct = [&](double corr) {
      const double alphacont = C.alpha[e];
      C.alpha[e] = C.alpha[e] + corr * sdt;
      if (C.alpha[e] > alpha_maxPosit) {
        C.alpha[e] = alpha_maxPosit;
        corr = (alpha_maxPosit - alphacont) * dt;
      }
      for (int z = 0; z < NV * nd; ++z) {
        U[z] = U[z] + corr * FF[z];
        Ut[z] = Ut[z] + (C.alpha[e] - alphacont) * FF[z];
      }
    };
    // density
    double corr = -eps;
    for (int z = 0; z < nd; ++z) {
      const double us0 = val(U[NV * z]) + dt * val(FF[NV * z]) * (1. - C.alpha[e]);
      const double a = C.P.posit_corr_factor * us0 - val(U[NV * z]);
      if (a > 0.) {
        if (std::fabs(val(FF[NV * z])) < eps) continue;
        corr = std::max(corr, a / val(FF[NV * z]));
      }
    }
    if (corr > 0.) correct(corr);
    // pressure
    corr = -eps;
    for (int z = 0; z < nd; ++z) {
      double pres = val(CorrPressure(C, &U[NV * z]));
      const double p_goal = C.P.posit_corr_factor * val(p_safe[z]);
      double ap = p_goal - pres;
      if (ap <= 0.) continue;
      real Uc[NVMAX], dp[NVMAX];
      for (int v = 0; v < NV; ++v) Uc[v] = U[NV * z + v];
      double corr1 = 0.0;
      for (int it = 1; it <= C.P.posit_max_iter; ++it) {
        CorrDpdU(C, Uc, dp);
        real dpa = 0.;
        for (int v = 0; v < NV; ++v) dpa = dpa + dp[v] * FF[NV * z + v];
        if (std::fabs(val(dpa)) < eps) break;
        corr1 = corr1 + ap / val(dpa);
        for (int v = 0; v < NV; ++v) Uc[v] = U[NV * z + v] + corr1 * FF[NV * z + v];
        pres = val(CorrPressure(C, Uc));
        ap = p_goal - pres;
        if (ap <= 2.220446049250313e-16 && ap > -NEWTON_ABSTOL * p_goal) break;
      }
      corr = std::max(corr, corr1);
    }
    if (corr > 0.) correct(corr);
  }
}

// TimeStepByLSERKW2, timedisc/timedisc.f90:424-480
// TimeStepByLSERKK3, timedisc.f90:489-542 (S2 and Uprev as extra registers)
void TimeStepLSERKK3(Case& C, double t, double dt) {
  const OrcRKTable& T = *C.rk;
  size_t nt = C.U.size();
  std::vector<double> b_dt(C.nRKStages + 1);
  for (int s = 1; s <= C.nRKStages; ++s) b_dt[s] = T.b[s] * dt;
  std::vector<real> Uprev(C.U.begin(), C.U.end()), S2(C.U.begin(), C.U.end());
  DGTimeDerivative(C, t);
  for (size_t z = 0; z < nt; ++z) C.U[z] = C.U[z] + C.Ut[z] * b_dt[1];
  for (int s = 2; s <= C.nRKStages; ++s) {
    DGTimeDerivative(C, t + dt * T.c[s]);
    for (size_t z = 0; z < nt; ++z) S2[z] = S2[z] + C.U[z] * T.delta[s];
    for (size_t z = 0; z < nt; ++z) C.U[z] = C.U[z] * T.g1[s] + S2[z] * T.g2[s];
    for (size_t z = 0; z < nt; ++z) C.U[z] = C.U[z] + Uprev[z] * T.g3[s];
    for (size_t z = 0; z < nt; ++z) C.U[z] = C.U[z] + C.Ut[z] * b_dt[s];
  }
}

// TimeStepBySSPRK2 (ssprk4-5), timedisc.f90:560-640
void TimeStepSSPRK2(Case& C, double t, double dt) {
  const OrcRKTable& T = *C.rk;
  const int n = C.nRKStages;
  size_t nt = C.U.size();
  std::vector<double> b_dt(n + 1);
  for (int s = 1; s <= n; ++s) b_dt[s] = T.b[s] * dt;
  std::vector<real> r0(C.U.begin(), C.U.end()), r1(nt, real(0.));
  const bool corr = C.P.nfvse && C.P.nfvse_corr;
  DGTimeDerivative(C, t);
  for (size_t z = 0; z < nt; ++z) C.U[z] = C.U[z] + C.Ut[z] * b_dt[1];
  if (corr) ApplyNFVSECorrection(C, b_dt[1]);
  for (int s = 2; s <= n - 1; ++s) {
    DGTimeDerivative(C, t + dt * T.c[s]);
    for (size_t z = 0; z < nt; ++z) C.U[z] = C.U[z] * T.d[s] + r0[z] * T.A[s] + C.Ut[z] * b_dt[s];
    if (corr) ApplyNFVSECorrection(C, b_dt[s]);
    for (size_t z = 0; z < nt; ++z) {
      if (s == 2) r1[z] = C.U[z] * T.e[s];
      else if (s == 3) r1[z] = r1[z] + C.U[z] * T.e[s];
      else if (s == 4) r1[z] = r1[z] + dt * C.Ut[z] * T.e[s];
    }
  }
  DGTimeDerivative(C, t + dt * T.c[n]);
  for (size_t z = 0; z < nt; ++z) C.U[z] = C.U[z] * T.d[n] + r0[z] * T.A[n] + C.Ut[z] * b_dt[n] + r1[z];
  if (corr) ApplyNFVSECorrection(C, b_dt[n]);
}

// TimeStepBySSPRK33, timedisc.f90:647-687
void TimeStepSSPRK33(Case& C, double t, double dt) {
  size_t nt = C.U.size();
  const double cc_dt[4] = {-0.75 * dt, 0.25 * dt, -1. / 12. * dt, 2. / 3. * dt};
  DGTimeDerivative(C, t);
  std::vector<real> tmp(C.Ut.begin(), C.Ut.end());
  for (size_t z = 0; z < nt; ++z) C.U[z] = C.U[z] + C.Ut[z] * dt;
  DGTimeDerivative(C, t + dt);
  for (size_t z = 0; z < nt; ++z) C.U[z] = C.U[z] + tmp[z] * cc_dt[0] + C.Ut[z] * cc_dt[1];
  for (size_t z = 0; z < nt; ++z) tmp[z] = tmp[z] + C.Ut[z];
  DGTimeDerivative(C, t + 0.5 * dt);
  for (size_t z = 0; z < nt; ++z) C.U[z] = C.U[z] + tmp[z] * cc_dt[2] + C.Ut[z] * cc_dt[3];
}

// TimeStepByLSERKW2, timedisc.f90:424-480; the other schemes dispatch from here (the TimeStep pointer)
void TimeStepLSERK(Case& C, double t, double dt) {
  if (C.rk->type == 1) { TimeStepLSERKK3(C, t, dt); return; }
  if (C.rk->type == 2) { TimeStepSSPRK2(C, t, dt); return; }
  if (C.rk->type == 3) { TimeStepSSPRK33(C, t, dt); return; }
  size_t nt = C.U.size();
  std::vector<double> b_dt(C.nRKStages + 1);
  for (int s = 1; s <= C.nRKStages; ++s) b_dt[s] = C.RKb[s] * dt;
  DGTimeDerivative(C, t);
  for (size_t z = 0; z < nt; ++z) C.UtTmp[z] = C.Ut[z];
  for (size_t z = 0; z < nt; ++z) C.U[z] = C.U[z] + C.Ut[z] * b_dt[1];
  if (C.P.nfvse && C.P.nfvse_corr) ApplyNFVSECorrection(C, b_dt[1]);
  for (int s = 2; s <= C.nRKStages; ++s) {
    double ts = t + dt * C.RKc[s];
    DGTimeDerivative(C, ts);
    for (size_t z = 0; z < nt; ++z) C.UtTmp[z] = C.Ut[z] - C.UtTmp[z] * C.RKA[s];  // VAXPBY ConstOut
    for (size_t z = 0; z < nt; ++z) C.U[z] = C.U[z] + C.UtTmp[z] * b_dt[s];
    if (C.P.nfvse && C.P.nfvse_corr) ApplyNFVSECorrection(C, b_dt[s]);
  }
}

}  // namespace

// ----------------------------------------------------------------------------------------------
// C interface
// ----------------------------------------------------------------------------------------------
static void* orc_create_impl(const orc_params* p, const HoprMesh* M) {
  try {
    Case* C = new Case();
    C->P = *p;
    C->N = p->N;
    C->np = p->N + 1;
    C->mhd = (p->eqn == 2 || p->eqn == 3);
    C->nVar = C->mhd ? 9 : 5;
    C->nAux = C->mhd ? 8 : 6;
    C->nDOFElem = C->np * C->np * C->np;
    C->parabolic = (p->eqn == 1 || p->eqn == 3);
    C->gauss = (p->node_type == 1);
    if (C->gauss && p->nfvse) throw std::runtime_error("Gauss nodes: NFVSE needs the LGL subcells");
    InitEquationAndTime(*C);
    InitBasis(*C);
    if (M) BuildMeshHOPR(*C, *M);
    else BuildMesh(*C);
    CalcMetrics(*C);
    if (p->nfvse) {  // InitNFVSE, nfvse.f90:106-260
      if (p->N < 2) throw std::runtime_error("NFVSE needs N >= 2 (shockcapturing.f90)");
      C->alpha.assign(C->nElems, 0.);
      if (p->compute_alpha == 20) {
        // RANDOM_NUMBER * alpha_max (nfvse.f90:1591-1596); the reference's stream is compiler-specific,
        // this one is SplitMix64 (Steele, Lea, Flood 2014) from state 0, one draw per element
        uint64_t st = 0;
        for (int e = 0; e < C->nElems; ++e) {
          uint64_t z = (st += 0x9e3779b97f4a7c15ULL);
          z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
          z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
          z ^= z >> 31;
          C->alpha[e] = (double)(z >> 11) / 9007199254740992.0 * p->alpha_max;
        }
      }
      C->alphaMaster.assign(C->nSides, 0.);
      C->alphaSlave.assign(C->nSides, 0.);
      ComputeSubcellMetrics(*C);
      const int sfm = p->sub_fv_method;
      if (sfm < 1 || sfm > 4) throw std::runtime_error("SubFVMethod not implemented");
      if (sfm >= 3 && !HasDissipMatrices(*C))
        throw std::runtime_error("SubFVMethod 3/4 need a Riemann solver with RiemannVolFluxAndDissipMatrices");
      if (p->nfvse_corr) {
        if (C->rk->type == 1)  // timedisc_vars.f90:111-114
          throw std::runtime_error("NFVSE correction is only implemented for LSERKW2 methods and ssprk4-5");
        C->FFVmFDG.assign((size_t)C->nVar * C->nDOFElem * C->nElems, 0.);
      }
    }
    size_t nt = (size_t)C->nVar * C->nDOFElem * C->nElems;
    size_t nf = (size_t)C->nVar * C->np * C->np * C->nSides;
    C->U.assign(nt, 0.); C->Ut.assign(nt, 0.); C->UtTmp.assign(nt, 0.);
    C->Umaster.assign(nf, 0.); C->Uslave.assign(nf, 0.); C->Fmaster.assign(nf, 0.); C->Fslave.assign(nf, 0.);
    if (C->parabolic) {
      C->gx.assign(nt, 0.); C->gy.assign(nt, 0.); C->gz.assign(nt, 0.);
      C->gxm.assign(nf, 0.); C->gym.assign(nf, 0.); C->gzm.assign(nf, 0.);
      C->gxs.assign(nf, 0.); C->gys.assign(nf, 0.); C->gzs.assign(nf, 0.);
      C->FX.assign(nf, 0.); C->FY.assign(nf, 0.); C->FZ.assign(nf, 0.);
    }
    // FillIni(IniExactFunc, U), equation.f90:545-568
    size_t nd = (size_t)C->nDOFElem * C->nElems;
    for (size_t z = 0; z < nd; ++z) {
      double r[NVMAX];
      if (p->ini_exact_func == 0) break;  // state set by the caller (orc_set_U)
      ExactFunc(*C, p->ini_exact_func, 0., &C->Elem_xGP[3 * z], r);
      for (int v = 0; v < C->nVar; ++v) C->U[C->nVar * z + v] = r[v];
    }
    return C;
  } catch (const std::exception& ex) {
    fprintf(stderr, "orc_create: %s\n", ex.what());
    return nullptr;
  }
}

extern "C" {

void* orc_create(const orc_params* p) { return orc_create_impl(p, nullptr); }

void* orc_create_hopr(const orc_params* p, int nElems, const int* ElemInfo, int nSideInfo, const int* SideInfo,
                      int nBCs, const int* BCType, int NGeo, int nodesGL, const double* NodeCoords, double meshScale,
                      int useCurveds) {
  if (!ElemInfo || !SideInfo || !BCType || !NodeCoords || nElems < 1 || NGeo < 1) return nullptr;
  HoprMesh M{nElems, nSideInfo, nBCs, NGeo, nodesGL, useCurveds, ElemInfo, SideInfo, BCType, NodeCoords, meshScale};
  return orc_create_impl(p, &M);
}

void orc_destroy(void* h) { delete (Case*)h; }

void orc_set_alpha(void* h, const double* alpha) {
  Case* C = (Case*)h;
  if (!C->alpha.empty()) std::copy(alpha, alpha + C->nElems, C->alpha.begin());
}

void orc_sizes(void* h, int* nElems, int* nSides, int* nVar, int* N) {
  Case* C = (Case*)h;
  *nElems = C->nElems; *nSides = C->nSides; *nVar = C->nVar; *N = C->N;
}

void orc_get_mesh(void* h, int* S2E, int* E2S, double* Mf, double* Mg, double* Mh, double* sJ, double* NormVec,
                  double* TangVec1, double* TangVec2, double* SurfElem, double* Elem_xGP) {
  Case* C = (Case*)h;
  if (S2E) std::copy(C->SideToElem.begin(), C->SideToElem.end(), S2E);
  if (E2S) std::copy(C->ElemToSide.begin(), C->ElemToSide.end(), E2S);
  if (Mf) std::copy(C->Mf.begin(), C->Mf.end(), Mf);
  if (Mg) std::copy(C->Mg.begin(), C->Mg.end(), Mg);
  if (Mh) std::copy(C->Mh.begin(), C->Mh.end(), Mh);
  if (sJ) std::copy(C->sJ.begin(), C->sJ.end(), sJ);
  if (NormVec) std::copy(C->NormVec.begin(), C->NormVec.end(), NormVec);
  if (TangVec1) std::copy(C->TangVec1.begin(), C->TangVec1.end(), TangVec1);
  if (TangVec2) std::copy(C->TangVec2.begin(), C->TangVec2.end(), TangVec2);
  if (SurfElem) std::copy(C->SurfElem.begin(), C->SurfElem.end(), SurfElem);
  if (Elem_xGP) std::copy(C->Elem_xGP.begin(), C->Elem_xGP.end(), Elem_xGP);
}

void orc_set_metrics(void* h, const double* Mf, const double* Mg, const double* Mh, const double* sJ,
                     const double* NormVec, const double* TangVec1, const double* TangVec2,
                     const double* SurfElem) {
  Case* C = (Case*)h;
  if (Mf) std::copy(Mf, Mf + C->Mf.size(), C->Mf.begin());
  if (Mg) std::copy(Mg, Mg + C->Mg.size(), C->Mg.begin());
  if (Mh) std::copy(Mh, Mh + C->Mh.size(), C->Mh.begin());
  if (sJ) std::copy(sJ, sJ + C->sJ.size(), C->sJ.begin());
  if (NormVec) std::copy(NormVec, NormVec + C->NormVec.size(), C->NormVec.begin());
  if (TangVec1) std::copy(TangVec1, TangVec1 + C->TangVec1.size(), C->TangVec1.begin());
  if (TangVec2) std::copy(TangVec2, TangVec2 + C->TangVec2.size(), C->TangVec2.begin());
  if (SurfElem) std::copy(SurfElem, SurfElem + C->SurfElem.size(), C->SurfElem.begin());
}

void orc_get_U(void* h, double* U) {
  Case* C = (Case*)h;
  for (size_t z = 0; z < C->U.size(); ++z) U[z] = val(C->U[z]);
}
void orc_set_U(void* h, const double* U) {
  Case* C = (Case*)h;
  for (size_t z = 0; z < C->U.size(); ++z) C->U[z] = U[z];
}

void orc_dg_time_derivative(void* h, double t, double* Ut) {
  Case* C = (Case*)h;
  DGTimeDerivative(*C, t);
  if (Ut)
    for (size_t z = 0; z < C->Ut.size(); ++z) Ut[z] = val(C->Ut[z]);
}

void orc_get_gradients(void* h, double* gx, double* gy, double* gz) {
  Case* C = (Case*)h;
  for (size_t z = 0; z < C->gx.size(); ++z) {
    if (gx) gx[z] = val(C->gx[z]);
    if (gy) gy[z] = val(C->gy[z]);
    if (gz) gz[z] = val(C->gz[z]);
  }
}

double orc_calc_timestep(void* h, int* errType) { return CalcTimeStep(*(Case*)h, errType); }

void orc_timestep(void* h, double t, double dt) { TimeStepLSERK(*(Case*)h, t, dt); }

double orc_run(void* h, double t, double tEnd, int maxIter, int* nSteps) {
  Case* C = (Case*)h;
  int it = 0;
  while (t < tEnd && (maxIter < 0 || it < maxIter)) {  // TimeDisc loop, timedisc.f90:274-359
    int err = 0;
    double dt = CalcTimeStep(*C, &err);
    if (err != 0) break;
    if (tEnd - t <= dt * (1. + 1.e-4)) dt = tEnd - t;
    TimeStepLSERK(*C, t, dt);
    t += dt;
    ++it;
  }
  if (nSteps) *nSteps = it;
  return t;
}

void orc_analyze(void* h, double t, double* L2, double* Linf, double* entropy, double* dSdU_Ut, double* ekin,
                 double* enstrophy) {
  Case* C = (Case*)h;
  int n = C->np, N = C->N;
  size_t nv = (size_t)n * n * n;
  std::vector<double> wVol(nv);
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) wVol[i + n * (j + n * k)] = C->wGP[i] * C->wGP[j] * C->wGP[k];
  double Vol = 0.;
  for (int e = 0; e < C->nElems; ++e)
    for (size_t z = 0; z < nv; ++z) Vol += wVol[z] / C->sJ[nv * e + z];
  if (L2 || Linf) {  // CalcErrorNorms, analyze.f90:557-632, NAnalyze = 2*(N+1)
    int NA = 2 * (N + 1), na = NA + 1;
    std::vector<double> xA(na), wA(na), V(na * n);
    LGLNodesWeights(NA, xA.data(), wA.data());
    InitVdm(N, NA, C->wBary.data(), C->xGP.data(), xA.data(), V.data());
    const int NV = C->nVar;
    double l2[NVMAX], li[NVMAX];
    for (int v = 0; v < NVMAX; ++v) { l2[v] = 0.; li[v] = -1e10; }
    std::vector<double> XA(3 * na * na * na), JN(nv), JA(na * na * na), Uin(NV * nv), UA(NV * na * na * na);
    for (int e = 0; e < C->nElems; ++e) {
      ChangeBasis3D(3, N, NA, V.data(), &C->Elem_xGP[3 * nv * e], XA.data());
      for (size_t z = 0; z < nv; ++z) JN[z] = 1. / C->sJ[nv * e + z];
      ChangeBasis3D(1, N, NA, V.data(), JN.data(), JA.data());
      for (size_t z = 0; z < NV * nv; ++z) Uin[z] = val(C->U[NV * nv * e + z]);
      ChangeBasis3D(NV, N, NA, V.data(), Uin.data(), UA.data());
      for (int m = 0; m < na; ++m)
        for (int l = 0; l < na; ++l)
          for (int k = 0; k < na; ++k) {
            size_t z = k + na * (l + (size_t)na * m);
            double ue[NVMAX];
            ExactFunc(*C, C->P.ini_exact_func, t, &XA[3 * z], ue);
            double w = wA[k] * wA[l] * wA[m] * JA[z];
            for (int v = 0; v < NV; ++v) {
              double d = UA[NV * z + v] - ue[v];
              li[v] = std::max(li[v], std::fabs(d));
              l2[v] += d * d * w;
            }
          }
    }
    for (int v = 0; v < NV; ++v) {
      if (L2) L2[v] = std::sqrt(l2[v] / Vol);
      if (Linf) Linf[v] = li[v];
    }
  }
  // CalcEntropy, navierstokes/analyze_equation.f90:549-599
  double S = 0., dS = 0., Ek = 0., En = 0.;
  if (C->mhd) {  // CalcEntropy, mhd/analyze_equation.f90:421-470
    for (int e = 0; e < C->nElems; ++e)
      for (size_t z = 0; z < nv; ++z) {
        size_t o = nv * e + z;
        double w = wVol[z] / C->sJ[o];
        real U[9], prim[9], W[9];
        for (int v = 0; v < 9; ++v) U[v] = C->U[9 * o + v];
        MHD_ConsToPrim(*C, U, prim);
        S += val(-prim[0] * (log(prim[4]) - C->kappa * log(prim[0]))) * w;
        MHD_ConsToEntropy(*C, U, W);
        double loc = 0.;
        for (int v = 0; v < 9; ++v) loc += val(W[v]) * val(C->Ut[9 * o + v]);
        dS += loc * w;
        double u = val(prim[1]), vv = val(prim[2]), ww = val(prim[3]);
        Ek += 0.5 * val(U[0]) * (u * u + vv * vv + ww * ww) * w;
      }
    if (entropy) *entropy = S * C->sKappaM1;
    if (dSdU_Ut) *dSdU_Ut = dS;
    if (ekin) *ekin = Ek / Vol;
    if (enstrophy) *enstrophy = 0.;
    return;
  }
  for (int e = 0; e < C->nElems; ++e)
    for (size_t z = 0; z < nv; ++z) {
      size_t o = nv * e + z;
      double w = wVol[z] / C->sJ[o];
      double U[5], prim[5];
      for (int v = 0; v < 5; ++v) U[v] = val(C->U[5 * o + v]);
      double sRho = 1. / U[0];
      prim[0] = U[0];
      for (int d = 0; d < 3; ++d) prim[1 + d] = U[1 + d] * sRho;
      prim[4] = C->kappaM1 * (U[4] - 0.5 * (U[1] * prim[1] + U[2] * prim[2] + U[3] * prim[3]));
      S += -prim[0] * (std::log(prim[4]) - C->kappa * std::log(prim[0])) * w;
      double u = prim[1], vv = prim[2], ww = prim[3];
      double v2s2 = 0.5 * (u * u + vv * vv + ww * ww);
      double rho_sp = U[0] / (C->kappaM1 * (U[4] - U[0] * v2s2));
      double s = -std::log(rho_sp * std::pow(U[0], C->kappaM1));
      double W[5] = {(C->kappa - s) * C->sKappaM1 - rho_sp * v2s2, rho_sp * u, rho_sp * vv, rho_sp * ww, -rho_sp};
      double loc = 0.;
      for (int v = 0; v < 5; ++v) loc += W[v] * val(C->Ut[5 * o + v]);
      dS += loc * w;
      Ek += 0.5 * U[0] * (u * u + vv * vv + ww * ww) * w;
    }
  if (C->parabolic && enstrophy) {  // TGV integrand 0.5*rho*|curl v|^2 from the lifted gradients
    for (int e = 0; e < C->nElems; ++e)
      for (size_t z = 0; z < nv; ++z) {
        size_t o = nv * e + z;
        double w = wVol[z] / C->sJ[o];
        const real* gx = &C->gx[5 * o];
        const real* gy = &C->gy[5 * o];
        const real* gz = &C->gz[5 * o];
        double wx = val(gy[3]) - val(gz[2]);
        double wy = val(gz[1]) - val(gx[3]);
        double wz = val(gx[2]) - val(gy[1]);
        En += 0.5 * val(C->U[5 * o]) * (wx * wx + wy * wy + wz * wz) * w;
      }
  }
  if (entropy) *entropy = S * C->sKappaM1;
  if (dSdU_Ut) *dSdU_Ut = dS;
  if (ekin) *ekin = Ek / Vol;
  if (enstrophy) *enstrophy = En / Vol;
}

void orc_exact_func(void* h, int func, double t, int n, const double* x, double* U) {
  Case* C = (Case*)h;
  for (int i = 0; i < n; ++i) ExactFunc(*C, func, t, x + 3 * i, U + C->nVar * i);
}

void orc_basis(int N, double* xGP, double* wGP, double* wBary, double* D, double* Dvolsurf, double* Dhat,
               double* Lminus, double* Lplus) {
  Case C;
  C.N = N; C.np = N + 1;
  InitBasis(C);
  int n = N + 1;
  if (xGP) std::copy(C.xGP.begin(), C.xGP.end(), xGP);
  if (wGP) std::copy(C.wGP.begin(), C.wGP.end(), wGP);
  if (wBary) std::copy(C.wBary.begin(), C.wBary.end(), wBary);
  if (D) std::copy(C.D.begin(), C.D.begin() + n * n, D);
  if (Dvolsurf) std::copy(C.Dvolsurf.begin(), C.Dvolsurf.end(), Dvolsurf);
  if (Dhat) std::copy(C.Dhat.begin(), C.Dhat.end(), Dhat);
  if (Lminus) std::copy(C.Lminus.begin(), C.Lminus.end(), Lminus);
  if (Lplus) std::copy(C.Lplus.begin(), C.Lplus.end(), Lplus);
}

uint64_t orc_flops(void) { return g_oracle_flops; }
uint64_t orc_phase_flops(int k) { return (k >= 0 && k < 8) ? g_phase[k] : 0; }
void orc_reset_flops(void) {
  g_oracle_flops = 0;
  for (int k = 0; k < 8; ++k) g_phase[k] = 0;
}

void orc_volume_flux(void* h, const double* UL, const double* UR, const double* mL, const double* mR, double* F) {
  Case* C = (Case*)h;
  const int NV = C->nVar;
  real uL[NVMAX], uR[NVMAX], aL[8], aR[8], ml[3], mr[3], f[NVMAX];
  for (int v = 0; v < NV; ++v) { uL[v] = UL[v]; uR[v] = UR[v]; }
  for (int d = 0; d < 3; ++d) { ml[d] = mL[d]; mr[d] = mR[d]; }
  Uaux(*C, uL, aL);
  Uaux(*C, uR, aR);
  if (C->mhd) MHD_VolumeFluxVec(*C, C->P.volume_flux, uL, uR, aL, aR, ml, mr, f);
  else VolumeFluxVec(*C, uL, uR, aL, aR, ml, mr, f);
  for (int v = 0; v < NV; ++v) F[v] = val(f[v]);
}

void orc_riemann_point(void* h, const double* UL, const double* UR, const double* nv, const double* t1,
                       const double* t2, double* F) {
  Case* C = (Case*)h;
  const int NV = C->nVar;
  real LL[NVMAX], RR[NVMAX], f[NVMAX];
  for (int v = 0; v < NV; ++v) { LL[v] = UL[v]; RR[v] = UR[v]; }
  for (int b = 1; b <= (C->mhd ? 5 : 1); b += 4) {  // momentum (and B for MHD)
    LL[b] = UL[b] * nv[0] + UL[b + 1] * nv[1] + UL[b + 2] * nv[2];
    LL[b + 1] = UL[b] * t1[0] + UL[b + 1] * t1[1] + UL[b + 2] * t1[2];
    LL[b + 2] = UL[b] * t2[0] + UL[b + 1] * t2[1] + UL[b + 2] * t2[2];
    RR[b] = UR[b] * nv[0] + UR[b + 1] * nv[1] + UR[b + 2] * nv[2];
    RR[b + 1] = UR[b] * t1[0] + UR[b + 1] * t1[1] + UR[b + 2] * t1[2];
    RR[b + 2] = UR[b] * t2[0] + UR[b + 1] * t2[1] + UR[b + 2] * t2[2];
  }
  if (C->mhd) MHD_Riemann(*C, LL, RR, f);
  else SolveRiemann(*C, 1, LL, RR, f);
  for (int v = 0; v < NV; ++v) F[v] = val(f[v]);
  for (int b = 1; b <= (C->mhd ? 5 : 1); b += 4) {
    real f2 = f[b], f3 = f[b + 1], f4 = f[b + 2];
    F[b] = val(nv[0] * f2 + t1[0] * f3 + t2[0] * f4);
    F[b + 1] = val(nv[1] * f2 + t1[1] * f3 + t2[1] * f4);
    F[b + 2] = val(nv[2] * f2 + t1[2] * f3 + t2[2] * f4);
  }
}

int orc_corr_error(void* h) { return ((Case*)h)->corrErr; }

void orc_get_surf_metrics(void* h, double* SM) {
  Case* C = (Case*)h;
  const size_t n = (size_t)3 * C->np * C->np * 6 * C->nElems;
  for (size_t z = 0; z < n; ++z) SM[z] = C->gauss ? C->SurfMetrics[z] : 0.;
}

void orc_get_alpha(void* h, double* alpha) {
  Case* C = (Case*)h;
  for (size_t e = 0; e < C->alpha.size(); ++e) alpha[e] = C->alpha[e];
}

void orc_set_glm_ch(void* h, double ch) { ((Case*)h)->GLM_ch = ch; }
double orc_get_glm_ch(void* h) { return ((Case*)h)->GLM_ch; }

double orc_ln_mean(double aL, double aR) { return val(LN_MEAN(real(aL), real(aR))); }

}  // extern "C"
