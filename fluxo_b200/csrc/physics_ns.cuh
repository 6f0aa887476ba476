// Compressible Euler / Navier-Stokes point physics in FP64 for the sm_100a kernels.
// Formulas follow the reference (src/equation/navierstokes/*) so that results agree
// with it to roundoff; each function names the routine it implements.
#pragma once
#include "common.cuh"

namespace fluxo {

// Logarithmic mean with the reference's series switch at f^2 < 1e-4
// (src/equation/navierstokes/flux_average.f90:1945-1965, LN_MEAN).
__device__ __forceinline__ double ln_mean(double aL, double aR) {
  double xi = aR / aL;
  double u = (xi * (xi - 2.) + 1.) / (xi * (xi + 2.) + 1.);
  if (u < 1.0e-4) return (aL + aR) * 52.5 / (105. + u * (35. + u * (21. + u * 15.)));
  return (aR - aL) / log(xi);
}

// Roe-type mean values returned by the 1D two-point fluxes (VolumeFluxAverage interface).
struct Hat { double u, v, w, a, H, p1, rho; };

// 1D two-point fluxes on rotated states (flux_average.f90), numbered like VolumeFlux: 2 and 8
// Kennedy-Gruber, 3 Ducros, 4 Morinishi, 5 EC-KEP, 6 approximate EC-KEP, 7 EC-KEP with pressure
// average, 9 Gassner-Winters-Walch, 10 Ismail-Roe, 32 Ranocha.
template <int W>
__device__ __forceinline__ void volume_flux_1d(const KParams& P, const double* UL, const double* UR, double* F,
                                               Hat& h) {
  double sRL = 1. / UL[0], sRR = 1. / UR[0];
  double uL = sRL * UL[1], vL = sRL * UL[2], wL = sRL * UL[3];
  double uR = sRR * UR[1], vR = sRR * UR[2], wR = sRR * UR[3];
  if constexpr (W == 10) {  // TwoPointEntropyConservingFlux :500-568
    double pL = P.kappaM1 * (UL[4] - 0.5 * (UL[1] * uL + UL[2] * vL + UL[3] * wL));
    double pR = P.kappaM1 * (UR[4] - 0.5 * (UR[1] * uR + UR[2] * vR + UR[3] * wR));
    double z1L = sqrt(UL[0] / pL), z1R = sqrt(UR[0] / pR);
    double z1M = 0.5 * (z1L + z1R);
    double z1LN = ln_mean(z1L, z1R);
    double z2M = 0.5 * (z1L * uL + z1R * uR);
    double z3M = 0.5 * (z1L * vL + z1R * vR);
    double z4M = 0.5 * (z1L * wL + z1R * wR);
    double z5L = pL * z1L, z5R = pR * z1R;
    double z5M = 0.5 * (z5L + z5R);
    double z5LN = ln_mean(z5L, z5R);
    h.rho = z1M * z5LN;
    double sz1M = 1. / z1M;
    h.u = z2M * sz1M; h.v = z3M * sz1M; h.w = z4M * sz1M;
    h.p1 = z5M * sz1M;
    double kp2 = 0.5 * (P.kappaP1 * (z5LN / z1LN) + P.kappaM1 * h.p1);
    h.a = sqrt(kp2 / h.rho);
    h.H = kp2 / (h.rho * P.kappaM1) + 0.5 * (h.u * h.u + h.v * h.v + h.w * h.w);
    F[0] = h.rho * h.u;
    F[1] = F[0] * h.u + h.p1;
    F[2] = F[0] * h.v;
    F[3] = F[0] * h.w;
    F[4] = F[0] * h.H;
  } else if constexpr (W == 5) {  // EntropyAndEnergyConservingFlux :1214-1269
    double v2s2L = 0.5 * (uL * uL + vL * vL + wL * wL), v2s2R = 0.5 * (uR * uR + vR * vR + wR * wR);
    double pL = P.kappaM1 * (UL[4] - UL[0] * v2s2L), pR = P.kappaM1 * (UR[4] - UR[0] * v2s2R);
    double bL = 0.5 * UL[0] / pL, bR = 0.5 * UR[0] / pR;
    double rhoM = 0.5 * (UL[0] + UR[0]);
    h.rho = ln_mean(UL[0], UR[0]);
    double bM = 0.5 * (bL + bR);
    double bHat = ln_mean(bL, bR);
    h.u = 0.5 * (uL + uR); h.v = 0.5 * (vL + vR); h.w = 0.5 * (wL + wR);
    h.a = sqrt(P.kappa * 0.5 * (pL + pR) / h.rho);
    h.H = P.kappa / (2. * P.kappaM1 * bHat) + 0.5 * (uL * uR + vL * vR + wL * wR);
    h.p1 = 0.5 * rhoM / bM;
    double v2M = v2s2L + v2s2R;
    F[0] = h.rho * h.u;
    F[1] = F[0] * h.u + h.p1;
    F[2] = F[0] * h.v;
    F[3] = F[0] * h.w;
    F[4] = F[0] * 0.5 * (P.sKappaM1 / bHat - v2M) + h.u * F[1] + h.v * F[2] + h.w * F[3];
  } else if constexpr (W == 32) {  // RanochaFlux :1806-1860
    double v2L = uL * uL + vL * vL + wL * wL, v2R = uR * uR + vR * vR + wR * wR;
    double pL = P.kappaM1 * (UL[4] - 0.5 * UL[0] * v2L), pR = P.kappaM1 * (UR[4] - 0.5 * UR[0] * v2R);
    h.rho = ln_mean(UL[0], UR[0]);
    h.u = 0.5 * (uL + uR); h.v = 0.5 * (vL + vR); h.w = 0.5 * (wL + wR);
    double v2zip = 0.5 * (uL * uR + vL * vR + wL * wR);
    h.p1 = 0.5 * (pL + pR);
    h.a = sqrt(P.kappa * h.p1 / h.rho);
    h.H = P.kappa * h.p1 * P.sKappaM1 / h.rho + 0.5 * (h.u * h.u + h.v * h.v + h.w * h.w);
    double rspM = ln_mean(UL[0] / pL, UR[0] / pR);
    F[0] = h.rho * h.u;
    F[1] = F[0] * h.u + h.p1;
    F[2] = F[0] * h.v;
    F[3] = F[0] * h.w;
    F[4] = F[0] * (v2zip + 1. / rspM * P.sKappaM1) + 0.5 * (pL * uR + pR * uL);
  } else if constexpr (W == 3) {  // DucrosFlux :937-979
    h.rho = 0.5 * (UL[0] + UR[0]);
    h.u = 0.5 * (uL + uR); h.v = 0.5 * (vL + vR); h.w = 0.5 * (wL + wR);
    h.p1 = 0.5 * P.kappaM1 *
           (UL[4] + UR[4] - 0.5 * (UL[1] * uL + UL[2] * vL + UL[3] * wL + UR[1] * uR + UR[2] * vR + UR[3] * wR));
    h.a = sqrt(P.kappa * h.p1 / h.rho);
    h.H = P.kappa * h.p1 / (h.rho * P.kappaM1) + 0.5 * (h.u * h.u + h.v * h.v + h.w * h.w);
    const double qLR = 0.5 * h.u;
    F[0] = h.rho * (qLR + qLR);
    F[1] = qLR * (UL[1] + UR[1]) + h.p1;
    F[2] = qLR * (UL[2] + UR[2]);
    F[3] = qLR * (UL[3] + UR[3]);
    F[4] = qLR * ((UL[4] + UR[4]) + (h.p1 + h.p1));
  } else if constexpr (W == 4) {  // MorinishiFlux :1066-1113
    const double vel2L = uL * uL + vL * vL + wL * wL, vel2R = uR * uR + vR * vR + wR * wR;
    const double pL = P.kappaM1 * (UL[4] - 0.5 * UL[0] * vel2L), pR = P.kappaM1 * (UR[4] - 0.5 * UR[0] * vel2R);
    h.rho = 0.5 * (UL[0] + UR[0]);
    h.u = 0.5 * (uL + uR); h.v = 0.5 * (vL + vR); h.w = 0.5 * (wL + wR);
    h.p1 = 0.5 * (pL + pR);
    h.a = sqrt(P.kappa * h.p1 / h.rho);
    h.H = P.kappa * h.p1 / (h.rho * P.kappaM1) + 0.5 * (h.u * h.u + h.v * h.v + h.w * h.w);
    const double rq2L = 0.5 * UL[0] * uL, rq2R = 0.5 * UR[0] * uR;
    F[0] = rq2L + rq2R;
    F[1] = F[0] * h.u + h.p1;
    F[2] = F[0] * h.v;
    F[3] = F[0] * h.w;
    F[4] = 0.5 * (P.kappa * P.sKappaM1 * (pL * uL + pR * uR) - (rq2L * vel2L + rq2R * vel2R)) +
           rq2L * (uL * h.u + vL * h.v + wL * h.w) + rq2R * (uR * h.u + vR * h.v + wR * h.w);
  } else if constexpr (W == 6 || W == 7) {
    // EntropyAndEnergyConservingFlux2 :1365-1419 (6) and ggFlux :1513-1567 (7); a = H = 0
    const double v2s2L = 0.5 * (uL * uL + vL * vL + wL * wL), v2s2R = 0.5 * (uR * uR + vR * vR + wR * wR);
    const double pL = P.kappaM1 * (UL[4] - UL[0] * v2s2L), pR = P.kappaM1 * (UR[4] - UR[0] * v2s2R);
    const double bL = 0.5 * UL[0] / pL, bR = 0.5 * UR[0] / pR;
    h.a = 0.; h.H = 0.;
    h.rho = ln_mean(UL[0], UR[0]);
    h.u = 0.5 * (uL + uR); h.v = 0.5 * (vL + vR); h.w = 0.5 * (wL + wR);
    double rhoF, sb;  // density of the mass flux, 1/beta of the energy flux
    if constexpr (W == 6) {
      const double rhoM = 0.5 * (UL[0] + UR[0]);
      sb = 2. / (bL + bR);
      h.p1 = 0.5 * rhoM * sb;
      rhoF = rhoM;
    } else {
      sb = 1. / ln_mean(bL, bR);
      h.p1 = 0.5 * (pL + pR);
      rhoF = h.rho;
    }
    F[0] = rhoF * h.u;
    F[1] = F[0] * h.u + h.p1;
    F[2] = F[0] * h.v;
    F[3] = F[0] * h.w;
    F[4] = F[0] * 0.5 * (P.sKappaM1 * sb - (v2s2L + v2s2R)) + h.u * F[1] + h.v * F[2] + h.w * F[3];
  } else if constexpr (W == 8) {  // KennedyAndGruberFlux2 :810-850
    const double pL = P.kappaM1 * (UL[4] - 0.5 * (UL[1] * uL + UL[2] * vL + UL[3] * wL));
    const double pR = P.kappaM1 * (UR[4] - 0.5 * (UR[1] * uR + UR[2] * vR + UR[3] * wR));
    h.rho = 0.5 * (UL[0] + UR[0]);
    h.u = 0.5 * (uL + uR); h.v = 0.5 * (vL + vR); h.w = 0.5 * (wL + wR);
    h.p1 = 0.5 * (pL + pR);
    h.a = sqrt(P.kappa * h.p1 / h.rho);
    h.H = 0.5 * ((UL[4] + pL) * sRL + (UR[4] + pR) * sRR);
    F[0] = h.rho * h.u;
    F[1] = F[0] * h.u + h.p1;
    F[2] = F[0] * h.v;
    F[3] = F[0] * h.w;
    F[4] = F[0] * h.H;
  } else if constexpr (W == 9) {  // GassnerWintersWalchFlux :1661-1716 (a = 0)
    const double pL = P.kappaM1 * (UL[4] - 0.5 * (UL[1] * uL + UL[2] * vL + UL[3] * wL));
    const double pR = P.kappaM1 * (UR[4] - 0.5 * (UR[1] * uR + UR[2] * vR + UR[3] * wR));
    const double w1L = sqrt(UL[0]), w1R = sqrt(UR[0]);
    h.rho = 0.5 * (w1L + w1R);
    h.u = 0.5 * (w1L * uL + w1R * uR);
    h.v = 0.5 * (w1L * vL + w1R * vR);
    h.w = 0.5 * (w1L * wL + w1R * wR);
    h.H = 0.5 * (w1L * (sRL * (UL[4] + pL)) + w1R * (sRR * (UR[4] + pR)));
    h.p1 = P.kappaM1 * P.sKappa * (h.rho * h.H - 0.5 * (h.u * h.u + h.v * h.v + h.w * h.w));
    h.a = 0.;
    F[0] = h.u * h.rho;
    F[1] = h.u * h.u + h.p1;
    F[2] = h.u * h.v;
    F[3] = h.u * h.w;
    F[4] = h.u * h.H;
  } else {  // W == 2: KennedyAndGruberFlux1 :680-721
    h.rho = 0.5 * (UL[0] + UR[0]);
    h.u = 0.5 * (uL + uR); h.v = 0.5 * (vL + vR); h.w = 0.5 * (wL + wR);
    h.p1 = 0.5 * P.kappaM1 *
           (UL[4] + UR[4] - 0.5 * (UL[1] * uL + UL[2] * vL + UL[3] * wL + UR[1] * uR + UR[2] * vR + UR[3] * wR));
    double eH = 0.5 * (sRL * UL[4] + sRR * UR[4]);
    h.a = sqrt(P.kappa * h.p1 / h.rho);
    h.H = P.kappa * h.p1 / (h.rho * P.kappaM1) + 0.5 * (h.u * h.u + h.v * h.v + h.w * h.w);
    F[0] = h.rho * h.u;
    F[1] = F[0] * h.u + h.p1;
    F[2] = F[0] * h.v;
    F[3] = F[0] * h.w;
    F[4] = F[0] * eH + h.p1 * h.u;
  }
}

// EvalEulerFlux1D (navierstokes/flux.f90:298-329)
__device__ __forceinline__ void euler_flux_1d(const KParams& P, const double* U, double* F) {
  double srho = 1. / U[0];
  double v1 = U[1] * srho, v2 = U[2] * srho, v3 = U[3] * srho;
  double p = P.kappaM1 * (U[4] - 0.5 * (U[1] * v1 + U[2] * v2 + U[3] * v3));
  F[0] = U[1];
  F[1] = U[1] * v1 + p;
  F[2] = U[1] * v2;
  F[3] = U[1] * v3;
  F[4] = (U[4] + p) * v1;
}

// SoundSpeed2 (navierstokes/equation_vars.f90:342-356)
__device__ __forceinline__ double sound_speed2(const KParams& P, const double* U) {
  return P.kappa * P.kappaM1 * (U[4] * U[0] - 0.5 * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3])) / (U[0] * U[0]);
}

__device__ __forceinline__ double lambda_max_pair(const KParams& P, const double* L, const double* R) {
  return fmax(fabs(L[1] / L[0]), fabs(R[1] / R[0])) + sqrt(fmax(sound_speed2(P, L), sound_speed2(P, R)));
}

__device__ __forceinline__ void primitive_pv(const KParams& P, const double* U, double* v, double& p) {
  double s = 1. / U[0];
  v[0] = U[1] * s; v[1] = U[2] * s; v[2] = U[3] * s;
  p = P.kappaM1 * (U[4] - 0.5 * (U[1] * v[0] + U[2] * v[1] + U[3] * v[2]));
}

// Point flux of the Riemann solvers that use RiemannSolver_VolumeFluxAverage (0: not such a
// solver), navierstokes/equation.f90:291-406
template <int RS>
__host__ __device__ constexpr int riemann_point_flux() {
  return RS == 5 ? 10 : RS == 6 ? 2 : RS == 7 ? 3 : RS == 8 ? 4 : RS == 9 ? 5 : RS == 10 ? 6 : RS == 11 ? 7
       : RS == 12 ? 8 : RS == 20 ? 9 : RS == 32 ? 32 : 0;
}
// ... and of those using RiemannSolver_VolumeFluxAverage_LLF
template <int RS>
__host__ __device__ constexpr int riemann_llf_point_flux() {
  return RS == 14 ? 2 : RS == 15 ? 3 : RS == 17 ? 7 : RS == 18 ? 8 : RS == 19 ? 4 : RS == 21 ? 9 : 0;
}

// RiemannSolver_EntropyStable_VolFluxAndDissipMatrices (riemann.f90:936-975): the solver's EC flux
// (4: Ismail-Roe, 44: EC-KEP, 33: Ranocha; equation.f90:381-404), the diagonal scaling DHat = |Lambda| S
// and the right eigenvectors Rh[row][col] at the flux's mean state, on rotated states
template <int RS>
__device__ __forceinline__ void es_matrices(const KParams& P, const double* L, const double* R, double* Fc,
                                            double* Dh, double (*Rh)[5]) {
  constexpr int W = (RS == 4) ? 10 : (RS == 44 ? 5 : 32);
  Hat h;
  volume_flux_1d<W>(P, L, R, Fc, h);
  const double rows[5][5] = {{1., 1., 0., 0., 1.},
                             {h.u - h.a, h.u, 0., 0., h.u + h.a},
                             {h.v, h.v, 1., 0., h.v},
                             {h.w, h.w, 0., 1., h.w},
                             {h.H - h.u * h.a, 0.5 * (h.u * h.u + h.v * h.v + h.w * h.w), h.v, h.w, h.H + h.u * h.a}};
#pragma unroll
  for (int r = 0; r < 5; ++r)
#pragma unroll
    for (int c = 0; c < 5; ++c) Rh[r][c] = rows[r][c];
  Dh[0] = 0.5 * fabs(h.u - h.a) * h.rho / P.kappa;
  Dh[1] = fabs(h.u) * (P.kappaM1 / P.kappa) * h.rho;
  Dh[2] = fabs(h.u) * h.p1;
  Dh[3] = Dh[2];
  Dh[4] = 0.5 * fabs(h.u + h.a) * h.rho / P.kappa;
}

// ConsToEntropy (equation_vars.f90:362-391); s = -log(rho_sp * rho^(kappa-1)) as two logarithms
__device__ __forceinline__ void cons_to_entropy_ns(const KParams& P, const double* U, double* V) {
  double srho = 1. / U[0];
  double u = U[1] * srho, v = U[2] * srho, w = U[3] * srho;
  double v2s2 = 0.5 * (u * u + v * v + w * w);
  double rho_sp = U[0] / (P.kappaM1 * (U[4] - U[0] * v2s2));
  double s = -(log(rho_sp) + P.kappaM1 * log(U[0]));
  V[0] = (P.kappa - s) * P.sKappaM1 - rho_sp * v2s2;
  V[1] = rho_sp * u; V[2] = rho_sp * v; V[3] = rho_sp * w;
  V[4] = -rho_sp;
}

// Riemann solvers on rotated states (navierstokes/riemann.f90).  lmm is the maximum wave speed
// over the side, used by the LLF-dissipation variants 13-19 and 21.
template <int RS>
__device__ __forceinline__ void riemann_rotated(const KParams& P, const double* L, const double* R, double lmm,
                                                double* F) {
  if constexpr (RS == 0) {  // RiemannSolverCentral :250-272
    double FL[5], FR[5];
    euler_flux_1d(P, L, FL);
    euler_flux_1d(P, R, FR);
    for (int v = 0; v < 5; ++v) F[v] = 0.5 * (FL[v] + FR[v]);
  } else if constexpr (RS == 1) {  // RiemannSolverByRusanov :279-313
    double lm = lambda_max_pair(P, L, R);
    double FL[5], FR[5];
    euler_flux_1d(P, L, FL);
    euler_flux_1d(P, R, FR);
    for (int v = 0; v < 5; ++v) F[v] = 0.5 * ((FL[v] + FR[v]) - lm * (R[v] - L[v]));
  } else if constexpr (RS == 22) {  // RiemannSolverByHLL :320-388
    double FL[5], FR[5];
    euler_flux_1d(P, L, FL);
    euler_flux_1d(P, R, FR);
    double vL[3], vR[3], pL, pR;
    primitive_pv(P, L, vL, pL);
    primitive_pv(P, R, vR, pR);
    double HL = (L[4] + pL) / L[0], HR = (R[4] + pR) / R[0];
    double sqL = sqrt(L[0]), sqR = sqrt(R[0]);
    double HT = (sqL * HL + sqR * HR) / (sqL + sqR);
    double vT = (sqL * vL[0] + sqR * vR[0]) / (sqL + sqR);
    double aT = sqrt((P.kappa - 1.) * (HT - 0.5 * (vT * vT)));
    double ssl = vT - aT, ssr = vT + aT;
    if (ssl >= 0. && ssr > 0.) {
      for (int v = 0; v < 5; ++v) F[v] = FL[v];
    } else if (ssr <= 0. && ssl < 0.) {
      for (int v = 0; v < 5; ++v) F[v] = FR[v];
    } else {
      for (int v = 0; v < 5; ++v) F[v] = (ssr * FL[v] - ssl * FR[v] + ssl * ssr * (R[v] - L[v])) / (ssr - ssl);
    }
  } else if constexpr (RS == 4 || RS == 44 || RS == 33) {
    // RiemannSolver_EntropyStable :874-931 with the dissipation matrices :936-975
    double Fc[5], Dh[5], Rh[5][5];
    es_matrices<RS>(P, L, R, Fc, Dh, Rh);
    double vL[3], vR[3], pL, pR;
    primitive_pv(P, L, vL, pL);
    primitive_pv(P, R, vR, pR);
    double sR = log(pR) - P.kappa * log(R[0]);
    double sL = log(pL) - P.kappa * log(L[0]);
    double rpR = R[0] / pR, rpL = L[0] / pL;
    double jump[5];
    jump[0] = ((P.kappa - sR) / P.kappaM1 - 0.5 * rpR * (vR[0] * vR[0] + vR[1] * vR[1] + vR[2] * vR[2])) -
              ((P.kappa - sL) / P.kappaM1 - 0.5 * rpL * (vL[0] * vL[0] + vL[1] * vL[1] + vL[2] * vL[2]));
    for (int d = 0; d < 3; ++d) jump[1 + d] = rpR * vR[d] - rpL * vL[d];
    jump[4] = -rpR + rpL;
    double diss[5];
#pragma unroll
    for (int c = 0; c < 5; ++c)
      diss[c] = Dh[c] * (Rh[0][c] * jump[0] + Rh[1][c] * jump[1] + Rh[2][c] * jump[2] + Rh[3][c] * jump[3] +
                         Rh[4][c] * jump[4]);
#pragma unroll
    for (int r = 0; r < 5; ++r)
      F[r] = Fc[r] - 0.5 * (Rh[r][0] * diss[0] + Rh[r][1] * diss[1] + Rh[r][2] * diss[2] + Rh[r][3] * diss[3] +
                            Rh[r][4] * diss[4]);
  } else if constexpr (riemann_point_flux<RS>() > 0) {
    // RiemannSolver_VolumeFluxAverage :980-1005
    Hat h;
    volume_flux_1d<riemann_point_flux<RS>()>(P, L, R, F, h);
  } else if constexpr (riemann_llf_point_flux<RS>() > 0) {  // RiemannSolver_VolumeFluxAverage_LLF :1117-1151
    double Fc[5];
    Hat h;
    volume_flux_1d<riemann_llf_point_flux<RS>()>(P, L, R, Fc, h);
    for (int v = 0; v < 5; ++v) F[v] = Fc[v] - 0.5 * lmm * (R[v] - L[v]);
  } else if constexpr (RS == 2) {  // RiemannSolverByHLLC :552-615
    double FL[5], FR[5];
    euler_flux_1d(P, L, FL);
    euler_flux_1d(P, R, FR);
    double vL[3], vR[3], pL, pR;
    primitive_pv(P, L, vL, pL);
    primitive_pv(P, R, vR, pR);
    const double sRL = 1. / L[0], sRR = 1. / R[0];
    const double ssl = vL[0] - sqrt(P.kappa * pL * sRL);
    const double ssr = vR[0] + sqrt(P.kappa * pR * sRR);
    if (ssl >= 0.) {
      for (int v = 0; v < 5; ++v) F[v] = FL[v];
    } else if (ssr <= 0.) {
      for (int v = 0; v < 5; ++v) F[v] = FR[v];
    } else {
      const double smuL = ssl - vL[0], smuR = ssr - vR[0];
      const double sStar = (pR - pL + L[1] * smuL - R[1] * smuR) / (L[0] * smuL - R[0] * smuR);
      const bool left = (ssl <= 0.) && (sStar >= 0.);
      const double* U = left ? L : R;
      const double* FF = left ? FL : FR;
      const double ss = left ? ssl : ssr, smu = left ? smuL : smuR, sr = left ? sRL : sRR, p = left ? pL : pR;
      const double vn = left ? vL[0] : vR[0];
      const double fac = U[0] * smu / (ss - sStar);
      const double Us[5] = {fac, fac * sStar, fac * (U[2] * sr), fac * (U[3] * sr),
                            fac * (U[4] * sr + (sStar - vn) * (sStar + p * sr / smu))};
      for (int v = 0; v < 5; ++v) F[v] = FF[v] + ss * (Us[v] - U[v]);
    }
  } else if constexpr (RS == 23 || RS == 24) {  // RiemannSolverByHLLE :393-462, ...HLLEM :466-547
    double FL[5], FR[5];
    euler_flux_1d(P, L, FL);
    euler_flux_1d(P, R, FR);
    double vL[3], vR[3], pL, pR;
    primitive_pv(P, L, vL, pL);
    primitive_pv(P, R, vR, pR);
    const double beta = sqrt(0.5 * P.kappaM1 / P.kappa);
    const double sRL = 1. / L[0], sRR = 1. / R[0];
    const double aL = sqrt(P.kappa * pL * sRL), aR = sqrt(P.kappa * pR * sRR);
    const double HL = (L[4] + pL) * sRL, HR = (R[4] + pR) * sRR;
    const double sqL = sqrt(L[0]), sqR = sqrt(R[0]);
    const double ssq = 1. / (sqL + sqR);
    double rv[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) rv[d] = (sqR * vR[d] + sqL * vL[d]) * ssq;
    const double rH = (sqR * HR + sqL * HL) * ssq;
    const double absVel = rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2];
    const double rc = sqrt(P.kappaM1 * (rH - 0.5 * absVel));
    const double ssl = fmin(fmin(rv[0] - rc, vL[0] - beta * aL), 0.);
    const double ssr = fmax(fmax(rv[0] + rc, vR[0] + beta * aR), 0.);
    if (ssl >= 0. && ssr > 0.) {
      for (int v = 0; v < 5; ++v) F[v] = FL[v];
    } else if (ssr <= 0. && ssl < 0.) {
      for (int v = 0; v < 5; ++v) F[v] = FR[v];
    } else if constexpr (RS == 23) {
      for (int v = 0; v < 5; ++v) F[v] = (ssr * FL[v] - ssl * FR[v] + ssl * ssr * (R[v] - L[v])) / (ssr - ssl);
    } else {  // HLLEM: anti-diffusion along the Roe-mean entropy and shear waves
      const double rd = sqrt(L[0] * R[0]);
      const double delta = rc / (rc + fabs(0.5 * (ssl + ssr)));
      const double al2 = (R[0] - L[0]) - (pR - pL) / (rc * rc);
      const double al3 = rd * (vR[1] - vL[1]), al4 = rd * (vR[2] - vL[2]);
      const double r2[5] = {1., rv[0], rv[1], rv[2], 0.5 * absVel};
      const double r3[5] = {0., 0., 1., 0., rv[1]};
      const double r4[5] = {0., 0., 0., 1., rv[2]};
      for (int v = 0; v < 5; ++v)
        F[v] = (ssr * FL[v] - ssl * FR[v] +
                ssl * ssr * (R[v] - L[v] - delta * (r2[v] * al2 + r3[v] * al3 + r4[v] * al4))) /
               (ssr - ssl);
    }
  } else if constexpr (RS == 3) {  // RiemannSolverByRoe :742-869 (baseline flux by the volume flux id)
    double FL[5], FR[5];
    euler_flux_1d(P, L, FL);
    euler_flux_1d(P, R, FR);
    const double sRL = 1. / L[0], sRR = 1. / R[0];
    const double vL[3] = {L[1] * sRL, L[2] * sRL, L[3] * sRL};
    const double vR[3] = {R[1] * sRR, R[2] * sRR, R[3] * sRR};
    const double HL = (L[4] + P.kappaM1 * (L[4] - 0.5 * (L[1] * vL[0] + L[2] * vL[1] + L[3] * vL[2]))) * sRL;
    const double HR = (R[4] + P.kappaM1 * (R[4] - 0.5 * (R[1] * vR[0] + R[2] * vR[1] + R[3] * vR[2]))) * sRR;
    const double sqL = sqrt(L[0]), sqR = sqrt(R[0]);
    const double ssq = 1. / (sqL + sqR);
    double rv[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) rv[d] = (sqR * vR[d] + sqL * vL[d]) * ssq;
    const double rH = (sqR * HR + sqL * HL) * ssq;
    const double v2 = rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2];
    const double rc = sqrt(P.kappaM1 * (rH - 0.5 * v2));
    double a1 = rv[0] - rc, a5 = rv[0] + rc;
    const double a2 = rv[0];
    const double r1[5] = {1., a1, rv[1], rv[2], rH - rv[0] * rc};
    const double r2[5] = {1., rv[0], rv[1], rv[2], 0.5 * v2};
    const double r5[5] = {1., a5, rv[1], rv[2], rH + rv[0] * rc};
    double dU[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) dU[v] = R[v] - L[v];
    const double dU6 = dU[4] - (dU[2] - rv[1] * dU[0]) * rv[1] - (dU[3] - rv[2] * dU[0]) * rv[2];
    const double al3 = dU[2] - rv[1] * dU[0];
    const double al4 = dU[3] - rv[2] * dU[0];
    const double al2 = P.kappaM1 / (rc * rc) * (dU[0] * (rH - rv[0] * rv[0]) - dU6 + rv[0] * dU[1]);
    const double al1 = 0.5 / rc * (dU[0] * (rv[0] + rc) - dU[1] - rc * al2);
    const double al5 = dU[0] - al1 - al2;
    double Fc[5];
    Hat h;
    if (P.volumeFlux == 2 || P.volumeFlux == 4) {
      // Kennedy-Gruber baseline (volume flux 4 is paired with the Pirozzoli variant here) with the
      // acoustic speeds replaced by their maximum (consistent kinetic energy dissipation)
      if (P.volumeFlux == 2) volume_flux_1d<2>(P, L, R, Fc, h);
      else volume_flux_1d<8>(P, L, R, Fc, h);
      a1 = fmax(fabs(rv[0] - rc), fabs(rv[0] + rc));
      a5 = a1;
    } else if (P.volumeFlux == 3) {
      volume_flux_1d<3>(P, L, R, Fc, h);
    } else {
#pragma unroll
      for (int v = 0; v < 5; ++v) Fc[v] = 0.5 * (FL[v] + FR[v]);
    }
    const double g1 = al1 * fabs(a1), g2 = al2 * fabs(a2), g3 = al3 * fabs(a2), g4 = al4 * fabs(a2),
                 g5 = al5 * fabs(a5);
    F[0] = Fc[0] - 0.5 * (g1 * r1[0] + g2 * r2[0] + g5 * r5[0]);
    F[1] = Fc[1] - 0.5 * (g1 * r1[1] + g2 * r2[1] + g5 * r5[1]);
    F[2] = Fc[2] - 0.5 * (g1 * r1[2] + g2 * r2[2] + g3 + g5 * r5[2]);
    F[3] = Fc[3] - 0.5 * (g1 * r1[3] + g2 * r2[3] + g4 + g5 * r5[3]);
    F[4] = Fc[4] - 0.5 * (g1 * r1[4] + g2 * r2[4] + g3 * rv[1] + g4 * rv[2] + g5 * r5[4]);
  } else if constexpr (RS == 13) {  // RiemannSolver_EC_LLF :1011-1110
    double Fc[5];
    Hat h;
    volume_flux_1d<10>(P, L, R, Fc, h);
    double vL[3], vR[3], pL, pR;
    primitive_pv(P, L, vL, pL);
    primitive_pv(P, R, vR, pR);
    double sL = log(pL) - P.kappa * log(L[0]);
    double sR = log(pR) - P.kappa * log(R[0]);
    double jump[5];
    jump[0] = -((P.kappa - sL) / P.kappaM1 - 0.5 * L[0] * (vL[0] * vL[0] + vL[1] * vL[1] + vL[2] * vL[2]) / pL) +
              ((P.kappa - sR) / P.kappaM1 - 0.5 * R[0] * (vR[0] * vR[0] + vR[1] * vR[1] + vR[2] * vR[2]) / pR);
    for (int d = 0; d < 3; ++d) jump[1 + d] = -L[0] * vL[d] / pL + R[0] * vR[d] / pR;
    jump[4] = L[0] / pL - R[0] / pR;
    double ra = h.rho, v1 = h.u, v2 = h.v, v3 = h.w, pa = h.p1, aa = h.a, Ha = h.H;
    double rhoea = pa / P.kappaM1 + 0.5 * ra * (v1 * v1 + v2 * v2 + v3 * v3);
    double H[5][5];
    H[0][0] = ra; H[1][1] = ra * v1 * v1 + pa; H[2][2] = ra * v2 * v2 + pa; H[3][3] = ra * v3 * v3 + pa;
    H[4][4] = ra * Ha * Ha - aa * aa * pa / P.kappaM1;
    H[0][1] = H[1][0] = ra * v1; H[0][2] = H[2][0] = ra * v2; H[0][3] = H[3][0] = ra * v3;
    H[0][4] = H[4][0] = rhoea;
    H[1][2] = H[2][1] = ra * v1 * v2; H[1][3] = H[3][1] = ra * v1 * v3; H[1][4] = H[4][1] = ra * v1 * Ha;
    H[2][3] = H[3][2] = ra * v2 * v3; H[2][4] = H[4][2] = ra * v2 * Ha; H[3][4] = H[4][3] = ra * v3 * Ha;
#pragma unroll
    for (int r = 0; r < 5; ++r)
      F[r] = Fc[r] - 0.5 * lmm * (H[r][0] * jump[0] + H[r][1] * jump[1] + H[r][2] * jump[2] + H[r][3] * jump[3] +
                                  H[r][4] * jump[4]);
  } else if constexpr (RS == 16) {  // RiemannSolver_ECKEP_LLF :1153-1209
    double Fc[5];
    Hat h;
    volume_flux_1d<5>(P, L, R, Fc, h);
    double vL[3], vR[3], pL, pR;
    primitive_pv(P, L, vL, pL);
    primitive_pv(P, R, vR, pR);
    double bL = 0.5 * L[0] / pL, bR = 0.5 * R[0] / pR;
    double ra = 0.5 * (R[0] + L[0]);
    double bLN = ln_mean(bL, bR);
    for (int v = 0; v < 4; ++v) F[v] = Fc[v] - 0.5 * lmm * (R[v] - L[v]);
    F[4] = Fc[4] - 0.5 * lmm *
                       ((0.5 / (P.kappaM1 * bLN) + 0.5 * (vL[0] * vR[0] + vL[1] * vR[1] + vL[2] * vR[2])) * (R[0] - L[0]) +
                        ra * (h.u * (vR[0] - vL[0]) + h.v * (vR[1] - vL[1]) + h.w * (vR[2] - vL[2]) +
                              0.5 / P.kappaM1 * (1. / bR - 1. / bL)));
  }
}

template <int RS>
__host__ __device__ constexpr bool riemann_needs_side_max() {
  return RS == 13 || RS == 16 || riemann_llf_point_flux<RS>() > 0;
}

// viscosity law (equation_vars.f90:672-692; flux.f90:470-480)
__device__ __forceinline__ double visc_mu(const KParams& P, double p, double srho) {
  if (P.visc == 0) return P.mu0;
  double T = p * srho / P.R;
  if (P.visc == 1) {
    double Tn = T * P.sTref;
    if (Tn >= P.Ts) return P.mu0 * pow(Tn, P.ExpoSuth) * (1 + P.Ts) / (Tn + P.Ts);
    return P.mu0 * Tn * P.cSuth;
  }
  return P.mu0 * pow(T, P.ExpoPow);
}

// EvalDiffFlux3D at one point (navierstokes/flux.f90:407-517); g* are primitive gradients.
// Only components 1..4 are returned (component 0 is zero): f[0..3] <-> f(2:5).
__device__ __forceinline__ void diff_flux_3d(const KParams& P, const double* U, const double* gX, const double* gY,
                                             const double* gZ, double* f, double* g, double* h) {
  double srho = 1. / U[0];
  double v1 = U[1] * srho, v2 = U[2] * srho, v3 = U[3] * srho;
  double p = P.kappaM1 * (U[4] - 0.5 * (U[1] * v1 + U[2] * v2 + U[3] * v3));
  double muS = visc_mu(P, p, srho);
  double lambda = muS * P.KappasPr;
  double divv = gX[1] + gY[2] + gZ[3];
  double cvTx = P.sKappaM1 * srho * (gX[4] - srho * p * gX[0]);
  double cvTy = P.sKappaM1 * srho * (gY[4] - srho * p * gY[0]);
  double cvTz = P.sKappaM1 * srho * (gZ[4] - srho * p * gZ[0]);
  f[0] = -muS * (2 * gX[1] - P.s23 * divv);
  f[1] = -muS * (gX[2] + gY[1]);
  f[2] = -muS * (gX[3] + gZ[1]);
  f[3] = v1 * f[0] + v2 * f[1] + v3 * f[2] - lambda * cvTx;
  g[0] = f[1];
  g[1] = -muS * (2 * gY[2] - P.s23 * divv);
  g[2] = -muS * (gY[3] + gZ[2]);
  g[3] = v1 * g[0] + v2 * g[1] + v3 * g[2] - lambda * cvTy;
  h[0] = f[2];
  h[1] = g[2];
  h[2] = -muS * (2 * gZ[3] - P.s23 * divv);
  h[3] = v1 * h[0] + v2 * h[1] + v3 * h[2] - lambda * cvTz;
}

// Lifting variable (EvalLiftingVolumeFlux, flux.f90:641-668): 1 cons, 2 prim, 3 entropy
// (ConsToEntropyVec, equation_vars.f90:397-429).
__device__ __forceinline__ void lifting_var(const KParams& P, const double* U, double* V) {
  if (P.lifting_var == 1) {
    for (int v = 0; v < 5; ++v) V[v] = U[v];
  } else if (P.lifting_var == 2) {
    double s = 1. / U[0];
    V[0] = U[0]; V[1] = U[1] * s; V[2] = U[2] * s; V[3] = U[3] * s;
    V[4] = P.kappaM1 * (U[4] - 0.5 * (U[1] * V[1] + U[2] * V[2] + U[3] * V[3]));
  } else {
    cons_to_entropy_ns(P, U, V);
  }
}

// ConvertToGradPrimVec at one point (equation_vars.f90:571-647)
__device__ __forceinline__ void to_grad_prim(const KParams& P, const double* U, double* g) {
  if (P.lifting_var == 1) {
    double sRho = 1. / U[0];
    double u = U[1] * sRho, v = U[2] * sRho, w = U[3] * sRho;
    double gi1 = g[0], gi5 = g[4];
    double gu = sRho * (g[1] - g[0] * u), gv = sRho * (g[2] - g[0] * v), gw = sRho * (g[3] - g[0] * w);
    g[1] = gu; g[2] = gv; g[3] = gw;
    g[4] = P.kappaM1 * (gi5 - (0.5 * gi1 * (u * u + v * v + w * w) + (U[1] * gu + U[2] * gv + U[3] * gw)));
  } else if (P.lifting_var == 3) {
    double sRho = 1. / U[0];
    double u = U[1] * sRho, v = U[2] * sRho, w = U[3] * sRho;
    double Ekin = 0.5 * (U[1] * u + U[2] * v + U[3] * w);
    double p = P.kappaM1 * (U[4] - Ekin);
    double rho_sp = U[0] / p;
    double p_srho = p * sRho;
    double gi1 = g[0], gi5 = g[4];
    double gu = p_srho * (g[1] + u * g[4]);
    double gv = p_srho * (g[2] + v * g[4]);
    double gw = p_srho * (g[3] + w * g[4]);
    g[0] = U[0] * gi1 - gi5 * (Ekin - p * P.sKappaM1) + rho_sp * (U[1] * gu + U[2] * gv + U[3] * gw);
    g[1] = gu; g[2] = gv; g[3] = gw;
    g[4] = p_srho * (g[0] + p * gi5);
  }
}

}  // namespace fluxo
