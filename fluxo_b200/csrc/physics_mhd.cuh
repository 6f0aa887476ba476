// Ideal / resistive MHD with GLM divergence cleaning (9 variables: rho, rho*v, E, B, psi): point
// physics in FP64 for the sm_100a kernels.  Formulas follow the reference's equation/mhd/* so
// that results agree with it to roundoff; each function names the routine it implements.
#pragma once
#include "common.cuh"
#include "physics_ns.cuh"

namespace fluxo {
namespace mhd {

constexpr int NV = 9;

// EvalAdvectionFlux1D, mhd/flux.f90:391-442 (rotated frame, GLM terms)
__device__ __forceinline__ void flux_1d(const KParams& P, double ch, const double* U, double* F) {
  const double srho = 1. / U[0];
  const double v1 = U[1] * srho, v2 = U[2] * srho, v3 = U[3] * srho;
  const double b1 = U[5], b2 = U[6], b3 = U[7];
  const double Et = U[4] - P.s2mu_0 * U[8] * U[8];
  const double vb = b1 * v1 + b2 * v2 + b3 * v3;
  const double pt = P.kappaM1 * (Et - 0.5 * U[0] * (v1 * v1 + v2 * v2 + v3 * v3)) -
                    P.kappaM2 * P.s2mu_0 * (b1 * b1 + b2 * b2 + b3 * b3);
  F[0] = U[1];
  F[1] = U[1] * v1 + pt - P.smu_0 * b1 * b1;
  F[2] = U[1] * v2 - P.smu_0 * b1 * b2;
  F[3] = U[1] * v3 - P.smu_0 * b1 * b3;
  F[4] = (Et + pt) * v1 - P.smu_0 * b1 * vb + P.smu_0 * ch * b1 * U[8];
  F[5] = ch * U[8];
  F[6] = v1 * b2 - b1 * v2;
  F[7] = v1 * b3 - b1 * v3;
  F[8] = ch * b1;
}

// ConsToPrim, mhd/equation_vars.f90:229-251 (gas pressure: magnetic and psi energy removed)
__device__ __forceinline__ void cons_to_prim(const KParams& P, const double* U, double* Q) {
  const double s = 1. / U[0];
  Q[0] = U[0];
  Q[1] = U[1] * s; Q[2] = U[2] * s; Q[3] = U[3] * s;
  Q[4] = P.kappaM1 * (U[4] - 0.5 * (U[1] * Q[1] + U[2] * Q[2] + U[3] * Q[3]) -
                      P.s2mu_0 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7] + U[8] * U[8]));
#pragma unroll
  for (int v = 5; v < 9; ++v) Q[v] = U[v];
}

// ConsToEntropy, mhd/equation_vars.f90:330-361
__device__ __forceinline__ void cons_to_entropy(const KParams& P, const double* U, double* W) {
  const double srho = 1. / U[0];
  const double u = U[1] * srho, v = U[2] * srho, w = U[3] * srho;
  const double v2s2 = 0.5 * (u * u + v * v + w * w);
  const double rho_sp = U[0] / (P.kappaM1 * (U[4] - U[0] * v2s2 -
                                             P.s2mu_0 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7] + U[8] * U[8])));
  const double s = -(log(rho_sp) + P.kappaM1 * log(U[0]));  // -log(rho_sp * rho^(kappa-1))
  W[0] = (P.kappa - s) * P.sKappaM1 - rho_sp * v2s2;
  W[1] = rho_sp * u; W[2] = rho_sp * v; W[3] = rho_sp * w;
  W[4] = -rho_sp;
#pragma unroll
  for (int z = 5; z < 9; ++z) W[z] = rho_sp * U[z];
}

// EntropyToCons, mhd/equation_vars.f90:366-401
__device__ __forceinline__ void entropy_to_cons(const KParams& P, const double* W, double* U) {
  const double rho_sp = -W[4];
  const double p_srho = 1. / rho_sp;
  const double u = W[1] * p_srho, v = W[2] * p_srho, w = W[3] * p_srho;
  const double v2s2 = 0.5 * (u * u + v * v + w * w);
  const double s = P.kappa - ((W[0] + rho_sp * v2s2) * P.kappaM1);
  U[0] = pow(exp(-s) * p_srho, P.sKappaM1);
  U[1] = u * U[0];
  U[2] = v * U[0];
  U[3] = w * U[0];
#pragma unroll
  for (int z = 5; z < 9; ++z) U[z] = W[z] * p_srho;
  U[4] = U[0] * (P.sKappaM1 * p_srho + v2s2) + P.s2mu_0 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7] + U[8] * U[8]);
}

// FastestWave1D, mhd/equation_vars.f90:663-684 (primitive input)
__device__ __forceinline__ double fastest_wave_1d(const KParams& P, const double* Q) {
  const double sRho = 1. / Q[0];
  const double c2 = P.kappa * Q[4] * sRho;
  const double ca2 = Q[5] * Q[5] * sRho * P.smu_0;
  const double va2 = (Q[6] * Q[6] + Q[7] * Q[7]) * sRho * P.smu_0 + ca2;
  const double astar = sqrt((c2 + va2) * (c2 + va2) - 4. * c2 * ca2);
  return sqrt(0.5 * (c2 + va2 + astar));
}

// FastestWave1D_Roe, mhd/equation_vars.f90:717-763
__device__ __forceinline__ void fastest_wave_1d_roe(const KParams& P, const double* UL, const double* UR,
                                                    const double* QL, const double* QR, double& RoeVelx,
                                                    double& cfRoe) {
  const double sqL = sqrt(QL[0]), sqR = sqrt(QR[0]);
  const double sS = 1. / (sqL + sqR);
  const double RL = sqL * sS, RR = sqR * sS;
  const double ptL = QL[4] + P.s2mu_0 * (QL[5] * QL[5] + QL[6] * QL[6] + QL[7] * QL[7]);
  const double ptR = QR[4] + P.s2mu_0 * (QR[5] * QR[5] + QR[6] * QR[6] + QR[7] * QR[7]);
  const double sRhoRoe = 1. / (sqL * sqR);
  double vR[3], BR[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { vR[d] = RL * QL[1 + d] + RR * QR[1 + d]; BR[d] = RL * QR[5 + d] + RR * QL[5 + d]; }
  const double HL = (UL[4] + ptL) / QL[0], HR = (UR[4] + ptR) / QR[0];
  const double RoeH = RL * HL + RR * HR;
  const double d0 = QL[5] - QR[5], d1 = QL[6] - QR[6], d2 = QL[7] - QR[7];
  const double XX = 0.5 * (d0 * d0 + d1 * d1 + d2 * d2) * (sS * sS);
  const double va2 = (BR[0] * BR[0] + BR[1] * BR[1] + BR[2] * BR[2]) * P.smu_0 * sRhoRoe;
  const double c2 = (2. - P.kappa) * XX +
                    (P.kappa - 1) * (RoeH - 0.5 * (vR[0] * vR[0] + vR[1] * vR[1] + vR[2] * vR[2]) - va2);
  const double ca2 = BR[0] * BR[0] * P.smu_0 * sRhoRoe;
  const double astar = sqrt((c2 + va2) * (c2 + va2) - 4. * c2 * ca2);
  cfRoe = sqrt(0.5 * (c2 + va2 + astar));
  RoeVelx = vR[0];
}

// StandardDGFlux (Riemann 0), mhd/flux_average.f90:421-484
__device__ __forceinline__ void standard_dg_flux(const KParams& P, double ch, const double* UL, const double* UR,
                                                 double* F) {
  const double EL = UL[4] - 0.5 * P.smu_0 * UL[8] * UL[8], ER = UR[4] - 0.5 * P.smu_0 * UR[8] * UR[8];
  const double sL = 1. / UL[0], sR = 1. / UR[0];
  const double v1L = sL * UL[1], v2L = sL * UL[2], v3L = sL * UL[3];
  const double v1R = sR * UR[1], v2R = sR * UR[2], v3R = sR * UR[3];
  const double b1L = UL[5], b2L = UL[6], b3L = UL[7], b1R = UR[5], b2R = UR[6], b3R = UR[7];
  const double bbL = b1L * b1L + b2L * b2L + b3L * b3L, bbR = b1R * b1R + b2R * b2R + b3R * b3R;
  const double ptL = P.kappaM1 * (EL - 0.5 * (UL[1] * v1L + UL[2] * v2L + UL[3] * v3L)) - P.kappaM2 * P.s2mu_0 * bbL;
  const double ptR = P.kappaM1 * (ER - 0.5 * (UR[1] * v1R + UR[2] * v2R + UR[3] * v3R)) - P.kappaM2 * P.s2mu_0 * bbR;
  const double vbL = v1L * b1L + v2L * b2L + v3L * b3L, vbR = v1R * b1R + v2R * b2R + v3R * b3R;
  const double qL = UL[0] * v1L, qR = UR[0] * v1R;
  F[0] = 0.5 * (qL + qR);
  F[1] = 0.5 * (qL * v1L + qR * v1R + (ptL + ptR) - P.smu_0 * (b1L * b1L + b1R * b1R));
  F[2] = 0.5 * (qL * v2L + qR * v2R - P.smu_0 * (b2L * b1L + b2R * b1R));
  F[3] = 0.5 * (qL * v3L + qR * v3R - P.smu_0 * (b3L * b1L + b3R * b1R));
  F[4] = 0.5 * ((EL + ptL) * v1L + (ER + ptR) * v1R - P.smu_0 * (b1L * vbL + b1R * vbR));
  F[6] = 0.5 * (v1L * b2L - b1L * v2L + v1R * b2R - b1R * v2R);
  F[7] = 0.5 * (v1L * b3L - b1L * v3L + v1R * b3R - b1R * v3R);
  F[4] = F[4] + 0.5 * P.smu_0 * ch * (b1L * UL[8] + b1R * UR[8]);
  F[5] = 0.5 * ch * (UL[8] + UR[8]);
  F[8] = 0.5 * ch * (b1L + b1R);
}

// EntropyAndKinEnergyConservingFlux_Derigs (1D), mhd/flux_average.f90:660-751
__device__ __forceinline__ void derigs_flux(const KParams& P, double ch, const double* UL, const double* UR, double* F) {
  const double smu0 = P.smu_0;
  const double EL = UL[4] - 0.5 * smu0 * UL[8] * UL[8], ER = UR[4] - 0.5 * smu0 * UR[8] * UR[8];
  double vL[3], vR[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { vL[d] = UL[1 + d] / UL[0]; vR[d] = UR[1 + d] / UR[0]; }
  const double v2L = vL[0] * vL[0] + vL[1] * vL[1] + vL[2] * vL[2], v2R = vR[0] * vR[0] + vR[1] * vR[1] + vR[2] * vR[2];
  const double B2L = UL[5] * UL[5] + UL[6] * UL[6] + UL[7] * UL[7], B2R = UR[5] * UR[5] + UR[6] * UR[6] + UR[7] * UR[7];
  const double pL = P.kappaM1 * (EL - 0.5 * (UL[0] * v2L + smu0 * B2L));
  const double pR = P.kappaM1 * (ER - 0.5 * (UR[0] * v2R + smu0 * B2R));
  const double bL = 0.5 * UL[0] / pL, bR = 0.5 * UR[0] / pR;
  const double rhoLN = ln_mean(UL[0], UR[0]);
  const double betaLN = ln_mean(bL, bR);
  double vA[3], BA[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { vA[d] = 0.5 * (vL[d] + vR[d]); BA[d] = 0.5 * (UL[5 + d] + UR[5 + d]); }
  const double v1B2 = 0.5 * (vL[0] * B2L + vR[0] * B2R);
  const double vBA = 0.5 * ((vL[0] * UL[5] + vL[1] * UL[6] + vL[2] * UL[7]) + (vR[0] * UR[5] + vR[1] * UR[6] + vR[2] * UR[7]));
  const double pTilde = 0.5 * ((UL[0] + UR[0]) / (bL + bR) + smu0 * 0.5 * (B2L + B2R));
  const double psiA = 0.5 * (UL[8] + UR[8]);
  F[0] = rhoLN * vA[0];
  F[1] = F[0] * vA[0] - smu0 * BA[0] * BA[0] + pTilde;
  F[2] = F[0] * vA[1] - smu0 * BA[0] * BA[1];
  F[3] = F[0] * vA[2] - smu0 * BA[0] * BA[2];
  F[6] = vA[0] * BA[1] - BA[0] * vA[1];
  F[7] = vA[0] * BA[2] - BA[0] * vA[2];
  F[5] = ch * psiA;
  F[8] = ch * BA[0];
  F[4] = F[0] * 0.5 * (P.sKappaM1 / betaLN - 0.5 * (v2L + v2R)) + (vA[0] * F[1] + vA[1] * F[2] + vA[2] * F[3]) +
         smu0 * ((BA[0] * F[5] + BA[1] * F[6] + BA[2] * F[7]) - 0.5 * v1B2 + BA[0] * vBA + F[8] * psiA -
                 ch * 0.5 * (UL[8] * UL[5] + UR[8] * UR[5]));
}

// EntropyAndKinEnergyConservingFlux_FloGor (1D), mhd/flux_average.f90:855-960
__device__ __forceinline__ void flogor_flux(const KParams& P, double ch, const double* UL, const double* UR, double* F) {
  const double smu0 = P.smu_0;
  const double EL = UL[4] - 0.5 * smu0 * UL[8] * UL[8], ER = UR[4] - 0.5 * smu0 * UR[8] * UR[8];
  const double sL = 1. / UL[0], sR = 1. / UR[0];
  double vL[3], vR[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { vL[d] = UL[1 + d] * sL; vR[d] = UR[1 + d] * sR; }
  const double v2L = vL[0] * vL[0] + vL[1] * vL[1] + vL[2] * vL[2], v2R = vR[0] * vR[0] + vR[1] * vR[1] + vR[2] * vR[2];
  const double B2L = UL[5] * UL[5] + UL[6] * UL[6] + UL[7] * UL[7], B2R = UR[5] * UR[5] + UR[6] * UR[6] + UR[7] * UR[7];
  const double pL = P.kappaM1 * (EL - 0.5 * (UL[0] * v2L + smu0 * B2L));
  const double pR = P.kappaM1 * (ER - 0.5 * (UR[0] * v2R + smu0 * B2R));
  const double ieL = pL * sL * P.sKappaM1, ieR = pR * sR * P.sKappaM1;
  const double rhoLN = ln_mean(UL[0], UR[0]);
  double vA[3], BA[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { vA[d] = 0.5 * (vL[d] + vR[d]); BA[d] = 0.5 * (UL[5 + d] + UR[5 + d]); }
  const double v2Z = vL[0] * vR[0] + vL[1] * vR[1] + vL[2] * vR[2];
  const double B2Z = UL[5] * UR[5] + UL[6] * UR[6] + UL[7] * UR[7];
  const double pA = 0.5 * (pL + pR);
  const double* BL = UL + 5;
  const double* BR = UR + 5;
  auto zip = [](double a, double b, double c, double d) { return 0.5 * (a * d + b * c); };
  F[0] = rhoLN * vA[0];
  F[1] = F[0] * vA[0] + pA + P.s2mu_0 * B2Z - smu0 * zip(BL[0], BR[0], BL[0], BR[0]);
  F[2] = F[0] * vA[1] - smu0 * zip(BL[0], BR[0], BL[1], BR[1]);
  F[3] = F[0] * vA[2] - smu0 * zip(BL[0], BR[0], BL[2], BR[2]);
  F[4] = F[0] * (0.5 * v2Z + ieL * ieR / ln_mean(ieL, ieR)) + zip(pL, pR, vL[0], vR[0]) +
         smu0 * (zip(vL[0] * BL[1], vR[0] * BR[1], BL[1], BR[1]) - zip(vL[1] * BL[0], vR[1] * BR[0], BL[1], BR[1]) +
                 zip(vL[0] * BL[2], vR[0] * BR[2], BL[2], BR[2]) - zip(vL[2] * BL[0], vR[2] * BR[0], BL[2], BR[2]) +
                 ch * zip(BL[0], BR[0], UL[8], UR[8]));
  F[5] = ch * 0.5 * (UL[8] + UR[8]);
  F[8] = ch * BA[0];
  F[6] = 0.5 * ((vL[0] * BL[1] - vL[1] * BL[0]) + (vR[0] * BR[1] - vR[1] * BR[0]));
  F[7] = 0.5 * ((vL[0] * BL[2] - vL[2] * BL[0]) + (vR[0] * BR[2] - vR[2] * BR[0]));
}

// jump of the entropy variables and the pressures / betas of both states (mhd/riemann.f90:1059-1089)
__device__ __forceinline__ void entropy_jump(const KParams& P, const double* UL, const double* UR, double& pL,
                                             double& pR, double& bL, double& bR, double* Vj) {
  const double EL = UL[4] - P.s2mu_0 * UL[8] * UL[8], ER = UR[4] - P.s2mu_0 * UR[8] * UR[8];
  const double sL = 1. / UL[0], sR = 1. / UR[0];
  double uL[3], uR[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { uL[d] = UL[1 + d] * sL; uR[d] = UR[1 + d] * sR; }
  const double u2L = uL[0] * uL[0] + uL[1] * uL[1] + uL[2] * uL[2], u2R = uR[0] * uR[0] + uR[1] * uR[1] + uR[2] * uR[2];
  const double B2L = UL[5] * UL[5] + UL[6] * UL[6] + UL[7] * UL[7], B2R = UR[5] * UR[5] + UR[6] * UR[6] + UR[7] * UR[7];
  pL = P.kappaM1 * (EL - 0.5 * (UL[0] * u2L + P.smu_0 * B2L));
  pR = P.kappaM1 * (ER - 0.5 * (UR[0] * u2R + P.smu_0 * B2R));
  bL = 0.5 * UL[0] / pL;
  bR = 0.5 * UR[0] / pR;
  Vj[0] = (P.kappa * log(UR[0] * sL) - log(pR / pL)) * P.sKappaM1 - (bR * u2R - bL * u2L);
#pragma unroll
  for (int d = 0; d < 3; ++d) Vj[1 + d] = 2.0 * (bR * uR[d] - bL * uL[d]);
  Vj[4] = -2.0 * (bR - bL);
#pragma unroll
  for (int z = 5; z < 9; ++z) Vj[z] = 2.0 * (bR * UR[z] - bL * UL[z]);
}

// EntropyStableByLLF (Riemann 10: Derigs, 13: FloGor), mhd/riemann.f90:1027-1211
template <bool FLOGOR>
__device__ __forceinline__ void es_llf(const KParams& P, double ch, const double* UL, const double* UR, double* F) {
  double Vj[9], pL, pR, bL, bR;
  entropy_jump(P, UL, UR, pL, pR, bL, bR, Vj);
  const double sL = 1. / UL[0], sR = 1. / UR[0];
  double uL[3], uR[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { uL[d] = UL[1 + d] * sL; uR[d] = UR[1 + d] * sR; }
  const double u2L = uL[0] * uL[0] + uL[1] * uL[1] + uL[2] * uL[2], u2R = uR[0] * uR[0] + uR[1] * uR[1] + uR[2] * uR[2];
  const double B2L = UL[5] * UL[5] + UL[6] * UL[6] + UL[7] * UL[7], B2R = UR[5] * UR[5] + UR[6] * UR[6] + UR[7] * UR[7];
  const double rhoLN = ln_mean(UL[0], UR[0]);
  const double sbetaLN = 1. / ln_mean(bL, bR);
  double uA[3], BA[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { uA[d] = 0.5 * (uL[d] + uR[d]); BA[d] = 0.5 * (UL[5 + d] + UR[5 + d]); }
  const double u2A = 0.5 * (u2L + u2R), B2A = 0.5 * (B2L + B2R);
  const double pA = 0.5 * (UL[0] + UR[0]) / (bL + bR);
  const double psiA = 0.5 * (UL[8] + UR[8]);
  if constexpr (FLOGOR) flogor_flux(P, ch, UL, UR, F);
  else derigs_flux(P, ch, UL, UR, F);
  const double pLN = 0.5 * rhoLN * sbetaLN;
  const double srhoLN = 1. / rhoLN;
  const double a2A = P.kappa * pA * srhoLN, va2A = B2A * srhoLN, ca2A = BA[0] * BA[0] * srhoLN;
  const double cfA = sqrt(0.5 * ((a2A + va2A) + sqrt((a2A + va2A) * (a2A + va2A) - 4.0 * a2A * ca2A)));
  const double LM = 0.5 * (fabs(uA[0]) + cfA);
  const double uA2 = uA[0] * uA[0] + uA[1] * uA[1] + uA[2] * uA[2];
  const double Eavg = pLN * P.sKappaM1 + 0.5 * rhoLN * (2.0 * uA2 - u2A);
  double H[5][5];
  H[0][0] = rhoLN; H[1][0] = rhoLN * uA[0]; H[2][0] = rhoLN * uA[1]; H[3][0] = rhoLN * uA[2]; H[4][0] = Eavg;
  H[0][1] = H[1][0]; H[1][1] = H[1][0] * uA[0] + pA; H[2][1] = H[2][0] * uA[0]; H[3][1] = H[3][0] * uA[0];
  H[4][1] = (Eavg + pA) * uA[0];
  H[0][2] = H[2][0]; H[1][2] = H[2][1]; H[2][2] = H[2][0] * uA[1] + pA; H[3][2] = H[3][0] * uA[1];
  H[4][2] = (Eavg + pA) * uA[1];
  H[0][3] = H[3][0]; H[1][3] = H[3][1]; H[2][3] = H[3][2]; H[3][3] = H[3][0] * uA[2] + pA;
  H[4][3] = (Eavg + pA) * uA[2];
  H[0][4] = H[4][0]; H[1][4] = H[4][1]; H[2][4] = H[4][2]; H[3][4] = H[4][3];
  const double tau = 1. / (bL + bR);
  H[4][4] = (pLN * pLN * P.sKappaM1 + Eavg * Eavg) * srhoLN + uA2 * pA +
            tau * ((BA[0] * BA[0] + BA[1] * BA[1] + BA[2] * BA[2]) + psiA * psiA);
#pragma unroll
  for (int r = 0; r < 4; ++r)
    F[r] = F[r] - LM * (H[r][0] * Vj[0] + H[r][1] * Vj[1] + H[r][2] * Vj[2] + H[r][3] * Vj[3] + H[r][4] * Vj[4]);
  const double s5 = H[0][4] * Vj[0] + H[1][4] * Vj[1] + H[2][4] * Vj[2] + H[3][4] * Vj[3] + H[4][4] * Vj[4];
  F[4] = F[4] - LM * (s5 + tau * ((BA[0] * Vj[5] + BA[1] * Vj[6] + BA[2] * Vj[7]) + psiA * Vj[8]));
#pragma unroll
  for (int d = 0; d < 3; ++d) F[5 + d] = F[5 + d] - (LM * tau) * (BA[d] * Vj[4] + Vj[5 + d]);
  F[8] = F[8] - (LM * tau) * (psiA * Vj[4] + Vj[8]);
}

// The mean state of the entropy-stable 9-wave solvers (Riemann 14 Derigs, 15 FloGor;
// EntropyStableDerigsFlux_VolFluxAndDissipMatrices mhd/riemann.f90:1287-1622 and the FloGor variant
// :1695-2042): the scalars of the right eigenvectors and the diagonal D (with the entropy scaling T).
// The eigenvector matrix is never stored: wave9_column forms column c (mhd/riemann.f90:1497-1586) from
// these scalars where it is used, which keeps the solver's live registers to a few dozen doubles.
struct Wave9 {
  double rhoLN, sqRho, sqRhoA, alf, als, cf, cs, be2, be3, sg, abeta, u2A, psiA, BA0;
  double uA[3];
  double psiSp, psiSm, psiFp, psiFm;
  double D[9];
};

// central flux F and the mean state W (the jump of the entropy variables in Vj)
template <bool FLOGOR>
__device__ __forceinline__ void wave9_setup(const KParams& P, double ch, const double* UL, const double* UR,
                                            double* F, double* Vj, Wave9& W) {
  double pL, pR, bL, bR;
  entropy_jump(P, UL, UR, pL, pR, bL, bR, Vj);
  const double sL = 1. / UL[0], sR = 1. / UR[0];
  double uL[3], uR[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { uL[d] = UL[1 + d] * sL; uR[d] = UR[1 + d] * sR; }
  const double rhoLN = ln_mean(UL[0], UR[0]);
  const double sbetaLN = 1. / ln_mean(bL, bR);
  double uA[3], BA[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { uA[d] = 0.5 * (uL[d] + uR[d]); BA[d] = 0.5 * (UL[5 + d] + UR[5 + d]); }
  const double betaA = 0.5 * (bL + bR);
  const double pA = 0.5 * (UL[0] + UR[0]) / (bL + bR);
  const double psiA = 0.5 * (UL[8] + UR[8]);
  if constexpr (FLOGOR) {
    flogor_flux(P, ch, UL, UR, F);
  } else {  // central flux as the Derigs dissipation routine writes it (:1346-1366)
    const double u2L = uL[0] * uL[0] + uL[1] * uL[1] + uL[2] * uL[2], u2R = uR[0] * uR[0] + uR[1] * uR[1] + uR[2] * uR[2];
    const double B2L = UL[5] * UL[5] + UL[6] * UL[6] + UL[7] * UL[7], B2R = UR[5] * UR[5] + UR[6] * UR[6] + UR[7] * UR[7];
    const double u2Av = 0.5 * (u2L + u2R), B2A = 0.5 * (B2L + B2R);
    const double u1B2 = 0.5 * (uL[0] * B2L + uR[0] * B2R);
    const double uBA = 0.5 * ((uL[0] * UL[5] + uL[1] * UL[6] + uL[2] * UL[7]) + (uR[0] * UR[5] + uR[1] * UR[6] + uR[2] * UR[7]));
    const double pTilde = pA + P.s2mu_0 * B2A;
    F[0] = rhoLN * uA[0];
    F[1] = F[0] * uA[0] - P.smu_0 * BA[0] * BA[0] + pTilde;
    F[2] = F[0] * uA[1] - P.smu_0 * BA[0] * BA[1];
    F[3] = F[0] * uA[2] - P.smu_0 * BA[0] * BA[2];
    F[6] = uA[0] * BA[1] - BA[0] * uA[1];
    F[7] = uA[0] * BA[2] - BA[0] * uA[2];
    F[5] = ch * psiA;
    F[8] = ch * BA[0];
    F[4] = F[0] * 0.5 * (P.sKappaM1 * sbetaLN - u2Av) + (uA[0] * F[1] + uA[1] * F[2] + uA[2] * F[3]) +
           P.smu_0 * ((BA[0] * F[5] + BA[1] * F[6] + BA[2] * F[7]) - 0.5 * u1B2 + BA[0] * uBA + F[8] * psiA -
                      ch * 0.5 * (UL[5] * UL[8] + UR[5] * UR[8]));
  }
  const double rhoA = 0.5 * (UL[0] + UR[0]);
  const double pLN = 0.5 * rhoLN * sbetaLN;
  const double u2A = uL[0] * uR[0] + uL[1] * uR[1] + uL[2] * uR[2];
  const double aA = sqrt(P.kappa * pA / rhoLN);
  const double aLN = sqrt(P.kappa * pLN / rhoLN);
  const double abeta = sqrt(0.5 * P.kappa / betaA);
  const double sqRho = sqrt(rhoLN), sqRhoA = sqrt(rhoA);
  const double bb1 = BA[0] / sqRho, bb2 = BA[1] / sqRho, bb3 = BA[2] / sqRho;
  const double bbA = sqrt(bb1 * bb1 + bb2 * bb2 + bb3 * bb3);
  const double aabb = aA * aA + bbA * bbA;
  const double ca = fabs(bb1);
  double xx = aabb * aabb - 4.0 * aA * aA * bb1 * bb1;
  if (xx < 0.0) xx = 0.0;
  double xxx = aabb + sqrt(xx);
  const double cf = sqrt(0.5 * xxx);
  xxx = aabb - sqrt(xx);
  if (xxx < 0.0) xxx = 0.0;
  const double cs = sqrt(0.5 * xxx);
  double bperp = sqrt(bb2 * bb2 + bb3 * bb3), be2, be3;
  if (bperp > 1.0E-14) { be2 = bb2 / bperp; be3 = bb3 / bperp; }
  else { bperp = 0.0; be2 = 1.0 / sqrt(2.0); be3 = 1.0 / sqrt(2.0); }
  xx = 0.0;
  if ((cf * cf - cs * cs) > 0.0) xx = (aA * aA - cs * cs) / (cf * cf - cs * cs);
  const double alf = (xx > 0.0) ? sqrt(xx) : 0.0;
  xx = 0.0;
  if ((cf * cf - cs * cs) > 0.0) xx = (cf * cf - aA * aA) / (cf * cf - cs * cs);
  const double als = (xx > 0.0) ? sqrt(xx) : 0.0;
  const double sg = copysign(1.0, bb1);  // SIGN(1.,bb1A)
  const double t23 = uA[1] * be2 + uA[2] * be3;
  const double psiSp = 0.5 * als * rhoLN * u2A - abeta * alf * rhoLN * bperp + als * rhoLN * aLN * aLN * P.sKappaM1 +
                       als * cs * rhoLN * uA[0] + alf * cf * rhoLN * sg * t23;
  const double psiSm = 0.5 * als * rhoLN * u2A - abeta * alf * rhoLN * bperp + als * rhoLN * aLN * aLN * P.sKappaM1 -
                       als * cs * rhoLN * uA[0] - alf * cf * rhoLN * sg * t23;
  const double psiFp = 0.5 * alf * rhoLN * u2A + abeta * als * rhoLN * bperp + alf * rhoLN * aLN * aLN * P.sKappaM1 +
                       alf * cf * rhoLN * uA[0] - als * cs * rhoLN * sg * t23;
  const double psiFm = 0.5 * alf * rhoLN * u2A + abeta * als * rhoLN * bperp + alf * rhoLN * aLN * aLN * P.sKappaM1 -
                       alf * cf * rhoLN * uA[0] + als * cs * rhoLN * sg * t23;
  W.rhoLN = rhoLN; W.sqRho = sqRho; W.sqRhoA = sqRhoA; W.alf = alf; W.als = als; W.cf = cf; W.cs = cs;
  W.be2 = be2; W.be3 = be3; W.sg = sg; W.abeta = abeta; W.u2A = u2A; W.psiA = psiA; W.BA0 = BA[0];
#pragma unroll
  for (int d = 0; d < 3; ++d) W.uA[d] = uA[d];
  W.psiSp = psiSp; W.psiSm = psiSm; W.psiFp = psiFp; W.psiFm = psiFm;
  const double ratio = pR * UR[0] / (pL * UL[0]);
  const double phi = sqrt(fabs(1.0 - ratio) / (1.0 + ratio));
  const double LM = fmax(fabs(uA[0] + cf), fabs(uA[0] - cf));
  const double wave[9] = {uA[0] + cf, uA[0] + ca, uA[0] + cs, uA[0] + ch, uA[0], uA[0] - ch, uA[0] - cs, uA[0] - ca,
                          uA[0] - cf};
  const double T1 = 0.5 / P.kappa / rhoLN, T2 = 0.25 / betaA / rhoLN / rhoLN, T4 = 0.25 / betaA,
               T5 = rhoLN * P.kappaM1 / P.kappa;
  const double Tm[9] = {T1, T2, T1, T4, T5, T4, T1, T2, T1};
#pragma unroll
  for (int c = 0; c < 9; ++c) W.D[c] = ((1. - phi) * fabs(wave[c]) + phi * LM) * Tm[c];
}

// column c of the right eigenvectors (c = 0..8 resolved at compile time under unrolled loops)
__device__ __forceinline__ void wave9_column(const Wave9& W, int c, double* col) {
  const double rhoLN = W.rhoLN, alf = W.alf, als = W.als, cf = W.cf, cs = W.cs, be2 = W.be2, be3 = W.be3,
               sg = W.sg, abeta = W.abeta, sqRho = W.sqRho, sqRhoA = W.sqRhoA;
  const double* uA = W.uA;
  switch (c) {
    case 0: {
      const double v[9] = {alf * rhoLN, alf * rhoLN * (uA[0] + cf), rhoLN * (alf * uA[1] - als * cs * be2 * sg),
                           rhoLN * (alf * uA[2] - als * cs * be3 * sg), W.psiFp, 0.0, als * abeta * be2 * sqRho,
                           als * abeta * be3 * sqRho, 0.0};
      for (int r = 0; r < 9; ++r) col[r] = v[r];
      return;
    }
    case 1: {
      const double v[9] = {0.0, 0.0, rhoLN * sqRhoA * be3, -rhoLN * sqRhoA * be2,
                           -rhoLN * sqRhoA * (be2 * uA[2] - be3 * uA[1]), 0.0, -rhoLN * be3, rhoLN * be2, 0.0};
      for (int r = 0; r < 9; ++r) col[r] = v[r];
      return;
    }
    case 2: {
      const double v[9] = {als * rhoLN, als * rhoLN * (uA[0] + cs), rhoLN * (als * uA[1] + alf * cf * be2 * sg),
                           rhoLN * (als * uA[2] + alf * cf * be3 * sg), W.psiSp, 0.0, -alf * abeta * be2 * sqRho,
                           -alf * abeta * be3 * sqRho, 0.0};
      for (int r = 0; r < 9; ++r) col[r] = v[r];
      return;
    }
    case 3: {
      const double v[9] = {0.0, 0.0, 0.0, 0.0, W.BA0 + W.psiA, 1.0, 0.0, 0.0, 1.0};
      for (int r = 0; r < 9; ++r) col[r] = v[r];
      return;
    }
    case 4: {
      const double v[9] = {1.0, uA[0], uA[1], uA[2], 0.5 * W.u2A, 0.0, 0.0, 0.0, 0.0};
      for (int r = 0; r < 9; ++r) col[r] = v[r];
      return;
    }
    case 5: {
      const double v[9] = {0.0, 0.0, 0.0, 0.0, W.BA0 - W.psiA, 1.0, 0.0, 0.0, -1.0};
      for (int r = 0; r < 9; ++r) col[r] = v[r];
      return;
    }
    case 6: {
      const double v[9] = {als * rhoLN, als * rhoLN * (uA[0] - cs), rhoLN * (als * uA[1] - alf * cf * be2 * sg),
                           rhoLN * (als * uA[2] - alf * cf * be3 * sg), W.psiSm, 0.0, -alf * abeta * be2 * sqRho,
                           -alf * abeta * be3 * sqRho, 0.0};
      for (int r = 0; r < 9; ++r) col[r] = v[r];
      return;
    }
    case 7: {
      const double v[9] = {0.0, 0.0, -rhoLN * sqRhoA * be3, rhoLN * sqRhoA * be2,
                           rhoLN * sqRhoA * (be2 * uA[2] - be3 * uA[1]), 0.0, -rhoLN * be3, rhoLN * be2, 0.0};
      for (int r = 0; r < 9; ++r) col[r] = v[r];
      return;
    }
    default: {
      const double v[9] = {alf * rhoLN, alf * rhoLN * (uA[0] - cf), rhoLN * (alf * uA[1] + als * cs * be2 * sg),
                           rhoLN * (alf * uA[2] + als * cs * be3 * sg), W.psiFm, 0.0, als * abeta * be2 * sqRho,
                           als * abeta * be3 * sqRho, 0.0};
      for (int r = 0; r < 9; ++r) col[r] = v[r];
      return;
    }
  }
}

// Flux and dissipation matrices (R[c] = column c) for the subcell schemes that need them explicitly
template <bool FLOGOR>
__device__ __forceinline__ void es_9wave_matrices(const KParams& P, double ch, const double* UL, const double* UR,
                                                  double* F, double* Dm, double (*R)[9]) {
  double Vj[9];
  Wave9 W;
  wave9_setup<FLOGOR>(P, ch, UL, UR, F, Vj, W);
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    Dm[c] = W.D[c];
    wave9_column(W, c, R[c]);
  }
}


// EntropyStableDerigsFlux / EntropyStableFloGorFlux (mhd/riemann.f90:1224-1283, :1633-1691):
// F - 1/2 R D R^T [v]
template <bool FLOGOR>
__device__ __forceinline__ void es_9wave(const KParams& P, double ch, const double* UL, const double* UR, double* F) {
  double Vj[9];
  Wave9 W;
  wave9_setup<FLOGOR>(P, ch, UL, UR, F, Vj, W);
  double w[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) {  // D * (R^T [v]), column by column
    double col[9];
    wave9_column(W, c, col);
    double s = 0.;
#pragma unroll
    for (int r = 0; r < 9; ++r) s += col[r] * Vj[r];
    w[c] = W.D[c] * s;
  }
  double acc[9] = {0., 0., 0., 0., 0., 0., 0., 0., 0.};  // R (D R^T [v]): row sums in column order
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    double col[9];
    wave9_column(W, c, col);
#pragma unroll
    for (int r = 0; r < 9; ++r) acc[r] += col[r] * w[c];
  }
#pragma unroll
  for (int r = 0; r < 9; ++r) F[r] = F[r] - 0.5 * acc[r];
}


template <int RS>
__host__ __device__ constexpr bool riemann_supported() {
  return (RS >= 0 && RS <= 5) || (RS >= 10 && RS <= 15);
}

// PrimToCons, mhd/equation_vars.f90:258-278
__device__ __forceinline__ void prim_to_cons(const KParams& P, const double* Q, double* U) {
  U[0] = Q[0];
  U[1] = Q[1] * Q[0]; U[2] = Q[2] * Q[0]; U[3] = Q[3] * Q[0];
  U[4] = P.sKappaM1 * Q[4] + 0.5 * (U[1] * Q[1] + U[2] * Q[2] + U[3] * Q[3]) +
         P.s2mu_0 * (Q[5] * Q[5] + Q[6] * Q[6] + Q[7] * Q[7] + Q[8] * Q[8]);
#pragma unroll
  for (int v = 5; v < 9; ++v) U[v] = Q[v];
}

// RiemannSolverByHLLC, mhd/riemann.f90:371-501 with the HLL state of EvalHLLState :733-757
__device__ __forceinline__ void hllc(const KParams& P, double ch, const double* UL, const double* UR, double* F) {
  double QL[9], QR[9], RoeVelx, cfRoe;
  cons_to_prim(P, UL, QL);
  cons_to_prim(P, UR, QR);
  const double cfL = fastest_wave_1d(P, QL);
  fastest_wave_1d_roe(P, UL, UR, QL, QR, RoeVelx, cfRoe);
  const double SL = fmin(QL[1] - cfL, RoeVelx - cfRoe);
  if (SL > 0.0) { flux_1d(P, ch, UL, F); return; }
  const double SR = fmax(RoeVelx + cfRoe, QR[1] + fastest_wave_1d(P, QR));
  if (SR < 0.0) { flux_1d(P, ch, UR, F); return; }
  double FL[9], FR[9], UH[9];
  flux_1d(P, ch, UL, FL);
  flux_1d(P, ch, UR, FR);
#pragma unroll
  for (int v = 0; v < 9; ++v) UH[v] = (SR * UR[v] - SL * UL[v] - FR[v] + FL[v]) / (SR - SL);
  const double ptotL = QL[4] + P.s2mu_0 * (QL[5] * QL[5] + QL[6] * QL[6] + QL[7] * QL[7]);
  const double sRhoH = 1. / UH[0];
  const double SM = UH[1] * sRhoH;
  const double Bx = UH[5], By = UH[6], Bz = UH[7];
  const double pS = ptotL + QL[0] * (QL[1] - SL) * (QL[1] - SM) - P.s2mu_0 * (QL[5] * QL[5] - Bx * Bx);
  const double ES = pS * SM + P.smu_0 * (-Bx * (UH[5] * UH[1] + UH[6] * UH[2] + UH[7] * UH[3]) * sRhoH +
                                         UH[8] * (ch * Bx - 0.5 * UH[8] * SM));
  const bool left = (SL <= 0.0) && (0.0 < SM);
  const double* U = left ? UL : UR;
  const double* Q = left ? QL : QR;
  const double* FF = left ? FL : FR;
  const double S = left ? SL : SR;
  const double sd = 1. / (S - SM);
  double Us[9];
  Us[0] = Q[0] * (S - Q[1]) * sd;
  Us[1] = Us[0] * SM;
  Us[2] = (U[2] * S - FF[2] - P.smu_0 * Bx * By) * sd;
  Us[3] = (U[3] * S - FF[3] - P.smu_0 * Bx * Bz) * sd;
  Us[4] = (ES + U[4] * S - FF[4]) * sd;
  Us[5] = Bx; Us[6] = By; Us[7] = Bz;
  Us[8] = U[8];
#pragma unroll
  for (int v = 0; v < 9; ++v) F[v] = FF[v] + S * (Us[v] - U[v]);
}

// RiemannSolverByHLLD, mhd/riemann.f90:511-729 (mu_0 = 1, checked at set-up; B_n made continuous)
__device__ __forceinline__ void hlld(const KParams& P, double ch, const double* ULin, const double* URin, double* F) {
  constexpr double eps = 1.0e-8, small = 1.0e-12;
  double QL[9], QR[9], UL[9], UR[9];
  cons_to_prim(P, ULin, QL);
  cons_to_prim(P, URin, QR);
  const double Bn = 0.5 * (QL[5] + QR[5]);
  QL[5] = Bn; QR[5] = Bn;
  prim_to_cons(P, QL, UL);
  prim_to_cons(P, QR, UR);
  const double FW = fmax(fastest_wave_1d(P, QL), fastest_wave_1d(P, QR));
  const double SL = fmin(QL[1], QR[1]) - FW;
  if (SL > 0.0) { flux_1d(P, ch, UL, F); return; }
  const double SR = fmax(QL[1], QR[1]) + FW;
  if (SR < 0.0) { flux_1d(P, ch, UR, F); return; }
  double FL[9], FR[9];
  flux_1d(P, ch, UL, FL);
  flux_1d(P, ch, UR, FR);
  const double rhoL = QL[0], rhoR = QR[0], unL = QL[1], unR = QR[1];
  const double ptotL = QL[4] + 0.5 * (QL[5] * QL[5] + QL[6] * QL[6] + QL[7] * QL[7]);
  const double ptotR = QR[4] + 0.5 * (QR[5] * QR[5] + QR[6] * QR[6] + QR[7] * QR[7]);
  const double SM = (rhoR * unR * (SR - unR) - rhoL * unL * (SL - unL) - ptotR + ptotL) /
                    (rhoR * (SR - unR) - rhoL * (SL - unL));
  const double sSL = 1. / (SL - SM), sSR = 1. / (SR - SM);
  const double rhoLS = rhoL * (SL - unL) * sSL, rhoRS = rhoR * (SR - unR) * sSR;
  const double sqLS = sqrt(rhoLS), sqRS = sqrt(rhoRS);
  const double SLS = SM - fabs(Bn) / sqLS, SRS = SM + fabs(Bn) / sqRS;
  const double ptotS = ptotL + rhoL * (SL - unL) * (SM - unL);
  // tangential velocity and field of the * states
  double utL1 = QL[2], utL2 = QL[3], BtL1 = QL[6], BtL2 = QL[7];
  double utR1 = QR[2], utR2 = QR[3], BtR1 = QR[6], BtR2 = QR[7];
  double temp = rhoL * (SL - unL) * (SL - SM) - Bn * Bn;
  if (!(fabs(temp) < eps)) {
    const double st = 1. / temp;
    const double a = Bn * (SM - unL) * st, b = (rhoL * (SL - unL) * (SL - unL) - Bn * Bn) * st;
    utL1 = utL1 - a * BtL1; utL2 = utL2 - a * BtL2;
    BtL1 = b * BtL1; BtL2 = b * BtL2;
  }
  double uBS = SM * Bn + utL1 * BtL1 + utL2 * BtL2;
  double uB = QL[1] * QL[5] + QL[2] * QL[6] + QL[3] * QL[7];
  const double eLS = (UL[4] * (SL - unL) + ptotS * SM - ptotL * unL + Bn * (uB - uBS)) * sSL;
  temp = rhoR * (SR - unR) * (SR - SM) - Bn * Bn;
  if (!(fabs(temp) < eps)) {
    const double st = 1. / temp;
    const double a = Bn * (SM - unR) * st, b = (rhoR * (SR - unR) * (SR - unR) - Bn * Bn) * st;
    utR1 = utR1 - a * BtR1; utR2 = utR2 - a * BtR2;
    BtR1 = b * BtR1; BtR2 = b * BtR2;
  }
  uBS = SM * Bn + utR1 * BtR1 + utR2 * BtR2;
  uB = QR[1] * QR[5] + QR[2] * QR[6] + QR[3] * QR[7];
  const double eRS = (UR[4] * (SR - unR) - ptotR * unR + ptotS * SM + Bn * (uB - uBS)) * sSR;
  const double ULS[9] = {rhoLS, rhoLS * SM, rhoLS * utL1, rhoLS * utL2, eLS, Bn, BtL1, BtL2, UL[8]};
  const double URS[9] = {rhoRS, rhoRS * SM, rhoRS * utR1, rhoRS * utR2, eRS, Bn, BtR1, BtR2, UR[8]};
  if (0.0 <= SLS) {
#pragma unroll
    for (int v = 0; v < 9; ++v) F[v] = FL[v] + SL * (ULS[v] - UL[v]);
    return;
  }
  if (0.0 > SRS) {
#pragma unroll
    for (int v = 0; v < 9; ++v) F[v] = FR[v] + SR * (URS[v] - UR[v]);
    return;
  }
  double ULSS[9], URSS[9];
#pragma unroll
  for (int v = 0; v < 9; ++v) { ULSS[v] = ULS[v]; URSS[v] = URS[v]; }
  if (!(fabs(Bn) < small)) {
    const double sgn = Bn < 0.0 ? -1.0 : 1.0;
    const double st = 1. / (sqLS + sqRS);
    const double ut1 = (sqLS * utL1 + sqRS * utR1 + sgn * (BtR1 - BtL1)) * st;
    const double ut2 = (sqLS * utL2 + sqRS * utR2 + sgn * (BtR2 - BtL2)) * st;
    const double bt1 = (sqLS * BtR1 + sqRS * BtL1 + sgn * (utR1 - utL1) * sqLS * sqRS) * st;
    const double bt2 = (sqLS * BtR2 + sqRS * BtL2 + sgn * (utR2 - utL2) * sqLS * sqRS) * st;
    const double uBSS = ut1 * bt1 + ut2 * bt2;
    ULSS[4] = eLS - sgn * sqLS * ((utL1 * BtL1 + utL2 * BtL2) - uBSS);
    URSS[4] = eRS + sgn * sqRS * ((utR1 * BtR1 + utR2 * BtR2) - uBSS);
    ULSS[1] = rhoLS * SM; ULSS[2] = rhoLS * ut1; ULSS[3] = rhoLS * ut2;
    URSS[1] = rhoRS * SM; URSS[2] = rhoRS * ut1; URSS[3] = rhoRS * ut2;
    ULSS[6] = bt1; ULSS[7] = bt2; URSS[6] = bt1; URSS[7] = bt2;
  }
  if (0.0 <= SM) {
#pragma unroll
    for (int v = 0; v < 9; ++v) F[v] = FL[v] + SLS * ULSS[v] - (SLS - SL) * ULS[v] - SL * UL[v];
  } else {
#pragma unroll
    for (int v = 0; v < 9; ++v) F[v] = FR[v] + SRS * URSS[v] - (SRS - SR) * URS[v] - SR * UR[v];
  }
}

// RiemannSolverByRoe, mhd/riemann.f90:764-1024: Cargo & Gallice Roe matrix, the dissipation
// sum_i eta_i |lambda_i| r_i over the 7 waves (entropy fix on the waves 1, 3, 6, 7 as in the reference)
__device__ __forceinline__ void roe(const KParams& P, double ch, const double* UL, const double* UR, double* F) {
  constexpr double efix = 1.0e-6, sefix = 1.0e6;
  double QL[9], QR[9];
  cons_to_prim(P, UL, QL);
  cons_to_prim(P, UR, QR);
  const double sqL = sqrt(QL[0]), sqR = sqrt(QR[0]);
  const double sS = 1. / (sqL + sqR);
  const double RL = sqL * sS, RR = sqR * sS;
  const double ptL = QL[4] + P.s2mu_0 * (QL[5] * QL[5] + QL[6] * QL[6] + QL[7] * QL[7]);
  const double ptR = QR[4] + P.s2mu_0 * (QR[5] * QR[5] + QR[6] * QR[6] + QR[7] * QR[7]);
  const double rhoRoe = sqL * sqR, sRhoRoe = 1. / rhoRoe;
  const double sqRoe = sqrt(rhoRoe), ssqRoe = 1. / sqRoe;
  double v[3], B[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { v[d] = RL * QL[1 + d] + RR * QR[1 + d]; B[d] = RL * QR[5 + d] + RR * QL[5 + d]; }
  const double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  const double B2 = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
  const double H = RL * ((UL[4] + ptL) / QL[0]) + RR * ((UR[4] + ptR) / QR[0]);
  const double dB0 = QL[5] - QR[5], dB1 = QL[6] - QR[6], dB2 = QL[7] - QR[7];
  const double XX = 0.5 * (dB0 * dB0 + dB1 * dB1 + dB2 * dB2) * (sS * sS);
  const double va2 = B2 * P.smu_0 * sRhoRoe;
  const double c2 = (2. - P.kappa) * XX + P.kappaM1 * (H - 0.5 * v2 - va2);
  const double sc2 = 1. / c2, c = sqrt(c2);
  const double ca2 = B[0] * B[0] * P.smu_0 * sRhoRoe, ca = sqrt(ca2);
  const double astar = sqrt((c2 + va2) * (c2 + va2) - 4. * c2 * ca2);
  const double cf2 = 0.5 * (c2 + va2 + astar), cf = sqrt(cf2);
  const double cs2 = 0.5 * (c2 + va2 - astar), cs = sqrt(cs2);
  flux_1d(P, ch, UL, F);
  double FR[9];
  flux_1d(P, ch, UR, FR);
#pragma unroll
  for (int z = 0; z < 9; ++z) F[z] = F[z] + FR[z];
  const double sBx = copysign(1.0, B[0]);
  const double Bt = sqrt(B[1] * B[1] + B[2] * B[2]);
  double by, bz;
  if (Bt > 1.0e-9) { by = B[1] / Bt; bz = B[2] / Bt; } else { by = sqrt(0.5); bz = by; }
  double af, as;
  if (cf2 == cs2) { af = 1.; as = 0.; }
  else if (c2 <= cs2) { af = 0.; as = 1.; }
  else if (cf2 <= c2) { af = 1.; as = 0.; }
  else {
    const double s = 1. / (cf2 - cs2);
    af = sqrt(fmax(0., (c2 - cs2) * s));
    as = sqrt(fmax(0., (cf2 - c2) * s));
  }
  const double drho = QR[0] - QL[0];
  const double dv0 = QR[1] - QL[1], dv1 = QR[2] - QL[2], dv2 = QR[3] - QL[3];
  const double dBy = QR[6] - QL[6], dBz = QR[7] - QL[7];
  const double dp = P.kappaM1 * ((0.5 * v2 - XX) * drho -
                                 (v[0] * (UR[1] - UL[1]) + v[1] * (UR[2] - UL[2]) + v[2] * (UR[3] - UL[3])) +
                                 (UR[4] - UL[4]) - P.smu_0 * (B[0] * (QR[5] - QL[5]) + B[1] * dBy + B[2] * dBz));
  // |lambda| with the entropy fix of the reference on the waves u-c_f, u-c_s, u+c_a, u+c_f
  auto fixed = [&](double l) { return fabs(l) < 0.5 * efix ? fabs(l * l * sefix + 0.25 * efix) : fabs(l); };
  const double l1 = fixed(v[0] - cf), l2 = fabs(v[0] - ca), l3 = fixed(v[0] - cs), l4 = fabs(v[0]);
  const double l5 = fabs(v[0] + cs), l6 = fixed(v[0] + ca), l7 = fixed(v[0] + cf);
  // fast waves
  double bv = by * v[1] + bz * v[2], bdv = by * dv1 + bz * dv2, bdB = by * dBy + bz * dBz;
  const double ascs = as * cs * sBx, asc = as * c * ssqRoe;
  const double fc = af * (XX * drho + dp);
  double g = 0.5 * sc2 * (fc + rhoRoe * (ascs * bdv - af * cf * dv0 + asc * bdB)) * l1;  // eta_1 |lambda_1|
  double h = 0.5 * sc2 * (fc - rhoRoe * (ascs * bdv - af * cf * dv0 - asc * bdB)) * l7;  // eta_7 |lambda_7|
  F[0] -= af * (g + h);
  F[1] -= af * ((v[0] - cf) * g + (v[0] + cf) * h);
  F[2] -= (af * v[1] + ascs * by) * g + (af * v[1] - ascs * by) * h;
  F[3] -= (af * v[2] + ascs * bz) * g + (af * v[2] - ascs * bz) * h;
  F[4] -= (af * (H - va2 - v[0] * cf) + ascs * bv + asc * Bt) * g +
          (af * (H - va2 + v[0] * cf) - ascs * bv + asc * Bt) * h;
  F[6] -= asc * by * (g + h);
  F[7] -= asc * bz * (g + h);
  // slow waves
  const double afcf = af * cf * sBx, afc = af * c * ssqRoe;
  const double sc = as * (XX * drho + dp);
  g = 0.5 * sc2 * (sc - rhoRoe * (afcf * bdv + as * cs * dv0 + afc * bdB)) * l3;
  h = 0.5 * sc2 * (sc + rhoRoe * (afcf * bdv + as * cs * dv0 - afc * bdB)) * l5;
  F[0] -= as * (g + h);
  F[1] -= as * ((v[0] - cs) * g + (v[0] + cs) * h);
  F[2] -= (as * v[1] - afcf * by) * g + (as * v[1] + afcf * by) * h;
  F[3] -= (as * v[2] - afcf * bz) * g + (as * v[2] + afcf * bz) * h;
  F[4] -= (as * (H - va2 - v[0] * cs) - afcf * bv - afc * Bt) * g +
          (as * (H - va2 + v[0] * cs) + afcf * bv - afc * Bt) * h;
  F[6] += afc * by * (g + h);
  F[7] += afc * bz * (g + h);
  // Alfven waves
  bv = bz * v[1] - by * v[2];
  bdv = bz * dv1 - by * dv2;
  bdB = bz * dBy - by * dBz;
  g = 0.5 * (-bdv - sBx * ssqRoe * bdB) * l2;
  h = 0.5 * (bdv - sBx * ssqRoe * bdB) * l6;
  F[2] -= -rhoRoe * bz * (g - h);
  F[3] -= rhoRoe * by * (g - h);
  F[4] -= -rhoRoe * bv * (g - h);
  F[6] -= -sBx * sqRoe * bz * (g + h);
  F[7] -= sBx * sqRoe * by * (g + h);
  // entropy wave
  g = sc2 * ((c2 - XX) * drho - dp) * l4;
  F[0] -= g;
  F[1] -= v[0] * g;
  F[2] -= v[1] * g;
  F[3] -= v[2] * g;
  F[4] -= (0.5 * v2 + P.kappaM2 * P.sKappaM1 * XX) * g;
#pragma unroll
  for (int z = 0; z < 9; ++z) F[z] = 0.5 * F[z];
}

// SolveRiemannProblem in the rotated frame, mhd/equation.f90:311-391
template <int RS>
__device__ __forceinline__ void riemann(const KParams& P, double ch, const double* UL, const double* UR, double* F) {
  if constexpr (RS == 0) {
    standard_dg_flux(P, ch, UL, UR, F);
  } else if constexpr (RS == 1) {  // RiemannSolverByRusanov, mhd/riemann.f90:273-308
    double FL[9], FR[9], QL[9], QR[9];
    flux_1d(P, ch, UL, FL);
    flux_1d(P, ch, UR, FR);
    cons_to_prim(P, UL, QL);
    cons_to_prim(P, UR, QR);
    const double LM = fmax(fabs(QL[1]) + fastest_wave_1d(P, QL), fabs(QR[1]) + fastest_wave_1d(P, QR));
#pragma unroll
    for (int v = 0; v < 9; ++v) F[v] = 0.5 * ((FL[v] + FR[v]) - LM * (UR[v] - UL[v]));
  } else if constexpr (RS == 4) {  // RiemannSolverByHLL, mhd/riemann.f90:314-364
    double QL[9], QR[9], RoeVelx, cfRoe;
    cons_to_prim(P, UL, QL);
    cons_to_prim(P, UR, QR);
    const double cfL = fastest_wave_1d(P, QL);
    fastest_wave_1d_roe(P, UL, UR, QL, QR, RoeVelx, cfRoe);
    const double SL = fmin(QL[1] - cfL, RoeVelx - cfRoe);
    if (SL > 0.0) { flux_1d(P, ch, UL, F); return; }
    const double SR = fmax(RoeVelx + cfRoe, QR[1] + fastest_wave_1d(P, QR));
    if (SR < 0.0) { flux_1d(P, ch, UR, F); return; }
    double FL[9], FR[9];
    flux_1d(P, ch, UL, FL);
    flux_1d(P, ch, UR, FR);
#pragma unroll
    for (int v = 0; v < 9; ++v) F[v] = (SR * FL[v] - SL * FR[v] + SL * SR * (UR[v] - UL[v])) / (SR - SL);
  } else if constexpr (RS == 2) {
    hllc(P, ch, UL, UR, F);
  } else if constexpr (RS == 3) {
    roe(P, ch, UL, UR, F);
  } else if constexpr (RS == 5) {
    hlld(P, ch, UL, UR, F);
  } else if constexpr (RS == 10) {
    es_llf<false>(P, ch, UL, UR, F);
  } else if constexpr (RS == 11) {
    derigs_flux(P, ch, UL, UR, F);
  } else if constexpr (RS == 12) {
    flogor_flux(P, ch, UL, UR, F);
  } else if constexpr (RS == 13) {
    es_llf<true>(P, ch, UL, UR, F);
  } else if constexpr (RS == 14) {
    es_9wave<false>(P, ch, UL, UR, F);
  } else if constexpr (RS == 15) {
    es_9wave<true>(P, ch, UL, UR, F);
  }
}

// lifting variable (EvalLiftingVolumeFlux / EvalLiftingSurfFlux, mhd/flux.f90:718-793)
template <int LV>
__device__ __forceinline__ void lift_var(const KParams& P, const double* U, double* V) {
  if constexpr (LV == 1) {
#pragma unroll
    for (int v = 0; v < 9; ++v) V[v] = U[v];
  } else if constexpr (LV == 2) {
    cons_to_prim(P, U, V);
  } else {
    cons_to_entropy(P, U, V);
  }
}

// ConvertToGradPrim, mhd/equation_vars.f90:547-628 (one point, in place)
template <int LV>
__device__ __forceinline__ void grad_prim(const KParams& P, const double* U, double* g) {
  if constexpr (LV == 1) {
    const double sRho = 1. / U[0];
    const double u = U[1] * sRho, v = U[2] * sRho, w = U[3] * sRho;
    const double gi1 = g[0];
    const double gu = sRho * (g[1] - g[0] * u), gv = sRho * (g[2] - g[0] * v), gw = sRho * (g[3] - g[0] * w);
    const double gi5 = g[4];
    g[1] = gu; g[2] = gv; g[3] = gw;
    g[4] = P.kappaM1 * (gi5 - (0.5 * gi1 * (u * u + v * v + w * w) + (U[1] * gu + U[2] * gv + U[3] * gw)) -
                        P.smu_0 * (U[5] * g[5] + U[6] * g[6] + U[7] * g[7] + U[8] * g[8]));
  } else if constexpr (LV == 3) {
    const double sRho = 1. / U[0];
    const double u = U[1] * sRho, v = U[2] * sRho, w = U[3] * sRho;
    const double Ekin = 0.5 * (U[1] * u + U[2] * v + U[3] * w);
    const double p = P.kappaM1 * (U[4] - Ekin - P.s2mu_0 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7] + U[8] * U[8]));
    const double rho_sp = U[0] / p;
    const double p_srho = p * sRho;
    const double gi1 = g[0];
    const double gu = p_srho * (g[1] + u * g[4]), gv = p_srho * (g[2] + v * g[4]), gw = p_srho * (g[3] + w * g[4]);
    const double gi5 = g[4];
    g[0] = U[0] * gi1 - gi5 * (Ekin - p * P.sKappaM1) + rho_sp * (U[1] * gu + U[2] * gv + U[3] * gw);
    g[1] = gu; g[2] = gv; g[3] = gw;
    g[4] = p_srho * (g[0] + p * gi5);
#pragma unroll
    for (int z = 5; z < 9; ++z) g[z] = p_srho * (g[z] + U[z] * gi5);
  }
}

__device__ __forceinline__ void lifting_var_rt(const KParams& P, const double* U, double* V) {
  if (P.lifting_var == 1) lift_var<1>(P, U, V);
  else if (P.lifting_var == 2) lift_var<2>(P, U, V);
  else lift_var<3>(P, U, V);
}
__device__ __forceinline__ void to_grad_prim_rt(const KParams& P, const double* U, double* g) {
  if (P.lifting_var == 1) grad_prim<1>(P, U, g);
  else if (P.lifting_var == 3) grad_prim<3>(P, U, g);
}

// EvalDiffFlux3D (one point), mhd/flux.f90:449-573: viscous (constant mu), heat and resistive
// fluxes of variables 2..8 (f[0..6] = variables 2..8; variables 1 and 9 have none)
__device__ __forceinline__ void visc_flux_3d(const KParams& P, const double* U, const double* gX, const double* gY,
                                             const double* gZ, double* f, double* g, double* h) {
  const double srho = 1. / U[0];
  const double v1 = U[1] * srho, v2 = U[2] * srho, v3 = U[3] * srho;
  const double b1 = U[5], b2 = U[6], b3 = U[7];
  const double p = P.kappaM1 * (U[4] - 0.5 * (U[0] * (v1 * v1 + v2 * v2 + v3 * v3)) -
                                P.s2mu_0 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7] + U[8] * U[8]));
  const double divv = gX[1] + gY[2] + gZ[3];
  const double lambda = P.muMHD * P.KappasPr;
  const double Qx = lambda * (P.sKappaM1 * srho * (gX[4] - srho * p * gX[0]));
  const double Qy = lambda * (P.sKappaM1 * srho * (gY[4] - srho * p * gY[0]));
  const double Qz = lambda * (P.sKappaM1 * srho * (gZ[4] - srho * p * gZ[0]));
  const double mu = P.muMHD, es = P.etasmu_0;
  // index k <-> variable k+2
  f[0] = -mu * (2 * gX[1] - P.s23 * divv);
  f[1] = -mu * (gX[2] + gY[1]);
  f[2] = -mu * (gX[3] + gZ[1]);
  f[4] = 0.;
  f[5] = -es * (gX[6] - gY[5]);
  f[6] = -es * (gX[7] - gZ[5]);
  f[3] = v1 * f[0] + v2 * f[1] + v3 * f[2] + P.smu_0 * (b1 * f[4] + b2 * f[5] + b3 * f[6]) - Qx;
  g[0] = f[1];
  g[1] = -mu * (2 * gY[2] - P.s23 * divv);
  g[2] = -mu * (gY[3] + gZ[2]);
  g[4] = -f[5];
  g[5] = 0.;
  g[6] = -es * (gY[7] - gZ[6]);
  g[3] = v1 * g[0] + v2 * g[1] + v3 * g[2] + P.smu_0 * (b1 * g[4] + b2 * g[5] + b3 * g[6]) - Qy;
  h[0] = f[2];
  h[1] = g[2];
  h[2] = -mu * (2 * gZ[3] - P.s23 * divv);
  h[4] = -f[6];
  h[5] = -g[6];
  h[6] = 0.;
  h[3] = v1 * h[0] + v2 * h[1] + v3 * h[2] + P.smu_0 * (b1 * h[4] + b2 * h[5] + b3 * h[6]) - Qz;
}

// Non-conservative surface term on the own side (AddNonConsFlux, mhd/riemann.f90:230-267):
// F[1..7] += Bn * phi(own) with Bn = 1/2 (B_own + B_nb).n, phi = Powell (B, v.B, v), Brackbill (B on
// momentum) or Janhunen (v on induction); the GLM part adds psi_own (v_own.nq) and v_own.nq with
// nq = 1/2 (psi_own + psi_nb) n.  Bn and nq arrive already multiplied by SurfElem.
__device__ __forceinline__ void add_noncons_surface(int NC, bool NCGLM, const double* U, double Bn, const double* nq,
                                                    double* F) {
  const double v0 = U[1] / U[0], v1 = U[2] / U[0], v2 = U[3] / U[0];
  if (NC == 1 || NC == 2) { F[1] += Bn * U[5]; F[2] += Bn * U[6]; F[3] += Bn * U[7]; }
  if (NC == 1) F[4] += Bn * (U[5] * v0 + U[6] * v1 + U[7] * v2);
  if (NC == 1 || NC == 3) { F[5] += Bn * v0; F[6] += Bn * v1; F[7] += Bn * v2; }
  if (NCGLM) {
    const double q = v0 * nq[0] + v1 * nq[1] + v2 * nq[2];
    F[4] += U[8] * q;
    F[8] += q;
  }
}

}  // namespace mhd
}  // namespace fluxo
