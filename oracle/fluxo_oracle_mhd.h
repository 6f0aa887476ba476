// ORACLE — test infrastructure only (part of fluxo_oracle.cpp, included inside its namespace).
// CPU restatement of the reference's ideal / resistive MHD equation system with GLM divergence
// cleaning (PP_GLM, nVar = 9) and the non-conservative Powell / Brackbill / Janhunen terms,
// equation/mhd/*.  Variables: rho, rho*v(3), E, B(3), psi.  Each routine names the file:line it
// restates; loops keep the reference's order of summation.

// EvalUaux, mhd/flux_average.f90:223-259: srho, v1, v2, v3, p_t (total pressure), |v|^2, |B|^2, v.B
inline void MHD_Uaux(const Case& C, const real* U, real* a) {
  real srho = 1. / U[0];
  real v1 = U[1] * srho, v2 = U[2] * srho, v3 = U[3] * srho;
  real v2s = v1 * v1 + v2 * v2 + v3 * v3;
  real B2 = U[5] * U[5] + U[6] * U[6] + U[7] * U[7];
  a[0] = srho; a[1] = v1; a[2] = v2; a[3] = v3;
  a[5] = v2s; a[6] = B2; a[7] = v1 * U[5] + v2 * U[6] + v3 * U[7];
  a[4] = C.kappaM1 * (U[4] - 0.5 * U[0] * v2s - C.s2mu_0 * U[8] * U[8]) - C.kappaM2 * C.s2mu_0 * B2;
}

// Two-point volume fluxes with metric terms (VolumeFluxAverageVec), mhd/flux_average.f90
void MHD_VolumeFluxVec(const Case& C, int which, const real* UL, const real* UR, const real* aL, const real* aR,
                       const real* mL, const real* mR, real* F) {
  const double ch = C.GLM_ch, smu0 = C.smu_0;
  switch (which) {
    case 0: {  // StandardDGFluxVec :492-567 (metrics not averaged)
      real EL = UL[4] - 0.5 * smu0 * UL[8] * UL[8], ER = UR[4] - 0.5 * smu0 * UR[8] * UR[8];
      real qvL = aL[1] * mL[0] + aL[2] * mL[1] + aL[3] * mL[2];
      real qbL = UL[5] * mL[0] + UL[6] * mL[1] + UL[7] * mL[2];
      real qvR = aR[1] * mR[0] + aR[2] * mR[1] + aR[3] * mR[2];
      real qbR = UR[5] * mR[0] + UR[6] * mR[1] + UR[7] * mR[2];
      F[0] = 0.5 * (UL[0] * qvL + UR[0] * qvR);
      F[1] = 0.5 * (UL[1] * qvL + UR[1] * qvR + mL[0] * aL[4] + mR[0] * aR[4] - smu0 * (qbL * UL[5] + qbR * UR[5]));
      F[2] = 0.5 * (UL[2] * qvL + UR[2] * qvR + mL[1] * aL[4] + mR[1] * aR[4] - smu0 * (qbL * UL[6] + qbR * UR[6]));
      F[3] = 0.5 * (UL[3] * qvL + UR[3] * qvR + mL[2] * aL[4] + mR[2] * aR[4] - smu0 * (qbL * UL[7] + qbR * UR[7]));
      F[4] = 0.5 * ((EL + aL[4]) * qvL + (ER + aR[4]) * qvR - smu0 * (qbL * aL[7] + qbR * aR[7]));
      F[5] = 0.5 * (qvL * UL[5] - qbL * aL[1] + qvR * UR[5] - qbR * aR[1]);
      F[6] = 0.5 * (qvL * UL[6] - qbL * aL[2] + qvR * UR[6] - qbR * aR[2]);
      F[7] = 0.5 * (qvL * UL[7] - qbL * aL[3] + qvR * UR[7] - qbR * aR[3]);
      F[4] = F[4] + 0.5 * smu0 * ch * (qbL * UL[8] + qbR * UR[8]);
      F[5] = F[5] + 0.5 * ch * (UL[8] * mL[0] + UR[8] * mR[0]);
      F[6] = F[6] + 0.5 * ch * (UL[8] * mL[1] + UR[8] * mR[1]);
      F[7] = F[7] + 0.5 * ch * (UL[8] * mL[2] + UR[8] * mR[2]);
      F[8] = 0.5 * ch * (qbL + qbR);
      return;
    }
    case 1: {  // StandardDGFluxDealiasedMetricVec :574-651
      real m[3] = {0.5 * (mL[0] + mR[0]), 0.5 * (mL[1] + mR[1]), 0.5 * (mL[2] + mR[2])};
      real EL = UL[4] - 0.5 * smu0 * UL[8] * UL[8], ER = UR[4] - 0.5 * smu0 * UR[8] * UR[8];
      real qvL = aL[1] * m[0] + aL[2] * m[1] + aL[3] * m[2];
      real qbL = UL[5] * m[0] + UL[6] * m[1] + UL[7] * m[2];
      real qvR = aR[1] * m[0] + aR[2] * m[1] + aR[3] * m[2];
      real qbR = UR[5] * m[0] + UR[6] * m[1] + UR[7] * m[2];
      F[0] = 0.5 * (UL[0] * qvL + UR[0] * qvR);
      F[1] = 0.5 * (UL[1] * qvL + UR[1] * qvR + m[0] * (aL[4] + aR[4]) - smu0 * (qbL * UL[5] + qbR * UR[5]));
      F[2] = 0.5 * (UL[2] * qvL + UR[2] * qvR + m[1] * (aL[4] + aR[4]) - smu0 * (qbL * UL[6] + qbR * UR[6]));
      F[3] = 0.5 * (UL[3] * qvL + UR[3] * qvR + m[2] * (aL[4] + aR[4]) - smu0 * (qbL * UL[7] + qbR * UR[7]));
      F[4] = 0.5 * ((EL + aL[4]) * qvL + (ER + aR[4]) * qvR - smu0 * (qbL * aL[7] + qbR * aR[7]));
      F[5] = 0.5 * (qvL * UL[5] - qbL * aL[1] + qvR * UR[5] - qbR * aR[1]);
      F[6] = 0.5 * (qvL * UL[6] - qbL * aL[2] + qvR * UR[6] - qbR * aR[2]);
      F[7] = 0.5 * (qvL * UL[7] - qbL * aL[3] + qvR * UR[7] - qbR * aR[3]);
      F[4] = F[4] + 0.5 * smu0 * ch * (qbL * UL[8] + qbR * UR[8]);
      real phiHat = 0.5 * ch * (UL[8] + UR[8]);
      F[5] = F[5] + phiHat * m[0];
      F[6] = F[6] + phiHat * m[1];
      F[7] = F[7] + phiHat * m[2];
      F[8] = 0.5 * ch * (qbL + qbR);
      return;
    }
    case 10: {  // EntropyAndKinEnergyConservingFluxVec_Derigs :761-848
      real m[3] = {0.5 * (mL[0] + mR[0]), 0.5 * (mL[1] + mR[1]), 0.5 * (mL[2] + mR[2])};
      real betaL = 0.5 * UL[0] / (aL[4] - C.s2mu_0 * aL[6]);
      real betaR = 0.5 * UR[0] / (aR[4] - C.s2mu_0 * aR[6]);
      real rhoLN = LN_MEAN(UL[0], UR[0]);
      real betaLN = LN_MEAN(betaL, betaR);
      real vA[3], BA[3];
      for (int d = 0; d < 3; ++d) { vA[d] = 0.5 * (aL[1 + d] + aR[1 + d]); BA[d] = 0.5 * (UL[5 + d] + UR[5 + d]); }
      real pTilde = 0.5 * ((UL[0] + UR[0]) / (betaL + betaR) + smu0 * 0.5 * (aL[6] + aR[6]));
      real vm = vA[0] * m[0] + vA[1] * m[1] + vA[2] * m[2];
      real Bm = BA[0] * m[0] + BA[1] * m[1] + BA[2] * m[2];
      real psiA = 0.5 * (UL[8] + UR[8]);
      F[0] = rhoLN * vm;
      for (int d = 0; d < 3; ++d) F[1 + d] = F[0] * vA[d] - (smu0 * Bm) * BA[d] + pTilde * m[d];
      for (int d = 0; d < 3; ++d) F[5 + d] = vm * BA[d] - Bm * vA[d] + (ch * psiA) * m[d];
      F[8] = ch * Bm;
      real sB = BA[0] * F[5] + BA[1] * F[6] + BA[2] * F[7];
      real b2v = (aL[6] * aL[1] + aR[6] * aR[1]) * m[0] + (aL[6] * aL[2] + aR[6] * aR[2]) * m[1] +
                 (aL[6] * aL[3] + aR[6] * aR[3]) * m[2];
      real pB = (UL[8] * UL[5] + UR[8] * UR[5]) * m[0] + (UL[8] * UL[6] + UR[8] * UR[6]) * m[1] +
                (UL[8] * UL[7] + UR[8] * UR[7]) * m[2];
      F[4] = F[0] * 0.5 * (C.sKappaM1 / betaLN - 0.5 * (aL[5] + aR[5])) +
             (vA[0] * F[1] + vA[1] * F[2] + vA[2] * F[3]) +
             smu0 * (sB - 0.25 * b2v + 0.5 * (aL[7] + aR[7]) * Bm + F[8] * psiA - (ch * 0.5) * pB);
      return;
    }
    case 12: {  // EntropyAndKinEnergyConservingFluxVec_FloGor :970-1074
      real m[3] = {0.5 * (mL[0] + mR[0]), 0.5 * (mL[1] + mR[1]), 0.5 * (mL[2] + mR[2])};
      real pL = aL[4] - C.s2mu_0 * aL[6], pR = aR[4] - C.s2mu_0 * aR[6];
      real ieL = pL / UL[0] * C.sKappaM1, ieR = pR / UR[0] * C.sKappaM1;
      real rhoLN = LN_MEAN(UL[0], UR[0]);
      real vA[3];
      for (int d = 0; d < 3; ++d) vA[d] = 0.5 * (aL[1 + d] + aR[1 + d]);
      real v2Z = aL[1] * aR[1] + aL[2] * aR[2] + aL[3] * aR[3];
      real B2Z = UL[5] * UR[5] + UL[6] * UR[6] + UL[7] * UR[7];
      real pA = 0.5 * (pL + pR);
      real vmL = aL[1] * m[0] + aL[2] * m[1] + aL[3] * m[2];
      real vmR = aR[1] * m[0] + aR[2] * m[1] + aR[3] * m[2];
      real BmL = UL[5] * m[0] + UL[6] * m[1] + UL[7] * m[2];
      real BmR = UR[5] * m[0] + UR[6] * m[1] + UR[7] * m[2];
      auto ZIP = [](real a, real b, real c, real d) { return 0.5 * (a * d + b * c); };
      F[0] = rhoLN * 0.5 * (vmL + vmR);
      for (int d = 0; d < 3; ++d)
        F[1 + d] = F[0] * vA[d] + m[d] * (pA + C.s2mu_0 * B2Z) - smu0 * ZIP(UL[5 + d], UR[5 + d], BmL, BmR);
      real s = 0.;
      for (int d = 0; d < 3; ++d)
        s = s + ZIP(vmL * UL[5 + d], vmR * UR[5 + d], UL[5 + d], UR[5 + d]) -
            ZIP(aL[1 + d] * BmL, aR[1 + d] * BmR, UL[5 + d], UR[5 + d]);
      F[4] = F[0] * (0.5 * v2Z + ieL * ieR / LN_MEAN(ieL, ieR)) + ZIP(pL, pR, vmL, vmR) +
             smu0 * (s + ch * ZIP(BmL, BmR, UL[8], UR[8]));
      for (int d = 0; d < 3; ++d)
        F[5 + d] = 0.5 * ((vmL * UL[5 + d] - aL[1 + d] * BmL) + (vmR * UR[5 + d] - aR[1 + d] * BmR) +
                          ch * (UL[8] + UR[8]) * m[d]);
      F[8] = ch * 0.5 * (BmL + BmR);
      return;
    }
    default: throw std::runtime_error("MHD volume flux not implemented in oracle");
  }
}

// Non-conservative terms of one node pair (AddNonConsFluxTilde3D, mhd/flux_average.f90:268-366):
// adds Phi(i) * (M_i.B_i + (M_i+M_l)/2 . B_l) [and the GLM part] to the flux at node i.
inline void MHD_NonConsPair(const Case& C, const real* Ui, const real* ai, const real* Ul, const real* Mi,
                            const real* Ml, real* F) {
  if (C.noncons == 0) return;
  real Bhat = Mi[0] * Ui[5] + Mi[1] * Ui[6] + Mi[2] * Ui[7];
  real t = Bhat + (0.5 * (Mi[0] + Ml[0]) * Ul[5] + 0.5 * (Mi[1] + Ml[1]) * Ul[6] + 0.5 * (Mi[2] + Ml[2]) * Ul[7]);
  if (C.noncons == 1) {  // Powell: 0.5*(B, v.B, v)
    real phi[7] = {0.5 * Ui[5], 0.5 * Ui[6], 0.5 * Ui[7], 0.5 * ai[7], 0.5 * ai[1], 0.5 * ai[2], 0.5 * ai[3]};
    for (int v = 0; v < 7; ++v) F[1 + v] = F[1 + v] + phi[v] * t;
  } else if (C.noncons == 2) {  // Brackbill: 0.5*B on momentum
    for (int v = 0; v < 3; ++v) F[1 + v] = F[1 + v] + 0.5 * Ui[5 + v] * t;
  } else {  // Janhunen: 0.5*v on induction
    for (int v = 0; v < 3; ++v) F[5 + v] = F[5 + v] + 0.5 * ai[1 + v] * t;
  }
  if (C.ncGLM) {
    real q = 0.5 * (Mi[0] * ai[1] + Mi[1] * ai[2] + Mi[2] * ai[3]);
    real s = Ui[8] + Ul[8];
    F[4] = F[4] + s * (q * Ui[8]);
    F[8] = F[8] + s * q;
  }
}

// EvalAdvectionFlux1D, mhd/flux.f90:391-442 (rotated frame)
inline void MHD_Flux1D(const Case& C, const real* U, real* F) {
  real srho = 1. / U[0];
  real v1 = U[1] * srho, v2 = U[2] * srho, v3 = U[3] * srho;
  real b1 = U[5], b2 = U[6], b3 = U[7];
  real Et = U[4] - C.s2mu_0 * U[8] * U[8];
  real vb = b1 * v1 + b2 * v2 + b3 * v3;
  real pt = C.kappaM1 * (Et - 0.5 * U[0] * (v1 * v1 + v2 * v2 + v3 * v3)) - C.kappaM2 * C.s2mu_0 * (b1 * b1 + b2 * b2 + b3 * b3);
  F[0] = U[1];
  F[1] = U[1] * v1 + pt - C.smu_0 * b1 * b1;
  F[2] = U[1] * v2 - C.smu_0 * b1 * b2;
  F[3] = U[1] * v3 - C.smu_0 * b1 * b3;
  F[4] = (Et + pt) * v1 - C.smu_0 * b1 * vb;
  F[5] = 0.;
  F[6] = v1 * b2 - b1 * v2;
  F[7] = v1 * b3 - b1 * v3;
  F[4] = F[4] + C.smu_0 * C.GLM_ch * b1 * U[8];
  F[5] = F[5] + C.GLM_ch * U[8];
  F[8] = C.GLM_ch * b1;
}

// ConsToPrim, mhd/equation_vars.f90:229-251 (pressure without magnetic and psi energy)
inline void MHD_ConsToPrim(const Case& C, const real* U, real* P) {
  real sRho = 1. / U[0];
  P[0] = U[0];
  P[1] = U[1] * sRho; P[2] = U[2] * sRho; P[3] = U[3] * sRho;
  P[4] = C.kappaM1 * (U[4] - 0.5 * (U[1] * P[1] + U[2] * P[2] + U[3] * P[3]) -
                      C.s2mu_0 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7] + U[8] * U[8]));
  for (int v = 5; v < 9; ++v) P[v] = U[v];
}

// PrimToCons, mhd/equation_vars.f90:258-278
template <typename T>
inline void MHD_PrimToCons(const Case& C, const T* P, T* U) {
  U[0] = P[0];
  U[1] = P[1] * P[0]; U[2] = P[2] * P[0]; U[3] = P[3] * P[0];
  U[4] = C.sKappaM1 * P[4] + 0.5 * (U[1] * P[1] + U[2] * P[2] + U[3] * P[3]) +
         C.s2mu_0 * (P[5] * P[5] + P[6] * P[6] + P[7] * P[7] + P[8] * P[8]);
  for (int v = 5; v < 9; ++v) U[v] = P[v];
}

// ConsToEntropy, mhd/equation_vars.f90:330-361
inline void MHD_ConsToEntropy(const Case& C, const real* U, real* W) {
  real srho = 1. / U[0];
  real u = U[1] * srho, v = U[2] * srho, w = U[3] * srho;
  real v2s2 = 0.5 * (u * u + v * v + w * w);
  real rho_sp = U[0] / (C.kappaM1 * (U[4] - U[0] * v2s2 -
                                     C.s2mu_0 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7] + U[8] * U[8])));
  real s = -log(rho_sp * pow(U[0], C.kappaM1));
  W[0] = (C.kappa - s) * C.sKappaM1 - rho_sp * v2s2;
  W[1] = rho_sp * u; W[2] = rho_sp * v; W[3] = rho_sp * w;
  W[4] = -rho_sp;
  for (int z = 5; z < 9; ++z) W[z] = rho_sp * U[z];
}

// EntropyToCons, mhd/equation_vars.f90:366-401
inline void MHD_EntropyToCons(const Case& C, const real* W, real* U) {
  real rho_sp = -W[4];
  real p_srho = 1. / rho_sp;
  real u = W[1] * p_srho, v = W[2] * p_srho, w = W[3] * p_srho;
  real v2s2 = 0.5 * (u * u + v * v + w * w);
  real s = C.kappa - ((W[0] + rho_sp * v2s2) * C.kappaM1);
  U[0] = pow(exp(-s) * p_srho, C.sKappaM1);
  U[1] = u * U[0];
  U[2] = v * U[0];
  U[3] = w * U[0];
  for (int z = 5; z < 9; ++z) U[z] = W[z] * p_srho;
  U[4] = U[0] * (C.sKappaM1 * p_srho + v2s2) +
         C.s2mu_0 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7] + U[8] * U[8]);
}

// FastestWave1D, mhd/equation_vars.f90:663-684 (primitive input, normal direction 1)
inline real MHD_FastestWave1D(const Case& C, const real* P) {
  real sRho = 1. / P[0];
  real c2 = C.kappa * P[4] * sRho;
  real ca2 = P[5] * P[5] * sRho * C.smu_0;
  real va2 = (P[6] * P[6] + P[7] * P[7]) * sRho * C.smu_0 + ca2;
  real astar = sqrt((c2 + va2) * (c2 + va2) - 4. * c2 * ca2);
  return sqrt(0.5 * (c2 + va2 + astar));
}

// FastestWave1D_Roe, mhd/equation_vars.f90:717-763
inline void MHD_FastestWave1D_Roe(const Case& C, const real* UL, const real* UR, const real* PL, const real* PR,
                                  real& RoeVelx, real& cfRoe) {
  real sqL = sqrt(PL[0]), sqR = sqrt(PR[0]);
  real sS = 1. / (sqL + sqR);
  real RL = sqL * sS, RR = sqR * sS;
  real ptL = PL[4] + C.s2mu_0 * (PL[5] * PL[5] + PL[6] * PL[6] + PL[7] * PL[7]);
  real ptR = PR[4] + C.s2mu_0 * (PR[5] * PR[5] + PR[6] * PR[6] + PR[7] * PR[7]);
  real sRhoRoe = 1. / (sqL * sqR);
  real vR[3], BR[3];
  for (int d = 0; d < 3; ++d) { vR[d] = RL * PL[1 + d] + RR * PR[1 + d]; BR[d] = RL * PR[5 + d] + RR * PL[5 + d]; }
  real HL = (UL[4] + ptL) / PL[0], HR = (UR[4] + ptR) / PR[0];
  real RoeH = RL * HL + RR * HR;
  real dB0 = PL[5] - PR[5], dB1 = PL[6] - PR[6], dB2 = PL[7] - PR[7];
  real XX = 0.5 * (dB0 * dB0 + dB1 * dB1 + dB2 * dB2) * (sS * sS);
  real va2 = (BR[0] * BR[0] + BR[1] * BR[1] + BR[2] * BR[2]) * C.smu_0 * sRhoRoe;
  real c2 = (2. - C.kappa) * XX + (C.kappa - 1) * (RoeH - 0.5 * (vR[0] * vR[0] + vR[1] * vR[1] + vR[2] * vR[2]) - va2);
  real ca2 = BR[0] * BR[0] * C.smu_0 * sRhoRoe;
  real astar = sqrt((c2 + va2) * (c2 + va2) - 4. * c2 * ca2);
  cfRoe = sqrt(0.5 * (c2 + va2 + astar));
  RoeVelx = vR[0];
}

// StandardDGFlux (Riemann 0), mhd/flux_average.f90:421-484
inline void MHD_StandardDGFlux(const Case& C, const real* UL, const real* UR, real* F) {
  real EL = UL[4] - 0.5 * C.smu_0 * UL[8] * UL[8], ER = UR[4] - 0.5 * C.smu_0 * UR[8] * UR[8];
  real sL = 1. / UL[0], sR = 1. / UR[0];
  real v1L = sL * UL[1], v2L = sL * UL[2], v3L = sL * UL[3];
  real v1R = sR * UR[1], v2R = sR * UR[2], v3R = sR * UR[3];
  real b1L = UL[5], b2L = UL[6], b3L = UL[7], b1R = UR[5], b2R = UR[6], b3R = UR[7];
  real bbL = b1L * b1L + b2L * b2L + b3L * b3L, bbR = b1R * b1R + b2R * b2R + b3R * b3R;
  real ptL = C.kappaM1 * (EL - 0.5 * (UL[1] * v1L + UL[2] * v2L + UL[3] * v3L)) - C.kappaM2 * C.s2mu_0 * bbL;
  real ptR = C.kappaM1 * (ER - 0.5 * (UR[1] * v1R + UR[2] * v2R + UR[3] * v3R)) - C.kappaM2 * C.s2mu_0 * bbR;
  real vbL = v1L * b1L + v2L * b2L + v3L * b3L, vbR = v1R * b1R + v2R * b2R + v3R * b3R;
  real qL = UL[0] * v1L, qR = UR[0] * v1R;
  F[0] = 0.5 * (qL + qR);
  F[1] = 0.5 * (qL * v1L + qR * v1R + (ptL + ptR) - C.smu_0 * (b1L * b1L + b1R * b1R));
  F[2] = 0.5 * (qL * v2L + qR * v2R - C.smu_0 * (b2L * b1L + b2R * b1R));
  F[3] = 0.5 * (qL * v3L + qR * v3R - C.smu_0 * (b3L * b1L + b3R * b1R));
  F[4] = 0.5 * ((EL + ptL) * v1L + (ER + ptR) * v1R - C.smu_0 * (b1L * vbL + b1R * vbR));
  F[5] = 0.;
  F[6] = 0.5 * (v1L * b2L - b1L * v2L + v1R * b2R - b1R * v2R);
  F[7] = 0.5 * (v1L * b3L - b1L * v3L + v1R * b3R - b1R * v3R);
  F[4] = F[4] + 0.5 * C.smu_0 * C.GLM_ch * (b1L * UL[8] + b1R * UR[8]);
  F[5] = F[5] + 0.5 * C.GLM_ch * (UL[8] + UR[8]);
  F[8] = 0.5 * C.GLM_ch * (b1L + b1R);
}

// EntropyAndKinEnergyConservingFlux_Derigs (1D), mhd/flux_average.f90:660-751
inline void MHD_DerigsFlux(const Case& C, const real* UL, const real* UR, real* F) {
  const double ch = C.GLM_ch, smu0 = C.smu_0;
  real EL = UL[4] - 0.5 * smu0 * UL[8] * UL[8], ER = UR[4] - 0.5 * smu0 * UR[8] * UR[8];
  real vL[3], vR[3];
  for (int d = 0; d < 3; ++d) { vL[d] = UL[1 + d] / UL[0]; vR[d] = UR[1 + d] / UR[0]; }
  real v2L = vL[0] * vL[0] + vL[1] * vL[1] + vL[2] * vL[2], v2R = vR[0] * vR[0] + vR[1] * vR[1] + vR[2] * vR[2];
  real B2L = UL[5] * UL[5] + UL[6] * UL[6] + UL[7] * UL[7], B2R = UR[5] * UR[5] + UR[6] * UR[6] + UR[7] * UR[7];
  real pL = C.kappaM1 * (EL - 0.5 * (UL[0] * v2L + smu0 * B2L));
  real pR = C.kappaM1 * (ER - 0.5 * (UR[0] * v2R + smu0 * B2R));
  real bL = 0.5 * UL[0] / pL, bR = 0.5 * UR[0] / pR;
  real rhoLN = LN_MEAN(UL[0], UR[0]);
  real betaLN = LN_MEAN(bL, bR);
  real vA[3], BA[3];
  for (int d = 0; d < 3; ++d) { vA[d] = 0.5 * (vL[d] + vR[d]); BA[d] = 0.5 * (UL[5 + d] + UR[5 + d]); }
  real v1B2 = 0.5 * (vL[0] * B2L + vR[0] * B2R);
  real vBA = 0.5 * ((vL[0] * UL[5] + vL[1] * UL[6] + vL[2] * UL[7]) + (vR[0] * UR[5] + vR[1] * UR[6] + vR[2] * UR[7]));
  real pTilde = 0.5 * ((UL[0] + UR[0]) / (bL + bR) + smu0 * 0.5 * (B2L + B2R));
  real psiA = 0.5 * (UL[8] + UR[8]);
  F[0] = rhoLN * vA[0];
  F[1] = F[0] * vA[0] - smu0 * BA[0] * BA[0] + pTilde;
  F[2] = F[0] * vA[1] - smu0 * BA[0] * BA[1];
  F[3] = F[0] * vA[2] - smu0 * BA[0] * BA[2];
  F[6] = vA[0] * BA[1] - BA[0] * vA[1];
  F[7] = vA[0] * BA[2] - BA[0] * vA[2];
  F[5] = ch * psiA;
  F[8] = ch * BA[0];
  F[4] = F[0] * 0.5 * (C.sKappaM1 / betaLN - 0.5 * (v2L + v2R)) + (vA[0] * F[1] + vA[1] * F[2] + vA[2] * F[3]) +
         smu0 * ((BA[0] * F[5] + BA[1] * F[6] + BA[2] * F[7]) - 0.5 * v1B2 + BA[0] * vBA + F[8] * psiA -
                 ch * 0.5 * (UL[8] * UL[5] + UR[8] * UR[5]));
}

// EntropyAndKinEnergyConservingFlux_FloGor (1D), mhd/flux_average.f90:855-960
inline void MHD_FloGorFlux(const Case& C, const real* UL, const real* UR, real* F) {
  const double ch = C.GLM_ch, smu0 = C.smu_0;
  real EL = UL[4] - 0.5 * smu0 * UL[8] * UL[8], ER = UR[4] - 0.5 * smu0 * UR[8] * UR[8];
  real sL = 1. / UL[0], sR = 1. / UR[0];
  real vL[3], vR[3];
  for (int d = 0; d < 3; ++d) { vL[d] = UL[1 + d] * sL; vR[d] = UR[1 + d] * sR; }
  real v2L = vL[0] * vL[0] + vL[1] * vL[1] + vL[2] * vL[2], v2R = vR[0] * vR[0] + vR[1] * vR[1] + vR[2] * vR[2];
  real B2L = UL[5] * UL[5] + UL[6] * UL[6] + UL[7] * UL[7], B2R = UR[5] * UR[5] + UR[6] * UR[6] + UR[7] * UR[7];
  real pL = C.kappaM1 * (EL - 0.5 * (UL[0] * v2L + smu0 * B2L));
  real pR = C.kappaM1 * (ER - 0.5 * (UR[0] * v2R + smu0 * B2R));
  real ieL = pL * sL * C.sKappaM1, ieR = pR * sR * C.sKappaM1;
  real rhoLN = LN_MEAN(UL[0], UR[0]);
  real vA[3], BA[3];
  for (int d = 0; d < 3; ++d) { vA[d] = 0.5 * (vL[d] + vR[d]); BA[d] = 0.5 * (UL[5 + d] + UR[5 + d]); }
  real v2Z = vL[0] * vR[0] + vL[1] * vR[1] + vL[2] * vR[2];
  real B2Z = UL[5] * UR[5] + UL[6] * UR[6] + UL[7] * UR[7];
  real pA = 0.5 * (pL + pR);
  auto ZIP = [](real a, real b, real c, real d) { return 0.5 * (a * d + b * c); };
  const real *BL = UL + 5, *BR = UR + 5;
  F[0] = rhoLN * vA[0];
  F[1] = F[0] * vA[0] + pA + C.s2mu_0 * B2Z - smu0 * ZIP(BL[0], BR[0], BL[0], BR[0]);
  F[2] = F[0] * vA[1] - smu0 * ZIP(BL[0], BR[0], BL[1], BR[1]);
  F[3] = F[0] * vA[2] - smu0 * ZIP(BL[0], BR[0], BL[2], BR[2]);
  F[4] = F[0] * (0.5 * v2Z + ieL * ieR / LN_MEAN(ieL, ieR)) + ZIP(pL, pR, vL[0], vR[0]) +
         smu0 * (ZIP(vL[0] * BL[1], vR[0] * BR[1], BL[1], BR[1]) - ZIP(vL[1] * BL[0], vR[1] * BR[0], BL[1], BR[1]) +
                 ZIP(vL[0] * BL[2], vR[0] * BR[2], BL[2], BR[2]) - ZIP(vL[2] * BL[0], vR[2] * BR[0], BL[2], BR[2]) +
                 ch * ZIP(BL[0], BR[0], UL[8], UR[8]));
  F[5] = ch * 0.5 * (UL[8] + UR[8]);
  F[8] = ch * BA[0];
  F[6] = 0.5 * ((vL[0] * BL[1] - vL[1] * BL[0]) + (vR[0] * BR[1] - vR[1] * BR[0]));
  F[7] = 0.5 * ((vL[0] * BL[2] - vL[2] * BL[0]) + (vR[0] * BR[2] - vR[2] * BR[0]));
}

// Entropy-variable jump [v] used by the entropy-stable solvers, mhd/riemann.f90:1085-1089, :1259-1263
inline void MHD_EntropyJump(const Case& C, const real* UL, const real* UR, real& pL, real& pR, real& bL, real& bR,
                            real* Vj) {
  real EL = UL[4] - C.s2mu_0 * UL[8] * UL[8], ER = UR[4] - C.s2mu_0 * UR[8] * UR[8];
  real sL = 1. / UL[0], sR = 1. / UR[0];
  real uL[3], uR[3];
  for (int d = 0; d < 3; ++d) { uL[d] = UL[1 + d] * sL; uR[d] = UR[1 + d] * sR; }
  real u2L = uL[0] * uL[0] + uL[1] * uL[1] + uL[2] * uL[2], u2R = uR[0] * uR[0] + uR[1] * uR[1] + uR[2] * uR[2];
  real B2L = UL[5] * UL[5] + UL[6] * UL[6] + UL[7] * UL[7], B2R = UR[5] * UR[5] + UR[6] * UR[6] + UR[7] * UR[7];
  pL = C.kappaM1 * (EL - 0.5 * (UL[0] * u2L + C.smu_0 * B2L));
  pR = C.kappaM1 * (ER - 0.5 * (UR[0] * u2R + C.smu_0 * B2R));
  bL = 0.5 * UL[0] / pL;
  bR = 0.5 * UR[0] / pR;
  Vj[0] = (C.kappa * (log(UR[0] * sL)) - log(pR / pL)) * C.sKappaM1 - (bR * u2R - bL * u2L);
  for (int d = 0; d < 3; ++d) Vj[1 + d] = 2.0 * (bR * uR[d] - bL * uL[d]);
  Vj[4] = -2.0 * (bR - bL);
  for (int z = 5; z < 9; ++z) Vj[z] = 2.0 * (bR * UR[z] - bL * UL[z]);
}

// EntropyStableByLLF (Riemann 10 with Derigs, 13 with FloGor), mhd/riemann.f90:1027-1211
inline void MHD_EntropyStableLLF(const Case& C, const real* UL, const real* UR, bool flogor, real* F) {
  real Vj[9], pL, pR, bL, bR;
  MHD_EntropyJump(C, UL, UR, pL, pR, bL, bR, Vj);
  real sL = 1. / UL[0], sR = 1. / UR[0];
  real uL[3], uR[3];
  for (int d = 0; d < 3; ++d) { uL[d] = UL[1 + d] * sL; uR[d] = UR[1 + d] * sR; }
  real u2L = uL[0] * uL[0] + uL[1] * uL[1] + uL[2] * uL[2], u2R = uR[0] * uR[0] + uR[1] * uR[1] + uR[2] * uR[2];
  real B2L = UL[5] * UL[5] + UL[6] * UL[6] + UL[7] * UL[7], B2R = UR[5] * UR[5] + UR[6] * UR[6] + UR[7] * UR[7];
  real rhoLN = LN_MEAN(UL[0], UR[0]);
  real sbetaLN = 1. / LN_MEAN(bL, bR);
  real uA[3], BA[3];
  for (int d = 0; d < 3; ++d) { uA[d] = 0.5 * (uL[d] + uR[d]); BA[d] = 0.5 * (UL[5 + d] + UR[5 + d]); }
  real u2A = 0.5 * (u2L + u2R);
  real B2A = 0.5 * (B2L + B2R);
  real pA = 0.5 * (UL[0] + UR[0]) / (bL + bR);
  real psiA = 0.5 * (UL[8] + UR[8]);
  if (flogor) MHD_FloGorFlux(C, UL, UR, F);
  else MHD_DerigsFlux(C, UL, UR, F);
  real pLN = 0.5 * rhoLN * sbetaLN;
  real srhoLN = 1. / rhoLN;
  real a2A = C.kappa * pA * srhoLN;
  real va2A = B2A * srhoLN;
  real ca2A = BA[0] * BA[0] * srhoLN;
  real cfA = sqrt(0.5 * ((a2A + va2A) + sqrt((a2A + va2A) * (a2A + va2A) - 4.0 * a2A * ca2A)));
  real LM = 0.5 * (fabs(uA[0]) + cfA);
  real uA2 = uA[0] * uA[0] + uA[1] * uA[1] + uA[2] * uA[2];
  real Eavg = pLN * C.sKappaM1 + 0.5 * rhoLN * (2.0 * uA2 - u2A);
  real H[5][5];  // H[row][col] = Hmatrix(row+1, col+1)
  H[0][0] = rhoLN; H[1][0] = rhoLN * uA[0]; H[2][0] = rhoLN * uA[1]; H[3][0] = rhoLN * uA[2]; H[4][0] = Eavg;
  H[0][1] = H[1][0]; H[1][1] = H[1][0] * uA[0] + pA; H[2][1] = H[2][0] * uA[0]; H[3][1] = H[3][0] * uA[0];
  H[4][1] = (Eavg + pA) * uA[0];
  H[0][2] = H[2][0]; H[1][2] = H[2][1]; H[2][2] = H[2][0] * uA[1] + pA; H[3][2] = H[3][0] * uA[1];
  H[4][2] = (Eavg + pA) * uA[1];
  H[0][3] = H[3][0]; H[1][3] = H[3][1]; H[2][3] = H[3][2]; H[3][3] = H[3][0] * uA[2] + pA;
  H[4][3] = (Eavg + pA) * uA[2];
  H[0][4] = H[4][0]; H[1][4] = H[4][1]; H[2][4] = H[4][2]; H[3][4] = H[4][3];
  real tau = 1. / (bL + bR);
  H[4][4] = (pLN * pLN * C.sKappaM1 + Eavg * Eavg) * srhoLN + uA2 * pA +
            tau * ((BA[0] * BA[0] + BA[1] * BA[1] + BA[2] * BA[2]) + psiA * psiA);
  for (int r = 0; r < 4; ++r) {
    real s = H[r][0] * Vj[0] + H[r][1] * Vj[1] + H[r][2] * Vj[2] + H[r][3] * Vj[3] + H[r][4] * Vj[4];
    F[r] = F[r] - LM * s;
  }
  real s5 = H[0][4] * Vj[0] + H[1][4] * Vj[1] + H[2][4] * Vj[2] + H[3][4] * Vj[3] + H[4][4] * Vj[4];
  F[4] = F[4] - LM * (s5 + tau * ((BA[0] * Vj[5] + BA[1] * Vj[6] + BA[2] * Vj[7]) + psiA * Vj[8]));
  for (int d = 0; d < 3; ++d) F[5 + d] = F[5 + d] - (LM * tau) * (BA[d] * Vj[4] + Vj[5 + d]);
  F[8] = F[8] - (LM * tau) * (psiA * Vj[4] + Vj[8]);
}

// Flux and dissipation matrices of the entropy-stable 9-wave solvers (Riemann 14 Derigs, 15 FloGor):
// EntropyStableDerigsFlux_VolFluxAndDissipMatrices mhd/riemann.f90:1287-1622 and
// EntropyStableFloGorFlux_VolFluxAndDissipMatrices :1695-2042: the EC flux F, the diagonal D and the
// right eigenvectors R[row][col] (the ES flux is F - 1/2 R D R^T [v]).
// pL, pR, bL, bR: the pressures and betas of MHD_EntropyJump
inline void MHD_ES9WaveMatrices(const Case& C, const real* UL, const real* UR, bool flogor, const real& pL,
                                const real& pR, const real& bL, const real& bR, real* F, real* Dm, real R[9][9]) {
  const double ch = C.GLM_ch;
  real sL = 1. / UL[0], sR = 1. / UR[0];
  real uL[3], uR[3];
  for (int d = 0; d < 3; ++d) { uL[d] = UL[1 + d] * sL; uR[d] = UR[1 + d] * sR; }
  real rhoLN = LN_MEAN(UL[0], UR[0]);
  real sbetaLN = 1. / LN_MEAN(bL, bR);
  real uA[3], BA[3];
  for (int d = 0; d < 3; ++d) { uA[d] = 0.5 * (uL[d] + uR[d]); BA[d] = 0.5 * (UL[5 + d] + UR[5 + d]); }
  real betaA = 0.5 * (bL + bR);
  real pA = 0.5 * (UL[0] + UR[0]) / (bL + bR);
  real psiA = 0.5 * (UL[8] + UR[8]);
  if (flogor) {
    MHD_FloGorFlux(C, UL, UR, F);
  } else {  // the central flux as EntropyStableDerigsFlux_VolFluxAndDissipMatrices writes it (:1346-1366)
    real u2L = uL[0] * uL[0] + uL[1] * uL[1] + uL[2] * uL[2], u2R = uR[0] * uR[0] + uR[1] * uR[1] + uR[2] * uR[2];
    real B2L = UL[5] * UL[5] + UL[6] * UL[6] + UL[7] * UL[7], B2R = UR[5] * UR[5] + UR[6] * UR[6] + UR[7] * UR[7];
    real u2Av = 0.5 * (u2L + u2R), B2A = 0.5 * (B2L + B2R);
    real u1B2 = 0.5 * (uL[0] * B2L + uR[0] * B2R);
    real uBA = 0.5 * ((uL[0] * UL[5] + uL[1] * UL[6] + uL[2] * UL[7]) + (uR[0] * UR[5] + uR[1] * UR[6] + uR[2] * UR[7]));
    real pTilde = pA + C.s2mu_0 * B2A;
    F[0] = rhoLN * uA[0];
    F[1] = F[0] * uA[0] - C.smu_0 * BA[0] * BA[0] + pTilde;
    F[2] = F[0] * uA[1] - C.smu_0 * BA[0] * BA[1];
    F[3] = F[0] * uA[2] - C.smu_0 * BA[0] * BA[2];
    F[6] = uA[0] * BA[1] - BA[0] * uA[1];
    F[7] = uA[0] * BA[2] - BA[0] * uA[2];
    F[5] = ch * psiA;
    F[8] = ch * BA[0];
    F[4] = F[0] * 0.5 * (C.sKappaM1 * sbetaLN - u2Av) + (uA[0] * F[1] + uA[1] * F[2] + uA[2] * F[3]) +
           C.smu_0 * ((BA[0] * F[5] + BA[1] * F[6] + BA[2] * F[7]) - 0.5 * u1B2 + BA[0] * uBA + F[8] * psiA -
                      ch * 0.5 * (UL[5] * UL[8] + UR[5] * UR[8]));
  }
  real rhoA = 0.5 * (UL[0] + UR[0]);
  real pLN = 0.5 * rhoLN * sbetaLN;
  real u2A = uL[0] * uR[0] + uL[1] * uR[1] + uL[2] * uR[2];
  real aA = sqrt(C.kappa * pA / rhoLN);
  real aLN = sqrt(C.kappa * pLN / rhoLN);
  real abeta = sqrt(0.5 * C.kappa / betaA);
  real bb1 = BA[0] / sqrt(rhoLN), bb2 = BA[1] / sqrt(rhoLN), bb3 = BA[2] / sqrt(rhoLN);
  real bbA = sqrt(bb1 * bb1 + bb2 * bb2 + bb3 * bb3);
  real aabb = aA * aA + bbA * bbA;
  real ca = fabs(bb1);
  real xx = aabb * aabb - 4.0 * aA * aA * bb1 * bb1;
  if (xx < 0.0) xx = 0.0;
  real xxx = aabb + sqrt(xx);
  real cf = sqrt(0.5 * xxx);
  xxx = aabb - sqrt(xx);
  if (xxx < 0.0) xxx = 0.0;
  real cs = sqrt(0.5 * xxx);
  real bperp = sqrt(bb2 * bb2 + bb3 * bb3);
  real be2, be3;
  if (bperp > 1.0E-14) { be2 = bb2 / bperp; be3 = bb3 / bperp; }
  else { bperp = 0.0; be2 = 1.0 / sqrt(2.0); be3 = 1.0 / sqrt(2.0); }
  xx = 0.0;
  if ((cf * cf - cs * cs) > 0.0) xx = (aA * aA - cs * cs) / (cf * cf - cs * cs);
  real alf = (xx > 0.0) ? sqrt(xx) : real(0.0);
  xx = 0.0;
  if ((cf * cf - cs * cs) > 0.0) xx = (cf * cf - aA * aA) / (cf * cf - cs * cs);
  real als = (xx > 0.0) ? sqrt(xx) : real(0.0);
  double sg = std::copysign(1., val(bb1));  // SIGN(1.,bb1A)
  real t23 = uA[1] * be2 + uA[2] * be3;
  real psiSp = 0.5 * als * rhoLN * u2A - abeta * alf * rhoLN * bperp + als * rhoLN * aLN * aLN * C.sKappaM1 +
               als * cs * rhoLN * uA[0] + alf * cf * rhoLN * sg * t23;
  real psiSm = 0.5 * als * rhoLN * u2A - abeta * alf * rhoLN * bperp + als * rhoLN * aLN * aLN * C.sKappaM1 -
               als * cs * rhoLN * uA[0] - alf * cf * rhoLN * sg * t23;
  real psiFp = 0.5 * alf * rhoLN * u2A + abeta * als * rhoLN * bperp + alf * rhoLN * aLN * aLN * C.sKappaM1 +
               alf * cf * rhoLN * uA[0] - als * cs * rhoLN * sg * t23;
  real psiFm = 0.5 * alf * rhoLN * u2A + abeta * als * rhoLN * bperp + alf * rhoLN * aLN * aLN * C.sKappaM1 -
               alf * cf * rhoLN * uA[0] + als * cs * rhoLN * sg * t23;
  real sqRho = sqrt(rhoLN), sqRhoA = sqrt(rhoA);
  // R[row][col] = Rmatrix(row+1, col+1)
  real c1[9] = {alf * rhoLN, alf * rhoLN * (uA[0] + cf), rhoLN * (alf * uA[1] - als * cs * be2 * sg),
                rhoLN * (alf * uA[2] - als * cs * be3 * sg), psiFp, 0.0, als * abeta * be2 * sqRho,
                als * abeta * be3 * sqRho, 0.0};
  real c2[9] = {0.0, 0.0, rhoLN * sqRhoA * be3, -rhoLN * sqRhoA * be2, -rhoLN * sqRhoA * (be2 * uA[2] - be3 * uA[1]),
                0.0, -rhoLN * be3, rhoLN * be2, 0.0};
  real c3[9] = {als * rhoLN, als * rhoLN * (uA[0] + cs), rhoLN * (als * uA[1] + alf * cf * be2 * sg),
                rhoLN * (als * uA[2] + alf * cf * be3 * sg), psiSp, 0.0, -alf * abeta * be2 * sqRho,
                -alf * abeta * be3 * sqRho, 0.0};
  real c4[9] = {0.0, 0.0, 0.0, 0.0, BA[0] + psiA, 1.0, 0.0, 0.0, 1.0};
  real c5[9] = {1.0, uA[0], uA[1], uA[2], 0.5 * u2A, 0.0, 0.0, 0.0, 0.0};
  real c6[9] = {0.0, 0.0, 0.0, 0.0, BA[0] - psiA, 1.0, 0.0, 0.0, -1.0};
  real c7[9] = {als * rhoLN, als * rhoLN * (uA[0] - cs), rhoLN * (als * uA[1] - alf * cf * be2 * sg),
                rhoLN * (als * uA[2] - alf * cf * be3 * sg), psiSm, 0.0, -alf * abeta * be2 * sqRho,
                -alf * abeta * be3 * sqRho, 0.0};
  real c8[9] = {0.0, 0.0, -rhoLN * sqRhoA * be3, rhoLN * sqRhoA * be2, rhoLN * sqRhoA * (be2 * uA[2] - be3 * uA[1]),
                0.0, -rhoLN * be3, rhoLN * be2, 0.0};
  real c9[9] = {alf * rhoLN, alf * rhoLN * (uA[0] - cf), rhoLN * (alf * uA[1] + als * cs * be2 * sg),
                rhoLN * (alf * uA[2] + als * cs * be3 * sg), psiFm, 0.0, als * abeta * be2 * sqRho,
                als * abeta * be3 * sqRho, 0.0};
  const real* cols[9] = {c1, c2, c3, c4, c5, c6, c7, c8, c9};
  for (int c = 0; c < 9; ++c)
    for (int r = 0; r < 9; ++r) R[r][c] = cols[c][r];
  real phi = sqrt(fabs(1.0 - (pR * UR[0] / (pL * UL[0]))) / (1.0 + (pR * UR[0] / (pL * UL[0]))));
  real LM = fmax(fabs(uA[0] + cf), fabs(uA[0] - cf));
  real wave[9] = {uA[0] + cf, uA[0] + ca, uA[0] + cs, uA[0] + ch, uA[0], uA[0] - ch, uA[0] - cs, uA[0] - ca,
                  uA[0] - cf};
  real T1 = 0.5 / C.kappa / rhoLN, T2 = 0.25 / betaA / rhoLN / rhoLN, T4 = 0.25 / betaA,
       T5 = rhoLN * C.kappaM1 / C.kappa;
  real Tm[9] = {T1, T2, T1, T4, T5, T4, T1, T2, T1};
  for (int z = 0; z < 9; ++z) Dm[z] = ((1. - phi) * fabs(wave[z]) + phi * LM) * Tm[z];
}

// EntropyStableDerigsFlux / EntropyStableFloGorFlux (Riemann 14 / 15), mhd/riemann.f90:1224-1283,
// :1633-1691: Fstar - 0.5*MATMUL(R, D*MATMUL(R^T, V_jump))
inline void MHD_EntropyStable9Wave(const Case& C, const real* UL, const real* UR, bool flogor, real* F) {
  real Vj[9], pL, pR, bL, bR;
  MHD_EntropyJump(C, UL, UR, pL, pR, bL, bR, Vj);
  real Dm[9], R[9][9];
  MHD_ES9WaveMatrices(C, UL, UR, flogor, pL, pR, bL, bR, F, Dm, R);
  real w[9];
  for (int c = 0; c < 9; ++c) {
    real s = 0.;
    for (int r = 0; r < 9; ++r) s = s + R[r][c] * Vj[r];
    w[c] = Dm[c] * s;
  }
  for (int r = 0; r < 9; ++r) {
    real s = 0.;
    for (int c = 0; c < 9; ++c) s = s + R[r][c] * w[c];
    F[r] = F[r] - 0.5 * s;
  }
}


// RiemannSolverByHLLC, mhd/riemann.f90:371-501 (with GLM), HLL state EvalHLLState :733-757
inline void MHD_HLLC(const Case& C, const real* UL, const real* UR, real* F) {
  real PL[9], PR[9];
  MHD_ConsToPrim(C, UL, PL);
  MHD_ConsToPrim(C, UR, PR);
  real cfL = MHD_FastestWave1D(C, PL), RoeVelx, cfRoe;
  MHD_FastestWave1D_Roe(C, UL, UR, PL, PR, RoeVelx, cfRoe);
  real SL = fmin(PL[1] - cfL, RoeVelx - cfRoe);
  if (SL > 0.0) { MHD_Flux1D(C, UL, F); return; }
  real cfR = MHD_FastestWave1D(C, PR);
  real SR = fmax(RoeVelx + cfRoe, PR[1] + cfR);
  if (SR < 0.0) { MHD_Flux1D(C, UR, F); return; }
  real FL[9], FR[9], UH[9];
  MHD_Flux1D(C, UL, FL);
  MHD_Flux1D(C, UR, FR);
  for (int v = 0; v < 9; ++v) UH[v] = (SR * UR[v] - SL * UL[v] - FR[v] + FL[v]) / (SR - SL);
  real ptotL = PL[4] + C.s2mu_0 * (PL[5] * PL[5] + PL[6] * PL[6] + PL[7] * PL[7]);
  real sRhoH = 1. / UH[0];
  real SM = UH[1] * sRhoH;
  real Bx = UH[5], By = UH[6], Bz = UH[7];
  real pS = ptotL + PL[0] * (PL[1] - SL) * (PL[1] - SM) - C.s2mu_0 * (PL[5] * PL[5] - Bx * Bx);
  real ES = pS * SM + C.smu_0 * (-Bx * (UH[5] * UH[1] + UH[6] * UH[2] + UH[7] * UH[3]) * sRhoH +
                                 UH[8] * (C.GLM_ch * Bx - 0.5 * UH[8] * SM));
  const bool left = (SL <= 0.0) && (0.0 < SM);
  const real* U = left ? UL : UR;
  const real* P = left ? PL : PR;
  const real* FF = left ? FL : FR;
  real S = left ? SL : SR;
  real s = 1. / (S - SM);
  real Us[9];
  Us[0] = P[0] * (S - P[1]) * s;
  Us[1] = Us[0] * SM;
  Us[2] = (U[2] * S - FF[2] - C.smu_0 * Bx * By) * s;
  Us[3] = (U[3] * S - FF[3] - C.smu_0 * Bx * Bz) * s;
  Us[4] = (ES + U[4] * S - FF[4]) * s;
  Us[5] = Bx; Us[6] = By; Us[7] = Bz;
  Us[8] = U[8];
  for (int v = 0; v < 9; ++v) F[v] = FF[v] + S * (Us[v] - U[v]);
}

// RiemannSolverByHLLD, mhd/riemann.f90:511-729 (mu_0 = 1; B_n made continuous first)
inline void MHD_HLLD(const Case& C, const real* ULin, const real* URin, real* F) {
  const double eps = 1.0e-8, small = 1.0e-12;
  real PL[9], PR[9], UL[9], UR[9];
  MHD_ConsToPrim(C, ULin, PL);
  MHD_ConsToPrim(C, URin, PR);
  real Bn = 0.5 * (PL[5] + PR[5]);
  PL[5] = Bn; PR[5] = Bn;
  MHD_PrimToCons(C, PL, UL);
  MHD_PrimToCons(C, PR, UR);
  real FW = fmax(MHD_FastestWave1D(C, PL), MHD_FastestWave1D(C, PR));
  real SL = fmin(PL[1], PR[1]) - FW;
  if (SL > 0.0) { MHD_Flux1D(C, UL, F); return; }
  real SR = fmax(PL[1], PR[1]) + FW;
  if (SR < 0.0) { MHD_Flux1D(C, UR, F); return; }
  real FL[9], FR[9];
  MHD_Flux1D(C, UL, FL);
  MHD_Flux1D(C, UR, FR);
  real rhoL = PL[0], rhoR = PR[0], unL = PL[1], unR = PR[1];
  real ptotL = PL[4] + 0.5 * (PL[5] * PL[5] + PL[6] * PL[6] + PL[7] * PL[7]);
  real ptotR = PR[4] + 0.5 * (PR[5] * PR[5] + PR[6] * PR[6] + PR[7] * PR[7]);
  real SM = (rhoR * unR * (SR - unR) - rhoL * unL * (SL - unL) - ptotR + ptotL) /
            (rhoR * (SR - unR) - rhoL * (SL - unL));
  real sSL = 1. / (SL - SM), sSR = 1. / (SR - SM);
  real rhoLS = rhoL * (SL - unL) * sSL, rhoRS = rhoR * (SR - unR) * sSR;
  real sqLS = sqrt(rhoLS), sqRS = sqrt(rhoRS);
  real SLS = SM - fabs(Bn) / sqLS, SRS = SM + fabs(Bn) / sqRS;
  real ptotS = ptotL + rhoL * (SL - unL) * (SM - unL);
  // tangential velocity and field of the * states (index 0 = normal, zero)
  real utLS[3] = {0., PL[2], PL[3]}, BtLS[3] = {0., PL[6], PL[7]};
  real utRS[3] = {0., PR[2], PR[3]}, BtRS[3] = {0., PR[6], PR[7]};
  real temp = rhoL * (SL - unL) * (SL - SM) - Bn * Bn;
  if (!(fabs(temp) < eps)) {
    real st = 1. / temp;
    real a = Bn * (SM - unL) * st, b = (rhoL * (SL - unL) * (SL - unL) - Bn * Bn) * st;
    for (int d = 1; d < 3; ++d) { utLS[d] = utLS[d] - a * BtLS[d]; BtLS[d] = b * BtLS[d]; }
  }
  real uBS = SM * Bn + utLS[1] * BtLS[1] + utLS[2] * BtLS[2];
  real uB = PL[1] * PL[5] + PL[2] * PL[6] + PL[3] * PL[7];
  real eLS = (UL[4] * (SL - unL) + ptotS * SM - ptotL * unL + Bn * (uB - uBS)) * sSL;
  real ULS[9] = {rhoLS, rhoLS * SM, rhoLS * utLS[1], rhoLS * utLS[2], eLS, Bn, BtLS[1], BtLS[2], UL[8]};
  temp = rhoR * (SR - unR) * (SR - SM) - Bn * Bn;
  if (!(fabs(temp) < eps)) {
    real st = 1. / temp;
    real a = Bn * (SM - unR) * st, b = (rhoR * (SR - unR) * (SR - unR) - Bn * Bn) * st;
    for (int d = 1; d < 3; ++d) { utRS[d] = utRS[d] - a * BtRS[d]; BtRS[d] = b * BtRS[d]; }
  }
  uBS = SM * Bn + utRS[1] * BtRS[1] + utRS[2] * BtRS[2];
  uB = PR[1] * PR[5] + PR[2] * PR[6] + PR[3] * PR[7];
  real eRS = (UR[4] * (SR - unR) - ptotR * unR + ptotS * SM + Bn * (uB - uBS)) * sSR;
  real URS[9] = {rhoRS, rhoRS * SM, rhoRS * utRS[1], rhoRS * utRS[2], eRS, Bn, BtRS[1], BtRS[2], UR[8]};
  real ULSS[9], URSS[9];
  for (int v = 0; v < 9; ++v) { ULSS[v] = ULS[v]; URSS[v] = URS[v]; }
  if (!(fabs(Bn) < small)) {
    real sgn = Bn < 0.0 ? -1.0 : 1.0;
    real st = 1. / (sqLS + sqRS);
    real utSS[3], BtSS[3];
    for (int d = 1; d < 3; ++d) {
      utSS[d] = (sqLS * utLS[d] + sqRS * utRS[d] + sgn * (BtRS[d] - BtLS[d])) * st;
      BtSS[d] = (sqLS * BtRS[d] + sqRS * BtLS[d] + sgn * (utRS[d] - utLS[d]) * sqLS * sqRS) * st;
    }
    uBS = utSS[1] * BtSS[1] + utSS[2] * BtSS[2];
    real eLSS = eLS - sgn * sqLS * ((utLS[1] * BtLS[1] + utLS[2] * BtLS[2]) - uBS);
    real eRSS = eRS + sgn * sqRS * ((utRS[1] * BtRS[1] + utRS[2] * BtRS[2]) - uBS);
    real uSS[3] = {SM, utSS[1], utSS[2]}, BSS[3] = {Bn, BtSS[1], BtSS[2]};
    for (int d = 0; d < 3; ++d) {
      ULSS[1 + d] = rhoLS * uSS[d]; URSS[1 + d] = rhoRS * uSS[d];
      ULSS[5 + d] = BSS[d]; URSS[5 + d] = BSS[d];
    }
    ULSS[4] = eLSS; URSS[4] = eRSS;
  }
  if (0.0 <= SLS) {
    for (int v = 0; v < 9; ++v) F[v] = FL[v] + SL * (ULS[v] - UL[v]);
  } else if (0.0 <= SM) {
    for (int v = 0; v < 9; ++v) F[v] = FL[v] + SLS * ULSS[v] - (SLS - SL) * ULS[v] - SL * UL[v];
  } else if (0.0 <= SRS) {
    for (int v = 0; v < 9; ++v) F[v] = FR[v] + SRS * URSS[v] - (SRS - SR) * URS[v] - SR * UR[v];
  } else {
    for (int v = 0; v < 9; ++v) F[v] = FR[v] + SR * (URS[v] - UR[v]);
  }
}

// RiemannSolverByRoe, mhd/riemann.f90:764-1024 (Cargo & Gallice Roe matrix, entropy fix on the
// waves 1, 3, 6, 7 as in the reference)
inline void MHD_Roe(const Case& C, const real* UL, const real* UR, real* F) {
  const double efix = 1.0e-6, sefix = 1.0e6;
  real PL[9], PR[9];
  MHD_ConsToPrim(C, UL, PL);
  MHD_ConsToPrim(C, UR, PR);
  real sqL = sqrt(PL[0]), sqR = sqrt(PR[0]);
  real sS = 1. / (sqL + sqR);
  real RL = sqL * sS, RR = sqR * sS;
  real ptL = PL[4] + C.s2mu_0 * (PL[5] * PL[5] + PL[6] * PL[6] + PL[7] * PL[7]);
  real ptR = PR[4] + C.s2mu_0 * (PR[5] * PR[5] + PR[6] * PR[6] + PR[7] * PR[7]);
  real rhoRoe = sqL * sqR;
  real sRhoRoe = 1. / rhoRoe;
  real sqRoe = sqrt(rhoRoe);
  real ssqRoe = 1. / sqRoe;
  real v[3], B[3];
  for (int d = 0; d < 3; ++d) { v[d] = RL * PL[1 + d] + RR * PR[1 + d]; B[d] = RL * PR[5 + d] + RR * PL[5 + d]; }
  real v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  real B2 = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
  real HL = (UL[4] + ptL) / PL[0], HR = (UR[4] + ptR) / PR[0];
  real H = RL * HL + RR * HR;
  real dB0 = PL[5] - PR[5], dB1 = PL[6] - PR[6], dB2 = PL[7] - PR[7];
  real XX = 0.5 * (dB0 * dB0 + dB1 * dB1 + dB2 * dB2) * (sS * sS);
  real va2 = B2 * C.smu_0 * sRhoRoe;
  real c2 = (2. - C.kappa) * XX + C.kappaM1 * (H - 0.5 * v2 - va2);
  real sc2 = 1. / c2;
  real c = sqrt(c2);
  real ca2 = B[0] * B[0] * C.smu_0 * sRhoRoe;
  real ca = sqrt(ca2);
  real astar = sqrt((c2 + va2) * (c2 + va2) - 4. * c2 * ca2);
  real cf2 = 0.5 * (c2 + va2 + astar), cf = sqrt(cf2);
  real cs2 = 0.5 * (c2 + va2 - astar), cs = sqrt(cs2);
  real FL[9], FR[9];
  MHD_Flux1D(C, UL, FL);
  MHD_Flux1D(C, UR, FR);
  real sBx = std::signbit(val(B[0])) ? -1.0 : 1.0;
  real Bt = sqrt(B[1] * B[1] + B[2] * B[2]);
  real by, bz;
  if (Bt > 1.0e-9) { by = B[1] / Bt; bz = B[2] / Bt; } else { by = sqrt(real(0.5)); bz = by; }
  real af, as;
  if (val(cf2) == val(cs2)) { af = 1.; as = 0.; }
  else if (c2 <= cs2) { af = 0.; as = 1.; }
  else if (cf2 <= c2) { af = 1.; as = 0.; }
  else {
    real s = 1. / (cf2 - cs2);
    af = sqrt(fmax(real(0.), (c2 - cs2) * s));
    as = sqrt(fmax(real(0.), (cf2 - c2) * s));
  }
  real drho = PR[0] - PL[0];
  real dv[3] = {PR[1] - PL[1], PR[2] - PL[2], PR[3] - PL[3]};
  real dB[3] = {PR[5] - PL[5], PR[6] - PL[6], PR[7] - PL[7]};
  real dp = C.kappaM1 * ((0.5 * v2 - XX) * drho -
                         (v[0] * (UR[1] - UL[1]) + v[1] * (UR[2] - UL[2]) + v[2] * (UR[3] - UL[3])) +
                         (UR[4] - UL[4]) - C.smu_0 * (B[0] * dB[0] + B[1] * dB[1] + B[2] * dB[2]));
  real lam[7] = {v[0] - cf, v[0] - ca, v[0] - cs, v[0], v[0] + cs, v[0] + ca, v[0] + cf};
  real eta[7];
  real bv = by * v[1] + bz * v[2], bdv = by * dv[1] + bz * dv[2], bdB = by * dB[1] + bz * dB[2];
  real ascs = as * cs * sBx, asc = as * c * ssqRoe;
  real EVr1[8] = {af, af * lam[0], af * v[1] + ascs * by, af * v[2] + ascs * bz,
                  af * (H - va2 - v[0] * cf) + ascs * bv + asc * Bt, 0., asc * by, asc * bz};
  real EVr7[8] = {af, af * lam[6], af * v[1] - ascs * by, af * v[2] - ascs * bz,
                  af * (H - va2 + v[0] * cf) - ascs * bv + asc * Bt, 0., asc * by, asc * bz};
  eta[0] = 0.5 * sc2 * (af * (XX * drho + dp) + rhoRoe * (ascs * bdv - af * cf * dv[0] + asc * bdB));
  eta[6] = 0.5 * sc2 * (af * (XX * drho + dp) - rhoRoe * (ascs * bdv - af * cf * dv[0] - asc * bdB));
  real afcf = af * cf * sBx, afc = af * c * ssqRoe;
  real EVr3[8] = {as, as * lam[2], as * v[1] - afcf * by, as * v[2] - afcf * bz,
                  as * (H - va2 - v[0] * cs) - afcf * bv - afc * Bt, 0., -afc * by, -afc * bz};
  real EVr5[8] = {as, as * lam[4], as * v[1] + afcf * by, as * v[2] + afcf * bz,
                  as * (H - va2 + v[0] * cs) + afcf * bv - afc * Bt, 0., -afc * by, -afc * bz};
  eta[2] = 0.5 * sc2 * (as * (XX * drho + dp) - rhoRoe * (afcf * bdv + as * cs * dv[0] + afc * bdB));
  eta[4] = 0.5 * sc2 * (as * (XX * drho + dp) + rhoRoe * (afcf * bdv + as * cs * dv[0] - afc * bdB));
  bv = bz * v[1] - by * v[2];
  bdv = bz * dv[1] - by * dv[2];
  bdB = bz * dB[1] - by * dB[2];
  real EVr2[8] = {0., 0., -rhoRoe * bz, rhoRoe * by, -rhoRoe * bv, 0., -sBx * sqRoe * bz, sBx * sqRoe * by};
  real EVr6[8] = {0., 0., rhoRoe * bz, -rhoRoe * by, rhoRoe * bv, 0., -sBx * sqRoe * bz, sBx * sqRoe * by};
  eta[1] = 0.5 * (-bdv - sBx * ssqRoe * bdB);
  eta[5] = 0.5 * (bdv - sBx * ssqRoe * bdB);
  real EVr4[8] = {1., v[0], v[1], v[2], 0.5 * v2 + C.kappaM2 * C.sKappaM1 * XX, 0., 0., 0.};
  eta[3] = sc2 * ((c2 - XX) * drho - dp);
  for (int z : {0, 6, 2, 5})
    if (fabs(lam[z]) < 0.5 * efix) lam[z] = lam[z] * lam[z] * sefix + 0.25 * efix;
  const real* EV7[7] = {EVr1, EVr2, EVr3, EVr4, EVr5, EVr6, EVr7};
  for (int v9 = 0; v9 < 9; ++v9) F[v9] = FL[v9] + FR[v9];
  for (int i = 0; i < 7; ++i) {
    real g = eta[i] * fabs(lam[i]);
    for (int r = 0; r < 8; ++r) F[r] = F[r] - g * EV7[i][r];
  }
  for (int v9 = 0; v9 < 9; ++v9) F[v9] = 0.5 * F[v9];
}

// SolveRiemannProblem (rotated frame) for the MHD solvers, mhd/equation.f90:311-391
inline void MHD_Riemann(const Case& C, const real* UL, const real* UR, real* F) {
  switch (C.P.riemann) {
    case 0: MHD_StandardDGFlux(C, UL, UR, F); return;
    case 1: {  // RiemannSolverByRusanov, mhd/riemann.f90:273-308
      real FL[9], FR[9], PL[9], PR[9];
      MHD_Flux1D(C, UL, FL);
      MHD_Flux1D(C, UR, FR);
      MHD_ConsToPrim(C, UL, PL);
      MHD_ConsToPrim(C, UR, PR);
      real cfL = MHD_FastestWave1D(C, PL), cfR = MHD_FastestWave1D(C, PR);
      real LM = fmax(fabs(PL[1]) + cfL, fabs(PR[1]) + cfR);
      for (int v = 0; v < 9; ++v) F[v] = 0.5 * ((FL[v] + FR[v]) - LM * (UR[v] - UL[v]));
      return;
    }
    case 4: {  // RiemannSolverByHLL, mhd/riemann.f90:314-364
      real PL[9], PR[9];
      MHD_ConsToPrim(C, UL, PL);
      MHD_ConsToPrim(C, UR, PR);
      real cfL = MHD_FastestWave1D(C, PL), RoeVelx, cfRoe;
      MHD_FastestWave1D_Roe(C, UL, UR, PL, PR, RoeVelx, cfRoe);
      real SL = fmin(PL[1] - cfL, RoeVelx - cfRoe);
      if (SL > 0.0) { MHD_Flux1D(C, UL, F); return; }
      real cfR = MHD_FastestWave1D(C, PR);
      real SR = fmax(RoeVelx + cfRoe, PR[1] + cfR);
      if (SR < 0.0) { MHD_Flux1D(C, UR, F); return; }
      real FL[9], FR[9];
      MHD_Flux1D(C, UL, FL);
      MHD_Flux1D(C, UR, FR);
      for (int v = 0; v < 9; ++v) F[v] = (SR * FL[v] - SL * FR[v] + SL * SR * (UR[v] - UL[v])) / (SR - SL);
      return;
    }
    case 2: MHD_HLLC(C, UL, UR, F); return;
    case 3: MHD_Roe(C, UL, UR, F); return;
    case 5: MHD_HLLD(C, UL, UR, F); return;
    case 10: MHD_EntropyStableLLF(C, UL, UR, false, F); return;
    case 11: MHD_DerigsFlux(C, UL, UR, F); return;
    case 12: MHD_FloGorFlux(C, UL, UR, F); return;
    case 13: MHD_EntropyStableLLF(C, UL, UR, true, F); return;
    case 14: MHD_EntropyStable9Wave(C, UL, UR, false, F); return;
    case 15: MHD_EntropyStable9Wave(C, UL, UR, true, F); return;
    default: throw std::runtime_error("MHD Riemann solver not implemented in oracle");
  }
}

// Surface non-conservative term on the UL side (AddNonConsFlux, mhd/riemann.f90:230-267),
// before the SurfElem scaling; nv is the master side's normal for both sides.
inline void MHD_NonConsSurf(const Case& C, const real* UL, const real* UR, const double* nv, real* F) {
  if (C.noncons == 0) return;
  real vL[3] = {UL[1] / UL[0], UL[2] / UL[0], UL[3] / UL[0]};
  real Bn = 0.5 * ((UL[5] + UR[5]) * nv[0] + (UL[6] + UR[6]) * nv[1] + (UL[7] + UR[7]) * nv[2]);
  if (C.noncons == 1) {
    real vB = UL[5] * vL[0] + UL[6] * vL[1] + UL[7] * vL[2];
    real phi[7] = {UL[5], UL[6], UL[7], vB, vL[0], vL[1], vL[2]};
    for (int v = 0; v < 7; ++v) F[1 + v] = F[1 + v] + Bn * phi[v];
  } else if (C.noncons == 2) {
    for (int v = 0; v < 3; ++v) F[1 + v] = F[1 + v] + Bn * UL[5 + v];
  } else {
    for (int v = 0; v < 3; ++v) F[5 + v] = F[5 + v] + Bn * vL[v];
  }
  if (C.ncGLM) {
    real q = 0.5 * (vL[0] * nv[0] + vL[1] * nv[1] + vL[2] * nv[2]);
    F[4] = F[4] + q * (UL[8] * (UR[8] + UL[8]));
    F[8] = F[8] + q * (UR[8] + UL[8]);
  }
}

// ConvertToGradPrim, mhd/equation_vars.f90:547-628 (one point, in place)
inline void MHD_ConvertToGradPrim(const Case& C, const real* U, real* g) {
  if (C.P.lifting_var == 1) {
    real sRho = 1. / U[0];
    real u = U[1] * sRho, v = U[2] * sRho, w = U[3] * sRho;
    real gi1 = g[0];
    real gu = sRho * (g[1] - g[0] * u), gv = sRho * (g[2] - g[0] * v), gw = sRho * (g[3] - g[0] * w);
    real gi5 = g[4];
    g[1] = gu; g[2] = gv; g[3] = gw;
    g[4] = C.kappaM1 * (gi5 - (0.5 * gi1 * (u * u + v * v + w * w) + (U[1] * gu + U[2] * gv + U[3] * gw)) -
                        C.smu_0 * (U[5] * g[5] + U[6] * g[6] + U[7] * g[7] + U[8] * g[8]));
  } else if (C.P.lifting_var == 2) {
    return;
  } else {
    real sRho = 1. / U[0];
    real u = U[1] * sRho, v = U[2] * sRho, w = U[3] * sRho;
    real Ekin = 0.5 * (U[1] * u + U[2] * v + U[3] * w);
    real p = C.kappaM1 * (U[4] - Ekin - C.s2mu_0 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7] + U[8] * U[8]));
    real rho_sp = U[0] / p;
    real p_srho = p * sRho;
    real gi1 = g[0];
    real gu = p_srho * (g[1] + u * g[4]), gv = p_srho * (g[2] + v * g[4]), gw = p_srho * (g[3] + w * g[4]);
    real gi5 = g[4];
    g[0] = U[0] * gi1 - gi5 * (Ekin - p * C.sKappaM1) + rho_sp * (U[1] * gu + U[2] * gv + U[3] * gw);
    g[1] = gu; g[2] = gv; g[3] = gw;
    g[4] = p_srho * (g[0] + p * gi5);
    for (int z = 5; z < 9; ++z) g[z] = p_srho * (g[z] + U[z] * gi5);
  }
}

// EvalDiffFlux3D (one point), mhd/flux.f90:449-573 (isotropic heat flux, constant mu)
inline void MHD_DiffFlux3D(const Case& C, const real* U, const real* gX, const real* gY, const real* gZ, real* f,
                           real* g, real* h) {
  real srho = 1. / U[0];
  real v1 = U[1] * srho, v2 = U[2] * srho, v3 = U[3] * srho;
  real b1 = U[5], b2 = U[6], b3 = U[7];
  real p = C.kappaM1 * (U[4] - 0.5 * (U[0] * (v1 * v1 + v2 * v2 + v3 * v3)) -
                        C.s2mu_0 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7] + U[8] * U[8]));
  real divv = gX[1] + gY[2] + gZ[3];
  real cvTx = C.sKappaM1 * srho * (gX[4] - srho * p * gX[0]);
  real cvTy = C.sKappaM1 * srho * (gY[4] - srho * p * gY[0]);
  real cvTz = C.sKappaM1 * srho * (gZ[4] - srho * p * gZ[0]);
  const double mu = C.muMHD, es = C.etasmu_0;
  real lambda = mu * C.KappasPr;
  real Qx = lambda * cvTx, Qy = lambda * cvTy, Qz = lambda * cvTz;
  f[0] = 0.;
  f[1] = -mu * (2 * gX[1] - C.s23 * divv);
  f[2] = -mu * (gX[2] + gY[1]);
  f[3] = -mu * (gX[3] + gZ[1]);
  f[5] = 0.;
  f[6] = -es * (gX[6] - gY[5]);
  f[7] = -es * (gX[7] - gZ[5]);
  f[4] = v1 * f[1] + v2 * f[2] + v3 * f[3] + C.smu_0 * (b1 * f[5] + b2 * f[6] + b3 * f[7]) - Qx;
  g[0] = 0.;
  g[1] = f[2];
  g[2] = -mu * (2 * gY[2] - C.s23 * divv);
  g[3] = -mu * (gY[3] + gZ[2]);
  g[5] = -f[6];
  g[6] = 0.;
  g[7] = -es * (gY[7] - gZ[6]);
  g[4] = v1 * g[1] + v2 * g[2] + v3 * g[3] + C.smu_0 * (b1 * g[5] + b2 * g[6] + b3 * g[7]) - Qy;
  h[0] = 0.;
  h[1] = f[3];
  h[2] = g[3];
  h[3] = -mu * (2 * gZ[3] - C.s23 * divv);
  h[5] = -f[7];
  h[6] = -g[7];
  h[7] = 0.;
  h[4] = v1 * h[1] + v2 * h[2] + v3 * h[3] + C.smu_0 * (b1 * h[5] + b2 * h[6] + b3 * h[7]) - Qz;
  f[8] = 0.; g[8] = 0.; h[8] = 0.;
}

// ExactFunc, mhd/equation.f90:544-1461 (the cases used by the tests and configs)
void MHD_ExactFunc(const Case& C, int func, double t, const double* x, double* resu) {
  const orc_params& P = C.P;
  double prim[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  switch (func) {
    case 1: {  // constant RefStateCons(IniRefState)
      for (int v = 0; v < 8; ++v) prim[v] = P.mhd_ref_state[0][v];
      MHD_PrimToCons(C, prim, resu);
      return;
    }
    case 3: {  // Alfven wave, domain [-1,1]^3, :596-639
      prim[4] = 1.;
      double Omega = 2. * PI * P.ini_frequency, r = 2., e = 0.2;
      double nx = 1. / std::sqrt(r * r + 1.), ny = r / std::sqrt(r * r + 1.), sqr = 1.;
      double Va = Omega / (ny * sqr);
      double phi = Omega / ny * (nx * (x[0] - 0.5 * r) + ny * (x[1] - 0.5 * r)) - Va * t;
      for (int v = 0; v < 9; ++v) resu[v] = 0.;
      resu[0] = 1.;
      resu[1] = -e * ny * std::cos(phi);
      resu[2] = e * nx * std::cos(phi);
      resu[3] = e * std::sin(phi);
      resu[4] = prim[4] * C.sKappaM1 + 0.5 * (resu[1] * resu[1] + resu[2] * resu[2] + resu[3] * resu[3]);
      resu[5] = nx - resu[1] * sqr;
      resu[6] = ny - resu[2] * sqr;
      resu[7] = -resu[3] * sqr;
      return;
    }
    case 201: {  // soft blast between RefState 1 (inside) and 2, :1239-1246
      double r2 = 0.;
      for (int d = 0; d < 3; ++d) r2 += (x[d] - P.ini_center[d]) * (x[d] - P.ini_center[d]);
      double a = std::exp(5. * (std::sqrt(r2) - P.ini_halfwidth) / P.ini_amplitude);
      a = a / (a + 1.);
      for (int v = 0; v < 8; ++v) prim[v] = (1. - a) * P.mhd_ref_state[0][v] + a * P.mhd_ref_state[1][v];
      MHD_PrimToCons(C, prim, resu);
      return;
    }
    case 311: {  // Orszag-Tang vortex, :1248-1256
      prim[0] = 1.;
      prim[1] = -std::sin(2. * PI * x[1]);
      prim[2] = std::sin(2. * PI * x[0]);
      prim[4] = 1. / C.kappa;
      prim[5] = -std::sin(2. * PI * x[1]) / C.kappa;
      prim[6] = std::sin(4. * PI * x[0]) / C.kappa;
      MHD_PrimToCons(C, prim, resu);
      return;
    }
    case 312: {  // 3D perturbed Orszag-Tang vortex, :1257-1266
      prim[0] = 1.;
      prim[1] = -(1. + 0.2 * std::sin(2. * PI * x[2])) * std::sin(2. * PI * x[1]);
      prim[2] = (1. + 0.2 * std::sin(2. * PI * x[2])) * std::sin(2. * PI * x[0]);
      prim[3] = 0.2 * std::sin(2. * PI * x[2]);
      prim[4] = 1. / C.kappa;
      prim[5] = -std::sin(2. * PI * x[1]) / C.kappa;
      prim[6] = std::sin(4. * PI * x[0]) / C.kappa;
      MHD_PrimToCons(C, prim, resu);
      return;
    }
    default: throw std::runtime_error("MHD ExactFunc not implemented in oracle");
  }
}

// InitTimeStep_GLM, mhd/calctimestep.f90:187-223: GLM_dtch1 = min over elements of CFL*2/sum(lambda)
inline void MHD_InitTimeStepGLM(Case& C) {
  const int n = C.np;
  C.GLM_dtch1 = 1.7976931348623157e308;
  for (int e = 0; e < C.nElems; ++e) {
    double ml[3] = {0., 0., 0.};
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          size_t o = C.nod(i, j, k, e);
          const double* M[3] = {&C.Mf[3 * o], &C.Mg[3 * o], &C.Mh[3 * o]};
          for (int d = 0; d < 3; ++d)
            ml[d] = std::max(ml[d], C.sJ[o] * std::sqrt(M[d][0] * M[d][0] + M[d][1] * M[d][1] + M[d][2] * M[d][2]));
        }
    C.GLM_dtch1 = std::min(C.GLM_dtch1, C.CFLScale * 2. / (ml[0] + ml[1] + ml[2]));
  }
  C.GLM_init = true;
}

// CALCTIMESTEP, mhd/calctimestep.f90:38-179 (convective with the fast magnetosonic speed, viscous
// and resistive), then GLM_ch = GLM_scale*GLM_dtch1/dt
inline double MHD_CalcTimeStep(Case& C, int* errType) {
  *errType = 0;
  const int n = C.np;
  double muKappasPr_max = C.muMHD * std::max(4. / 3., C.KappasPr);
  double diffC_max = C.etasmu_0;
  double mlv = 0.;
  if (!C.GLM_init) MHD_InitTimeStepGLM(C);
  double dtConv = 1.7976931348623157e308, dtVisc = 1.7976931348623157e308;
  for (int e = 0; e < C.nElems; ++e) {
    double ml[3] = {0., 0., 0.};
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          size_t o = C.nod(i, j, k, e);
          double U[9], P[9];
          for (int v = 0; v < 9; ++v) U[v] = val(C.U[9 * o + v]);
          if (std::isnan(U[0])) *errType = 1;
          double sRho = 1. / U[0];
          double s2 = C.s2mu_0;
          P[0] = U[0];
          P[1] = U[1] * sRho; P[2] = U[2] * sRho; P[3] = U[3] * sRho;
          P[4] = C.kappaM1 * (U[4] - 0.5 * (U[1] * P[1] + U[2] * P[2] + U[3] * P[3]) -
                              s2 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7] + U[8] * U[8]));
          if (P[4] <= 0.) *errType = 2;
          // FastestWave3D, mhd/equation_vars.f90:690-709
          double cf = std::sqrt((C.kappa * P[4] + (U[5] * U[5] + U[6] * U[6] + U[7] * U[7]) * C.smu_0) / P[0]);
          const double* M[3] = {&C.Mf[3 * o], &C.Mg[3 * o], &C.Mh[3 * o]};
          double sj = C.sJ[o];
          for (int d = 0; d < 3; ++d)
            ml[d] = std::max(ml[d], sj * (std::fabs(M[d][0] * P[1] + M[d][1] * P[2] + M[d][2] * P[3]) +
                                          cf * std::sqrt(M[d][0] * M[d][0] + M[d][1] * M[d][1] + M[d][2] * M[d][2])));
          if (C.parabolic) {
            double lv = 0.;
            for (int d = 0; d < 3; ++d) {
              double a = M[d][0] * sj, b = M[d][1] * sj, c = M[d][2] * sj;
              lv += a * a + b * b + c * c;
            }
            mlv = std::max(mlv, std::max(diffC_max, sRho * muKappasPr_max) * lv);
          }
        }
    double dtE = C.CFLScale * 2. / (ml[0] + ml[1] + ml[2]);
    dtConv = std::min(dtConv, dtE);
    if (std::isnan(dtConv)) *errType = 3;
    if (C.parabolic) {
      if (mlv > 0.) dtVisc = std::min(dtVisc, C.DFLScale * 4. / mlv);
      if (std::isnan(dtVisc)) *errType = 4;
      mlv = 0.;
    }
    if (*errType != 0) break;
  }
  double dt = std::min(dtConv, dtVisc);
  C.GLM_ch = C.GLM_scale * (C.GLM_dtch1 / dt);
  return dt;
}
