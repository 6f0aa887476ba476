// ORACLE — test infrastructure only (part of fluxo_oracle.cpp, included inside its namespace).
// CPU restatement of the reference's NFVSE shock capturing (shockcapturing/nfvse.f90,
// nfvse_mpi.f90, indicators/indicators.f90): Persson-Peraire indicator, blending coefficient,
// its space propagation, the subcell finite-volume volume integral on the LGL subcells (SubFVMethod
// 1 first order, 2 TVD, 3 TVD-ES, 4 TVD-Fjordholm), its blending with the split-form volume integral
// and the positivity correction of NFVSE_CORR (Apply_NFVSE_Correction).

// Sub-cell metrics, nfvse.f90:261-378: for direction d, subcell face f = -1..N and transverse
// point (a,b): normal, tangents and the norm of the (unnormalised) face metric
inline size_t SubcellIdx(const Case& C, int e, int d, int f, int a, int b) {
  const int n = C.np;
  return ((((size_t)e * 3 + d) * (n + 1) + (f + 1)) * n + b) * n + a;
}

void ComputeSubcellMetrics(Case& C) {
  const int n = C.np, N = C.N;
  const size_t cnt = (size_t)C.nElems * 3 * (n + 1) * n * n;
  C.scNv.assign(3 * cnt, 0.); C.scT1.assign(3 * cnt, 0.); C.scT2.assign(3 * cnt, 0.); C.scNorm.assign(cnt, 0.);
  for (int e = 0; e < C.nElems; ++e)
    for (int d = 0; d < 3; ++d) {
      // metric of the normal (Ja^d) and of the first tangent (Ja^(d+1)) at line position x, point (a,b)
      const std::vector<double>& Mn = (d == 0) ? C.Mf : (d == 1 ? C.Mg : C.Mh);
      const std::vector<double>& Mt = (d == 0) ? C.Mg : (d == 1 ? C.Mh : C.Mf);
      auto node = [&](int x, int a, int b) -> size_t {  // (a,b) = (j,k) for xi, (i,k) for eta, (i,j) for zeta
        if (d == 0) return C.nod(x, a, b, e);
        if (d == 1) return C.nod(a, x, b, e);
        return C.nod(a, b, x, e);
      };
      for (int f = -1; f <= N; ++f)
        for (int b = 0; b < n; ++b)
          for (int a = 0; a < n; ++a) {
            double nv[3], t1[3];
            for (int c = 0; c < 3; ++c) { nv[c] = Mn[3 * node(0, a, b) + c]; t1[c] = Mt[3 * node(0, a, b) + c]; }
            for (int m = 0; m <= N; ++m)
              for (int l = 0; l <= f; ++l)
                for (int c = 0; c < 3; ++c) {
                  nv[c] = nv[c] + C.wGP[l] * C.D[l + n * m] * Mn[3 * node(m, a, b) + c];
                  t1[c] = t1[c] + C.wGP[l] * C.D[l + n * m] * Mt[3 * node(m, a, b) + c];
                }
            const double norm = std::sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
            for (int c = 0; c < 3; ++c) nv[c] = nv[c] / norm;
            const double tn = t1[0] * nv[0] + t1[1] * nv[1] + t1[2] * nv[2];
            for (int c = 0; c < 3; ++c) t1[c] = t1[c] - tn * nv[c];
            const double tl = std::sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
            for (int c = 0; c < 3; ++c) t1[c] = t1[c] / tl;
            const double t2[3] = {nv[1] * t1[2] - nv[2] * t1[1], nv[2] * t1[0] - nv[0] * t1[2],
                                  nv[0] * t1[1] - nv[1] * t1[0]};
            const size_t s = SubcellIdx(C, e, d, f, a, b);
            for (int c = 0; c < 3; ++c) { C.scNv[3 * s + c] = nv[c]; C.scT1[3 * s + c] = t1[c]; C.scT2[3 * s + c] = t2[c]; }
            C.scNorm[s] = norm;
          }
    }
}

// indicator quantity (SetIndicatorFunction, navierstokes/equation_vars.f90:735-790, mhd/equation_vars.f90:764-808)
inline double IndicatorQuantity(const Case& C, const double* U) {
  const int q = C.P.indicator_quantity;
  const double ke = (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / U[0];
  double p = C.kappaM1 * (U[4] - 0.5 * ke);
  if (C.mhd) p = C.kappaM1 * (U[4] - 0.5 * ke - C.s2mu_0 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7] + U[8] * U[8]));
  switch (q) {
    case 1: return U[0];
    case 2: return p;
    case 4: return C.mhd ? 0.5 * ke + C.s2mu_0 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7]) : ke;
    default: return U[0] * p;
  }
}

// CalcBlendingCoefficient (nfvse.f90:1537-1620) with PerssonPeraire_Compute (indicators.f90:108-173)
// and ProlongBlendingCoeffToFaces (nfvse_mpi.f90:31-58)
void CalcBlendingCoefficient(Case& C) {
  const int n = C.np, N = C.N;
  const size_t nv = (size_t)n * n * n;
  const orc_params& P = C.P;
  if (P.compute_alpha == 1) {
    std::vector<double> Uind(nv), Umod(nv), Vdm(n * n), sVdm(n * n);
    LegendreVdm(N, C.xGP.data(), Vdm.data(), sVdm.data());
    const double sharpness = std::log((1.0 - 1.e-4) / 1.e-4);
    const double threshold = (P.modal_threshold == 2) ? 0.5 * std::pow(10.0, -1.8 * std::pow((double)N, 0.25))
                                                      : 0.5 * std::pow(10.0, -1.8 * std::pow(N + 1., 0.25));
    for (int e = 0; e < C.nElems; ++e) {
      for (size_t z = 0; z < nv; ++z) {
        double U[NVMAX];
        for (int v = 0; v < C.nVar; ++v) U[v] = val(C.U[C.nVar * (nv * e + z) + v]);
        Uind[z] = IndicatorQuantity(C, U);
      }
      ChangeBasis3D(1, N, N, sVdm.data(), Uind.data(), Umod.data());
      double LU = 0., LUM1 = 0., LUM2 = 0.;
      for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
          for (int i = 0; i < n; ++i) {
            const double m2 = Umod[i + n * (j + n * k)] * Umod[i + n * (j + n * k)];
            LU += m2;
            if (i < N && j < N && k < N) LUM1 += m2;
            if (i < N - 1 && j < N - 1 && k < N - 1) LUM2 += m2;
          }
      double eta = std::max((LU - LUM1) / LU, (LUM1 - LUM2) / LUM1);
      if (eta < REALTOL) eta = REALTOL;
      C.alpha[e] = std::max(P.time_rel_factor * C.alpha[e],
                            1.0 / (1.0 + std::exp(-sharpness * (eta - threshold) / threshold)));
    }
  } else if (P.compute_alpha == 3) {
    for (int e = 0; e < C.nElems; ++e) C.alpha[e] = P.shock_blend_coef;
  } else if (P.compute_alpha == 20) {
    // random values drawn once (at creation or by orc_set_alpha) and kept, nfvse.f90:1591-1596
  } else {
    throw std::runtime_error("ComputeAlpha not implemented in oracle");
  }
  for (int e = 0; e < C.nElems; ++e) {
    if (C.alpha[e] < P.alpha_min) C.alpha[e] = 0.0;
    else if (C.alpha[e] >= P.alpha_max) C.alpha[e] = P.alpha_max;
  }
  if (P.space_prop_sweeps > 0) {  // ProlongBlendingCoeffToFaces
    for (int s = 0; s < C.nSides; ++s) {
      C.alphaMaster[s] = C.alpha[C.SideToElem[5 * s] - 1];
      C.alphaSlave[s] = C.alpha[C.SideToElem[5 * s + 1] - 1];
    }
  }
}

// PropagateBlendingCoeff, nfvse_mpi.f90:62-131 (conforming inner sides)
void PropagateBlendingCoeff(Case& C) {
  for (int s = 0; s < C.nSides; ++s) {
    const double m = C.P.space_prop_factor * std::max(C.alphaMaster[s], C.alphaSlave[s]);
    const int e = C.SideToElem[5 * s] - 1, nb = C.SideToElem[5 * s + 1] - 1;
    if (C.alpha[e] < m) C.alpha[e] = m;
    if (C.alpha[nb] < m) C.alpha[nb] = m;
  }
}

// Rotated Riemann flux of one subcell face plane (AdvRiemann, riemann.f90), npts points
void SubcellRiemann(const Case& C, int npts, const real* UL, const real* UR, const double* nv, const double* t1,
                    const double* t2, real* F) {
  const int NV = C.nVar;
  std::vector<real> L((size_t)NV * npts), R((size_t)NV * npts);
  for (int z = 0; z < npts; ++z) {
    const real* a = UL + NV * z;
    const real* b = UR + NV * z;
    for (int v = 0; v < NV; ++v) { L[NV * z + v] = a[v]; R[NV * z + v] = b[v]; }
    for (int o = 1; o <= (C.mhd ? 5 : 1); o += 4) {
      L[NV * z + o] = a[o] * nv[3 * z] + a[o + 1] * nv[3 * z + 1] + a[o + 2] * nv[3 * z + 2];
      L[NV * z + o + 1] = a[o] * t1[3 * z] + a[o + 1] * t1[3 * z + 1] + a[o + 2] * t1[3 * z + 2];
      L[NV * z + o + 2] = a[o] * t2[3 * z] + a[o + 1] * t2[3 * z + 1] + a[o + 2] * t2[3 * z + 2];
      R[NV * z + o] = b[o] * nv[3 * z] + b[o + 1] * nv[3 * z + 1] + b[o + 2] * nv[3 * z + 2];
      R[NV * z + o + 1] = b[o] * t1[3 * z] + b[o + 1] * t1[3 * z + 1] + b[o + 2] * t1[3 * z + 2];
      R[NV * z + o + 2] = b[o] * t2[3 * z] + b[o + 1] * t2[3 * z + 1] + b[o + 2] * t2[3 * z + 2];
    }
  }
  if (C.mhd) {
    for (int z = 0; z < npts; ++z) MHD_Riemann(C, &L[NV * z], &R[NV * z], F + NV * z);
  } else {
    SolveRiemann(C, npts, L.data(), R.data(), F);
  }
  for (int z = 0; z < npts; ++z)
    for (int o = 1; o <= (C.mhd ? 5 : 1); o += 4) {
      real f2 = F[NV * z + o], f3 = F[NV * z + o + 1], f4 = F[NV * z + o + 2];
      for (int c = 0; c < 3; ++c)
        F[NV * z + o + c] = nv[3 * z + c] * f2 + t1[3 * z + c] * f3 + t2[3 * z + c] * f4;
    }
}

inline void FV_ConsToPrim(const Case& C, const real* U, real* P) {
  if (C.mhd) MHD_ConsToPrim(C, U, P);
  else ConsToPrim(C, U, P);
}
inline void FV_PrimToCons(const Case& C, const real* P, real* U) {  // PrimToConsVec (both systems)
  if (C.mhd) { MHD_PrimToCons(C, P, U); return; }
  U[0] = P[0];
  U[1] = P[1] * P[0]; U[2] = P[2] * P[0]; U[3] = P[3] * P[0];
  U[4] = C.sKappaM1 * P[4] + 0.5 * (U[1] * P[1] + U[2] * P[2] + U[3] * P[3]);
}
// minmod limiter, nfvse.f90:1514-1529
inline real MinMod(real a, real b) {
  if (fabs(a) < fabs(b) && a * b > 0.0) return a;
  if (fabs(b) < fabs(a) && a * b > 0.0) return b;
  return real(0.);
}

// Second-order (TVD) reconstruction along one line, ReconstructSolution_2nd_Order nfvse.f90:1448-1510
// with the node spacings and sub-cell offsets of InitNFVSE :218-238.  pr[x*NV+v]: primitive variables
// of the line; ext[0|1]: the neighbour elements' boundary states beyond node 0 / node N (ReconsBoundaries
// 3); outputs primR (right face of the subcell of node x, x = 0..N-1) and primL (left face, x = 1..N).
void ReconstructLine(const Case& C, const real* pr, const real* extL, const real* extR, real* pR, real* pL) {
  const int N = C.N, NV = C.nVar;
  std::vector<double> sdxR(N), sdxL(N), rL(N), rR(N);
  double sumWm1 = C.wGP[0] - 1.;
  for (int i = 1; i <= N - 1; ++i) {
    sdxR[i] = 1.0 / (C.xGP[i + 1] - C.xGP[i]);
    sdxL[i] = 1.0 / (C.xGP[i] - C.xGP[i - 1]);
    rL[i] = sumWm1 - C.xGP[i];
    sumWm1 = sumWm1 + C.wGP[i];
    rR[i] = sumWm1 - C.xGP[i];
  }
  const int rb = C.P.recons_boundaries;
  for (int v = 0; v < NV; ++v) {
    auto P = [&](int i) { return pr[i * NV + v]; };
    // first node
    if (rb == 1) pR[v] = P(0);
    else if (rb == 2) pR[v] = P(0) + (P(1) - P(0)) * sdxL[1] * C.wGP[0];
    else pR[v] = P(0) + MinMod(sdxL[1] * (P(1) - P(0)), sdxL[1] * (P(1) - extL[v])) * C.wGP[0];
    for (int i = 1; i <= N - 1; ++i) {
      real sigma = MinMod(sdxR[i] * (P(i + 1) - P(i)), sdxL[i] * (P(i) - P(i - 1)));
      pR[i * NV + v] = P(i) + sigma * rR[i];
      pL[i * NV + v] = P(i) + sigma * rL[i];
    }
    // last node
    if (rb == 1) pL[N * NV + v] = P(N);
    else if (rb == 2) pL[N * NV + v] = P(N) - (P(N) - P(N - 1)) * sdxL[1] * C.wGP[N];
    else pL[N * NV + v] = P(N) - MinMod(sdxL[1] * (P(N) - P(N - 1)), sdxL[1] * (extR[v] - P(N - 1))) * C.wGP[0];
  }
}

// RotateState / RotateFluxBack (navierstokes/riemann.f90:218-246, mhd/riemann.f90:185-217): the
// momentum (and for MHD the magnetic field) into the frame (nv, t1, t2) and back
inline void FV_Rotate(const Case& C, const real* a, const double* nv, const double* t1, const double* t2, real* o) {
  for (int v = 0; v < C.nVar; ++v) o[v] = a[v];
  for (int b = 1; b <= (C.mhd ? 5 : 1); b += 4) {
    o[b] = a[b] * nv[0] + a[b + 1] * nv[1] + a[b + 2] * nv[2];
    o[b + 1] = a[b] * t1[0] + a[b + 1] * t1[1] + a[b + 2] * t1[2];
    o[b + 2] = a[b] * t2[0] + a[b + 1] * t2[1] + a[b + 2] * t2[2];
  }
}
inline void FV_RotateBack(const Case& C, real* F, const double* nv, const double* t1, const double* t2) {
  for (int b = 1; b <= (C.mhd ? 5 : 1); b += 4) {
    real f2 = F[b], f3 = F[b + 1], f4 = F[b + 2];
    for (int c = 0; c < 3; ++c) F[b + c] = nv[c] * f2 + t1[c] * f3 + t2[c] * f4;
  }
}
// ConsToEntropy of the equation system (navierstokes/equation_vars.f90:362-391, mhd/equation_vars.f90:330-361)
inline void FV_ConsToEntropy(const Case& C, const real* U, real* W) {
  if (C.mhd) MHD_ConsToEntropy(C, U, W);
  else ConsToEntropy(C, U, W);
}
// Whether the Riemann solver provides RiemannVolFluxAndDissipMatrices (navierstokes/equation.f90:381-404:
// 4, 44, 33; mhd/equation.f90:367-386: 14, 15), which SubFVMethod 3 and 4 need (nfvse.f90:174-187)
inline bool HasDissipMatrices(const Case& C) {
  const int rs = C.P.riemann;
  return C.mhd ? (rs == 14 || rs == 15) : (rs == 4 || rs == 44 || rs == 33);
}
// RiemannVolFluxAndDissipMatrices on rotated states: EC flux F, diagonal D, right eigenvectors R[row][col]
inline void FV_DissipMatrices(const Case& C, const real* L, const real* R, real* F, real* D, real Rm[NVMAX][NVMAX]) {
  if (C.mhd) {
    real R9[9][9], Vj[9], pL, pR, bL, bR;
    MHD_EntropyJump(C, L, R, pL, pR, bL, bR, Vj);
    MHD_ES9WaveMatrices(C, L, R, C.P.riemann == 15, pL, pR, bL, bR, F, D, R9);
    for (int r = 0; r < 9; ++r)
      for (int c = 0; c < 9; ++c) Rm[r][c] = R9[r][c];
  } else {
    real R5[5][5];
    ES_VolFluxAndDissipMatrices(C, C.P.riemann, L, R, F, D, R5);
    for (int r = 0; r < 5; ++r)
      for (int c = 0; c < 5; ++c) Rm[r][c] = R5[r][c];
  }
}
// x = R^T v: x(c) = sum_r R(r,c) v(r) (matmul(RmatT, v))
inline void FV_RT(int NV, const real Rm[NVMAX][NVMAX], const real* v, real* x) {
  for (int c = 0; c < NV; ++c) {
    real s = 0.;
    for (int r = 0; r < NV; ++r) s = s + Rm[r][c] * v[r];
    x[c] = s;
  }
}
// F = F - 0.5 R (D x) (matmul(Rmat, Dmat*x))
inline void FV_Dissipate(int NV, const real Rm[NVMAX][NVMAX], const real* D, const real* x, real* F) {
  real y[NVMAX];
  for (int c = 0; c < NV; ++c) y[c] = D[c] * x[c];
  for (int r = 0; r < NV; ++r) {
    real s = 0.;
    for (int c = 0; c < NV; ++c) s = s + Rm[r][c] * y[c];
    F[r] = F[r] - 0.5 * s;
  }
}

// AdvRiemannRecons (nfvse.f90:1036-1090) of one subcell face plane, SubFVMethod 3: the EC flux and the
// dissipation matrices of the nodal states, and the dissipation of the entropy jump of the reconstructed
// states (UL_r, UR_r) unless, in some component, it has the opposite sign to the nodal jump (beyond
// -1e-10), in which case the nodal jump is used.  Output rotated back to the physical frame.
void SubcellTVD2ES(const Case& C, int npts, const real* UL, const real* UR, const real* ULr, const real* URr,
                   const double* nv, const double* t1, const double* t2, real* F) {
  const int NV = C.nVar;
  for (int z = 0; z < npts; ++z) {
    const double *n = nv + 3 * z, *a = t1 + 3 * z, *b = t2 + 3 * z;
    real L[NVMAX], R[NVMAX], Lr[NVMAX], Rr[NVMAX];
    FV_Rotate(C, UL + NV * z, n, a, b, L);
    FV_Rotate(C, UR + NV * z, n, a, b, R);
    FV_Rotate(C, ULr + NV * z, n, a, b, Lr);
    FV_Rotate(C, URr + NV * z, n, a, b, Rr);
    real D[NVMAX], Rm[NVMAX][NVMAX];
    real* Fz = F + NV * z;
    FV_DissipMatrices(C, L, R, Fz, D, Rm);
    real vL[NVMAX], vR[NVMAX], vLr[NVMAX], vRr[NVMAX], dv[NVMAX], dvr[NVMAX], x[NVMAX], xr[NVMAX];
    FV_ConsToEntropy(C, L, vL);
    FV_ConsToEntropy(C, R, vR);
    FV_ConsToEntropy(C, Lr, vLr);
    FV_ConsToEntropy(C, Rr, vRr);
    for (int v = 0; v < NV; ++v) { dv[v] = vR[v] - vL[v]; dvr[v] = vRr[v] - vLr[v]; }
    FV_RT(NV, Rm, dv, x);
    FV_RT(NV, Rm, dvr, xr);
    bool notES = false;
    for (int v = 0; v < NV; ++v)
      if (x[v] * xr[v] < -1.e-10) notES = true;
    FV_Dissipate(NV, Rm, D, notES ? x : xr, Fz);
    FV_RotateBack(C, Fz, n, a, b);
  }
}

// External states of ReconsBoundaries 3 (Get_externalU, nfvse.f90:1621-1683) as conservative variables
// at [(a + n*b)*NV] (ExternalPrim below converts them to primitive variables)
void ExternalCons(const Case& C, int e, int s, std::vector<real>& ext) {
  const int n = C.np, N = C.N, NV = C.nVar;
  ext.assign((size_t)n * n * NV, real(0.));
  const int sideID = C.ElemToSide[2 * (6 * e + (s - 1))] - 1;
  const int flipE = C.ElemToSide[2 * (6 * e + (s - 1)) + 1];
  const bool master = flipE == 0;  // master sides have flip 0
  static const int tan1[6] = {0, 0, 1, 0, 1, 0}, tan2[6] = {1, 2, 2, 2, 2, 1};  // TanDirs1/2 - 1
  for (int q = 0; q <= N; ++q)
    for (int p = 0; p <= N; ++p) {
      int ijk[3];
      SideToVol(N, 0, p, q, master ? 0 : flipE, s, ijk);
      const real* Uf = master ? &C.Uslave[C.fac(0, p, q, sideID)] : &C.Umaster[C.fac(0, p, q, sideID)];
      const int a = ijk[tan1[s - 1]], b = ijk[tan2[s - 1]];
      for (int v = 0; v < NV; ++v) ext[(a + n * b) * NV + v] = Uf[v];
    }
}

// External state of ReconsBoundaries 3 (Get_externalU, nfvse.f90:1621-1683): at the boundary node of
// local side s of element e, the neighbour's face state (U_slave on a master side, U_master on a
// slave side); returned as primitive variables at [(a + n*b)*NV], (a,b) the tangential node indexes
void ExternalPrim(const Case& C, int e, int s, std::vector<real>& ext) {
  const int NV = C.nVar;
  std::vector<real> cons;
  ExternalCons(C, e, s, cons);
  ext.assign(cons.size(), real(0.));
  for (size_t z = 0; z < cons.size() / NV; ++z) FV_ConsToPrim(C, &cons[z * NV], &ext[z * NV]);
}

// Compute_FVFluxes_1D_TVD_Fjordholm (nfvse.f90:1187-1386) for one direction of element e: node(x, a, b)
// gives the volume index of the line position x at the transverse point (a,b); Fout[(x*npt + p)*NV] the
// rotated-back ES fluxes of the subcell faces x = 0..N-1 (before the non-conservative terms and the norm).
// The central EC flux uses the nodal states; the dissipation acts on the jump of the minmod-reconstructed
// scaled entropy variables w = R^T v, each face's w computed with that face's eigenvectors.
template <class NodeFn>
void FjordholmDirection(const Case& C, int e, int d, NodeFn node, const std::vector<real>& extL,
                        const std::vector<real>& extR, std::vector<real>& Fout) {
  const int n = C.np, N = C.N, NV = C.nVar, npt = n * n;
  std::vector<double> sdxR(N), sdxL(N), rL(N), rR(N);
  double sumWm1 = C.wGP[0] - 1.;
  for (int i = 1; i <= N - 1; ++i) {  // InitNFVSE :218-238
    sdxR[i] = 1.0 / (C.xGP[i + 1] - C.xGP[i]);
    sdxL[i] = 1.0 / (C.xGP[i] - C.xGP[i - 1]);
    rL[i] = sumWm1 - C.xGP[i];
    sumWm1 = sumWm1 + C.wGP[i];
    rR[i] = sumWm1 - C.xGP[i];
  }
  const int rb = C.P.recons_boundaries;
  auto metric = [&](int f, int a, int b, double* nvv, double* t1v, double* t2v) {
    const size_t s = SubcellIdx(C, e, d, f, a, b);
    for (int c = 0; c < 3; ++c) { nvv[c] = C.scNv[3 * s + c]; t1v[c] = C.scT1[3 * s + c]; t2v[c] = C.scT2[3 * s + c]; }
  };
  // per face x and point p: EC flux, D, R and the scaled entropy variables of both nodes
  std::vector<real> Fc((size_t)N * npt * NV), Dd((size_t)N * npt * NV), Rr((size_t)N * npt * NVMAX * NVMAX),
      wL((size_t)N * npt * NV), wR((size_t)N * npt * NV);
  for (int x = 0; x < N; ++x)
    for (int b = 0; b < n; ++b)
      for (int a = 0; a < n; ++a) {
        const int p = a + n * b;
        const size_t o = ((size_t)x * npt + p) * NV;
        double nvv[3], t1v[3], t2v[3];
        metric(x, a, b, nvv, t1v, t2v);
        real L[NVMAX], R[NVMAX], Rm[NVMAX][NVMAX], vL[NVMAX], vR[NVMAX];
        FV_Rotate(C, &C.U[NV * node(x, a, b)], nvv, t1v, t2v, L);
        FV_Rotate(C, &C.U[NV * node(x + 1, a, b)], nvv, t1v, t2v, R);
        FV_DissipMatrices(C, L, R, &Fc[o], &Dd[o], Rm);
        for (int r = 0; r < NV; ++r)
          for (int c = 0; c < NV; ++c) Rr[((size_t)x * npt + p) * NVMAX * NVMAX + r * NVMAX + c] = Rm[r][c];
        FV_ConsToEntropy(C, L, vL);
        FV_ConsToEntropy(C, R, vR);
        FV_RT(NV, Rm, vL, &wL[o]);
        FV_RT(NV, Rm, vR, &wR[o]);
      }
  // scaled entropy variables of the neighbour's boundary state (ReconsBoundaries 3) across the element
  // face: U_ext and node 1 (left, face -1 metrics), node N-1 and U_ext (right, face N metrics)
  auto boundaryW = [&](int f, int a, int b, const real* Ua, const real* Ub, real* w0L, real* w0R) {
    double nvv[3], t1v[3], t2v[3];
    metric(f, a, b, nvv, t1v, t2v);
    real L[NVMAX], R[NVMAX], Fd[NVMAX], D0[NVMAX], R0[NVMAX][NVMAX], vL[NVMAX], vR[NVMAX];
    FV_Rotate(C, Ua, nvv, t1v, t2v, L);
    FV_Rotate(C, Ub, nvv, t1v, t2v, R);
    FV_ConsToEntropy(C, L, vL);
    FV_ConsToEntropy(C, R, vR);
    FV_DissipMatrices(C, L, R, Fd, D0, R0);
    FV_RT(NV, R0, vL, w0L);
    FV_RT(NV, R0, vR, w0R);
  };
  std::vector<real> wtR((size_t)n * npt * NV, real(0.)), wtL((size_t)n * npt * NV, real(0.));
  auto at = [&](int x, int p) { return ((size_t)x * npt + p) * NV; };
  for (int b = 0; b < n; ++b)
    for (int a = 0; a < n; ++a) {
      const int p = a + n * b;
      real w0L[NVMAX], w0R[NVMAX];
      // first DOF
      if (rb == 3) boundaryW(-1, a, b, &extL[(size_t)p * NV], &C.U[NV * node(1, a, b)], w0L, w0R);
      for (int v = 0; v < NV; ++v) {
        const real jl = wR[at(0, p) + v] - wL[at(0, p) + v];
        if (rb == 1) wtR[at(0, p) + v] = wL[at(0, p) + v];
        else if (rb == 2) wtR[at(0, p) + v] = wL[at(0, p) + v] + jl * sdxL[1] * C.wGP[0];
        else wtR[at(0, p) + v] = wL[at(0, p) + v] + MinMod(sdxL[1] * jl, sdxL[1] * (w0R[v] - w0L[v])) * C.wGP[0];
      }
      // middle DOFs
      for (int i = 1; i <= N - 1; ++i)
        for (int v = 0; v < NV; ++v) {
          const real sg = MinMod(sdxR[i] * (wR[at(i, p) + v] - wL[at(i, p) + v]),
                                 sdxL[i] * (wR[at(i - 1, p) + v] - wL[at(i - 1, p) + v]));
          wtR[at(i, p) + v] = wL[at(i, p) + v] + sg * rR[i];
          wtL[at(i, p) + v] = wR[at(i - 1, p) + v] + sg * rL[i];
        }
      // last DOF
      if (rb == 3) boundaryW(N, a, b, &C.U[NV * node(N - 1, a, b)], &extR[(size_t)p * NV], w0L, w0R);
      for (int v = 0; v < NV; ++v) {
        const real jr = wR[at(N - 1, p) + v] - wL[at(N - 1, p) + v];
        if (rb == 1) wtL[at(N, p) + v] = wR[at(N - 1, p) + v];
        else if (rb == 2) wtL[at(N, p) + v] = wR[at(N - 1, p) + v] - jr * sdxL[1] * C.wGP[N];
        else wtL[at(N, p) + v] = wR[at(N - 1, p) + v] - MinMod(sdxL[1] * jr, sdxL[1] * (w0R[v] - w0L[v])) * C.wGP[N];
      }
    }
  Fout.assign((size_t)N * npt * NV, real(0.));
  for (int x = 0; x < N; ++x)
    for (int b = 0; b < n; ++b)
      for (int a = 0; a < n; ++a) {
        const int p = a + n * b;
        const size_t o = at(x, p);
        real Rm[NVMAX][NVMAX], jw[NVMAX];
        for (int r = 0; r < NV; ++r)
          for (int c = 0; c < NV; ++c) Rm[r][c] = Rr[((size_t)x * npt + p) * NVMAX * NVMAX + r * NVMAX + c];
        for (int v = 0; v < NV; ++v) { Fout[o + v] = Fc[o + v]; jw[v] = wtL[at(x + 1, p) + v] - wtR[o + v]; }
        FV_Dissipate(NV, Rm, &Dd[o], jw, &Fout[o]);
        double nvv[3], t1v[3], t2v[3];
        metric(x, a, b, nvv, t1v, t2v);
        FV_RotateBack(C, &Fout[o], nvv, t1v, t2v);
      }
}

// VolInt_NFVSE (nfvse.f90:475-565) with Compute_FVFluxes_1st_Order (:566-673), Compute_FVFluxes_TVD
// (:674-815), Compute_FVFluxes_TVD2ES (:826-1090) or Compute_FVFluxes_TVD_Fjordholm (:1101-1386) and
// Compute_FVFluxes_1D (:1389-1447): Ut = (1-alpha) Ut + alpha F_FV on the blended elements; with
// NFVSE_CORR on every element, keeping FFV_m_FDG = (F_FV - Ut) (-sJ) for Apply_NFVSE_Correction
void VolIntNFVSE(Case& C) {
  const int n = C.np, N = C.N, NV = C.nVar, npt = n * n;
  if (C.P.space_prop_sweeps > 0) {
    PropagateBlendingCoeff(C);
    for (int sw = 2; sw <= C.P.space_prop_sweeps; ++sw) {
      for (int s = 0; s < C.nSides; ++s) {
        C.alphaMaster[s] = C.alpha[C.SideToElem[5 * s] - 1];
        C.alphaSlave[s] = C.alpha[C.SideToElem[5 * s + 1] - 1];
      }
      PropagateBlendingCoeff(C);
    }
  }
  std::vector<double> sW(n);
  for (int i = 0; i < n; ++i) sW[i] = 1.0 / C.wGP[i];
  // per direction: left flux FL(x) and right flux FR(x) of subcell face x = -1..N at (a,b)
  std::vector<real> FL((size_t)3 * (n + 1) * npt * NV), FR((size_t)3 * (n + 1) * npt * NV);
  std::vector<real> UL((size_t)npt * NV), UR((size_t)npt * NV), F((size_t)npt * NV), G((size_t)npt * NV);
  // TVD: reconstructed face states of the Riemann problems, per direction and line
  const int sfm = C.P.sub_fv_method;
  const bool tvd = sfm == 2 || sfm == 3;  // primitive-variable reconstruction (TVD2ES: for the ES switch)
  const bool corr = C.P.nfvse_corr != 0;
  std::vector<real> extCL, extCR, Fj;
  std::vector<real> RL((size_t)npt * NV), RR((size_t)npt * NV), pr((size_t)n * NV), pRl((size_t)n * NV),
      pLl((size_t)n * NV), recR((size_t)3 * n * npt * NV), recL((size_t)3 * n * npt * NV);
  std::vector<real> extL, extR;
  static const int sideMinus[3] = {XI_MINUS, ETA_MINUS, ZETA_MINUS}, sidePlus[3] = {XI_PLUS, ETA_PLUS, ZETA_PLUS};
  std::vector<double> nvb(3 * npt), t1b(3 * npt), t2b(3 * npt);
  auto fi = [&](int d, int x, int p) { return ((size_t)(d * (n + 1) + (x + 1)) * npt + p) * NV; };
  for (int e = 0; e < C.nElems; ++e) {
    if (!corr && AlmostEqual(C.alpha[e], 0.0)) continue;
    std::fill(FL.begin(), FL.end(), real(0.));
    std::fill(FR.begin(), FR.end(), real(0.));
    for (int d = 0; d < 3; ++d) {
      auto node = [&](int x, int a, int b) -> size_t {
        if (d == 0) return C.nod(x, a, b, e);
        if (d == 1) return C.nod(a, x, b, e);
        return C.nod(a, b, x, e);
      };
      if (tvd) {  // reconstruct every line of this direction: recR/recL[(x*npt + p)*NV + v]
        if (C.P.recons_boundaries == 3) {
          ExternalPrim(C, e, sideMinus[d], extL);
          ExternalPrim(C, e, sidePlus[d], extR);
        }
        for (int b = 0; b < n; ++b)
          for (int a = 0; a < n; ++a) {
            for (int x = 0; x <= N; ++x) FV_ConsToPrim(C, &C.U[NV * node(x, a, b)], &pr[x * NV]);
            const real* eL = C.P.recons_boundaries == 3 ? &extL[(a + n * b) * NV] : nullptr;
            const real* eR = C.P.recons_boundaries == 3 ? &extR[(a + n * b) * NV] : nullptr;
            ReconstructLine(C, pr.data(), eL, eR, pRl.data(), pLl.data());
            for (int x = 0; x <= N; ++x) {
              FV_PrimToCons(C, &pRl[x * NV], &recR[((size_t)x * npt + a + n * b) * NV]);
              FV_PrimToCons(C, &pLl[x * NV], &recL[((size_t)x * npt + a + n * b) * NV]);
            }
          }
      }
      if (sfm == 4) {
        if (C.P.recons_boundaries == 3) {
          ExternalCons(C, e, sideMinus[d], extCL);
          ExternalCons(C, e, sidePlus[d], extCR);
        }
        FjordholmDirection(C, e, d, node, extCL, extCR, Fj);
      }
      for (int x = 0; x < N; ++x) {
        for (int b = 0; b < n; ++b)
          for (int a = 0; a < n; ++a) {
            const int p = a + n * b;
            for (int v = 0; v < NV; ++v) {
              UL[NV * p + v] = C.U[NV * node(x, a, b) + v];
              UR[NV * p + v] = C.U[NV * node(x + 1, a, b) + v];
            }
            const size_t s = SubcellIdx(C, e, d, x, a, b);
            for (int c = 0; c < 3; ++c) {
              nvb[3 * p + c] = C.scNv[3 * s + c]; t1b[3 * p + c] = C.scT1[3 * s + c]; t2b[3 * p + c] = C.scT2[3 * s + c];
            }
          }
        if (sfm == 4) {
          for (int z = 0; z < npt * NV; ++z) F[z] = Fj[(size_t)x * npt * NV + z];
        } else if (tvd) {
          for (int z = 0; z < npt * NV; ++z) {
            RL[z] = recR[(size_t)x * npt * NV + z];
            RR[z] = recL[(size_t)(x + 1) * npt * NV + z];
          }
          if (sfm == 3)
            SubcellTVD2ES(C, npt, UL.data(), UR.data(), RL.data(), RR.data(), nvb.data(), t1b.data(), t2b.data(),
                          F.data());
          else
            SubcellRiemann(C, npt, RL.data(), RR.data(), nvb.data(), t1b.data(), t2b.data(), F.data());
        } else {
          SubcellRiemann(C, npt, UL.data(), UR.data(), nvb.data(), t1b.data(), t2b.data(), F.data());
        }
        for (size_t z = 0; z < F.size(); ++z) G[z] = F[z];  // FR_ = F_ before the non-conservative terms
        if (C.mhd && C.noncons) {
          for (int p = 0; p < npt; ++p) {
            MHD_NonConsSurf(C, &UR[NV * p], &UL[NV * p], &nvb[3 * p], &F[NV * p]);  // left flux of node x+1
            MHD_NonConsSurf(C, &UL[NV * p], &UR[NV * p], &nvb[3 * p], &G[NV * p]);  // right flux of node x
          }
        }
        for (int b = 0; b < n; ++b)
          for (int a = 0; a < n; ++a) {
            const int p = a + n * b;
            const double nrm = C.scNorm[SubcellIdx(C, e, d, x, a, b)];
            for (int v = 0; v < NV; ++v) {
              FL[fi(d, x, p) + v] = F[NV * p + v] * nrm;
              FR[fi(d, x, p) + v] = (C.mhd && C.noncons) ? G[NV * p + v] * nrm : F[NV * p + v] * nrm;
            }
          }
      }
    }
    const double al = C.alpha[e];
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
          for (int v = 0; v < NV; ++v) {
            real ffv = sW[i] * (FR[fi(0, i, j + n * k) + v] - FL[fi(0, i - 1, j + n * k) + v]) +
                       sW[j] * (FR[fi(1, j, i + n * k) + v] - FL[fi(1, j - 1, i + n * k) + v]) +
                       sW[k] * (FR[fi(2, k, i + n * j) + v] - FL[fi(2, k - 1, i + n * j) + v]);
            real& ut = C.Ut[C.vol(v, i, j, k, e)];
            if (corr) C.FFVmFDG[C.vol(v, i, j, k, e)] = (ffv - ut) * (-C.sJ[C.nod(i, j, k, e)]);
            ut = (1. - al) * ut + al * ffv;
          }
  }
}
