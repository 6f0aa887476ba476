// NFVSE shock capturing (shockcapturing/nfvse.f90, nfvse_mpi.f90, indicators/indicators.f90) on
// the sm_100a path for the Euler / Navier-Stokes and the MHD systems, LGL nodes, subcell finite
// volumes of first order (SubFVMethod = 1), TVD (2), TVD-ES (3) or TVD-Fjordholm (4):
//   alpha_kernel      Persson-Peraire indicator of rho*p (or rho, p, kinetic energy) from its modal
//                     Legendre coefficients, alpha = 1/(1+exp(-s (eta-T)/T)), clipping;
//   propagate_kernel  alpha_e = max(alpha_e, SpacePropFactor * max over its sides of the two
//                     element values) and the list of blended elements (alpha > 2*EPSILON);
//   fv_kernel         per blended element: the subcell FV volume integral with sub-cell metrics built
//                     from the element's metrics on the fly (nfvse.f90:261-378), the Riemann solver of
//                     the face kernel (SubFVMethod 1, 2) or the entropy-stable flux built from its
//                     dissipation matrices (3, 4), and the non-conservative terms, written as
//                     alpha * F_FV (NFVSE_CORR: F_FV, every element) for the volume kernel to blend with;
//   corr_kernel       NFVSE_CORR: Apply_NFVSE_Correction after an RK stage update.
#pragma once
#include "common.cuh"
#include "kernels.cuh"
#include "mhd_kernels.cuh"
#include "physics_mhd.cuh"

namespace fluxo {
namespace nfvse {

constexpr double kTiny = 2. * 2.220446049250313e-16;  // ALMOSTEQUAL(alpha, 0), basis.f90:673-690

// indicator quantity (SetIndicatorFunction, navierstokes/equation_vars.f90:735-790, mhd/equation_vars.f90:764-808)
template <int NV>
__device__ __forceinline__ double indicator_quantity(const KParams& P, const double* U) {
  const double ke = (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / U[0];
  double p;
  if constexpr (NV == 9)
    p = P.kappaM1 * (U[4] - 0.5 * ke - P.s2mu_0 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7] + U[8] * U[8]));
  else
    p = P.kappaM1 * (U[4] - 0.5 * ke);
  switch (P.indicatorQuantity) {
    case 1: return U[0];
    case 2: return p;
    case 4:
      if constexpr (NV == 9) return 0.5 * ke + P.s2mu_0 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7]);
      else return ke;
    default: return U[0] * p;
  }
}

// CalcBlendingCoefficient (nfvse.f90:1537-1620) with PerssonPeraire_Compute (indicators.f90:108-173);
// EPB elements per block, one thread per node; the modal energies are summed by one thread per
// element in node order, so the result does not depend on thread scheduling
template <int NP, int NV>
__global__ void __launch_bounds__(512) alpha_kernel(KParams P) {
  if (halted(P)) return;
  constexpr int NP3 = NP * NP * NP, NPT = NP * NP, N = NP - 1;
  constexpr int EPB = (256 / NP3) > 0 ? (256 / NP3) : 1;
  __shared__ double sV[NPT];
  __shared__ double sA[EPB][NP3], sB[EPB][NP3];
  const int eb = threadIdx.x / NP3, t = threadIdx.x - eb * NP3;
  const int e = blockIdx.x * EPB + eb;
  const bool valid = e < P.nElems;
  if (blockIdx.x == 0 && threadIdx.x == 0) *P.blendCount = 0;  // the list kernels run after this one
  for (int z = threadIdx.x; z < NPT; z += blockDim.x) sV[z] = P.sVdm[z];
  const int i = t % NP, j = (t / NP) % NP, k = t / NPT;
  if (valid) {
    double U[NV];
    const double* Ug = P.U + NV * ((size_t)e * NP3 + t);
#pragma unroll
    for (int v = 0; v < NV; ++v) U[v] = Ug[v];
    sA[eb][t] = indicator_quantity<NV>(P, U);
  }
  __syncthreads();
  // modal coefficients Umod(m1,m2,m3) = sum sVdm(m1,i) sVdm(m2,j) sVdm(m3,k) Uind(i,j,k), one index at a time
  if (valid) {
    double s = 0.;
    for (int l = 0; l < NP; ++l) s += sV[i * NP + l] * sA[eb][l + NP * (j + NP * k)];
    sB[eb][t] = s;
  }
  __syncthreads();
  if (valid) {
    double s = 0.;
    for (int l = 0; l < NP; ++l) s += sV[j * NP + l] * sB[eb][i + NP * (l + NP * k)];
    sA[eb][t] = s;
  }
  __syncthreads();
  if (valid) {
    double s = 0.;
    for (int l = 0; l < NP; ++l) s += sV[k * NP + l] * sA[eb][i + NP * (j + NP * l)];
    sB[eb][t] = s * s;
  }
  __syncthreads();
  if (!valid || t != 0) return;
  double a;
  if (P.computeAlpha == 1) {
    double LU = 0., LUM1 = 0., LUM2 = 0.;
    for (int z = 0; z < NP3; ++z) {
      const int zi = z % NP, zj = (z / NP) % NP, zk = z / NPT;
      const double m2 = sB[eb][z];
      LU += m2;
      if (zi < N && zj < N && zk < N) LUM1 += m2;
      if (zi < N - 1 && zj < N - 1 && zk < N - 1) LUM2 += m2;
    }
    double eta = fmax((LU - LUM1) / LU, (LUM1 - LUM2) / LUM1);
    if (eta < 2.220446049250313e-16) eta = 2.220446049250313e-16;
    a = fmax(P.timeRelFactor * P.alpha[e], 1.0 / (1.0 + exp(-P.sharpness * (eta - P.threshold) / P.threshold)));
  } else if (P.computeAlpha == 20) {  // random values drawn once, kept over time (nfvse.f90:1591-1596)
    a = P.alpha[e];
  } else {
    a = P.shockBlendCoef;
  }
  if (a < P.alphaMin) a = 0.0;
  else if (a >= P.alphaMax) a = P.alphaMax;
  P.alphaRaw[e] = a;
}

// PropagateBlendingCoeff (nfvse_mpi.f90:62-131) for one sweep from `src` into alpha; the last
// sweep also lists the blended elements (NFVSE_CORR: every element, nfvse.f90:525-528)
static __global__ void propagate_kernel(KParams P, const double* src, bool last) {
  if (halted(P)) return;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= P.nElems) return;
  double a = src[e];
  for (int ls = 0; ls < 6; ++ls) {
    const int s = P.e2s[2 * (6 * e + ls)];
    const double m = P.propFactor * fmax(src[P.s2e[5 * s]], src[P.s2e[5 * s + 1]]);
    if (a < m) a = m;
  }
  P.alpha[e] = a;
  if (last && (a > kTiny || P.nfvseCorr)) P.blendList[atomicAdd(P.blendCount, 1)] = e;
}

// no propagation (SpacePropSweeps = 0): alpha = raw value, list the blended elements
static __global__ void list_kernel(KParams P) {
  if (halted(P)) return;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= P.nElems) return;
  const double a = P.alphaRaw[e];
  P.alpha[e] = a;
  if (a > kTiny || P.nfvseCorr) P.blendList[atomicAdd(P.blendCount, 1)] = e;
}

// minmod limiter (nfvse.f90:1514-1529)
__device__ __forceinline__ double minmod(double a, double b) {
  if (fabs(a) < fabs(b) && a * b > 0.0) return a;
  if (fabs(b) < fabs(a) && a * b > 0.0) return b;
  return 0.;
}

// The TVD reconstruction is evaluated without multiply-add contraction, each operation rounded as in
// the reference's formula: the limiter's decisions (|a| < |b|, a*b > 0) are discontinuous, and for
// data continuous across an element face its two slopes tie, so a last-bit difference would select
// another branch.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// ConsToPrim / PrimToCons of MHD (mhd/equation_vars.f90:229-278), uncontracted
__device__ __forceinline__ void cons_to_prim_rn(const KParams& P, const double* U, double* Q) {
  const double s = 1. / U[0];
  Q[0] = U[0];
  Q[1] = mul_rn(U[1], s); Q[2] = mul_rn(U[2], s); Q[3] = mul_rn(U[3], s);
  const double mv = add_rn(add_rn(mul_rn(U[1], Q[1]), mul_rn(U[2], Q[2])), mul_rn(U[3], Q[3]));
  const double b2 = add_rn(add_rn(add_rn(mul_rn(U[5], U[5]), mul_rn(U[6], U[6])), mul_rn(U[7], U[7])), mul_rn(U[8], U[8]));
  Q[4] = mul_rn(P.kappaM1, sub_rn(sub_rn(U[4], mul_rn(0.5, mv)), mul_rn(P.s2mu_0, b2)));
#pragma unroll
  for (int v = 5; v < 9; ++v) Q[v] = U[v];
}
// ConsToPrim / PrimToCons of Euler / Navier-Stokes (navierstokes/equation_vars.f90:243-290), uncontracted
__device__ __forceinline__ void cons_to_prim_ns_rn(const KParams& P, const double* U, double* Q) {
  const double s = 1. / U[0];
  Q[0] = U[0];
  Q[1] = mul_rn(U[1], s); Q[2] = mul_rn(U[2], s); Q[3] = mul_rn(U[3], s);
  const double mv = add_rn(add_rn(mul_rn(U[1], Q[1]), mul_rn(U[2], Q[2])), mul_rn(U[3], Q[3]));
  Q[4] = mul_rn(P.kappaM1, sub_rn(U[4], mul_rn(0.5, mv)));
}
__device__ __forceinline__ void prim_to_cons_ns_rn(const KParams& P, const double* Q, double* U) {
  U[0] = Q[0];
  U[1] = mul_rn(Q[1], Q[0]); U[2] = mul_rn(Q[2], Q[0]); U[3] = mul_rn(Q[3], Q[0]);
  const double mv = add_rn(add_rn(mul_rn(U[1], Q[1]), mul_rn(U[2], Q[2])), mul_rn(U[3], Q[3]));
  U[4] = add_rn(mul_rn(P.sKappaM1, Q[4]), mul_rn(0.5, mv));
}
template <int NV>
__device__ __forceinline__ void c2p_rn(const KParams& P, const double* U, double* Q) {
  if constexpr (NV == 9) cons_to_prim_rn(P, U, Q);
  else cons_to_prim_ns_rn(P, U, Q);
}

__device__ __forceinline__ void prim_to_cons_rn(const KParams& P, const double* Q, double* U) {
  U[0] = Q[0];
  U[1] = mul_rn(Q[1], Q[0]); U[2] = mul_rn(Q[2], Q[0]); U[3] = mul_rn(Q[3], Q[0]);
  const double mv = add_rn(add_rn(mul_rn(U[1], Q[1]), mul_rn(U[2], Q[2])), mul_rn(U[3], Q[3]));
  const double b2 = add_rn(add_rn(add_rn(mul_rn(Q[5], Q[5]), mul_rn(Q[6], Q[6])), mul_rn(Q[7], Q[7])), mul_rn(Q[8], Q[8]));
  U[4] = add_rn(add_rn(mul_rn(P.sKappaM1, Q[4]), mul_rn(0.5, mv)), mul_rn(P.s2mu_0, b2));
#pragma unroll
  for (int v = 5; v < 9; ++v) U[v] = Q[v];
}

// Primitive state of the neighbour element's node that coincides with the boundary node `node` of
// element e on the minus (plus = false) or plus side of direction dir (Get_externalU: U_slave on a
// master side, U_master on a slave side, which are the neighbour's boundary nodes for LGL)
template <int NP, int NV>
__device__ __forceinline__ const double* ext_node(const KParams& P, int e, int dir, bool plus, int node) {
  constexpr int N = NP - 1, NP3 = NP * NP * NP;
  const int s = dir == 0 ? (plus ? XI_PLUS : XI_MINUS) : (dir == 1 ? (plus ? ETA_PLUS : ETA_MINUS)
                                                                   : (plus ? ZETA_PLUS : ZETA_MINUS));
  const int i = node % NP, j = (node / NP) % NP, k = node / (NP * NP);
  const int* es = P.e2s + 2 * (6 * (size_t)e + (s - 1));
  const int side = es[0], flip = es[1];
  const int pt = node_side_point(N, s, flip, i, j, k), p = pt % NP, q = pt / NP;
  const int* se5 = P.s2e + 5 * side;
  const int nb = flip == 0 ? se5[1] : se5[0];
  const int nn = flip == 0 ? side_node(N, p, q, se5[4], se5[3]) : side_node(N, p, q, 0, se5[2]);
  return P.U + NV * ((size_t)nb * NP3 + nn);
}
template <int NP, int NV>
__device__ __forceinline__ void ext_prim(const KParams& P, int e, int dir, bool plus, int node, double* pr) {
  c2p_rn<NV>(P, ext_node<NP, NV>(P, e, dir, plus, node), pr);
}

// TVD states of subcell face x of a line (ReconstructSolution_2nd_Order, nfvse.f90:1448-1510):
// cL = cons(primR(x)), cR = cons(primL(x+1)); pr = the line's primitive records (stride st doubles)
template <int NP, int NV>
__device__ __forceinline__ void tvd_states(const KParams& P, const double* pr, int st, int x, const double* sdxR,
                                           const double* sdxL, const double* rL, const double* rR,
                                           const double* w, const double* extL, const double* extR, double* cL,
                                           double* cR) {
  constexpr int N = NP - 1;
  const int rb = P.reconsBoundaries;
  double pl[NV], prr[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    auto Q = [&](int m) { return pr[m * st + v]; };
    // right face of the subcell of node x
    if (x == 0) {
      if (rb == 1) pl[v] = Q(0);
      else if (rb == 2) pl[v] = add_rn(Q(0), mul_rn(mul_rn(sub_rn(Q(1), Q(0)), sdxL[1]), w[0]));
      else pl[v] = add_rn(Q(0), mul_rn(minmod(mul_rn(sdxL[1], sub_rn(Q(1), Q(0))), mul_rn(sdxL[1], sub_rn(Q(1), extL[v]))), w[0]));
    } else {
      const double sg = minmod(mul_rn(sdxR[x], sub_rn(Q(x + 1), Q(x))), mul_rn(sdxL[x], sub_rn(Q(x), Q(x - 1))));
      pl[v] = add_rn(Q(x), mul_rn(sg, rR[x]));
    }
    // left face of the subcell of node x+1
    const int y = x + 1;
    if (y == N) {
      if (rb == 1) prr[v] = Q(N);
      else if (rb == 2) prr[v] = sub_rn(Q(N), mul_rn(mul_rn(sub_rn(Q(N), Q(N - 1)), sdxL[1]), w[N]));
      else prr[v] = sub_rn(Q(N), mul_rn(minmod(mul_rn(sdxL[1], sub_rn(Q(N), Q(N - 1))), mul_rn(sdxL[1], sub_rn(extR[v], Q(N - 1)))), w[0]));
    } else {
      const double sg = minmod(mul_rn(sdxR[y], sub_rn(Q(y + 1), Q(y))), mul_rn(sdxL[y], sub_rn(Q(y), Q(y - 1))));
      prr[v] = add_rn(Q(y), mul_rn(sg, rL[y]));
    }
  }
  if constexpr (NV == 9) {
    prim_to_cons_rn(P, pl, cL);
    prim_to_cons_rn(P, prr, cR);
  } else {
    prim_to_cons_ns_rn(P, pl, cL);
    prim_to_cons_ns_rn(P, prr, cR);
  }
}

// Whether the Riemann solver provides RiemannVolFluxAndDissipMatrices (navierstokes/equation.f90:381-404,
// mhd/equation.f90:367-386), which SubFVMethod 3 and 4 need (nfvse.f90:174-187)
template <bool MHD, int RS>
__host__ __device__ constexpr bool has_dissip_matrices() {
  return MHD ? (RS == 14 || RS == 15) : (RS == 4 || RS == 44 || RS == 33);
}

// EC flux, dissipation diagonal and right eigenvectors (Rc[c] = column c) on rotated states
template <bool MHD, int RS, int NV>
__device__ __forceinline__ void fv_matrices(const KParams& P, double ch, const double* L, const double* R, double* F,
                                            double* D, double (*Rc)[NV]) {
  if constexpr (MHD) {
    mhd::es_9wave_matrices<RS == 15>(P, ch, L, R, F, D, Rc);
  } else {
    double Rh[5][5];
    es_matrices<RS>(P, L, R, F, D, Rh);
#pragma unroll
    for (int c = 0; c < 5; ++c)
#pragma unroll
      for (int r = 0; r < 5; ++r) Rc[c][r] = Rh[r][c];
  }
}
template <bool MHD>
__device__ __forceinline__ void fv_entropy(const KParams& P, const double* U, double* W) {
  if constexpr (MHD) mhd::cons_to_entropy(P, U, W);
  else cons_to_entropy_ns(P, U, W);
}
// RotateState (riemann.f90:218-231, mhd :185-200)
template <bool MHD, int NV>
__device__ __forceinline__ void fv_rotate(const double* a, const double* nv, const double* t1, const double* t2,
                                          double* o) {
#pragma unroll
  for (int v = 0; v < NV; ++v) o[v] = a[v];
#pragma unroll
  for (int b = 1; b <= (MHD ? 5 : 1); b += 4) {
    o[b] = a[b] * nv[0] + a[b + 1] * nv[1] + a[b + 2] * nv[2];
    o[b + 1] = a[b] * t1[0] + a[b + 1] * t1[1] + a[b + 2] * t1[2];
    o[b + 2] = a[b] * t2[0] + a[b + 1] * t2[1] + a[b + 2] * t2[2];
  }
}
// x = R^T v and F -= 1/2 R (D x), R given by its columns
template <int NV>
__device__ __forceinline__ void fv_rt(const double (*Rc)[NV], const double* v, double* x) {
#pragma unroll
  for (int c = 0; c < NV; ++c) {
    double s = 0.;
#pragma unroll
    for (int r = 0; r < NV; ++r) s += Rc[c][r] * v[r];
    x[c] = s;
  }
}
template <int NV>
__device__ __forceinline__ void fv_dissipate(const double (*Rc)[NV], const double* D, const double* x, double* F) {
  double y[NV];
#pragma unroll
  for (int c = 0; c < NV; ++c) y[c] = D[c] * x[c];
#pragma unroll
  for (int r = 0; r < NV; ++r) {
    double s = 0.;
#pragma unroll
    for (int c = 0; c < NV; ++c) s += Rc[c][r] * y[c];
    F[r] = F[r] - 0.5 * s;
  }
}

// Sub-cell metrics of face x = -1..N of the line through node n0 (position 0) of direction dir
// (ComputeSubcellMetrics, nfvse.f90:261-378): nv from Ja^dir, t1 from Ja^(dir+1), normalised, t2 = nv x t1
template <int NP>
__device__ __forceinline__ void face_metrics(const double* sM, const double* sW, const double* sD, int dir, int x,
                                             int n0, int stride, double* nv, double* t1, double* t2, double& norm) {
  constexpr int NP3 = NP * NP * NP;
  const double* Mn = sM + (3 * dir) * NP3;
  const double* Mt = sM + (3 * ((dir + 1) % 3)) * NP3;
#pragma unroll
  for (int c = 0; c < 3; ++c) { nv[c] = Mn[c * NP3 + n0]; t1[c] = Mt[c * NP3 + n0]; }
  for (int m = 0; m < NP; ++m)
    for (int l = 0; l <= x; ++l) {
      const double wd = sW[l] * sD[l * NP + m];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        nv[c] += wd * Mn[c * NP3 + n0 + m * stride];
        t1[c] += wd * Mt[c * NP3 + n0 + m * stride];
      }
    }
  norm = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
#pragma unroll
  for (int c = 0; c < 3; ++c) nv[c] = nv[c] / norm;
  const double tn = t1[0] * nv[0] + t1[1] * nv[1] + t1[2] * nv[2];
#pragma unroll
  for (int c = 0; c < 3; ++c) t1[c] = t1[c] - tn * nv[c];
  const double tl = sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
#pragma unroll
  for (int c = 0; c < 3; ++c) t1[c] = t1[c] / tl;
  t2[0] = nv[1] * t1[2] - nv[2] * t1[1];
  t2[1] = nv[2] * t1[0] - nv[0] * t1[2];
  t2[2] = nv[0] * t1[1] - nv[1] * t1[0];
}

// Scaled entropy variables w = R^T v of the two states of a face with the face's own eigenvectors
// (Compute_FVFluxes_1D_TVD_Fjordholm, nfvse.f90:1240-1256); F and D of the face are returned as well
template <bool MHD, int RS, int NV>
__device__ __forceinline__ void fj_face(const KParams& P, double ch, const double* uA, const double* uB,
                                        const double* nv, const double* t1, const double* t2, double* F, double* D,
                                        double (*Rc)[NV], double* wA, double* wB) {
  double L[NV], R[NV], vL[NV], vR[NV];
  fv_rotate<MHD, NV>(uA, nv, t1, t2, L);
  fv_rotate<MHD, NV>(uB, nv, t1, t2, R);
  fv_matrices<MHD, RS, NV>(P, ch, L, R, F, D, Rc);
  fv_entropy<MHD>(P, L, vL);
  fv_entropy<MHD>(P, R, vR);
  fv_rt<NV>(Rc, vL, wA);
  fv_rt<NV>(Rc, vR, wB);
}

// ES = 0: SubFVMethod 1 / 2 (P.subFV); 3: TVD-ES; 4: TVD-Fjordholm (both need has_dissip_matrices)
template <int NP, int ES>
__host__ __device__ constexpr size_t fv_smem_bytes() {
  return sizeof(double) * (size_t)(NP * NP + 6 * NP + (ES == 4 ? 45 : 36) * NP * NP * NP);
}

// Subcell FV volume integral (Compute_FVFluxes_1st_Order nfvse.f90:566-673, _TVD :674-815, _TVD2ES
// :826-1090, _TVD_Fjordholm :1101-1386, Compute_FVFluxes_1D :1389-1447) on the listed elements: one
// element per block iteration, one thread per node.  Per direction each node evaluates the flux on its
// right subcell face (x, x+1), keeps its own share (with its own non-conservative part) and hands the
// right neighbour's share over in shared memory.  F_FV(x) = (FR(x) - FL(x-1)) / w_x.
//   TVD-ES: EC flux and dissipation matrices of the nodal states; the dissipation acts on the entropy
//   jump of the TVD states unless, in some characteristic component, it has the opposite sign to the
//   nodal jump (below -1e-10), then on the nodal jump.
//   TVD-Fjordholm: every face first stores the scaled entropy variables w = R^T v of its two nodes (its
//   own eigenvectors) in shared memory; after a barrier each face reconstructs w at its two sides with
//   the minmod slopes of the neighbouring faces and dissipates the jump of the reconstructed values.
// resident blocks per SM the register allocation must allow: the MHD kernels hold the 9-variable states
// and the ES solver's mean state; 3 blocks of (N+1)^3 <= 128 threads keep 12 warps per SM at a few
// spilled doubles instead of 8 warps at 228+ registers
template <int NP, bool MHD>
__host__ __device__ constexpr int fv_minb() { return (MHD && NP * NP * NP <= 128) ? 3 : 1; }

template <int NP, int RS, bool MHD, int ES>
__global__ void __launch_bounds__(NP * NP * NP, fv_minb<NP, MHD>()) fv_kernel(KParams P) {
  if (halted(P)) return;
  constexpr int NP3 = NP * NP * NP, NPT = NP * NP, N = NP - 1, NV = MHD ? 9 : 5;
  static_assert(ES == 0 || has_dissip_matrices<MHD, RS>(), "SubFVMethod 3/4 need dissipation matrices");
  // LLF-dissipation solvers of Euler / Navier-Stokes: the largest wave speed over each subcell face
  // plane (AdvRiemann on the plane's points), per direction and face
  constexpr bool planeMax = !MHD && ES == 0 && riemann_needs_side_max<RS>();
  __shared__ unsigned long long sLam[3][NP];
  extern __shared__ double smem[];
  double* sD = smem;          // D(l,m) at [l*NP+m]
  double* sW = sD + NPT;      // wGP
  double* sIW = sW + NP;      // 1/wGP
  double* sU = sIW + NP;      // [node][9] state
  double* sM = sU + 9 * NP3;  // [9][node] metrics
  double* sA = sM + 9 * NP3;  // [node][9] left-face flux handed over by the left neighbour
  double* sPr = sA + 9 * NP3;  // [node][9] primitive variables (TVD reconstruction); Fjordholm: w of the left node
  double* sWB = sPr + 9 * NP3;  // Fjordholm: [node][9] w of the right node of the face at the node
  // TVD: node spacings and sub-cell offsets of InitNFVSE (nfvse.f90:218-238), index 1..N-1
  double* sdxR = sPr + (ES == 4 ? 18 : 9) * NP3;
  double* sdxL = sdxR + NP;
  double* rL = sdxL + NP;
  double* rR = rL + NP;
  const int t = threadIdx.x;
  for (int z = t; z < NPT; z += blockDim.x) sD[z] = P.basis->D[z];
  if (t < NP) { sW[t] = P.basis->wGP[t]; sIW[t] = 1.0 / P.basis->wGP[t]; }
  if (t == 0) {
    const double* x = P.basis->xGP;
    double sumWm1 = P.basis->wGP[0] - 1.;
    for (int m = 1; m <= N - 1; ++m) {
      sdxR[m] = 1.0 / (x[m + 1] - x[m]);
      sdxL[m] = 1.0 / (x[m] - x[m - 1]);
      rL[m] = sumWm1 - x[m];
      sumWm1 = sumWm1 + P.basis->wGP[m];
      rR[m] = sumWm1 - x[m];
    }
  }
  const bool tvd = ES == 3 || (ES == 0 && P.subFV == 2);
  const int i = t % NP, j = (t / NP) % NP, k = t / NPT;
  const double ch = MHD ? glm_ch(P) : 0.;
  const int count = *P.blendCount;
  for (int li = blockIdx.x; li < count; li += gridDim.x) {
    const int e = P.blendList[li];
    __syncthreads();  // the previous element is done with the shared arrays
    {
      const double* Ug = P.U + NV * ((size_t)e * NP3 + t);
#pragma unroll
      for (int v = 0; v < NV; ++v) sU[NV * t + v] = Ug[v];
      const double* Mg = P.metrics + (size_t)e * 9 * NP3 + t;
#pragma unroll
      for (int c = 0; c < 9; ++c) sM[c * NP3 + t] = Mg[c * NP3];
      if (tvd) c2p_rn<NV>(P, sU + NV * t, sPr + NV * t);
      if (planeMax && t < 3 * NP) sLam[t / NP][t % NP] = 0ull;
    }
    __syncthreads();
    double ffv[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) ffv[v] = 0.;
#pragma unroll 1
    for (int dir = 0; dir < 3; ++dir) {
      const int x = dir == 0 ? i : (dir == 1 ? j : k);
      const int stride = dir == 0 ? 1 : (dir == 1 ? NP : NPT);
      const int n0 = t - x * stride;  // node at position 0 of this node's line
      double nv[3], t1[3], t2[3], norm = 0., L[NV], R[NV];
      const double* uL = sU + NV * t;
      const double* uR = sU + NV * (t + (x < N ? stride : 0));
      if (x < N) face_metrics<NP>(sM, sW, sD, dir, x, n0, stride, nv, t1, t2, norm);
      double F[NV];
      if constexpr (ES == 4) {
        // phase 1: scaled entropy variables of both nodes of face x
        double Fc[NV], Dd[NV], Rc[NV][NV];
        if (x < N) fj_face<MHD, RS, NV>(P, ch, uL, uR, nv, t1, t2, Fc, Dd, Rc, sPr + NV * t, sWB + NV * t);
        __syncthreads();
        if (x < N) {
          const int rb = P.reconsBoundaries;
          const double* wLx = sPr + NV * t;  // w_L(x), w_R(x): nodes x, x+1 with face x's eigenvectors
          const double* wRx = sWB + NV * t;
          double wtR[NV], wtL[NV];
          // reconstructed value on the right of subcell x (wTildeR(x))
          if (x == 0) {
            double w0L[NV], w0R[NV];
            if (rb == 3) {  // the neighbour's state beyond node 0 and node 1, face -1 (nfvse.f90:1272-1290)
              double nb[3], tb1[3], tb2[3], nrm, Fd[NV], D0[NV], R0[NV][NV];
              face_metrics<NP>(sM, sW, sD, dir, -1, n0, stride, nb, tb1, tb2, nrm);
              fj_face<MHD, RS, NV>(P, ch, ext_node<NP, NV>(P, e, dir, false, t), sU + NV * (t + stride), nb, tb1, tb2,
                                   Fd, D0, R0, w0L, w0R);
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) {
              const double jl = wRx[v] - wLx[v];
              if (rb == 1) wtR[v] = wLx[v];
              else if (rb == 2) wtR[v] = wLx[v] + jl * sdxL[1] * sW[0];
              else wtR[v] = wLx[v] + minmod(sdxL[1] * jl, sdxL[1] * (w0R[v] - w0L[v])) * sW[0];
            }
          } else {
            const double* wLm = sPr + NV * (t - stride);  // face x-1
            const double* wRm = sWB + NV * (t - stride);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
              const double sg = minmod(sdxR[x] * (wRx[v] - wLx[v]), sdxL[x] * (wRm[v] - wLm[v]));
              wtR[v] = wLx[v] + sg * rR[x];
            }
          }
          // reconstructed value on the left of subcell x+1 (wTildeL(x+1))
          if (x + 1 == N) {
            double w0L[NV], w0R[NV];
            if (rb == 3) {  // node N-1 and the neighbour's state beyond node N, face N (nfvse.f90:1317-1335)
              double nb[3], tb1[3], tb2[3], nrm, Fd[NV], D0[NV], R0[NV][NV];
              face_metrics<NP>(sM, sW, sD, dir, N, n0, stride, nb, tb1, tb2, nrm);
              fj_face<MHD, RS, NV>(P, ch, sU + NV * t, ext_node<NP, NV>(P, e, dir, true, t + stride), nb, tb1, tb2,
                                   Fd, D0, R0, w0L, w0R);
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) {
              const double jr = wRx[v] - wLx[v];
              if (rb == 1) wtL[v] = wRx[v];
              else if (rb == 2) wtL[v] = wRx[v] - jr * sdxL[1] * sW[N];
              else wtL[v] = wRx[v] - minmod(sdxL[1] * jr, sdxL[1] * (w0R[v] - w0L[v])) * sW[N];
            }
          } else {
            const double* wLp = sPr + NV * (t + stride);  // face x+1
            const double* wRp = sWB + NV * (t + stride);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
              const double sg = minmod(sdxR[x + 1] * (wRp[v] - wLp[v]), sdxL[x + 1] * (wRx[v] - wLx[v]));
              wtL[v] = wRx[v] + sg * rL[x + 1];
            }
          }
          double jw[NV];
#pragma unroll
          for (int v = 0; v < NV; ++v) { F[v] = Fc[v]; jw[v] = wtL[v] - wtR[v]; }
          fv_dissipate<NV>(Rc, Dd, jw, F);
        }
      } else {
        if (x < N) {
          // states of the subcell Riemann problem: the nodal values (first order) or the TVD
          // reconstruction primR(x), primL(x+1) of the line (Compute_FVFluxes_TVD nfvse.f90:674-815)
          double cL[NV], cR[NV];
          if (tvd) {
            double extL[NV], extR[NV];
            if (P.reconsBoundaries == 3) {  // Get_externalU (nfvse.f90:1621-1683): the neighbours' nodes
              if (x == 0) ext_prim<NP, NV>(P, e, dir, false, t, extL);
              if (x + 1 == N) ext_prim<NP, NV>(P, e, dir, true, t + stride, extR);
            }
            tvd_states<NP, NV>(P, sPr + NV * (t - x * stride), NV * stride, x, sdxR, sdxL, rL, rR, sW, extL, extR, cL,
                               cR);
          } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) { cL[v] = uL[v]; cR[v] = uR[v]; }
          }
          fv_rotate<MHD, NV>(cL, nv, t1, t2, L);
          fv_rotate<MHD, NV>(cR, nv, t1, t2, R);
        }
        double lmm = 0.;
        if constexpr (planeMax) {
          if (x < N) atomicMax(&sLam[dir][x], (unsigned long long)__double_as_longlong(lambda_max_pair(P, L, R)));
          __syncthreads();
          if (x < N) lmm = __longlong_as_double((long long)sLam[dir][x]);
        }
        if (x < N) {
          if constexpr (ES == 3) {  // AdvRiemannRecons (nfvse.f90:1036-1090)
            double Ln[NV], Rn[NV], Dd[NV], Rc[NV][NV], va[NV], vb[NV], dv[NV], dvr[NV], xs[NV], xr[NV];
            fv_rotate<MHD, NV>(uL, nv, t1, t2, Ln);
            fv_rotate<MHD, NV>(uR, nv, t1, t2, Rn);
            fv_matrices<MHD, RS, NV>(P, ch, Ln, Rn, F, Dd, Rc);
            fv_entropy<MHD>(P, Ln, va);
            fv_entropy<MHD>(P, Rn, vb);
#pragma unroll
            for (int v = 0; v < NV; ++v) dv[v] = vb[v] - va[v];
            fv_entropy<MHD>(P, L, va);
            fv_entropy<MHD>(P, R, vb);
#pragma unroll
            for (int v = 0; v < NV; ++v) dvr[v] = vb[v] - va[v];
            fv_rt<NV>(Rc, dv, xs);
            fv_rt<NV>(Rc, dvr, xr);
            bool notES = false;
#pragma unroll
            for (int v = 0; v < NV; ++v) notES = notES || (xs[v] * xr[v] < -1.e-10);
            fv_dissipate<NV>(Rc, Dd, notES ? xs : xr, F);
          } else {
            if constexpr (MHD) mhd::riemann<RS>(P, ch, L, R, F);
            else riemann_rotated<RS>(P, L, R, lmm, F);
          }
        }
      }
      if (x < N) {
#pragma unroll
        for (int b = 1; b <= (MHD ? 5 : 1); b += 4) {  // RotateFluxBack, riemann.f90:235-246 (MHD :204-217)
          const double f2 = F[b], f3 = F[b + 1], f4 = F[b + 2];
          F[b] = nv[0] * f2 + t1[0] * f3 + t2[0] * f4;
          F[b + 1] = nv[1] * f2 + t1[1] * f3 + t2[1] * f4;
          F[b + 2] = nv[2] * f2 + t1[2] * f3 + t2[2] * f4;
        }
        double FR[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) FR[v] = F[v];
        if constexpr (MHD) {
          if (P.noncons != 0) {  // AddNonConsFlux on both nodes of the face (Compute_FVFluxes_1D :1420-1436)
            const bool ncg = P.ncGLM != 0;
            const double Bn = 0.5 * ((uL[5] + uR[5]) * nv[0] + (uL[6] + uR[6]) * nv[1] + (uL[7] + uR[7]) * nv[2]);
            const double ps = 0.5 * (uL[8] + uR[8]);
            const double nq[3] = {ps * nv[0], ps * nv[1], ps * nv[2]};
            mhd::add_noncons_surface(P.noncons, ncg, uR, Bn, nq, F);
            mhd::add_noncons_surface(P.noncons, ncg, uL, Bn, nq, FR);
          }
        }
        double* A = sA + NV * (t + stride);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          A[v] = F[v] * norm;
          ffv[v] += sIW[x] * (FR[v] * norm);
        }
      }
      __syncthreads();
      if (x > 0) {
#pragma unroll
        for (int v = 0; v < NV; ++v) ffv[v] -= sIW[x] * sA[NV * t + v];
      }
      __syncthreads();
    }
    // NFVSE_CORR keeps F_FV itself: the volume kernel also needs F_FV - Ut_DG of every element
    const double a = P.nfvseCorr ? 1.0 : P.alpha[e];
    double* O = P.fv + (size_t)e * NV * NP3 + t;
#pragma unroll
    for (int v = 0; v < NV; ++v) O[v * NP3] = a * ffv[v];
  }
}

// Get_Pressure / Get_dpdU (navierstokes/equation_vars.f90:752-760, 792-809; mhd/equation_vars.f90:803-812,
// 844-862)
template <int NV>
__device__ __forceinline__ double corr_pressure(const KParams& P, const double* U) {
  const double m2 = U[1] * U[1] + U[2] * U[2] + U[3] * U[3];
  if constexpr (NV == 9)
    return P.kappaM1 * (U[4] - 0.5 * (m2 / U[0]) - P.s2mu_0 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7] + U[8] * U[8]));
  else
    return P.kappaM1 * (U[4] - 0.5 * (m2 / U[0]));
}
template <int NV>
__device__ __forceinline__ void corr_dpdu(const KParams& P, const double* U, double* d) {
  const double vel[3] = {U[1] / U[0], U[2] / U[0], U[3] / U[0]};
  d[0] = 0.5 * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
#pragma unroll
  for (int c = 0; c < 3; ++c) d[1 + c] = -vel[c];
  d[4] = 1.0;
  if constexpr (NV == 9) {
#pragma unroll
    for (int z = 5; z < 9; ++z) d[z] = -P.smu_0 * U[z];
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) d[v] = d[v] * P.kappaM1;
}

// maximum over the block of NT threads (all call it; every thread gets the result): a tree in shared
// memory, so that partial warps (NT = 27, 125, 343) need no shuffles across missing lanes
template <int NT>
__device__ __forceinline__ double block_max(double v, double* red) {
  constexpr int P2 = NT <= 1 ? 1 : NT <= 2 ? 2 : NT <= 4 ? 4 : NT <= 8 ? 8 : NT <= 16 ? 16 : NT <= 32 ? 32
                   : NT <= 64 ? 64 : NT <= 128 ? 128 : NT <= 256 ? 256 : 512;
  static_assert(NT <= 512, "block_max: at most 512 threads");
  const int t = threadIdx.x;
  __syncthreads();  // the previous reduction's result has been read
  red[t] = v;
  __syncthreads();
#pragma unroll
  for (int s = P2 / 2; s > 0; s >>= 1) {
    if (t < s && t + s < NT) red[t] = fmax(red[t], red[t + s]);
    __syncthreads();
  }
  return red[0];
}

// Apply_NFVSE_Correction (nfvse.f90:1688-1883) after an RK stage update of U with step dt = b_dt(stage):
// one element per block, one thread per node.  Per element the smallest increase of alpha (a correction
// of U along FFV_m_FDG) that keeps the density, then the pressure (Newton iterations per node), at
// PositCorrFactor of the values of the safe state U + dt (1-alpha) FFV_m_FDG; alpha <= 1.  Ut (when
// `ut` is non-null) gets the matching change.  A safe state with negative density or pressure records
// elem*8 + 5 in errKey (the reference stops the run there).  Each node's Newton loop is bounded by
// PositMaxIter; the maxima are exact, so the result does not depend on thread order.
template <int NP, int NV>
__global__ void __launch_bounds__(NP * NP * NP) corr_kernel(KParams P, double* ut, double bStage, int* errKey) {
  if (halted(P)) return;
  constexpr int NP3 = NP * NP * NP;
  constexpr double eps = 1.e-14, NEWTON_ABSTOL = 1.e-8, alpha_maxPosit = 1.0;
  __shared__ double red[NP3];
  const int e = blockIdx.x, t = threadIdx.x;
  const double dt = bStage * (P.dtDev ? P.dtDev[0] : P.dt);
  if (!(dt > 0.)) return;  // a finished step (dt = 0) has nothing to correct
  const double sdt = 1. / dt;
  double alpha = P.alpha[e];
  if (fabs(alpha - alpha_maxPosit) < eps) return;
  double* Un = P.U + NV * ((size_t)e * NP3 + t);
  double* Utn = ut ? ut + NV * ((size_t)e * NP3 + t) : nullptr;
  const double* FF = P.ffvmfdg + NV * ((size_t)e * NP3 + t);
  double u[NV], ff[NV], us[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    u[v] = Un[v];
    ff[v] = FF[v];
    us[v] = u[v] + dt * ff[v] * (1. - alpha);
  }
  const double p_safe = corr_pressure<NV>(P, us);
  if (p_safe < 0. || us[0] < 0.) atomicMin(errKey, e * 8 + 5);
  auto correct = [&](double corr) {
    const double alphacont = alpha;
    alpha = alpha + corr * sdt;
    if (alpha > alpha_maxPosit) {
      alpha = alpha_maxPosit;
      corr = (alpha_maxPosit - alphacont) * dt;
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) u[v] = u[v] + corr * ff[v];
    if (Utn) {
#pragma unroll
      for (int v = 0; v < NV; ++v) Utn[v] = Utn[v] + (alpha - alphacont) * ff[v];
    }
  };
  // density
  double corr = -eps;
  {
    const double a = P.positCorrFactor * us[0] - u[0];
    if (a > 0. && !(fabs(ff[0]) < eps)) corr = a / ff[0];
  }
  corr = block_max<NP3>(corr, red);
  if (corr > 0.) correct(corr);
  // pressure
  corr = -eps;
  {
    double pres = corr_pressure<NV>(P, u);
    const double p_goal = P.positCorrFactor * p_safe;
    double ap = p_goal - pres;
    if (ap > 0.) {
      double Uc[NV], dp[NV], corr1 = 0.0;
#pragma unroll
      for (int v = 0; v < NV; ++v) Uc[v] = u[v];
      for (int it = 1; it <= P.positMaxIter; ++it) {
        corr_dpdu<NV>(P, Uc, dp);
        double dpa = 0.;
#pragma unroll
        for (int v = 0; v < NV; ++v) dpa = dpa + dp[v] * ff[v];
        if (fabs(dpa) < eps) break;
        corr1 = corr1 + ap / dpa;
#pragma unroll
        for (int v = 0; v < NV; ++v) Uc[v] = u[v] + corr1 * ff[v];
        pres = corr_pressure<NV>(P, Uc);
        ap = p_goal - pres;
        if (ap <= 2.220446049250313e-16 && ap > -NEWTON_ABSTOL * p_goal) break;
      }
      corr = fmax(corr, corr1);
    }
  }
  corr = block_max<NP3>(corr, red);
  if (corr > 0.) correct(corr);
#pragma unroll
  for (int v = 0; v < NV; ++v) Un[v] = u[v];
  if (t == 0) P.alpha[e] = alpha;
}

}  // namespace nfvse
}  // namespace fluxo
