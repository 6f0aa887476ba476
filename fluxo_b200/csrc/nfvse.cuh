// NFVSE shock capturing (shockcapturing/nfvse.f90, nfvse_mpi.f90, indicators/indicators.f90) on
// the sm_100a path for the Euler / Navier-Stokes and the MHD systems, LGL nodes, first-order
// (SubFVMethod = 1) or TVD (SubFVMethod = 2) subcell finite volumes:
//   alpha_kernel      Persson-Peraire indicator of rho*p (or rho, p, kinetic energy) from its modal
//                     Legendre coefficients, alpha = 1/(1+exp(-s (eta-T)/T)), clipping;
//   propagate_kernel  alpha_e = max(alpha_e, SpacePropFactor * max over its sides of the two
//                     element values) and the list of blended elements (alpha > 2*EPSILON);
//   fv_kernel         per blended element: first-order or TVD subcell FV volume integral with sub-cell
//                     metrics built from the element's metrics on the fly (nfvse.f90:261-378),
//                     the Riemann solver of the face kernel and the non-conservative terms,
//                     written as alpha * F_FV for the volume kernel to blend with.
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
  } else {
    a = P.shockBlendCoef;
  }
  if (a < P.alphaMin) a = 0.0;
  else if (a >= P.alphaMax) a = P.alphaMax;
  P.alphaRaw[e] = a;
}

// PropagateBlendingCoeff (nfvse_mpi.f90:62-131) for one sweep from `src` into alpha; the last
// sweep also lists the blended elements
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
  if (last && a > kTiny) P.blendList[atomicAdd(P.blendCount, 1)] = e;
}

// no propagation (SpacePropSweeps = 0): alpha = raw value, list the blended elements
static __global__ void list_kernel(KParams P) {
  if (halted(P)) return;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= P.nElems) return;
  const double a = P.alphaRaw[e];
  P.alpha[e] = a;
  if (a > kTiny) P.blendList[atomicAdd(P.blendCount, 1)] = e;
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
__device__ __forceinline__ void ext_prim(const KParams& P, int e, int dir, bool plus, int node, double* pr) {
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
  c2p_rn<NV>(P, P.U + NV * ((size_t)nb * NP3 + nn), pr);
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

template <int NP>
__host__ __device__ constexpr size_t fv_smem_bytes() {
  return sizeof(double) * (size_t)(NP * NP + 6 * NP + 36 * NP * NP * NP);
}

// First-order subcell FV volume integral (Compute_FVFluxes_1st_Order nfvse.f90:566-673,
// Compute_FVFluxes_1D :1389-1447) of the MHD equations on the listed elements: one element per
// block iteration, one thread per node.  Per direction each node evaluates the flux on its right
// subcell face (x, x+1), keeps its own share (with its own non-conservative part) and hands the
// right neighbour's share over in shared memory.  F_FV(x) = (FR(x) - FL(x-1)) / w_x.
template <int NP, int RS, bool MHD>
__global__ void __launch_bounds__(NP * NP * NP) fv_kernel(KParams P) {
  if (halted(P)) return;
  constexpr int NP3 = NP * NP * NP, NPT = NP * NP, N = NP - 1, NV = MHD ? 9 : 5;
  // LLF-dissipation solvers of Euler / Navier-Stokes: the largest wave speed over each subcell face
  // plane (AdvRiemann on the plane's points), per direction and face
  constexpr bool planeMax = !MHD && riemann_needs_side_max<RS>();
  __shared__ unsigned long long sLam[3][NP];
  extern __shared__ double smem[];
  double* sD = smem;          // D(l,m) at [l*NP+m]
  double* sW = sD + NPT;      // wGP
  double* sIW = sW + NP;      // 1/wGP
  double* sU = sIW + NP;      // [node][9] state
  double* sM = sU + 9 * NP3;  // [9][node] metrics
  double* sA = sM + 9 * NP3;  // [node][9] left-face flux handed over by the left neighbour
  double* sPr = sA + 9 * NP3;  // [node][9] primitive variables (TVD reconstruction)
  // TVD: node spacings and sub-cell offsets of InitNFVSE (nfvse.f90:218-238), index 1..N-1
  double* sdxR = sPr + 9 * NP3;
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
  const bool tvd = P.subFV == 2;
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
      if (x < N) {
        // sub-cell metrics of face x (nfvse.f90:261-378): nv from Ja^dir, t1 from Ja^(dir+1)
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
#pragma unroll
        for (int v = 0; v < NV; ++v) { L[v] = cL[v]; R[v] = cR[v]; }
#pragma unroll
        for (int b = 1; b <= (MHD ? 5 : 1); b += 4) {  // RotateState, riemann.f90:218-231 (MHD :185-200)
          L[b] = cL[b] * nv[0] + cL[b + 1] * nv[1] + cL[b + 2] * nv[2];
          L[b + 1] = cL[b] * t1[0] + cL[b + 1] * t1[1] + cL[b + 2] * t1[2];
          L[b + 2] = cL[b] * t2[0] + cL[b + 1] * t2[1] + cL[b + 2] * t2[2];
          R[b] = cR[b] * nv[0] + cR[b + 1] * nv[1] + cR[b + 2] * nv[2];
          R[b + 1] = cR[b] * t1[0] + cR[b + 1] * t1[1] + cR[b + 2] * t1[2];
          R[b + 2] = cR[b] * t2[0] + cR[b + 1] * t2[1] + cR[b + 2] * t2[2];
        }
      }
      double lmm = 0.;
      if constexpr (planeMax) {
        if (x < N) atomicMax(&sLam[dir][x], (unsigned long long)__double_as_longlong(lambda_max_pair(P, L, R)));
        __syncthreads();
        if (x < N) lmm = __longlong_as_double((long long)sLam[dir][x]);
      }
      if (x < N) {
        double F[NV];
        if constexpr (MHD) mhd::riemann<RS>(P, ch, L, R, F);
        else riemann_rotated<RS>(P, L, R, lmm, F);
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
    const double a = P.alpha[e];
    double* O = P.fv + (size_t)e * NV * NP3 + t;
#pragma unroll
    for (int v = 0; v < NV; ++v) O[v * NP3] = a * ffv[v];
  }
}

}  // namespace nfvse
}  // namespace fluxo
