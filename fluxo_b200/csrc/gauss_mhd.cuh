// Gauss-node (PP_NodeType = 1) surface integral of the MHD + GLM right-hand side on sm_100a.
//
// The entropy-stable Gauss collocation of surfint.f90:118-175, 196-253 with the MHD two-point fluxes
// (mhd/flux_average.f90) and the non-conservative terms: for node l of the line through a side point,
//   FluxB(l)      = F#(U_l, U_side; Ja_l, SurfMetrics) + phi^<>(U_l -> U_side)
//   FluxB_sum     = sum_l [F#(U_l, U_side; ...) + phi^<>(U_side -> U_l)] L_Minus(l)
//   Ut(l)        += (Flux_side -+ (FluxB_sum - FluxB(l)) NormalSign) L_HatMinus(l)      (master + / slave -)
// where phi^<>(L -> R) is AddNonConsFluxVec (mhd/flux_average.f90:378-418) and Flux_side the side's own
// numerical flux: the conservative Riemann flux plus its non-conservative surface term from its own face
// state (AddNonConsFlux, mhd/riemann.f90:230-267, fillflux.f90:87-99).  The face states U_master /
// U_slave come from gauss::prolong_kernel (9 variables per point).  Output: [elem][9][node] for the MHD
// volume kernel, which adds it in place of its LGL surface terms.
#pragma once
#include "gauss.cuh"
#include "mhd_kernels.cuh"

namespace fluxo {
namespace gauss {

// phi^<>(L -> R) added to F, with the side records of mhd::Rec<VF> (B, psi and v at the record's offsets)
template <int VF>
__device__ __forceinline__ void nc_pair_rec(int NC, bool NCGLM, const double* rL, const double* rR,
                                            const double* mL, const double* mR, double* F) {
  constexpr int IB = mhd::Rec<VF>::B, IPSI = mhd::Rec<VF>::PSI, IV = mhd::Rec<VF>::V;
  const double bL0 = rL[IB], bL1 = rL[IB + 1], bL2 = rL[IB + 2];
  const double vL0 = rL[IV], vL1 = rL[IV + 1], vL2 = rL[IV + 2];
  const double h = 0.5 * ((mL[0] * bL0 + mL[1] * bL1 + mL[2] * bL2) +
                          (0.5 * (mL[0] + mR[0]) * rR[IB] + 0.5 * (mL[1] + mR[1]) * rR[IB + 1] +
                           0.5 * (mL[2] + mR[2]) * rR[IB + 2]));
  if (NC == 1 || NC == 2) { F[1] += h * bL0; F[2] += h * bL1; F[3] += h * bL2; }
  if (NC == 1) F[4] += h * (bL0 * vL0 + bL1 * vL1 + bL2 * vL2);
  if (NC == 1 || NC == 3) { F[5] += h * vL0; F[6] += h * vL1; F[7] += h * vL2; }
  if (NCGLM) {
    const double q = 0.5 * (rL[IPSI] + rR[IPSI]) * (mL[0] * vL0 + mL[1] * vL1 + mL[2] * vL2);
    F[4] += q * rL[IPSI];
    F[8] += q;
  }
}

// per side point of the element: record (NQ), SurfMetrics (3), the side's own flux (9); odd stride
template <int VF>
__host__ __device__ constexpr int surf_mhd_stride() { return (mhd::Rec<VF>::NQ + 12) | 1; }
template <int NP, int VF>
__host__ __device__ constexpr size_t surf_mhd_smem_bytes() {
  return sizeof(double) * (size_t)(6 * NP * NP * surf_mhd_stride<VF>() + 9 * NP * NP * NP);
}

// One element per block, one thread per node (as gauss::surf_kernel).
template <int NP, int VF>
__global__ void __launch_bounds__(NP * NP * NP, 1) surf_mhd_kernel(KParams P) {
  if (halted(P)) return;
  constexpr int NV9 = 9, NP3 = NP * NP * NP, NPT = NP * NP, N = NP - 1, NQ = mhd::Rec<VF>::NQ;
  constexpr int FS = surf_mhd_stride<VF>();
  extern __shared__ double smem[];
  double* sP = smem;               // [6 * NPT][FS]
  double* sB = sP + 6 * NPT * FS;  // [var][node] (FluxB(l) + phi(side -> l)) L_Minus(l) of the current side
  __shared__ double sLm[NP], sLh[NP];
  __shared__ int sE2S[12];
  const int NC = P.noncons;
  const bool NCGLM = NC != 0 && P.ncGLM != 0;
  const double ch = glm_ch(P);
  const int e = blockIdx.x, t = threadIdx.x;
  const int i = t % NP, j = (t / NP) % NP, k = t / NPT;
  if (t < NP) { sLm[t] = P.basis->Lminus[t]; sLh[t] = P.basis->LhatMinus[t]; }
  for (int z = t; z < 12; z += NP3) sE2S[z] = P.e2s[12 * (size_t)e + z];  // NP3 = 8 for N = 1
  double rN[NQ];
  {
    const double* Ug = P.U + NV9 * ((size_t)e * NP3 + t);
    double u[NV9];
#pragma unroll
    for (int v = 0; v < NV9; ++v) u[v] = Ug[v];
    mhd::make_rec<VF>(P, u, rN);
  }
  double m[9];
  {
    const double* M = P.metrics + (size_t)e * 9 * NP3 + t;
#pragma unroll
    for (int c = 0; c < 9; ++c) m[c] = M[c * NP3];
  }
  __syncthreads();
  for (int task = t; task < 6 * NPT; task += NP3) {
    const int s = task / NPT + 1, ab = task - (s - 1) * NPT, a = ab % NP, b = ab / NP;
    const int side = sE2S[2 * (s - 1)], flip = sE2S[2 * (s - 1) + 1], role = flip == 0 ? 0 : 1;
    const int pt = face_point_of(NP, s, flip, a, b);
    double* o = sP + task * FS;
    const double* uf = uface_at(P, NPT, side, role, pt, NV9);
    double us[NV9];
#pragma unroll
    for (int v = 0; v < NV9; ++v) us[v] = uf[v];
    {
      double r[NQ];
      mhd::make_rec<VF>(P, us, r);
#pragma unroll
      for (int z = 0; z < NQ; ++z) o[z] = r[z];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) o[NQ + c] = P.surfMet[(((size_t)e * 6 + (s - 1)) * 3 + c) * NPT + pt];
    const double* Fs = P.flux + (size_t)side * mhd::NF * NPT + pt;
    double F[NV9];
#pragma unroll
    for (int v = 0; v < NV9; ++v) F[v] = Fs[v * NPT];
    if (NC != 0) {
      const double nq[3] = {Fs[10 * NPT], Fs[11 * NPT], Fs[12 * NPT]};
      mhd::add_noncons_surface(NC, NCGLM, us, Fs[9 * NPT], nq, F);
    }
#pragma unroll
    for (int v = 0; v < NV9; ++v) o[NQ + 3 + v] = F[v];
  }
  double ut[NV9];
#pragma unroll
  for (int v = 0; v < NV9; ++v) ut[v] = 0.;
  __syncthreads();
#pragma unroll 1
  for (int s = 1; s <= 6; ++s) {
    int l, a, b;
    line_of_node(N, s, i, j, k, l, a, b);
    const int role = sE2S[2 * (s - 1) + 1] == 0 ? 0 : 1;
    const int dir = (s == XI_MINUS || s == XI_PLUS) ? 0 : ((s == ETA_MINUS || s == ETA_PLUS) ? 1 : 2);
    const double sg = (s == ZETA_MINUS || s == ETA_MINUS || s == XI_MINUS) ? -1. : 1.;  // NormalSigns
    const double* o = sP + ((s - 1) * NPT + a + NP * b) * FS;
    double mN[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) mN[c] = dir == 0 ? m[c] : (dir == 1 ? m[3 + c] : m[6 + c]);
    double FB[NV9], FC[NV9];
    mhd::pair_flux_mhd<VF>(P, ch, rN, o, mN, o + NQ, FB);
#pragma unroll
    for (int v = 0; v < NV9; ++v) FC[v] = FB[v];
    if (NC != 0) {
      nc_pair_rec<VF>(NC, NCGLM, o, rN, o + NQ, mN, FC);  // side state -> node l
      nc_pair_rec<VF>(NC, NCGLM, rN, o, mN, o + NQ, FB);  // node l -> side state
    }
#pragma unroll
    for (int v = 0; v < NV9; ++v) sB[v * NP3 + t] = FC[v] * sLm[l];
    __syncthreads();
    double sum[NV9];
#pragma unroll
    for (int v = 0; v < NV9; ++v) sum[v] = 0.;
    for (int ll = 0; ll < NP; ++ll) {
      const int nd = line_node_of(NP, s, a, b, ll);
#pragma unroll
      for (int v = 0; v < NV9; ++v) sum[v] = sum[v] + sB[v * NP3 + nd];
    }
    const double lh = sLh[l];
#pragma unroll
    for (int v = 0; v < NV9; ++v) {
      const double corr = (sum[v] - FB[v]) * sg;
      const double f = o[NQ + 3 + v];
      if (role == 0) ut[v] = ut[v] + (f - corr) * lh;
      else ut[v] = ut[v] - (f + corr) * lh;
    }
    __syncthreads();  // sB is rewritten by the next side
  }
  double* O = P.utsurf + (size_t)e * NV9 * NP3 + t;
#pragma unroll
  for (int v = 0; v < NV9; ++v) O[v * NP3] = ut[v];
}

}  // namespace gauss
}  // namespace fluxo
