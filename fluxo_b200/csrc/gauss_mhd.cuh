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
//
// The resistive / viscous terms with Gauss nodes (mhd_lift_visc_kernel): BR1 / BR2 gradients of the
// lifting variable with the surface terms at every node of each line (L_HatMinus(l)), the face traces of
// the gradient interpolated to the 6 sides and converted with the face states into each side's share
// n.F_v of the face flux (7 components, br1.f90:318-350, br2_surfint.f90:109-148), and the viscous /
// resistive volume integral of variables 2..8 (volint.f90:228-271), as gauss::lift_visc_kernel does for
// the Navier-Stokes equations.
#pragma once
#include "gauss.cuh"
#include "mhd_kernels.cuh"
#include "mhd_lifting.cuh"

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
// resident blocks per SM the register allocation must allow: one element per block leaves small-N blocks
// of (N+1)^3 threads, so for N <= 4 four of them (a register cap of 128), else one
template <int NP>
__host__ __device__ constexpr int surf_mhd_minb() { return NP * NP * NP <= 125 ? 4 : 1; }

template <int NP, int VF>
__global__ void __launch_bounds__(NP * NP * NP, surf_mhd_minb<NP>()) surf_mhd_kernel(KParams P) {
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

// shared memory of the MHD lifting kernel: operators, sJ, the 27 gradient rows (slot n + n / NP), and one
// area used in turn for the lifting variable [9][node], the staged side products [side point][27] and
// the contravariant fluxes [21][node]
template <int NP>
__host__ __device__ constexpr int mlift_area() {
  constexpr int a = 9 * NP * NP * NP, b = 27 * 6 * NP * NP, c = 21 * NP * NP * NP;
  return a > b ? (a > c ? a : c) : (b > c ? b : c);
}
template <int NP>
__host__ __device__ constexpr size_t mlift_smem_bytes() {
  return sizeof(double) * (size_t)(2 * NP * NP + 2 * NP + NP * NP * NP + 27 * lift_gstride<NP>() + mlift_area<NP>());
}

// resident blocks per SM for the lifting kernel: for N <= 4 three (as many as its shared memory allows at
// N = 4, a register cap of 170), else one
template <int NP>
__host__ __device__ constexpr int mlift_minb() { return NP * NP * NP <= 125 ? 3 : 1; }

template <int NP, int LIFT>
__global__ void __launch_bounds__(NP * NP * NP, mlift_minb<NP>()) mhd_lift_visc_kernel(KParams P) {
  if (halted(P)) return;
  constexpr int NV9 = 9, NP3 = NP * NP * NP, NPT = NP * NP, N = NP - 1, GS = lift_gstride<NP>();
  extern __shared__ double smem[];
  double* sD = smem;              // D(i,l) at [i*NP+l]
  double* sDhat = sD + NPT;       // D_hat(i,l)
  double* sLm = sDhat + NPT;      // L_Minus(l)
  double* sLh = sLm + NP;         // L_HatMinus(l)
  double* sSJ = sLh + NP;         // [node] sJ
  double* sG = sSJ + NP3;         // [27][slot] gradient of the lifting variable that is prolonged
  double* sA = sG + 27 * GS;      // lifting variable, then staged side products, then contravariant fluxes
  __shared__ int sE2S[12];
  const int e = blockIdx.x, t = threadIdx.x;
  const int i = t % NP, j = (t / NP) % NP, k = t / NPT;
  for (int z = t; z < NPT; z += NP3) { sD[z] = P.basis->D[z]; sDhat[z] = P.basis->Dhat[z]; }
  if (t < NP) { sLm[t] = P.basis->Lminus[t]; sLh[t] = P.basis->LhatMinus[t]; }
  for (int z = t; z < 12; z += NP3) sE2S[z] = P.e2s[12 * (size_t)e + z];  // NP3 = 8 for N = 1
  double u[NV9];
  const double sj = P.sJ[(size_t)e * NP3 + t];
  const int gs = lift_gslot(NP, t);
  {
    const double* Ug = P.U + NV9 * ((size_t)e * NP3 + t);
#pragma unroll
    for (int v = 0; v < NV9; ++v) u[v] = Ug[v];
    double V[NV9];
    mhd::lifting_var_rt(P, u, V);
#pragma unroll
    for (int v = 0; v < NV9; ++v) sA[v * NP3 + t] = V[v];
    sSJ[t] = sj;
  }
  __syncthreads();
  const double* M = P.metrics + (size_t)e * 9 * NP3 + t;
  double g[3][NV9];
  {
    // Lifting_VolInt (br1_volint.f90:45-98): the derivatives along the lines, metric terms
    double dx[NV9], de[NV9], dz[NV9];
#pragma unroll
    for (int v = 0; v < NV9; ++v) { dx[v] = 0.; de[v] = 0.; dz[v] = 0.; }
#pragma unroll
    for (int l = 0; l < NP; ++l) {
      const double a = sD[i * NP + l], b = sD[j * NP + l], c = sD[k * NP + l];
#pragma unroll
      for (int v = 0; v < NV9; ++v) {
        dx[v] += a * sA[v * NP3 + l + NP * (j + NP * k)];
        de[v] += b * sA[v * NP3 + i + NP * (l + NP * k)];
        dz[v] += c * sA[v * NP3 + i + NP * (j + NP * l)];
      }
    }
    double m[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) m[c] = M[c * NP3];
#pragma unroll
    for (int v = 0; v < NV9; ++v)
#pragma unroll
      for (int d = 0; d < 3; ++d) g[d][v] = m[0 + d] * dx[v] + m[3 + d] * de[v] + m[6 + d] * dz[v];
  }
  if constexpr (LIFT == 2) {  // br2_volint.f90: the volume part carries sJ; it is what is prolonged
#pragma unroll
    for (int v = 0; v < NV9; ++v)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        g[d][v] *= sj;
        sG[(NV9 * d + v) * GS + gs] = g[d][v];
      }
  }
  __syncthreads();  // the lifting variable is read; the area takes the staged side products
  // surface terms: every node of the line of each side takes the lifting flux times L_HatMinus(l); the 27
  // products (flux x normal) of each side point are staged once, [side point][3 x 9]
  for (int task = t; task < 6 * NPT; task += NP3) {
    const int s = task / NPT + 1, ab = task - (s - 1) * NPT, a = ab % NP, b = ab / NP;
    const int side = sE2S[2 * (s - 1)], flip = sE2S[2 * (s - 1) + 1];
    const int pt = face_point_of(NP, s, flip, a, b);
    const double* nvec = P.facegeo + (size_t)side * 10 * NPT + pt;
    const double* F = P.lflux + (size_t)side * NV9 * NPT + pt;
    const double n0 = nvec[0], n1 = nvec[NPT], n2 = nvec[2 * NPT];
#pragma unroll
    for (int v = 0; v < NV9; ++v) {
      const double f = F[v * NPT];
      sA[task * 27 + v] = f * n0;
      sA[task * 27 + 9 + v] = f * n1;
      sA[task * 27 + 18 + v] = f * n2;
    }
  }
  __syncthreads();
#pragma unroll 1
  for (int s = 1; s <= 6; ++s) {
    int l, a, b;
    line_of_node(N, s, i, j, k, l, a, b);
    const double* Fn = sA + ((s - 1) * NPT + a + NP * b) * 27;
    const double lh = sLh[l];
#pragma unroll
    for (int v = 0; v < NV9; ++v) {
      if constexpr (LIFT == 2) {
        const double fl = sj * lh;
        g[0][v] += fl * Fn[v]; g[1][v] += fl * Fn[9 + v]; g[2][v] += fl * Fn[18 + v];
      } else {
        g[0][v] += Fn[v] * lh; g[1][v] += Fn[9 + v] * lh; g[2][v] += Fn[18 + v] * lh;
      }
    }
  }
  if constexpr (LIFT == 1) {
#pragma unroll
    for (int v = 0; v < NV9; ++v)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        g[d][v] *= sj;
        sG[(NV9 * d + v) * GS + gs] = g[d][v];
      }
  }
  __syncthreads();  // the staged products are read; the gradient rows are complete
  // face traces: the gradient interpolated to each side's points (BR2: plus etaBR2 L_Minus(l) times the
  // own side's surface terms), converted with the side's state, n.F_v for the face kernel
  for (int task = t; task < 6 * NPT; task += NP3) {
    const int s = task / NPT + 1, ab = task - (s - 1) * NPT, a = ab % NP, b = ab / NP;
    const int side = sE2S[2 * (s - 1)], flip = sE2S[2 * (s - 1) + 1], role = flip == 0 ? 0 : 1;
    const int pt = face_point_of(NP, s, flip, a, b);
    const double* nvec = P.facegeo + (size_t)side * 10 * NPT + pt;
    const double n0 = nvec[0], n1 = nvec[NPT], n2 = nvec[2 * NPT];
    double tr[3][NV9];
    {
      const int nd = lift_gslot(NP, line_node_of(NP, s, a, b, 0));
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int v = 0; v < NV9; ++v) tr[d][v] = sG[(NV9 * d + v) * GS + nd] * sLm[0];
    }
    for (int l = 1; l < NP; ++l) {
      const int nd = lift_gslot(NP, line_node_of(NP, s, a, b, l));
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int v = 0; v < NV9; ++v) tr[d][v] = tr[d][v] + sG[(NV9 * d + v) * GS + nd] * sLm[l];
    }
    if constexpr (LIFT == 2) {
      const double* F = P.lflux + (size_t)side * NV9 * NPT + pt;
      double f[NV9];
#pragma unroll
      for (int v = 0; v < NV9; ++v) f[v] = F[v * NPT];
      for (int l = 0; l < NP; ++l) {
        const double w = P.etaBR2 * sLm[l], fl = sSJ[line_node_of(NP, s, a, b, l)] * sLh[l];
#pragma unroll
        for (int v = 0; v < NV9; ++v) {
          tr[0][v] = tr[0][v] + w * (fl * (f[v] * n0));
          tr[1][v] = tr[1][v] + w * (fl * (f[v] * n1));
          tr[2][v] = tr[2][v] + w * (fl * (f[v] * n2));
        }
      }
    }
    const double* uf = uface_at(P, NPT, side, role, pt, NV9);
    double us[NV9];
#pragma unroll
    for (int v = 0; v < NV9; ++v) us[v] = uf[v];
#pragma unroll
    for (int d = 0; d < 3; ++d) mhd::to_grad_prim_rt(P, us, tr[d]);
    double kf[7], kg[7], kh[7];
    mhd::visc_flux_3d(P, us, tr[0], tr[1], tr[2], kf, kg, kh);
    double* T = P.gtrace + ((size_t)side * 2 + role) * 7 * NPT + pt;
#pragma unroll
    for (int v = 0; v < 7; ++v) T[(size_t)v * NPT] = n0 * kf[v] + n1 * kg[v] + n2 * kh[v];
  }
  // volume: primitive gradients of the node, contravariant viscous / resistive fluxes
#pragma unroll
  for (int d = 0; d < 3; ++d) mhd::to_grad_prim_rt(P, u, g[d]);
  if (P.grad) {
    double* G = P.grad + 27 * ((size_t)e * NP3 + t);
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int v = 0; v < NV9; ++v) G[9 * d + v] = g[d][v];
  }
  {
    double f[7], gg[7], h[7];
    mhd::visc_flux_3d(P, u, g[0], g[1], g[2], f, gg, h);
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
      const double m0 = M[(3 * dir + 0) * NP3], m1 = M[(3 * dir + 1) * NP3], m2 = M[(3 * dir + 2) * NP3];
#pragma unroll
      for (int v = 0; v < 7; ++v) sA[(7 * dir + v) * NP3 + t] = f[v] * m0 + gg[v] * m1 + h[v] * m2;
    }
  }
  __syncthreads();
  double r[7] = {0., 0., 0., 0., 0., 0., 0.};
#pragma unroll
  for (int l = 0; l < NP; ++l) {
    const double a = sDhat[i * NP + l], b = sDhat[j * NP + l], c = sDhat[k * NP + l];
#pragma unroll
    for (int v = 0; v < 7; ++v)
      r[v] += a * sA[v * NP3 + l + NP * (j + NP * k)] + b * sA[(7 + v) * NP3 + i + NP * (l + NP * k)] +
              c * sA[(14 + v) * NP3 + i + NP * (j + NP * l)];
  }
  double* O = P.utvisc + (size_t)e * 7 * NP3 + t;
#pragma unroll
  for (int v = 0; v < 7; ++v) O[v * NP3] = r[v];
}

}  // namespace gauss
}  // namespace fluxo
