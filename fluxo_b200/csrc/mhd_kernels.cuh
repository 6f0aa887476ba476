// sm_100a FP64 kernels of the MHD + GLM right-hand side (9 variables), LGL nodes, split form.
//
// Per RHS evaluation (dg/dg.f90:282-452, all sides inner sides):
//   ideal MHD:  face  ->  volume (split form + non-conservative terms + surface integral + Jacobian
//                                  + GLM damping [+ RK stage])
//   resistive:  lift_flux  ->  lifting + viscous (mhd_lifting.cuh)  ->  face (+ viscous)  ->  volume
// Face buffer per side point ([side][13][pt]): the conservative flux times SurfElem (9), then
// Bn*SurfElem with Bn = 1/2 (B_master + B_slave).n (the non-conservative surface term's weight,
// mhd/riemann.f90:230-267) and 1/2 (psi_master + psi_slave) n SurfElem (its GLM part, 3 values).
// The volume kernel adds each side's own non-conservative part from its boundary node's state.
#pragma once
#include "common.cuh"
#include "kernels.cuh"
#include "physics_mhd.cuh"

namespace fluxo {
namespace mhd {

constexpr int NF = 13;  // face buffer entries per point

// ------------------------------------------------------------------------------------------------
// Face kernel: ProlongToFace (LGL copy) + FillFlux (fillflux.f90:41-110): rotate (B too), Riemann,
// rotate back, + 1/2 n.(F_v(L) + F_v(R)) (mhd/riemann.f90:120-141), x SurfElem.
// ------------------------------------------------------------------------------------------------
template <int RS, bool VISC>
__global__ void face_kernel(KParams P, int NP) {
  if (halted(P)) return;
  const int npts = NP * NP;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)P.nSides * npts) return;
  const int side = (int)(idx / npts), pt = (int)(idx - (size_t)side * npts);
  const int* se5 = P.s2e + 5 * side;
  const int eM = se5[0], eS = se5[1];
  const int nM = side_node(NP - 1, pt % NP, pt / NP, 0, se5[2]);
  const int nS = side_node(NP - 1, pt % NP, pt / NP, se5[4], se5[3]);
  const size_t NP3 = (size_t)NP * NP * NP;
  // LGL: the sides' boundary nodes; Gauss nodes: the interpolated face states [side][master|slave][pt][9]
  const double* UM = P.uface ? P.uface + ((size_t)side * 2 * npts + pt) * NV : P.U + NV * ((size_t)eM * NP3 + nM);
  const double* US = P.uface ? P.uface + (((size_t)side * 2 + 1) * npts + pt) * NV : P.U + NV * ((size_t)eS * NP3 + nS);
  const double* g = P.facegeo + (size_t)side * 10 * npts + pt;
  double nv[3], t1[3], t2[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { nv[d] = g[d * npts]; t1[d] = g[(3 + d) * npts]; t2[d] = g[(6 + d) * npts]; }
  const double se = g[9 * npts];
  double uL[NV], uR[NV], L[NV], R[NV], F[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) { uL[v] = UM[v]; uR[v] = US[v]; L[v] = uL[v]; R[v] = uR[v]; }
  // RotateState, mhd/riemann.f90:185-200
#pragma unroll
  for (int b = 1; b <= 5; b += 4) {
    L[b] = uL[b] * nv[0] + uL[b + 1] * nv[1] + uL[b + 2] * nv[2];
    L[b + 1] = uL[b] * t1[0] + uL[b + 1] * t1[1] + uL[b + 2] * t1[2];
    L[b + 2] = uL[b] * t2[0] + uL[b + 1] * t2[1] + uL[b + 2] * t2[2];
    R[b] = uR[b] * nv[0] + uR[b + 1] * nv[1] + uR[b + 2] * nv[2];
    R[b + 1] = uR[b] * t1[0] + uR[b + 1] * t1[1] + uR[b + 2] * t1[2];
    R[b + 2] = uR[b] * t2[0] + uR[b + 1] * t2[1] + uR[b + 2] * t2[2];
  }
  riemann<RS>(P, glm_ch(P), L, R, F);
  // RotateFluxBack, mhd/riemann.f90:204-217
#pragma unroll
  for (int b = 1; b <= 5; b += 4) {
    const double f2 = F[b], f3 = F[b + 1], f4 = F[b + 2];
    F[b] = nv[0] * f2 + t1[0] * f3 + t2[0] * f4;
    F[b + 1] = nv[1] * f2 + t1[1] * f3 + t2[1] * f4;
    F[b + 2] = nv[2] * f2 + t1[2] * f3 + t2[2] * f4;
  }
  if constexpr (VISC) {  // + 1/2 (n.F_v(L) + n.F_v(R)); each side's share from its lifting kernel
    const double* tM = P.gtrace + ((size_t)side * 2 + 0) * 7 * npts + pt;
    const double* tS = P.gtrace + ((size_t)side * 2 + 1) * 7 * npts + pt;
#pragma unroll
    for (int v = 1; v < 8; ++v) F[v] = F[v] + 0.5 * (tM[(v - 1) * npts] + tS[(v - 1) * npts]);
  }
  double* out = P.flux + (size_t)side * NF * npts + pt;
#pragma unroll
  for (int v = 0; v < NV; ++v) out[v * npts] = F[v] * se;
  const double Bn = 0.5 * ((uL[5] + uR[5]) * nv[0] + (uL[6] + uR[6]) * nv[1] + (uL[7] + uR[7]) * nv[2]);
  out[9 * npts] = Bn * se;
  const double ps = 0.5 * (uL[8] + uR[8]) * se;
  out[10 * npts] = ps * nv[0];
  out[11 * npts] = ps * nv[1];
  out[12 * npts] = ps * nv[2];
}

// Lifting surface flux 1/2 (V_slave - V_master) SurfElem of the 9 lifting variables
// (Lifting_FillFlux br1_fillflux.f90:49-91 with EvalLiftingSurfFlux mhd/flux.f90:754-793)
template <int LV>
__global__ void lift_flux_kernel(KParams P, int NP) {
  if (halted(P)) return;
  const int npts = NP * NP;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)P.nSides * npts) return;
  const int side = (int)(idx / npts), pt = (int)(idx - (size_t)side * npts);
  const int* se5 = P.s2e + 5 * side;
  const int nM = side_node(NP - 1, pt % NP, pt / NP, 0, se5[2]);
  const int nS = side_node(NP - 1, pt % NP, pt / NP, se5[4], se5[3]);
  const size_t NP3 = (size_t)NP * NP * NP;
  const double* UM = P.uface ? P.uface + ((size_t)side * 2 * npts + pt) * NV : P.U + NV * ((size_t)se5[0] * NP3 + nM);
  const double* US = P.uface ? P.uface + (((size_t)side * 2 + 1) * npts + pt) * NV : P.U + NV * ((size_t)se5[1] * NP3 + nS);
  double uM[NV], uS[NV], VM[NV], VS[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) { uM[v] = UM[v]; uS[v] = US[v]; }
  lift_var<LV>(P, uM, VM);
  lift_var<LV>(P, uS, VS);
  const double se = P.facegeo[(size_t)side * 10 * npts + 9 * npts + pt];
  double* o = P.lflux + (size_t)side * NV * npts + pt;
#pragma unroll
  for (int v = 0; v < NV; ++v) o[v * npts] = 0.5 * (VS[v] - VM[v]) * se;
}

// ------------------------------------------------------------------------------------------------
// Split-form volume records and pair fluxes (VolumeFluxAverageVec, mhd/flux_average.f90)
// ------------------------------------------------------------------------------------------------
template <int VF> struct Rec;
// standard DG (0) / dealiased metric (1): rho, rho v(3), E - psi^2/(2mu0), p_t, v(3), B(3), psi, v.B
// (NQ state entries, then the metrics of the three directions; B, PSI, V: offsets of B, psi, v)
template <> struct Rec<0> { static constexpr int NQ = 15, RS = 24, B = 9, PSI = 12, V = 6; };
template <> struct Rec<1> { static constexpr int NQ = 15, RS = 24, B = 9, PSI = 12, V = 6; };
// Derigs (10): rho, beta, v(3), B(3), psi, |v|^2, |B|^2, v.B, log rho, log beta
template <> struct Rec<10> { static constexpr int NQ = 14, RS = 23, B = 5, PSI = 8, V = 2; };
// FloGor (12): rho, p, e_in, v(3), B(3), psi, log rho, log e_in
template <> struct Rec<12> { static constexpr int NQ = 12, RS = 21, B = 6, PSI = 9, V = 3; };

constexpr int NACC = NV + 2;  // accumulator per node: Ut (9), non-conservative MHD and GLM line sums

template <int VF>
__device__ __forceinline__ void make_rec(const KParams& P, const double* U, double* r) {
  // EvalUaux, mhd/flux_average.f90:223-259
  const double srho = 1. / U[0];
  const double v1 = U[1] * srho, v2 = U[2] * srho, v3 = U[3] * srho;
  const double v2s = v1 * v1 + v2 * v2 + v3 * v3;
  const double B2 = U[5] * U[5] + U[6] * U[6] + U[7] * U[7];
  const double vB = v1 * U[5] + v2 * U[6] + v3 * U[7];
  const double pt = P.kappaM1 * (U[4] - 0.5 * U[0] * v2s - P.s2mu_0 * U[8] * U[8]) - P.kappaM2 * P.s2mu_0 * B2;
  if constexpr (VF == 0 || VF == 1) {
    r[0] = U[0]; r[1] = U[1]; r[2] = U[2]; r[3] = U[3];
    r[4] = U[4] - 0.5 * P.smu_0 * U[8] * U[8]; r[5] = pt;
    r[6] = v1; r[7] = v2; r[8] = v3;
    r[9] = U[5]; r[10] = U[6]; r[11] = U[7]; r[12] = U[8]; r[13] = vB; r[14] = 0.;
  } else if constexpr (VF == 10) {
    const double beta = 0.5 * U[0] / (pt - P.s2mu_0 * B2);
    r[0] = U[0]; r[1] = beta; r[2] = v1; r[3] = v2; r[4] = v3;
    r[5] = U[5]; r[6] = U[6]; r[7] = U[7]; r[8] = U[8];
    r[9] = v2s; r[10] = B2; r[11] = vB; r[12] = log(U[0]); r[13] = log(beta);
  } else if constexpr (VF == 12) {
    const double p = pt - P.s2mu_0 * B2;
    const double ie = p / U[0] * P.sKappaM1;
    r[0] = U[0]; r[1] = p; r[2] = ie; r[3] = v1; r[4] = v2; r[5] = v3;
    r[6] = U[5]; r[7] = U[6]; r[8] = U[7]; r[9] = U[8]; r[10] = log(U[0]); r[11] = log(ie);
  }
}

// F = F#(L, R; metrics), symmetric in (L, R)
template <int VF>
__device__ __forceinline__ void pair_flux_mhd(const KParams& P, double ch, const double* L, const double* R,
                                          const double* mL, const double* mR, double* F) {
  const double smu0 = P.smu_0;
  if constexpr (VF == 0) {  // StandardDGFluxVec :492-567
    const double qvL = L[6] * mL[0] + L[7] * mL[1] + L[8] * mL[2], qbL = L[9] * mL[0] + L[10] * mL[1] + L[11] * mL[2];
    const double qvR = R[6] * mR[0] + R[7] * mR[1] + R[8] * mR[2], qbR = R[9] * mR[0] + R[10] * mR[1] + R[11] * mR[2];
    F[0] = 0.5 * (L[0] * qvL + R[0] * qvR);
#pragma unroll
    for (int d = 0; d < 3; ++d)
      F[1 + d] = 0.5 * (L[1 + d] * qvL + R[1 + d] * qvR + mL[d] * L[5] + mR[d] * R[5] - smu0 * (qbL * L[9 + d] + qbR * R[9 + d]));
    F[4] = 0.5 * ((L[4] + L[5]) * qvL + (R[4] + R[5]) * qvR - smu0 * (qbL * L[13] + qbR * R[13]));
#pragma unroll
    for (int d = 0; d < 3; ++d) F[5 + d] = 0.5 * (qvL * L[9 + d] - qbL * L[6 + d] + qvR * R[9 + d] - qbR * R[6 + d]);
    F[4] = F[4] + 0.5 * smu0 * ch * (qbL * L[12] + qbR * R[12]);
#pragma unroll
    for (int d = 0; d < 3; ++d) F[5 + d] = F[5 + d] + 0.5 * ch * (L[12] * mL[d] + R[12] * mR[d]);
    F[8] = 0.5 * ch * (qbL + qbR);
  } else {
    const double m[3] = {0.5 * (mL[0] + mR[0]), 0.5 * (mL[1] + mR[1]), 0.5 * (mL[2] + mR[2])};
    if constexpr (VF == 1) {  // StandardDGFluxDealiasedMetricVec :574-651
      const double qvL = L[6] * m[0] + L[7] * m[1] + L[8] * m[2], qbL = L[9] * m[0] + L[10] * m[1] + L[11] * m[2];
      const double qvR = R[6] * m[0] + R[7] * m[1] + R[8] * m[2], qbR = R[9] * m[0] + R[10] * m[1] + R[11] * m[2];
      F[0] = 0.5 * (L[0] * qvL + R[0] * qvR);
#pragma unroll
      for (int d = 0; d < 3; ++d)
        F[1 + d] = 0.5 * (L[1 + d] * qvL + R[1 + d] * qvR + m[d] * (L[5] + R[5]) - smu0 * (qbL * L[9 + d] + qbR * R[9 + d]));
      F[4] = 0.5 * ((L[4] + L[5]) * qvL + (R[4] + R[5]) * qvR - smu0 * (qbL * L[13] + qbR * R[13]));
#pragma unroll
      for (int d = 0; d < 3; ++d) F[5 + d] = 0.5 * (qvL * L[9 + d] - qbL * L[6 + d] + qvR * R[9 + d] - qbR * R[6 + d]);
      F[4] = F[4] + 0.5 * smu0 * ch * (qbL * L[12] + qbR * R[12]);
      const double phiHat = 0.5 * ch * (L[12] + R[12]);
#pragma unroll
      for (int d = 0; d < 3; ++d) F[5 + d] = F[5 + d] + phiHat * m[d];
      F[8] = 0.5 * ch * (qbL + qbR);
    } else if constexpr (VF == 10) {  // EntropyAndKinEnergyConservingFluxVec_Derigs :761-848
      double nr, dr, nb, db;
      ln_mean_nd(L, R, 0, 12, nr, dr);
      ln_mean_nd(L, R, 1, 13, nb, db);
      const double sr = L[0] + R[0], sb = L[1] + R[1];
      const double inv = 1. / (dr * nb * sb);
      const double rhoLN = nr * nb * sb * inv;    // LN(rho)
      const double sbLN = db * dr * sb * inv;     // 1/LN(beta)
      const double rsb = sr * dr * nb * inv;      // (rho_L+rho_R)/(beta_L+beta_R)
      double vA[3], BA[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) { vA[d] = 0.5 * (L[2 + d] + R[2 + d]); BA[d] = 0.5 * (L[5 + d] + R[5 + d]); }
      const double pTilde = 0.5 * (rsb + smu0 * 0.5 * (L[10] + R[10]));
      const double vm = vA[0] * m[0] + vA[1] * m[1] + vA[2] * m[2];
      const double Bm = BA[0] * m[0] + BA[1] * m[1] + BA[2] * m[2];
      const double psiA = 0.5 * (L[8] + R[8]);
      F[0] = rhoLN * vm;
#pragma unroll
      for (int d = 0; d < 3; ++d) F[1 + d] = F[0] * vA[d] - (smu0 * Bm) * BA[d] + pTilde * m[d];
#pragma unroll
      for (int d = 0; d < 3; ++d) F[5 + d] = vm * BA[d] - Bm * vA[d] + (ch * psiA) * m[d];
      F[8] = ch * Bm;
      const double sB = BA[0] * F[5] + BA[1] * F[6] + BA[2] * F[7];
      const double b2v = (L[10] * L[2] + R[10] * R[2]) * m[0] + (L[10] * L[3] + R[10] * R[3]) * m[1] +
                         (L[10] * L[4] + R[10] * R[4]) * m[2];
      const double pB = (L[8] * L[5] + R[8] * R[5]) * m[0] + (L[8] * L[6] + R[8] * R[6]) * m[1] +
                        (L[8] * L[7] + R[8] * R[7]) * m[2];
      F[4] = F[0] * 0.5 * (P.sKappaM1 * sbLN - 0.5 * (L[9] + R[9])) + (vA[0] * F[1] + vA[1] * F[2] + vA[2] * F[3]) +
             smu0 * (sB - 0.25 * b2v + 0.5 * (L[11] + R[11]) * Bm + F[8] * psiA - (ch * 0.5) * pB);
    } else if constexpr (VF == 12) {  // EntropyAndKinEnergyConservingFluxVec_FloGor :970-1074
      double nr, dr, ne, de;
      ln_mean_nd(L, R, 0, 10, nr, dr);
      ln_mean_nd(L, R, 2, 11, ne, de);
      const double inv = 1. / (dr * ne);
      const double rhoLN = nr * ne * inv;
      const double ieT = L[2] * R[2] * de * dr * inv;  // e_L e_R / LN(e)
      double vA[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) vA[d] = 0.5 * (L[3 + d] + R[3 + d]);
      const double v2Z = L[3] * R[3] + L[4] * R[4] + L[5] * R[5];
      const double B2Z = L[6] * R[6] + L[7] * R[7] + L[8] * R[8];
      const double pA = 0.5 * (L[1] + R[1]);
      const double vmL = L[3] * m[0] + L[4] * m[1] + L[5] * m[2], vmR = R[3] * m[0] + R[4] * m[1] + R[5] * m[2];
      const double BmL = L[6] * m[0] + L[7] * m[1] + L[8] * m[2], BmR = R[6] * m[0] + R[7] * m[1] + R[8] * m[2];
      auto zip = [](double a, double b, double c, double d) { return 0.5 * (a * d + b * c); };
      F[0] = rhoLN * 0.5 * (vmL + vmR);
#pragma unroll
      for (int d = 0; d < 3; ++d)
        F[1 + d] = F[0] * vA[d] + m[d] * (pA + P.s2mu_0 * B2Z) - smu0 * zip(L[6 + d], R[6 + d], BmL, BmR);
      double s = 0.;
#pragma unroll
      for (int d = 0; d < 3; ++d)
        s = s + zip(vmL * L[6 + d], vmR * R[6 + d], L[6 + d], R[6 + d]) - zip(L[3 + d] * BmL, R[3 + d] * BmR, L[6 + d], R[6 + d]);
      F[4] = F[0] * (0.5 * v2Z + ieT) + zip(L[1], R[1], vmL, vmR) + smu0 * (s + ch * zip(BmL, BmR, L[9], R[9]));
#pragma unroll
      for (int d = 0; d < 3; ++d)
        F[5 + d] = 0.5 * ((vmL * L[6 + d] - L[3 + d] * BmL) + (vmR * R[6 + d] - R[3 + d] * BmR) + ch * (L[9] + R[9]) * m[d]);
      F[8] = ch * 0.5 * (BmL + BmR);
    }
  }
}

// ------------------------------------------------------------------------------------------------
// Volume kernel: split-form volume integral with the non-conservative terms (volint.f90:173-218,
// mhd/flux_average.f90:112-186 and AddNonConsFluxTilde3D :268-366), viscous / resistive volume
// integral (from the lifting kernel), surface integral with each side's own non-conservative part,
// Jacobian, GLM damping (mhd/equation.f90:1698-1706), optional LSERK stage.
//
// The non-conservative term of node i along one line is Phi(i) * sum_l Dvs(i,l) (Bhat_i +
// (M_i+M_l)/2 . B_l) = Phi(i) * (Bhat_i rowsum_i + M_i/2 . sum_l Dvs B_l + 1/2 sum_l Dvs Bhat_l): four
// line sums per direction, accumulated over the directions into one scalar per node.
// ------------------------------------------------------------------------------------------------
template <int NP>
__host__ __device__ constexpr int epb() { return (256 / (NP * NP * NP)) > 0 ? (256 / (NP * NP * NP)) : 1; }

// node slot of the records and accumulators: for N+1 = 5 (6 lines of 5 lanes per warp, 23-double
// records) four spare slots after every 25 nodes, from a lane-by-lane model of the own, partner and
// line-sum loads (1.12x the minimum shared wavefronts against 1.24x for one spare slot every 16
// nodes); other N+1 keep the 16-node padding
template <int NP>
__host__ __device__ constexpr int mpad(int n) { return NP == 5 ? n + 4 * (n / 25) : vol_slot(n); }
template <int NP>
__host__ __device__ constexpr int mpad_slots() { return mpad<NP>(NP * NP * NP - 1) + 1; }

template <int NP, int VF>
__host__ __device__ constexpr size_t vol_smem_bytes() {
  return sizeof(double) * (size_t)(NP * NP + NP + epb<NP>() * (Rec<VF>::RS + NACC) * mpad_slots<NP>());
}

// Pair-phase schedule: lines contiguous in the thread index when N+1 divides 32, otherwise
// floor(32/(N+1)) lines packed whole into each warp (the rounds are warp shuffles either way; see the
// Euler / Navier-Stokes volume kernel)
template <int NP>
__host__ __device__ constexpr int vol_lpw() { return 32 % NP == 0 ? 0 : 32 / NP; }

template <int NP>
__host__ __device__ constexpr int vol_threads() { return VolShape<NP, epb<NP>(), vol_lpw<NP>()>::THREADS; }

// resident blocks per SM the register allocation must allow: 2 for blocks of up to 320 threads
// (at most 102 registers: more resident warps than the unconstrained ~160), else 1
template <int NP>
__host__ __device__ constexpr int vol_minb() { return vol_threads<NP>() <= 320 ? 2 : 1; }

template <int NP, int VF>
__global__ void __launch_bounds__(vol_threads<NP>(), vol_minb<NP>()) volume_kernel(KParams P) {
  if (halted(P)) return;
  const int NC = P.noncons;
  const bool NCGLM = NC != 0 && P.ncGLM != 0;
  constexpr int NP3 = NP * NP * NP, N = NP - 1, NPT = NP * NP, EPB = epb<NP>(), LPW = vol_lpw<NP>();
  constexpr int RS = Rec<VF>::RS, NQ = Rec<VF>::NQ, IB = Rec<VF>::B, IPSI = Rec<VF>::PSI, IV = Rec<VF>::V;
  constexpr int NS = mpad_slots<NP>();
  extern __shared__ double smem[];
  double* sDvs = smem;        // Dvolsurf(i,l) at [i*NP+l]
  double* sRow = sDvs + NPT;  // sum_l Dvolsurf(i,l)
  // node phases: thread -> (element slot eb, node t); with packed lines the threads past EPB*NP3 idle
  const bool nodeThread = threadIdx.x < EPB * NP3;
  const int eb = nodeThread ? threadIdx.x / NP3 : 0, t = nodeThread ? threadIdx.x - eb * NP3 : 0;
  const int e = blockIdx.x * EPB + eb;
  const bool valid = nodeThread && e < P.nElems;
  double* rec = sRow + NP + (size_t)eb * (RS + NACC) * NS;  // [slot][RS]
  double* acc = rec + (size_t)RS * NS;                       // [slot][NACC]
  for (int z = threadIdx.x; z < NPT; z += blockDim.x) sDvs[z] = P.basis->Dvs[z];
  if (threadIdx.x < NP) {
    double s = 0.;
    for (int l = 0; l < NP; ++l) s += P.basis->Dvs[threadIdx.x * NP + l];
    sRow[threadIdx.x] = s;
  }
  const double ch = glm_ch(P);
  double u[NV];
  if (valid) {
    const double* Ug = P.U + NV * ((size_t)e * NP3 + t);
#pragma unroll
    for (int v = 0; v < NV; ++v) u[v] = Ug[v];
    prefetch_l2(P.sJ + (size_t)e * NP3 + t);
    double* r = rec + mpad<NP>(t) * RS;
    make_rec<VF>(P, u, r);
    const double* Mg = P.metrics + (size_t)e * 9 * NP3 + t;
#pragma unroll
    for (int c = 0; c < 9; ++c) r[NQ + c] = Mg[c * NP3];
#pragma unroll
    for (int v = 0; v < NACC; ++v) acc[mpad<NP>(t) * NACC + v] = 0.;
  }
  __syncthreads();
  {
    // this thread's (element slot pe, line Ln, position p) in the pair phase; lv: it holds a position
    // of a line of an existing element (idle lanes keep in-range indexes and only join the shuffles)
    int pe, p, Ln, lbase;
    bool lv;
    const int lane = threadIdx.x & 31;
    if constexpr (LPW == 0) {
      pe = eb; p = t % NP; Ln = t / NP; lv = valid; lbase = lane - p;
    } else {
      constexpr int G = 32 / LPW, WPE = VolShape<NP, EPB, LPW>::WPE;
      const int wi = threadIdx.x >> 5, slot = lane / G;
      pe = wi / WPE;
      p = lane - slot * G;
      Ln = (wi - pe * WPE) * LPW + slot;
      lv = slot < LPW && p < NP && Ln < NPT && (int)blockIdx.x * EPB + pe < P.nElems;
      lbase = slot * G;
      if (!lv) { p = 0; Ln = 0; }
    }
    const int la = Ln % NP, lb = Ln / NP;
    double* prec = sRow + NP + (size_t)pe * (RS + NACC) * NS;
    double* pacc = prec + (size_t)RS * NS;
#pragma unroll 1
    for (int dir = 0; dir < 3; ++dir) {
      const int stride = dir == 0 ? 1 : (dir == 1 ? NP : NPT);
      const int base = dir == 0 ? NP * (la + NP * lb) : (dir == 1 ? la + NPT * lb : la + NP * lb);
      const int own = base + p * stride, os = mpad<NP>(own);
      double ro[NQ], mo[3], racc[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) racc[v] = 0.;
      if (lv) {
#pragma unroll
        for (int z = 0; z < NQ; ++z) ro[z] = prec[os * RS + z];
#pragma unroll
        for (int c = 0; c < 3; ++c) mo[c] = prec[os * RS + NQ + 3 * dir + c];
      }
#pragma unroll
      for (int d = 1; d <= NP / 2; ++d) {
        const bool active = lv && (2 * d < NP || p < d);
        int q = p + d;
        if (q >= NP) q -= NP;
        double F[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) F[v] = 0.;
        if (active) {
          // the partner's record is read in place (the log-mean logarithms only when needed)
          const double* rq = prec + mpad<NP>(base + q * stride) * RS;
          pair_flux_mhd<VF>(P, ch, ro, rq, mo, rq + NQ + 3 * dir, F);
        }
        const double dOwn = sDvs[p * NP + q], dPart = sDvs[q * NP + p];
        int src = p - d;
        if (src < 0) src += NP;
        const bool receive = lv && (2 * d < NP || p >= d);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          racc[v] += active ? dOwn * F[v] : 0.;
          const double got = __shfl_sync(0xffffffffu, dPart * F[v], (lbase + src) & 31);
          racc[v] += receive ? got : 0.;
        }
      }
      double ncMHD = 0., ncGLM = 0.;  // this direction's non-conservative line sums of node `own`
      {
        if (lv && NC != 0) {
          double sB0 = 0., sB1 = 0., sB2 = 0., sBh = 0., sPsi = 0.;
#pragma unroll
          for (int l = 0; l < NP; ++l) {
            const double* rl = prec + mpad<NP>(base + l * stride) * RS;
            const double dl = sDvs[p * NP + l];
            const double b0 = rl[IB], b1 = rl[IB + 1], b2 = rl[IB + 2];
            const double* ml = rl + NQ + 3 * dir;
            sB0 += dl * b0; sB1 += dl * b1; sB2 += dl * b2;
            sBh += dl * (ml[0] * b0 + ml[1] * b1 + ml[2] * b2);
            sPsi += dl * rl[IPSI];
          }
          const double bhat = mo[0] * ro[IB] + mo[1] * ro[IB + 1] + mo[2] * ro[IB + 2];
          ncMHD = bhat * sRow[p] + 0.5 * (mo[0] * sB0 + mo[1] * sB1 + mo[2] * sB2) + 0.5 * sBh;
          if (NCGLM) {
            const double vm = mo[0] * ro[IV] + mo[1] * ro[IV + 1] + mo[2] * ro[IV + 2];
            ncGLM = 0.5 * vm * (ro[IPSI] * sRow[p] + sPsi);
          }
        }
      }
      if (lv) {
#pragma unroll
        for (int v = 0; v < NV; ++v) pacc[os * NACC + v] += racc[v];
        pacc[os * NACC + NV] += ncMHD;
        pacc[os * NACC + NV + 1] += ncGLM;
      }
      __syncthreads();
    }
  }
  double ut[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) ut[v] = valid ? acc[mpad<NP>(t) * NACC + v] : 0.;
  const double ncMHD = valid ? acc[mpad<NP>(t) * NACC + NV] : 0.;
  const double ncGLM = valid ? acc[mpad<NP>(t) * NACC + NV + 1] : 0.;
  const int i = t % NP, j = (t / NP) % NP, k = t / NPT;
  if (!valid) return;
  if (NC != 0) {  // Phi(i) * sum of the line terms (Powell / Brackbill / Janhunen)
    const double srho = 1. / u[0];
    const double v0 = u[1] * srho, v1 = u[2] * srho, v2 = u[3] * srho;
    const double h = 0.5 * ncMHD;
    if (NC == 1 || NC == 2) { ut[1] += h * u[5]; ut[2] += h * u[6]; ut[3] += h * u[7]; }
    if (NC == 1) ut[4] += h * (v0 * u[5] + v1 * u[6] + v2 * u[7]);
    if (NC == 1 || NC == 3) { ut[5] += h * v0; ut[6] += h * v1; ut[7] += h * v2; }
    if (NCGLM) { ut[4] += u[8] * ncGLM; ut[8] += ncGLM; }
  }
  if (P.nfvse) {  // VolInt_NFVSE (nfvse.f90:475-565): blend with alpha * F_FV of the subcell FV kernel
    const double a = P.alpha[e];
    const double* FV = P.fv + (size_t)e * NV * NP3 + t;
    if (P.nfvseCorr) {  // F_FV of every element; FFV_m_FDG = (F_FV - Ut) (-sJ) for the correction
      const double sjn = P.sJ[(size_t)e * NP3 + t];
      double* FF = P.ffvmfdg + NV * ((size_t)e * NP3 + t);
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const double f = FV[v * NP3];
        FF[v] = (f - ut[v]) * (-sjn);
        ut[v] = (1. - a) * ut[v] + a * f;
      }
    } else if (a > 4.440892098500626e-16) {
#pragma unroll
      for (int v = 0; v < NV; ++v) ut[v] = (1. - a) * ut[v] + FV[v * NP3];
    }
  }
  if (P.parabolic) {  // viscous / resistive volume integral of variables 2..8 (lifting kernel)
    const double* V = P.utvisc + (size_t)e * 7 * NP3 + t;
#pragma unroll
    for (int v = 0; v < 7; ++v) ut[1 + v] += V[v * NP3];
  }
  if (P.utsurf) {  // Gauss nodes: the surface integral of every node, formed by gauss::surf_mhd_kernel
    const double* S = P.utsurf + (size_t)e * NV * NP3 + t;
#pragma unroll
    for (int v = 0; v < NV; ++v) ut[v] += S[v * NP3];
  }
  // surface integral at the boundary nodes (LGL), with the own side's non-conservative part
  int sides[3];
  const int ns = P.utsurf ? 0 : boundary_sides(i, j, k, N, sides);
  const double lh = P.basis->LhatM0;
  for (int z = 0; z < ns; ++z) {
    const int s = sides[z];
    const int* es = P.e2s + 2 * (6 * (size_t)e + (s - 1));
    const int side = es[0], flip = es[1];
    const int pt = node_side_point(N, s, flip, i, j, k);
    const double* Fs = P.flux + (size_t)side * NF * NPT + pt;
    double F[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) F[v] = Fs[v * NPT];
    if (NC != 0) {
      const double nq[3] = {Fs[10 * NPT], Fs[11 * NPT], Fs[12 * NPT]};
      add_noncons_surface(NC, NCGLM, u, Fs[9 * NPT], nq, F);
    }
    const double sg = (flip == 0) ? lh : -lh;
#pragma unroll
    for (int v = 0; v < NV; ++v) ut[v] += sg * F[v];
  }
  const double sj = P.sJ[(size_t)e * NP3 + t];
#pragma unroll
  for (int v = 0; v < NV; ++v) ut[v] = ut[v] * (-sj);
  if (P.source) ut[8] = ut[8] - P.glmScr * ch * u[8];  // GLM damping
  const size_t o = NV * ((size_t)e * NP3 + t);
  if (P.stage == 0) {
#pragma unroll
    for (int v = 0; v < NV; ++v) P.Ut[o + v] = ut[v];
  } else {
    const double dt = stage_dt(P, e);
    const double bdt = P.rkB * dt;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double tmp = (P.stage == 1) ? ut[v] : ut[v] - P.UtTmp[o + v] * P.rkA;
      P.UtTmp[o + v] = tmp;
      P.U[o + v] = u[v] + tmp * bdt;
    }
  }
}

// ------------------------------------------------------------------------------------------------
// CALCTIMESTEP (mhd/calctimestep.f90:38-179): fast magnetosonic speed (FastestWave3D), the
// viscous / resistive limit max(eta/mu0, mu max(4/3,kappa/Pr)/rho) * sum |Ja sJ|^2, global min dt,
// error code of the first bad element.  Same outputs as the Navier-Stokes kernel.
// ------------------------------------------------------------------------------------------------
template <int NP, bool VISC>
__global__ void __launch_bounds__(512) timestep_kernel(KParams P, unsigned long long* dtBits, int* errKey) {
  if (halted(P)) return;
  constexpr int NP3 = NP * NP * NP;
  constexpr int EPB = (256 / NP3) > 0 ? (256 / NP3) : 1;
  constexpr int RSTART = (NP3 > 256) ? 256 : (NP3 > 128) ? 128 : (NP3 > 64) ? 64 : (NP3 > 32) ? 32 : (NP3 > 16) ? 16 : (NP3 > 8) ? 8 : 4;
  __shared__ double s_l[EPB][4][NP3];
  __shared__ int s_err[EPB];
  const int eb = threadIdx.x / NP3, n = threadIdx.x - eb * NP3;
  const int e = blockIdx.x * EPB + eb;
  const bool valid = e < P.nElems;
  if (n == 0) s_err[eb] = -1;
  __syncthreads();
  double lam[4] = {0., 0., 0., 0.};
  int code = 0;
  if (valid) {
    const double* U = P.U + NV * ((size_t)e * NP3 + n);
    double u[NV], q[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) u[v] = U[v];
    if (isnan(u[0])) code = 1;
    const double sRho = 1. / u[0];
    cons_to_prim(P, u, q);
    if (q[4] <= 0.) code = 2;
    const double cf = sqrt((P.kappa * q[4] + (q[5] * q[5] + q[6] * q[6] + q[7] * q[7]) * P.smu_0) / q[0]);
    const double* M = P.metrics + (size_t)e * 9 * NP3 + n;
    const double sj = P.sJ[(size_t)e * NP3 + n];
    double lv = 0.;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double m0 = M[(3 * d + 0) * NP3], m1 = M[(3 * d + 1) * NP3], m2 = M[(3 * d + 2) * NP3];
      lam[d] = sj * (fabs(m0 * q[1] + m1 * q[2] + m2 * q[3]) + cf * sqrt(m0 * m0 + m1 * m1 + m2 * m2));
      if (VISC) {
        const double a = m0 * sj, b = m1 * sj, c = m2 * sj;
        lv += a * a + b * b + c * c;
      }
    }
    if (VISC) lam[3] = fmax(P.etasmu_0, sRho * P.KappasPrMax) * lv;
  }
  if (code != 0) atomicMax(&s_err[eb], n * 8 + code);
#pragma unroll
  for (int d = 0; d < 4; ++d) s_l[eb][d][n] = lam[d];
  __syncthreads();
  for (int stride = RSTART; stride > 0; stride >>= 1) {
    if (n < stride && n + stride < NP3)
#pragma unroll
      for (int d = 0; d < 4; ++d) s_l[eb][d][n] = fmax(s_l[eb][d][n], s_l[eb][d][n + stride]);
    __syncthreads();
  }
  if (n != 0 || !valid) return;
#pragma unroll
  for (int d = 0; d < 4; ++d) lam[d] = s_l[eb][d][0];
  int err = (s_err[eb] >= 0) ? (s_err[eb] & 7) : 0;
  double dtE = P.CFLScale * 2. / (lam[0] + lam[1] + lam[2]);
  if (isnan(dtE)) err = 3;
  if (VISC && lam[3] > 0.) dtE = fmin(dtE, P.DFLScale * 4. / lam[3]);
  reduce_timestep(P, e, dtE, err, dtBits, errKey);
}

}  // namespace mhd
}  // namespace fluxo
