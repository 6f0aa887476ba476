// Lifting + viscous volume kernel of the Navier-Stokes right-hand side (LGL nodes).
//
// Per element (one thread per volume node) it computes
//   1. the BR1/BR2 gradients of the lifting variable: strong-form volume derivative
//      (br1_volint.f90:45-98, br2_volint.f90:45-103), surface integral of the lifting flux
//      (br1_surfint.f90:52-131, br2_surfint.f90:53-148), Jacobian, conversion to gradients of the
//      primitive variables (equation_vars.f90:571-647);
//   2. each side's share n.F_v(U, gradP trace) of the viscous face flux 1/2 n.(F_v(L) + F_v(R))
//      (riemann.f90:155-168), from the face trace of the gradient (BR1: the volume gradient at the
//      boundary node, ProlongToFace; BR2: volume part + etaBR2 * own-side surface part): 4 values
//      per side and face point instead of the 15 gradient components, written side-major so the
//      face kernel reads them coalesced;
//   3. the viscous volume integral sum_l D_hat(i,l) (f~,g~,h~)(l) of the contravariant viscous
//      fluxes (volint.f90:228-271 with EvalDiffFluxTilde3D flux.f90:523-635), written as 4 values per
//      node for the volume kernel.
// Both operator applications are node-centric: every thread forms the derivatives (and later the
// divergence) of its own node from the N+1 nodes of its three lines, so the gradient flows straight
// from the derivative sums into the flux evaluation and the divergence straight into the global
// store, with two block barriers in all and the same work on every thread.  Reads of a line are
// broadcasts or consecutive doubles within a warp (no bank conflicts, no padding), and every
// shared-memory address is a per-thread base plus a compile-time offset.
#pragma once
#include "common.cuh"
#include "physics_ns.cuh"

namespace fluxo {

template <int NP>
__host__ __device__ constexpr int lv_epb() { return (256 / (NP * NP * NP)) > 0 ? (256 / (NP * NP * NP)) : 1; }
// padded node slots of the MHD lifting kernel's line-blocked arrays
template <int NP>
__host__ __device__ constexpr int lv_slots() { return (NP * NP * NP - 1) + ((NP * NP * NP - 1) >> 4) + 1; }
// per element: the 5 lifting variables, then the 12 contravariant viscous fluxes (4 per direction)
// row stride of the operator copies in shared memory: odd, so that the rows D(i,.) that the 8 lanes
// of a line read at once fall into different banks
template <int NP>
__host__ __device__ constexpr int lv_row() { return NP | 1; }
template <int NP>
__host__ __device__ constexpr size_t lv_smem_bytes() {
  return sizeof(double) * (size_t)(2 * NP * lv_row<NP>() + lv_epb<NP>() * 17 * NP * NP * NP);
}

__device__ __forceinline__ int lv_slot(int n) { return n + (n >> 4); }

// node index of position x on line (a,b) of direction dir
template <int NP>
__device__ __forceinline__ int line_node(int dir, int a, int b, int x) {
  return dir == 0 ? x + NP * (a + NP * b) : (dir == 1 ? a + NP * (x + NP * b) : a + NP * (b + NP * x));
}

template <int LV>
__device__ __forceinline__ void lifting_var_t(const KParams& P, const double* U, double* V) {
  if constexpr (LV == 1) {
    for (int v = 0; v < 5; ++v) V[v] = U[v];
  } else if constexpr (LV == 2) {
    const double s = 1. / U[0];
    V[0] = U[0]; V[1] = U[1] * s; V[2] = U[2] * s; V[3] = U[3] * s;
    V[4] = P.kappaM1 * (U[4] - 0.5 * (U[1] * V[1] + U[2] * V[2] + U[3] * V[3]));
  } else {  // ConsToEntropyVec (equation_vars.f90:397-429)
    const double srho = 1. / U[0];
    const double u = U[1] * srho, v = U[2] * srho, w = U[3] * srho;
    const double v2s2 = 0.5 * (u * u + v * v + w * w);
    const double rho_sp = U[0] / (P.kappaM1 * (U[4] - U[0] * v2s2));
    const double s = -(log(rho_sp) + P.kappaM1 * log(U[0]));  // -log(rho_sp * rho^(kappa-1))
    V[0] = (P.kappa - s) * P.sKappaM1 - rho_sp * v2s2;
    V[1] = rho_sp * u; V[2] = rho_sp * v; V[3] = rho_sp * w;
    V[4] = -rho_sp;
  }
}

// resident blocks per SM the register allocation must allow: 2, except BR2 for N+1 >= 7, whose
// per-side traces need more than the 64 registers of two 512-thread blocks
template <int NP, int LIFT>
__host__ __device__ constexpr int lv_minb() { return (LIFT == 2 && NP >= 7) ? 1 : 2; }

// Node phase of the lifting kernel: from the derivatives (dx, de, dz along xi, eta, zeta) of the lifting
// variable at node t of element e to the primitive gradient (metric terms, surface lift, Jacobian,
// conversion), the face traces n.F_v of the node's sides (gtrace) and the contravariant viscous fluxes
// of the node, stored as sF[q * fstride + slot], q = 4*dir + v.  e2s is the element's ElemToSide
// (side, flip per local side) in shared memory.
template <int NP, int LIFT, int LV>
__device__ __forceinline__ void lv_node_fluxes(const KParams& P, int e, int t, int i, int j, int k, const double* u,
                                               const double* dx, const double* de, const double* dz, const int* e2s,
                                               double* sF, int fstride, int slot) {
  constexpr int NP3 = NP * NP * NP, NPT = NP * NP, N = NP - 1;
  const double* M = P.metrics + (size_t)e * 9 * NP3 + t;
  const double sj = P.sJ[(size_t)e * NP3 + t];
  double g[3][5];
  {
    double m[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) m[c] = M[c * NP3];
#pragma unroll
    for (int v = 0; v < 5; ++v)
#pragma unroll
      for (int d = 0; d < 3; ++d) g[d][v] = m[0 + d] * dx[v] + m[3 + d] * de[v] + m[6 + d] * dz[v];
  }
  int sides[3];
  const int ns = boundary_sides(i, j, k, N, sides);
  const double lh = P.basis->LhatM0;
  if constexpr (LIFT == 2) {
    // g is the volume part of the gradient, the base of every face trace.  First pass: each side's
    // trace (volume part + etaBR2 * own-side surface part) and its share n.F_v(U, trace) of the
    // viscous face flux (riemann.f90:155-168); second pass: the plain surface terms into g.  Two
    // passes (the face data read twice) keep only one gradient copy live beside the trace.
#pragma unroll
    for (int v = 0; v < 5; ++v)
#pragma unroll
      for (int d = 0; d < 3; ++d) g[d][v] *= sj;
#pragma unroll 1
    for (int z = 0; z < ns; ++z) {
      const int s = sides[z], side = e2s[2 * (s - 1)], flip = e2s[2 * (s - 1) + 1];
      const int pt = node_side_point(N, s, flip, i, j, k);
      const double* nvec = P.facegeo + (size_t)side * 10 * NPT + pt;
      const double* F = P.lflux + (size_t)side * 5 * NPT + pt;
      const double n0 = nvec[0], n1 = nvec[NPT], n2 = nvec[2 * NPT];
      double tr[3][5];
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        const double fl = sj * lh * F[v * NPT];
        tr[0][v] = g[0][v] + P.etaBR2 * (fl * n0);
        tr[1][v] = g[1][v] + P.etaBR2 * (fl * n1);
        tr[2][v] = g[2][v] + P.etaBR2 * (fl * n2);
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) to_grad_prim(P, u, tr[d]);
      double kf[4], kg[4], kh[4];
      diff_flux_3d(P, u, tr[0], tr[1], tr[2], kf, kg, kh);
      double* T = P.gtrace + ((size_t)side * 2 + (flip == 0 ? 0 : 1)) * 4 * NPT + pt;
#pragma unroll
      for (int v = 0; v < 4; ++v) T[(size_t)v * NPT] = n0 * kf[v] + n1 * kg[v] + n2 * kh[v];
    }
  }
  for (int z = 0; z < ns; ++z) {
    const int s = sides[z], side = e2s[2 * (s - 1)], flip = e2s[2 * (s - 1) + 1];
    const int pt = node_side_point(N, s, flip, i, j, k);
    const double* nvec = P.facegeo + (size_t)side * 10 * NPT + pt;
    const double* F = P.lflux + (size_t)side * 5 * NPT + pt;
    const double n0 = nvec[0], n1 = nvec[NPT], n2 = nvec[2 * NPT];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      if constexpr (LIFT == 2) {  // volume gradient gets the plain surface term
        const double fl = sj * lh * F[v * NPT];
        g[0][v] += fl * n0; g[1][v] += fl * n1; g[2][v] += fl * n2;
      } else {
        const double fl = F[v * NPT] * lh;
        g[0][v] += fl * n0; g[1][v] += fl * n1; g[2][v] += fl * n2;
      }
    }
  }
  if constexpr (LIFT == 1) {
#pragma unroll
    for (int v = 0; v < 5; ++v)
#pragma unroll
      for (int d = 0; d < 3; ++d) g[d][v] *= sj;
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) to_grad_prim(P, u, g[d]);
  if (P.grad) {  // volume gradients kept for analysis (DGTimeDerivative calls only)
    double* G = P.grad + 15 * ((size_t)e * NP3 + t);
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int v = 0; v < 5; ++v) G[5 * d + v] = g[d][v];
  }
  double f[4], gg[4], h[4];
  diff_flux_3d(P, u, g[0], g[1], g[2], f, gg, h);
  if constexpr (LIFT == 1) {
    // BR1: the face trace of the gradient is the volume gradient at the boundary node, so this
    // side's share of the viscous face flux is n.F_v of the node (riemann.f90:155-168)
    for (int z = 0; z < ns; ++z) {
      const int s = sides[z], side = e2s[2 * (s - 1)], flip = e2s[2 * (s - 1) + 1];
      const int pt = node_side_point(N, s, flip, i, j, k);
      const double* nvec = P.facegeo + (size_t)side * 10 * NPT + pt;
      const double n0 = nvec[0], n1 = nvec[NPT], n2 = nvec[2 * NPT];
      double* T = P.gtrace + ((size_t)side * 2 + (flip == 0 ? 0 : 1)) * 4 * NPT + pt;
#pragma unroll
      for (int v = 0; v < 4; ++v) T[(size_t)v * NPT] = n0 * f[v] + n1 * gg[v] + n2 * h[v];
    }
  }
  // contravariant fluxes (metrics re-read rather than held across the gradient work)
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    const double m0 = M[(3 * dir + 0) * NP3], m1 = M[(3 * dir + 1) * NP3], m2 = M[(3 * dir + 2) * NP3];
#pragma unroll
    for (int v = 0; v < 4; ++v) sF[(4 * dir + v) * fstride + slot] = f[v] * m0 + gg[v] * m1 + h[v] * m2;
  }
}

template <int NP, int LIFT, int LV>
__global__ void __launch_bounds__(lv_epb<NP>() * NP * NP * NP, lv_minb<NP, LIFT>()) lift_visc_kernel(KParams P) {
  if (halted(P)) return;
  constexpr int NP3 = NP * NP * NP, NPT = NP * NP, N = NP - 1, EPB = lv_epb<NP>(), R = lv_row<NP>();
  extern __shared__ double smem[];
  double* sD = smem;             // D(i,l) at [i*R+l]
  double* sDhat = sD + NP * R;   // D_hat(i,l)
  const int eb = threadIdx.x / NP3, t = threadIdx.x - eb * NP3;
  const int e = blockIdx.x * EPB + eb;
  const bool valid = e < P.nElems;
  double* sV = sDhat + NP * R + (size_t)eb * 17 * NP3;  // [5][node] lifting variable
  double* sF = sV + 5 * NP3;                         // [12][node] contravariant fluxes, 4 per direction
  __shared__ int sE2S[EPB][12];  // the element's ElemToSide (side, flip per local side)
  for (int z = threadIdx.x; z < NPT; z += blockDim.x) {
    const int r = z / NP, c = z - r * NP;
    sD[r * R + c] = P.basis->D[z];
    sDhat[r * R + c] = P.basis->Dhat[z];
  }
  const int i = t % NP, j = (t / NP) % NP, k = t / NPT;
  // first node of the own xi / eta / zeta line; the line's nodes follow at strides 1, NP, NP^2
  const int bx = t - i, be = t - NP * j, bz = t - NPT * k;
  if (P.pfTiles > 0 && threadIdx.x == 0) {  // the tile one wave ahead: its inputs into L2
    const size_t en = ((size_t)blockIdx.x + P.pfTiles) * EPB;
    if (en < (size_t)P.nElems) {
      const size_t ne = ((size_t)P.nElems - en < (size_t)EPB ? (size_t)P.nElems - en : (size_t)EPB) * NP3;
      prefetch_l2_bulk(P.U + 5 * en * NP3, 5 * ne * sizeof(double));
      prefetch_l2_bulk(P.metrics + 9 * en * NP3, 9 * ne * sizeof(double));
      prefetch_l2_bulk(P.sJ + en * NP3, ne * sizeof(double));
    }
  }
  double u[5];
  if (valid) {
    for (int z = t; z < 12; z += NP3) sE2S[eb][z] = P.e2s[12 * (size_t)e + z];  // NP3 = 8 for N = 1
    const double* Ug = P.U + 5 * ((size_t)e * NP3 + t);
#pragma unroll
    for (int v = 0; v < 5; ++v) u[v] = Ug[v];
#pragma unroll
    for (int c = 0; c < 9; ++c) prefetch_l2(P.metrics + (size_t)e * 9 * NP3 + c * NP3 + t);
    prefetch_l2(P.sJ + (size_t)e * NP3 + t);
    double V[5];
    lifting_var_t<LV>(P, u, V);
#pragma unroll
    for (int v = 0; v < 5; ++v) sV[v * NP3 + t] = V[v];
  }
  __syncthreads();
  if (valid) {
    // derivatives of the lifting variable along xi, eta, zeta at the own node, l = 0..N
    double dx[5], de[5], dz[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) { dx[v] = 0.; de[v] = 0.; dz[v] = 0.; }
    const double* Di = sD + i * R;
    const double* Dj = sD + j * R;
    const double* Dk = sD + k * R;
#pragma unroll
    for (int l = 0; l < NP; ++l) {
      const double a = Di[l], b = Dj[l], c = Dk[l];
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        dx[v] += a * sV[v * NP3 + bx + l];
        de[v] += b * sV[v * NP3 + be + NP * l];
        dz[v] += c * sV[v * NP3 + bz + NPT * l];
      }
    }
    lv_node_fluxes<NP, LIFT, LV>(P, e, t, i, j, k, u, dx, de, dz, sE2S[eb], sF, NP3, t);
  }
  __syncthreads();
  // viscous volume integral at the own node: sum_l D_hat(i,l) f~(l,j,k) + D_hat(j,l) g~(i,l,k) +
  // D_hat(k,l) h~(i,j,l), l = 0..N
  if (valid) {
    double r[4] = {0., 0., 0., 0.};
    const double* Hi = sDhat + i * R;
    const double* Hj = sDhat + j * R;
    const double* Hk = sDhat + k * R;
#pragma unroll
    for (int l = 0; l < NP; ++l) {
      const double a = Hi[l], b = Hj[l], c = Hk[l];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        r[v] += a * sF[v * NP3 + bx + l];
        r[v] += b * sF[(4 + v) * NP3 + be + NP * l];
        r[v] += c * sF[(8 + v) * NP3 + bz + NPT * l];
      }
    }
    double* O = P.utvisc + (size_t)e * 4 * NP3 + t;
#pragma unroll
    for (int v = 0; v < 4; ++v) O[v * NP3] = r[v];
  }
}

}  // namespace fluxo
