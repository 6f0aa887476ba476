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
// The derivative sums are line-blocked: one thread loads a whole line of one variable into registers
// and produces all N+1 outputs, so a shared-memory load serves N+1 multiply-adds.
#pragma once
#include "common.cuh"
#include "physics_ns.cuh"

namespace fluxo {

template <int NP>
__host__ __device__ constexpr int lv_epb() { return (256 / (NP * NP * NP)) > 0 ? (256 / (NP * NP * NP)) : 1; }
template <int NP>
__host__ __device__ constexpr int lv_slots() { return (NP * NP * NP - 1) + ((NP * NP * NP - 1) >> 4) + 1; }
// per element: 5 lifting variables + 15 derivatives, later 12 contravariant fluxes + 12 directional
// divergences
template <int NP>
__host__ __device__ constexpr size_t lv_smem_bytes() {
  return sizeof(double) * (size_t)(2 * NP * NP + lv_epb<NP>() * 24 * lv_slots<NP>());
}

__device__ __forceinline__ int lv_slot(int n) { return n + (n >> 4); }

// node index of position x on line (a,b) of direction dir
template <int NP>
__device__ __forceinline__ int line_node(int dir, int a, int b, int x) {
  return dir == 0 ? x + NP * (a + NP * b) : (dir == 1 ? a + NP * (x + NP * b) : a + NP * (b + NP * x));
}

// sum_l row[l] x[l] for a row of an (N+1)^2 operator in shared memory, in the order l = 0..N.  For
// even N+1 the row is read with 16-byte loads (half the load instructions; every lane reads the same
// address, a broadcast).  FRESH: the row is re-read on every call, so the compiler cannot hoist the
// whole operator out of a loop into registers (which spills).
template <int NP, bool FRESH>
__device__ __forceinline__ double row_dot(const double* row, const double* x) {
  double s = 0.;
  if constexpr (NP % 2 == 0) {
#pragma unroll
    for (int l = 0; l < NP; l += 2) {
      double a, b;
      if constexpr (FRESH) {
        const unsigned addr = static_cast<unsigned>(__cvta_generic_to_shared(row + l));
        asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(a), "=d"(b) : "r"(addr));
      } else {
        const double2 r2 = *reinterpret_cast<const double2*>(row + l);
        a = r2.x; b = r2.y;
      }
      s += a * x[l];
      s += b * x[l + 1];
    }
  } else {
    const volatile double* vrow = row;
#pragma unroll
    for (int l = 0; l < NP; ++l) s += (FRESH ? vrow[l] : row[l]) * x[l];
  }
  return s;
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

template <int NP, int LIFT, int LV>
#ifndef FLUXO_LV_MINB
#define FLUXO_LV_MINB 2  // resident blocks per SM the register allocation must allow
#endif
__global__ void __launch_bounds__(lv_epb<NP>() * NP * NP * NP, FLUXO_LV_MINB)
lift_visc_kernel(KParams P) {
  if (halted(P)) return;
  constexpr int NP3 = NP * NP * NP, NPT = NP * NP, N = NP - 1, EPB = lv_epb<NP>(), NS = lv_slots<NP>();
  extern __shared__ double smem[];
  double* sD = smem;           // D(i,l) at [i*NP+l]
  double* sDhat = sD + NPT;    // D_hat(i,l)
  const int eb = threadIdx.x / NP3, t = threadIdx.x - eb * NP3;
  const int e = blockIdx.x * EPB + eb;
  const bool valid = e < P.nElems;
  // per element 24 arrays of NS: [0,5) lifting variable, [5,20) xi/eta/zeta derivatives; later
  // [5,17) contravariant fluxes and the 12 directional divergences in [0,5) and [17,24)
  double* sV = sDhat + NPT + (size_t)eb * 24 * NS;
  double* sW = sV + 5 * NS;
  __shared__ int sE2S[EPB][12];  // the element's ElemToSide (side, flip per local side)
  for (int z = threadIdx.x; z < NPT; z += blockDim.x) {
    sD[z] = P.basis->D[z];
    sDhat[z] = P.basis->Dhat[z];
  }
  double u[5];
  if (valid) {
    for (int z = t; z < 12; z += NP3) sE2S[eb][z] = P.e2s[12 * (size_t)e + z];  // NP3 = 8 for N = 1
    const double* Ug = P.U + 5 * ((size_t)e * NP3 + t);
#pragma unroll
    for (int v = 0; v < 5; ++v) u[v] = Ug[v];
    // metrics and Jacobian are read after the derivative phase: start them towards L2 now
#pragma unroll
    for (int c = 0; c < 9; ++c) prefetch_l2(P.metrics + (size_t)e * 9 * NP3 + c * NP3 + t);
    prefetch_l2(P.sJ + (size_t)e * NP3 + t);
    double V[5];
    lifting_var_t<LV>(P, u, V);
#pragma unroll
    for (int v = 0; v < 5; ++v) sV[v * NS + lv_slot(t)] = V[v];
  }
  __syncthreads();
  // derivatives of the lifting variable along xi, eta, zeta: tasks (dir, var, line)
  if (valid) {
    for (int task = t; task < 15 * NPT; task += NP3) {
      const int dir = task / (5 * NPT), rem = task - dir * 5 * NPT, v = rem / NPT, L = rem - v * NPT;
      const int a = L % NP, b = L / NP;
      double x[NP];
#pragma unroll
      for (int l = 0; l < NP; ++l) x[l] = sV[v * NS + lv_slot(line_node<NP>(dir, a, b, l))];
#pragma unroll
      for (int o = 0; o < NP; ++o) sW[(dir * 5 + v) * NS + lv_slot(line_node<NP>(dir, a, b, o))] = row_dot<NP, true>(sD + o * NP, x);
    }
  }
  __syncthreads();
  // Each thread reads only its own node's derivatives and overwrites the same node's slots with its
  // contravariant fluxes, so no barrier separates the two.  The metrics are read twice (gradient
  // transform, flux transform) rather than held across the gradient work: fewer live registers.
  if (valid) {
    const double* M = P.metrics + (size_t)e * 9 * NP3 + t;
    const double sj = P.sJ[(size_t)e * NP3 + t];
    double g[3][5];
    {
      double m[9];
#pragma unroll
      for (int c = 0; c < 9; ++c) m[c] = M[c * NP3];
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        const double gx = sW[(0 + v) * NS + lv_slot(t)], ge = sW[(5 + v) * NS + lv_slot(t)],
                     gz = sW[(10 + v) * NS + lv_slot(t)];
#pragma unroll
        for (int d = 0; d < 3; ++d) g[d][v] = m[0 + d] * gx + m[3 + d] * ge + m[6 + d] * gz;
      }
    }
    double gv[3][5];  // BR2: volume part of the gradient, the base of every face trace
    if constexpr (LIFT == 2) {
#pragma unroll
      for (int v = 0; v < 5; ++v)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          g[d][v] *= sj;
          gv[d][v] = g[d][v];
        }
    }
    const int i = t % NP, j = (t / NP) % NP, k = t / NPT;
    int sides[3];
    const int ns = boundary_sides(i, j, k, N, sides);
    const double lh = P.basis->LhatM0;
    for (int z = 0; z < ns; ++z) {
      const int s = sides[z], side = sE2S[eb][2 * (s - 1)], flip = sE2S[eb][2 * (s - 1) + 1];
      const int pt = node_side_point(N, s, flip, i, j, k);
      const double* nvec = P.facegeo + (size_t)side * 10 * NPT + pt;
      const double* F = P.lflux + (size_t)side * 5 * NPT + pt;
      const double n0 = nvec[0], n1 = nvec[NPT], n2 = nvec[2 * NPT];
      if constexpr (LIFT == 2) {
        double tr[3][5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const double fl = sj * lh * F[v * NPT];
          const double sx = fl * n0, sy = fl * n1, sz = fl * n2;
          tr[0][v] = gv[0][v] + P.etaBR2 * sx;
          tr[1][v] = gv[1][v] + P.etaBR2 * sy;
          tr[2][v] = gv[2][v] + P.etaBR2 * sz;
          g[0][v] += sx; g[1][v] += sy; g[2][v] += sz;  // volume gradient gets the plain surface term
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) to_grad_prim(P, u, tr[d]);
        // this side's share of the viscous face flux: n.F_v(U, trace) (riemann.f90:155-168)
        double kf[4], kg[4], kh[4];
        diff_flux_3d(P, u, tr[0], tr[1], tr[2], kf, kg, kh);
        double* T = P.gtrace + ((size_t)side * 2 + (flip == 0 ? 0 : 1)) * 4 * NPT + pt;
#pragma unroll
        for (int v = 0; v < 4; ++v) T[(size_t)v * NPT] = n0 * kf[v] + n1 * kg[v] + n2 * kh[v];
      } else {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
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
        const int s = sides[z], side = sE2S[eb][2 * (s - 1)], flip = sE2S[eb][2 * (s - 1) + 1];
        const int pt = node_side_point(N, s, flip, i, j, k);
        const double* nvec = P.facegeo + (size_t)side * 10 * NPT + pt;
        const double n0 = nvec[0], n1 = nvec[NPT], n2 = nvec[2 * NPT];
        double* T = P.gtrace + ((size_t)side * 2 + (flip == 0 ? 0 : 1)) * 4 * NPT + pt;
#pragma unroll
        for (int v = 0; v < 4; ++v) T[(size_t)v * NPT] = n0 * f[v] + n1 * gg[v] + n2 * h[v];
      }
    }
    const int st = lv_slot(t);
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
      const double m0 = M[(3 * dir + 0) * NP3], m1 = M[(3 * dir + 1) * NP3], m2 = M[(3 * dir + 2) * NP3];
#pragma unroll
      for (int v = 0; v < 4; ++v) sW[(4 * dir + v) * NS + st] = f[v] * m0 + gg[v] * m1 + h[v] * m2;
    }
  }
  __syncthreads();
  // viscous volume integral: sum_l D_hat(o,l) f~(l) along each direction, tasks (dir, var, line) of
  // all three directions at once, each (dir, var) into its own array (array dv -> sV index
  // dv < 5 ? dv : dv + 12, around the fluxes in [5,17))
  if (valid) {
    for (int task = t; task < 12 * NPT; task += NP3) {
      const int dv = task / NPT, L = task - dv * NPT, a = L % NP, b = L / NP, dir = dv >> 2;
      double x[NP];
#pragma unroll
      for (int l = 0; l < NP; ++l) x[l] = sW[dv * NS + lv_slot(line_node<NP>(dir, a, b, l))];
      double* out = sV + (dv < 5 ? dv : dv + 12) * NS;
      // D_hat re-read per row: hoisting its NP^2 entries out of the task loop spills
#pragma unroll
      for (int o = 0; o < NP; ++o) out[lv_slot(line_node<NP>(dir, a, b, o))] = row_dot<NP, true>(sDhat + o * NP, x);
    }
  }
  __syncthreads();
  if (valid) {
    double* O = P.utvisc + (size_t)e * 4 * NP3 + t;
    const int st = lv_slot(t);
    // divergence arrays of (dir, v): dv = 4 dir + v at sV index dv < 5 ? dv : dv + 12
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int d1 = 4 + v, d2 = 8 + v;
      O[v * NP3] = (sV[v * NS + st] + sV[(d1 < 5 ? d1 : d1 + 12) * NS + st]) + sV[(d2 + 12) * NS + st];
    }
  }
}

}  // namespace fluxo
