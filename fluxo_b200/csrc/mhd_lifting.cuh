// Lifting + viscous / resistive volume kernel of the MHD right-hand side (9 variables, LGL nodes).
// Same structure as the Navier-Stokes kernel (lifting.cuh): per element, one thread per node,
//   1. BR1/BR2 gradients of the lifting variable (strong-form volume derivative br1_volint.f90:45-98 /
//      br2_volint.f90:45-103, surface lifting br1_surfint.f90:52-131 / br2_surfint.f90:53-148,
//      Jacobian, ConvertToGradPrim mhd/equation_vars.f90:547-628);
//   2. each side's share n.F_v(U, gradP trace) of the viscous / resistive face flux (7 components,
//      side-major [side][master|slave][7][pt]) from the face trace of the gradient;
//   3. the viscous / resistive volume integral sum_l D_hat(i,l) (f~,g~,h~)(l) of variables 2..8
//      (volint.f90:228-271 with EvalDiffFluxTilde3D mhd/flux.f90:579-712), 7 values per node.
#pragma once
#include "common.cuh"
#include "kernels.cuh"
#include "lifting.cuh"
#include "mhd_kernels.cuh"
#include "physics_mhd.cuh"

namespace fluxo {
namespace mhd {

template <int NP>
__host__ __device__ constexpr size_t lv_smem_bytes() {
  return sizeof(double) * (size_t)(2 * NP * NP + epb<NP>() * 36 * lv_slots<NP>());
}

// resident blocks per SM the register allocation must allow: 2 for BR1 blocks of up to 320 threads
// (more resident warps than the ~150 registers it would take unconstrained), else 1
template <int NP, int LIFT>
__host__ __device__ constexpr int lv_minb() { return (LIFT == 1 && epb<NP>() * NP * NP * NP <= 320) ? 2 : 1; }

template <int NP, int LIFT>
__global__ void __launch_bounds__(epb<NP>() * NP * NP * NP, lv_minb<NP, LIFT>()) lift_visc_kernel(KParams P) {
  if (halted(P)) return;
  constexpr int NP3 = NP * NP * NP, NPT = NP * NP, N = NP - 1, EPB = epb<NP>(), NS = lv_slots<NP>();
  extern __shared__ double smem[];
  double* sD = smem;
  double* sDhat = sD + NPT;
  const int eb = threadIdx.x / NP3, t = threadIdx.x - eb * NP3;
  const int e = blockIdx.x * EPB + eb;
  const bool valid = e < P.nElems;
  double* sV = sDhat + NPT + (size_t)eb * 36 * NS;  // [9][NS] lifting variable; later [7][NS] sums
  double* sW = sV + 9 * NS;                          // [27][NS] derivatives; later [21][NS] fluxes
  for (int z = threadIdx.x; z < NPT; z += blockDim.x) {
    sD[z] = P.basis->D[z];
    sDhat[z] = P.basis->Dhat[z];
  }
  double u[NV];
  if (valid) {
    const double* Ug = P.U + NV * ((size_t)e * NP3 + t);
#pragma unroll
    for (int v = 0; v < NV; ++v) u[v] = Ug[v];
#pragma unroll
    for (int c = 0; c < 9; ++c) prefetch_l2(P.metrics + (size_t)e * 9 * NP3 + c * NP3 + t);
    prefetch_l2(P.sJ + (size_t)e * NP3 + t);
    double V[NV];
    lifting_var_rt(P, u, V);
#pragma unroll
    for (int v = 0; v < NV; ++v) sV[v * NS + lv_slot(t)] = V[v];
  }
  __syncthreads();
  if (valid) {  // line-blocked derivatives: tasks (dir, var, line)
    for (int task = t; task < 27 * NPT; task += NP3) {
      const int dir = task / (9 * NPT), rem = task - dir * 9 * NPT, v = rem / NPT, L = rem - v * NPT;
      const int a = L % NP, b = L / NP;
      double x[NP];
#pragma unroll
      for (int l = 0; l < NP; ++l) x[l] = sV[v * NS + lv_slot(line_node<NP>(dir, a, b, l))];
#pragma unroll
      for (int o = 0; o < NP; ++o) {
        double s = 0.;
#pragma unroll
        for (int l = 0; l < NP; ++l) s += sD[o * NP + l] * x[l];
        sW[(dir * 9 + v) * NS + lv_slot(line_node<NP>(dir, a, b, o))] = s;
      }
    }
  }
  __syncthreads();
  double ft[21];
  if (valid) {
    const double* M = P.metrics + (size_t)e * 9 * NP3 + t;
    double m[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) m[c] = M[c * NP3];
    const double sj = P.sJ[(size_t)e * NP3 + t];
    double g[3][NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double gx = sW[v * NS + lv_slot(t)], ge = sW[(9 + v) * NS + lv_slot(t)], gz = sW[(18 + v) * NS + lv_slot(t)];
#pragma unroll
      for (int d = 0; d < 3; ++d) g[d][v] = m[0 + d] * gx + m[3 + d] * ge + m[6 + d] * gz;
    }
    const int i = t % NP, j = (t / NP) % NP, k = t / NPT;
    int sides[3];
    const int ns = boundary_sides(i, j, k, N, sides);
    const double lh = P.basis->LhatM0;
    if constexpr (LIFT == 2) {
      // g is the volume part of the gradient.  First pass: each side's trace (volume part + etaBR2 *
      // own-side surface part) and its share n.F_v(U, trace) of the viscous / resistive face flux;
      // second pass: the plain surface terms into g (one gradient copy live beside the trace)
#pragma unroll
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int d = 0; d < 3; ++d) g[d][v] *= sj;
#pragma unroll 1
      for (int z = 0; z < ns; ++z) {
        const int s = sides[z];
        const int* es = P.e2s + 2 * (6 * (size_t)e + (s - 1));
        const int side = es[0], flip = es[1];
        const int pt = node_side_point(N, s, flip, i, j, k);
        const double* nvec = P.facegeo + (size_t)side * 10 * NPT + pt;
        const double* F = P.lflux + (size_t)side * NV * NPT + pt;
        const double n0 = nvec[0], n1 = nvec[NPT], n2 = nvec[2 * NPT];
        double tr[3][NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const double fl = sj * lh * F[v * NPT];
          tr[0][v] = g[0][v] + P.etaBR2 * (fl * n0);
          tr[1][v] = g[1][v] + P.etaBR2 * (fl * n1);
          tr[2][v] = g[2][v] + P.etaBR2 * (fl * n2);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) to_grad_prim_rt(P, u, tr[d]);
        double kf[7], kg[7], kh[7];
        visc_flux_3d(P, u, tr[0], tr[1], tr[2], kf, kg, kh);
        double* T = P.gtrace + ((size_t)side * 2 + (flip == 0 ? 0 : 1)) * 7 * NPT + pt;
#pragma unroll
        for (int v = 0; v < 7; ++v) T[(size_t)v * NPT] = n0 * kf[v] + n1 * kg[v] + n2 * kh[v];
      }
    }
    for (int z = 0; z < ns; ++z) {
      const int s = sides[z];
      const int* es = P.e2s + 2 * (6 * (size_t)e + (s - 1));
      const int side = es[0];
      const int pt = node_side_point(N, s, es[1], i, j, k);
      const double* nvec = P.facegeo + (size_t)side * 10 * NPT + pt;
      const double* F = P.lflux + (size_t)side * NV * NPT + pt;
      const double n0 = nvec[0], n1 = nvec[NPT], n2 = nvec[2 * NPT];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const double fl = LIFT == 2 ? sj * lh * F[v * NPT] : F[v * NPT] * lh;
        g[0][v] += fl * n0; g[1][v] += fl * n1; g[2][v] += fl * n2;
      }
    }
    if constexpr (LIFT == 1) {
#pragma unroll
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int d = 0; d < 3; ++d) g[d][v] *= sj;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) to_grad_prim_rt(P, u, g[d]);
    if (P.grad) {
      double* G = P.grad + 27 * ((size_t)e * NP3 + t);
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int v = 0; v < NV; ++v) G[9 * d + v] = g[d][v];
    }
    double f[7], gg[7], h[7];
    visc_flux_3d(P, u, g[0], g[1], g[2], f, gg, h);
    if constexpr (LIFT == 1) {
      // BR1: the face trace of the gradient is the volume gradient at the boundary node, so this
      // side's share of the viscous / resistive face flux is n.F_v of the node
      for (int z = 0; z < ns; ++z) {
        const int s = sides[z];
        const int* es = P.e2s + 2 * (6 * (size_t)e + (s - 1));
        const int side = es[0], flip = es[1];
        const int pt = node_side_point(N, s, flip, i, j, k);
        const double* nvec = P.facegeo + (size_t)side * 10 * NPT + pt;
        const double n0 = nvec[0], n1 = nvec[NPT], n2 = nvec[2 * NPT];
        double* T = P.gtrace + ((size_t)side * 2 + (flip == 0 ? 0 : 1)) * 7 * NPT + pt;
#pragma unroll
        for (int v = 0; v < 7; ++v) T[(size_t)v * NPT] = n0 * f[v] + n1 * gg[v] + n2 * h[v];
      }
    }
#pragma unroll
    for (int v = 0; v < 7; ++v) {
      ft[0 + v] = f[v] * m[0] + gg[v] * m[1] + h[v] * m[2];
      ft[7 + v] = f[v] * m[3] + gg[v] * m[4] + h[v] * m[5];
      ft[14 + v] = f[v] * m[6] + gg[v] * m[7] + h[v] * m[8];
    }
  }
  __syncthreads();
  if (valid) {
#pragma unroll
    for (int c = 0; c < 21; ++c) sW[c * NS + lv_slot(t)] = ft[c];
#pragma unroll
    for (int v = 0; v < 7; ++v) sV[v * NS + lv_slot(t)] = 0.;
  }
  __syncthreads();
#pragma unroll 1
  for (int dir = 0; dir < 3; ++dir) {
    if (valid) {
      for (int task = t; task < 7 * NPT; task += NP3) {
        const int v = task / NPT, L = task - v * NPT, a = L % NP, b = L / NP;
        double x[NP];
#pragma unroll
        for (int l = 0; l < NP; ++l) x[l] = sW[(dir * 7 + v) * NS + lv_slot(line_node<NP>(dir, a, b, l))];
#pragma unroll
        for (int o = 0; o < NP; ++o) {
          double s = 0.;
#pragma unroll
          for (int l = 0; l < NP; ++l) s += sDhat[o * NP + l] * x[l];
          sV[v * NS + lv_slot(line_node<NP>(dir, a, b, o))] += s;
        }
      }
    }
    __syncthreads();
  }
  if (valid) {
    double* O = P.utvisc + (size_t)e * 7 * NP3 + t;
#pragma unroll
    for (int v = 0; v < 7; ++v) O[v * NP3] = sV[v * NS + lv_slot(t)];
  }
}

}  // namespace mhd
}  // namespace fluxo
