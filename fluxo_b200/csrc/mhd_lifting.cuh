// Lifting + viscous / resistive volume kernel of the MHD right-hand side (9 variables, LGL nodes).
// Same node-centric structure as the Navier-Stokes kernel (lifting.cuh): per element, one thread per
// node, two block barriers,
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

// operators at an odd row stride, then per element the 9 lifting variables and the 21 contravariant
// viscous / resistive fluxes (7 per direction), node-major
template <int NP>
__host__ __device__ constexpr size_t lv_smem_bytes() {
  return sizeof(double) * (size_t)(2 * NP * lv_row<NP>() + epb<NP>() * 30 * NP * NP * NP);
}

// resident blocks per SM the register allocation must allow: 2 for BR1 blocks of up to 320 threads
// (more resident warps than the ~150 registers it would take unconstrained), else 1
template <int NP, int LIFT>
__host__ __device__ constexpr int lv_minb() { return (LIFT == 1 && epb<NP>() * NP * NP * NP <= 320) ? 2 : 1; }

template <int NP, int LIFT>
__global__ void __launch_bounds__(epb<NP>() * NP * NP * NP, lv_minb<NP, LIFT>()) lift_visc_kernel(KParams P) {
  if (halted(P)) return;
  constexpr int NP3 = NP * NP * NP, NPT = NP * NP, N = NP - 1, EPB = epb<NP>(), R = lv_row<NP>();
  extern __shared__ double smem[];
  double* sD = smem;             // D(i,l) at [i*R+l]
  double* sDhat = sD + NP * R;   // D_hat(i,l)
  const int eb = threadIdx.x / NP3, t = threadIdx.x - eb * NP3;
  const int e = blockIdx.x * EPB + eb;
  const bool valid = e < P.nElems;
  double* sV = sDhat + NP * R + (size_t)eb * 30 * NP3;  // [9][node] lifting variable
  double* sF = sV + 9 * NP3;                            // [21][node] contravariant fluxes, 7 per direction
  for (int z = threadIdx.x; z < NPT; z += blockDim.x) {
    const int r = z / NP, c = z - r * NP;
    sD[r * R + c] = P.basis->D[z];
    sDhat[r * R + c] = P.basis->Dhat[z];
  }
  const int i = t % NP, j = (t / NP) % NP, k = t / NPT;
  // first node of the own xi / eta / zeta line; the line's nodes follow at strides 1, NP, NP^2
  const int bx = t - i, be = t - NP * j, bz = t - NPT * k;
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
    for (int v = 0; v < NV; ++v) sV[v * NP3 + t] = V[v];
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
    {
      // derivatives of the lifting variable along xi, eta, zeta at the own node, l = 0..N
      double dx[NV], de[NV], dz[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) { dx[v] = 0.; de[v] = 0.; dz[v] = 0.; }
      const double* Di = sD + i * R;
      const double* Dj = sD + j * R;
      const double* Dk = sD + k * R;
#pragma unroll
      for (int l = 0; l < NP; ++l) {
        const double a = Di[l], b = Dj[l], c = Dk[l];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          dx[v] += a * sV[v * NP3 + bx + l];
          de[v] += b * sV[v * NP3 + be + NP * l];
          dz[v] += c * sV[v * NP3 + bz + NPT * l];
        }
      }
#pragma unroll
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int d = 0; d < 3; ++d) g[d][v] = m[0 + d] * dx[v] + m[3 + d] * de[v] + m[6 + d] * dz[v];
    }
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
    // contravariant fluxes of the own node
#pragma unroll
    for (int c = 0; c < 21; ++c) sF[c * NP3 + t] = ft[c];
  }
  __syncthreads();
  // viscous / resistive volume integral at the own node: sum_l D_hat(i,l) f~(l,j,k) + D_hat(j,l) g~(i,l,k)
  // + D_hat(k,l) h~(i,j,l), l = 0..N
  if (valid) {
    double r[7] = {0., 0., 0., 0., 0., 0., 0.};
    const double* Hi = sDhat + i * R;
    const double* Hj = sDhat + j * R;
    const double* Hk = sDhat + k * R;
#pragma unroll
    for (int l = 0; l < NP; ++l) {
      const double a = Hi[l], b = Hj[l], c = Hk[l];
#pragma unroll
      for (int v = 0; v < 7; ++v) {
        r[v] += a * sF[v * NP3 + bx + l];
        r[v] += b * sF[(7 + v) * NP3 + be + NP * l];
        r[v] += c * sF[(14 + v) * NP3 + bz + NPT * l];
      }
    }
    double* O = P.utvisc + (size_t)e * 7 * NP3 + t;
#pragma unroll
    for (int v = 0; v < 7; ++v) O[v * NP3] = r[v];
  }
}

}  // namespace mhd
}  // namespace fluxo
