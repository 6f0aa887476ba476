// Gauss-node (PP_NodeType = 1) kernels of the Euler / Navier-Stokes right-hand side on sm_100a.
//
// With Gauss nodes no volume node lies on the element faces, so the face states are interpolated along
// the lines normal to each side, every node of a line takes a share of the surface terms, and the
// split form needs a correction at the faces (the entropy-stable Gauss collocation of dg.f90:458-511,
// prolongtoface.f90:103-132, surfint.f90:118-175, br1.f90:318-350, br2_surfint.f90:109-148):
//   prolong_kernel   per element: the 6 x (N+1)^2 face states U_master / U_slave, interpolated with
//                    L_Minus along the lines, from the entropy variables when the volume flux is entropy
//                    conservative (useEntropyProlongToFace) and converted back; written as
//                    [side][master|slave][pt][5] for the face kernels;
//   lift_visc_kernel per element (Navier-Stokes): BR1/BR2 gradients of the lifting variable with the
//                    surface terms at every node of each line (L_HatMinus(l)), the face traces of the
//                    gradient interpolated to the 6 sides, converted with the face states and turned
//                    into each side's share n.F_v of the viscous face flux, and the viscous volume
//                    integral (as the LGL lifting kernel);
//   surf_kernel      per element: the surface integral sum over the 6 sides of
//                    (F* -+ (FluxB_sum - FluxB(l)) NormalSign) L_HatMinus(l), where FluxB(l) is the
//                    two-point volume flux between node l and the side's state (node metric and
//                    SurfMetrics averaged) and FluxB_sum = sum_l FluxB(l) L_Minus(l); written as
//                    [elem][5][node] for the volume kernel.
// All three keep one element in shared memory with one thread per node; line sums run in the order of
// the reference's loops (l = 0..N from the side).
#pragma once
#include "common.cuh"
#include "kernels.cuh"
#include "lifting.cuh"
#include "physics_mhd.cuh"
#include "physics_ns.cuh"
#include "volume_pairs.cuh"

namespace fluxo {
namespace gauss {

// Volume node at distance l from local side s on the line through face point (a,b) of that side, (a,b)
// being the side's two tangential volume indices in increasing order (xi sides: (j,k), eta: (i,k),
// zeta: (i,j)).  l = 0 is the node next to the side.
__device__ __forceinline__ int line_node_of(int NP, int s, int a, int b, int l) {
  const int N = NP - 1;
  int i, j, k;
  switch (s) {
    case XI_MINUS: i = l; j = a; k = b; break;
    case XI_PLUS: i = N - l; j = a; k = b; break;
    case ETA_MINUS: i = a; j = l; k = b; break;
    case ETA_PLUS: i = a; j = N - l; k = b; break;
    case ZETA_MINUS: i = a; j = b; k = l; break;
    default: i = a; j = b; k = N - l; break;
  }
  return i + NP * (j + NP * k);
}

// distance of node (i,j,k) from local side s, and the side's tangential indices (a,b) of its line
__device__ __forceinline__ void line_of_node(int N, int s, int i, int j, int k, int& l, int& a, int& b) {
  switch (s) {
    case XI_MINUS: l = i; a = j; b = k; break;
    case XI_PLUS: l = N - i; a = j; b = k; break;
    case ETA_MINUS: l = j; a = i; b = k; break;
    case ETA_PLUS: l = N - j; a = i; b = k; break;
    case ZETA_MINUS: l = k; a = i; b = j; break;
    default: l = N - k; a = i; b = j; break;
  }
}

// face point (master frame) of the line (a,b) of local side s stored with flip `flip`
__device__ __forceinline__ int face_point_of(int NP, int s, int flip, int a, int b) {
  const int n0 = line_node_of(NP, s, a, b, 0);
  const int i = n0 % NP, j = (n0 / NP) % NP, k = n0 / (NP * NP);
  return node_side_point(NP - 1, s, flip, i, j, k);
}

// EntropyToCons (navierstokes/equation_vars.f90:434-469)
__device__ __forceinline__ void entropy_to_cons(const KParams& P, const double* W, double* U) {
  const double rho_sp = -W[4];
  const double p_srho = 1. / rho_sp;
  const double u = W[1] * p_srho, v = W[2] * p_srho, w = W[3] * p_srho;
  const double v2s2 = 0.5 * (u * u + v * v + w * w);
  const double s = P.kappa - ((W[0] + rho_sp * v2s2) * P.kappaM1);
  U[0] = pow(exp(-s) * p_srho, P.sKappaM1);
  U[1] = u * U[0];
  U[2] = v * U[0];
  U[3] = w * U[0];
  U[4] = U[0] * (p_srho * P.sKappaM1 + v2s2);
}

// face-state slot of (side, role, point), nv variables per point
__device__ __forceinline__ double* uface_at(const KParams& P, int NPT, int side, int role, int pt, int nv = 5) {
  return P.uface + (((size_t)side * 2 + role) * NPT + pt) * nv;
}

// ProlongToFace_U (dg.f90:458-511) with the Gauss interpolation of prolongtoface.f90:103-132; ENT: the
// entropy variables are interpolated and the face values converted back (useEntropyProlongToFace);
// NVT = 5 (Euler / Navier-Stokes) or 9 (MHD + GLM, mhd/equation_vars.f90:330-401).
template <int NP, bool ENT, int NVT>
__global__ void __launch_bounds__(NP * NP * NP) prolong_kernel(KParams P) {
  if (halted(P)) return;
  constexpr int NP3 = NP * NP * NP, NPT = NP * NP, XS = NP3 + NPT;
  __shared__ double sX[NVT * XS];  // [var][slot], node n at slot n + n / NP (the lines of a warp's side
                                   // points spread over the banks)
  __shared__ double sL[NP];
  __shared__ int sE2S[12];
  const int e = blockIdx.x, t = threadIdx.x;
  for (int z = t; z < 12; z += NP3) sE2S[z] = P.e2s[12 * (size_t)e + z];  // NP3 = 8 for N = 1
  if (t < NP) sL[t] = P.basis->Lminus[t];
  {
    const double* Ug = P.U + NVT * ((size_t)e * NP3 + t);
    double u[NVT], x[NVT];
#pragma unroll
    for (int v = 0; v < NVT; ++v) u[v] = Ug[v];
    if constexpr (ENT && NVT == 9) {
      mhd::cons_to_entropy(P, u, x);
    } else if constexpr (ENT) {
      cons_to_entropy_ns(P, u, x);
    } else {
#pragma unroll
      for (int v = 0; v < NVT; ++v) x[v] = u[v];
    }
#pragma unroll
    for (int v = 0; v < NVT; ++v) sX[v * XS + t + t / NP] = x[v];
  }
  __syncthreads();
  for (int task = t; task < 6 * NPT; task += NP3) {
    const int s = task / NPT + 1, ab = task - (s - 1) * NPT, a = ab % NP, b = ab / NP;
    const int side = sE2S[2 * (s - 1)], flip = sE2S[2 * (s - 1) + 1];
    double acc[NVT];
    {
      const int n0 = line_node_of(NP, s, a, b, 0);
#pragma unroll
      for (int v = 0; v < NVT; ++v) acc[v] = sX[v * XS + n0 + n0 / NP] * sL[0];
    }
#pragma unroll
    for (int l = 1; l < NP; ++l) {
      const int n = line_node_of(NP, s, a, b, l);
#pragma unroll
      for (int v = 0; v < NVT; ++v) acc[v] = acc[v] + sX[v * XS + n + n / NP] * sL[l];
    }
    double c[NVT];
    if constexpr (ENT && NVT == 9) {
      mhd::entropy_to_cons(P, acc, c);
    } else if constexpr (ENT) {
      entropy_to_cons(P, acc, c);
    } else {
#pragma unroll
      for (int v = 0; v < NVT; ++v) c[v] = acc[v];
    }
    double* o = uface_at(P, NPT, side, flip == 0 ? 0 : 1, face_point_of(NP, s, flip, a, b), NVT);
#pragma unroll
    for (int v = 0; v < NVT; ++v) o[v] = c[v];
  }
}

// the flux area of the lifting kernel: the 12 contravariant fluxes per node, and before them the 15 staged
// surface products of each of the 6 (N+1)^2 side points
template <int NP>
__host__ __device__ constexpr int lift_farea() {
  return 12 * NP * NP * NP > 90 * NP * NP ? 12 * NP * NP * NP : 90 * NP * NP;
}
// gradient rows of the lifting kernel: node n at slot n + n / NP (row stride NP^3 + NP^2), so that the
// face-trace sums of the side points of a warp spread over the banks
template <int NP>
__host__ __device__ constexpr int lift_gstride() { return NP * NP * NP + NP * NP; }
__device__ __forceinline__ int lift_gslot(int NP, int n) { return n + n / NP; }
template <int NP>
__host__ __device__ constexpr size_t lift_smem_bytes() {
  return sizeof(double) * (size_t)(2 * NP * NP + 2 * NP + 6 * NP * NP * NP + 15 * lift_gstride<NP>() + lift_farea<NP>());
}

// BR1 / BR2 lifting with Gauss nodes (br1.f90:154-364, br1_surfint.f90:100-128, br2_surfint.f90:109-148),
// the viscous face-flux shares of both sides of every face point of the element (riemann.f90:155-168) and
// the viscous volume integral (volint.f90:228-271).  One element per block, one thread per node.
template <int NP, int LIFT, int LV>
__global__ void __launch_bounds__(NP * NP * NP) lift_visc_kernel(KParams P) {
  if (halted(P)) return;
  constexpr int NP3 = NP * NP * NP, NPT = NP * NP, N = NP - 1;
  extern __shared__ double smem[];
  double* sD = smem;              // D(i,l) at [i*NP+l]
  double* sDhat = sD + NPT;       // D_hat(i,l)
  double* sLm = sDhat + NPT;      // L_Minus(l)
  double* sLh = sLm + NP;         // L_HatMinus(l)
  double* sV = sLh + NP;          // [5][node] lifting variable
  constexpr int GS = lift_gstride<NP>();
  double* sG = sV + 5 * NP3;      // [15][slot] gradient of the lifting variable that is prolonged
  double* sF = sG + 15 * GS;      // [12][node] contravariant viscous fluxes (first: staged side products)
  double* sSJ = sF + lift_farea<NP>();  // [node] sJ
  __shared__ int sE2S[12];
  const int e = blockIdx.x, t = threadIdx.x;
  const int i = t % NP, j = (t / NP) % NP, k = t / NPT;
  for (int z = t; z < NPT; z += NP3) { sD[z] = P.basis->D[z]; sDhat[z] = P.basis->Dhat[z]; }
  if (t < NP) { sLm[t] = P.basis->Lminus[t]; sLh[t] = P.basis->LhatMinus[t]; }
  for (int z = t; z < 12; z += NP3) sE2S[z] = P.e2s[12 * (size_t)e + z];  // NP3 = 8 for N = 1
  double u[5];
  const double sj = P.sJ[(size_t)e * NP3 + t];
  const int gs = lift_gslot(NP, t);
  {
    const double* Ug = P.U + 5 * ((size_t)e * NP3 + t);
#pragma unroll
    for (int v = 0; v < 5; ++v) u[v] = Ug[v];
    double V[5];
    lifting_var_t<LV>(P, u, V);
#pragma unroll
    for (int v = 0; v < 5; ++v) sV[v * NP3 + t] = V[v];
    sSJ[t] = sj;
  }
  __syncthreads();
  const double* M = P.metrics + (size_t)e * 9 * NP3 + t;
  double g[3][5];
  {
    // Lifting_VolInt (br1_volint.f90:45-98): the derivatives along the lines, metric terms
    double dx[5], de[5], dz[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) { dx[v] = 0.; de[v] = 0.; dz[v] = 0.; }
#pragma unroll
    for (int l = 0; l < NP; ++l) {
      const double a = sD[i * NP + l], b = sD[j * NP + l], c = sD[k * NP + l];
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        dx[v] += a * sV[v * NP3 + l + NP * (j + NP * k)];
        de[v] += b * sV[v * NP3 + i + NP * (l + NP * k)];
        dz[v] += c * sV[v * NP3 + i + NP * (j + NP * l)];
      }
    }
    double m[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) m[c] = M[c * NP3];
#pragma unroll
    for (int v = 0; v < 5; ++v)
#pragma unroll
      for (int d = 0; d < 3; ++d) g[d][v] = m[0 + d] * dx[v] + m[3 + d] * de[v] + m[6 + d] * dz[v];
  }
  if constexpr (LIFT == 2) {  // br2_volint.f90: the volume part carries sJ; it is what is prolonged
#pragma unroll
    for (int v = 0; v < 5; ++v)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        g[d][v] *= sj;
        sG[(5 * d + v) * GS + gs] = g[d][v];
      }
  }
  // surface terms: every node of the line of each side takes the lifting flux times L_HatMinus(l).  The
  // 15 products (flux x normal) of each of the element's 6 (N+1)^2 side points are staged once in the
  // flux area (free until the volume fluxes), [side point][3 x 5]
  for (int task = t; task < 6 * NPT; task += NP3) {
    const int s = task / NPT + 1, ab = task - (s - 1) * NPT, a = ab % NP, b = ab / NP;
    const int side = sE2S[2 * (s - 1)], flip = sE2S[2 * (s - 1) + 1];
    const int pt = face_point_of(NP, s, flip, a, b);
    const double* nvec = P.facegeo + (size_t)side * 10 * NPT + pt;
    const double* F = P.lflux + (size_t)side * 5 * NPT + pt;
    const double n0 = nvec[0], n1 = nvec[NPT], n2 = nvec[2 * NPT];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const double f = F[v * NPT];
      sF[task * 15 + v] = f * n0;
      sF[task * 15 + 5 + v] = f * n1;
      sF[task * 15 + 10 + v] = f * n2;
    }
  }
  __syncthreads();
#pragma unroll 1
  for (int s = 1; s <= 6; ++s) {
    int l, a, b;
    line_of_node(N, s, i, j, k, l, a, b);
    const double* Fn = sF + ((s - 1) * NPT + a + NP * b) * 15;
    const double lh = sLh[l];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      if constexpr (LIFT == 2) {
        const double fl = sj * lh;
        g[0][v] += fl * Fn[v]; g[1][v] += fl * Fn[5 + v]; g[2][v] += fl * Fn[10 + v];
      } else {
        g[0][v] += Fn[v] * lh; g[1][v] += Fn[5 + v] * lh; g[2][v] += Fn[10 + v] * lh;
      }
    }
  }
  if constexpr (LIFT == 1) {
#pragma unroll
    for (int v = 0; v < 5; ++v)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        g[d][v] *= sj;
        sG[(5 * d + v) * GS + gs] = g[d][v];
      }
  }
  __syncthreads();
  // face traces: the gradient interpolated to each side's points (BR2: plus etaBR2 L_Minus(l) times the
  // own side's surface terms), converted with the side's state, n.F_v for the face kernel
  for (int task = t; task < 6 * NPT; task += NP3) {
    const int s = task / NPT + 1, ab = task - (s - 1) * NPT, a = ab % NP, b = ab / NP;
    const int side = sE2S[2 * (s - 1)], flip = sE2S[2 * (s - 1) + 1], role = flip == 0 ? 0 : 1;
    const int pt = face_point_of(NP, s, flip, a, b);
    const double* nvec = P.facegeo + (size_t)side * 10 * NPT + pt;
    const double n0 = nvec[0], n1 = nvec[NPT], n2 = nvec[2 * NPT];
    double tr[3][5];
    {
      const int nd = lift_gslot(NP, line_node_of(NP, s, a, b, 0));
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int v = 0; v < 5; ++v) tr[d][v] = sG[(5 * d + v) * GS + nd] * sLm[0];
    }
    for (int l = 1; l < NP; ++l) {
      const int nd = lift_gslot(NP, line_node_of(NP, s, a, b, l));
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int v = 0; v < 5; ++v) tr[d][v] = tr[d][v] + sG[(5 * d + v) * GS + nd] * sLm[l];
    }
    if constexpr (LIFT == 2) {
      const double* F = P.lflux + (size_t)side * 5 * NPT + pt;
      double f[5];
#pragma unroll
      for (int v = 0; v < 5; ++v) f[v] = F[v * NPT];
      for (int l = 0; l < NP; ++l) {
        const double w = P.etaBR2 * sLm[l], fl = sSJ[line_node_of(NP, s, a, b, l)] * sLh[l];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          tr[0][v] = tr[0][v] + w * (fl * (f[v] * n0));
          tr[1][v] = tr[1][v] + w * (fl * (f[v] * n1));
          tr[2][v] = tr[2][v] + w * (fl * (f[v] * n2));
        }
      }
    }
    const double* uf = uface_at(P, NPT, side, role, pt);
    double us[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) us[v] = uf[v];
#pragma unroll
    for (int d = 0; d < 3; ++d) to_grad_prim(P, us, tr[d]);
    double kf[4], kg[4], kh[4];
    diff_flux_3d(P, us, tr[0], tr[1], tr[2], kf, kg, kh);
    double* T = P.gtrace + ((size_t)side * 2 + role) * 4 * NPT + pt;
#pragma unroll
    for (int v = 0; v < 4; ++v) T[(size_t)v * NPT] = n0 * kf[v] + n1 * kg[v] + n2 * kh[v];
  }
  // volume: primitive gradients of the node, contravariant viscous fluxes
#pragma unroll
  for (int d = 0; d < 3; ++d) to_grad_prim(P, u, g[d]);
  if (P.grad) {
    double* G = P.grad + 15 * ((size_t)e * NP3 + t);
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int v = 0; v < 5; ++v) G[5 * d + v] = g[d][v];
  }
  {
    double f[4], gg[4], h[4];
    diff_flux_3d(P, u, g[0], g[1], g[2], f, gg, h);
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
      const double m0 = M[(3 * dir + 0) * NP3], m1 = M[(3 * dir + 1) * NP3], m2 = M[(3 * dir + 2) * NP3];
#pragma unroll
      for (int v = 0; v < 4; ++v) sF[(4 * dir + v) * NP3 + t] = f[v] * m0 + gg[v] * m1 + h[v] * m2;
    }
  }
  __syncthreads();
  double r[4] = {0., 0., 0., 0.};
#pragma unroll
  for (int l = 0; l < NP; ++l) {
    const double a = sDhat[i * NP + l], b = sDhat[j * NP + l], c = sDhat[k * NP + l];
#pragma unroll
    for (int v = 0; v < 4; ++v)
      r[v] += a * sF[v * NP3 + l + NP * (j + NP * k)] + b * sF[(4 + v) * NP3 + i + NP * (l + NP * k)] +
              c * sF[(8 + v) * NP3 + i + NP * (j + NP * l)];
  }
  double* O = P.utvisc + (size_t)e * 4 * NP3 + t;
#pragma unroll
  for (int v = 0; v < 4; ++v) O[v * NP3] = r[v];
}

// shared memory of the surface kernel: per side point of the element the side state's record (NQ), the
// halved SurfMetrics (3) and the surface flux (5); the line buffer [5][node]
// stride of a side point's data: record (NQ), metric (3), flux (5), made odd so that the records of
// consecutive side points fall into different banks
template <int VF>
__host__ __device__ constexpr int surf_stride() { return (VolRec<VF>::NQ + 8) | 1; }
template <int NP, int VF>
__host__ __device__ constexpr size_t surf_smem_bytes() {
  return sizeof(double) * (size_t)(6 * NP * NP * surf_stride<VF>() + 5 * NP * NP * NP);
}

// SurfInt with Gauss nodes and the split-form correction (surfint.f90:118-175, 196-253).  One element per
// block, one thread per node.  The records of the side states (their logarithms included), the surface
// metrics and the surface fluxes of the element's 6 (N+1)^2 side points are formed once in shared memory;
// then per local side every node forms FluxB(l) with its line's side state, the line sum
// FluxB_sum = sum_l FluxB(l) L_Minus(l) (shared memory, l = 0..N), and its share of the side's terms.
template <int NP, int VF>
__global__ void __launch_bounds__(NP * NP * NP, NP == 8 ? 2 : 1) surf_kernel(KParams P) {
  if (halted(P)) return;
  constexpr int NP3 = NP * NP * NP, NPT = NP * NP, N = NP - 1, RS = VolRec<VF>::RS, NQ = VolRec<VF>::NQ;
  constexpr int FS = surf_stride<VF>();  // per side point: record, metric (3), flux (5), padding
  extern __shared__ double smem[];
  double* sP = smem;               // [6 * NPT][FS]
  double* sB = sP + 6 * NPT * FS;  // [var][node] FluxB(l) L_Minus(l) of the current side
  __shared__ double sLm[NP], sLh[NP];
  __shared__ int sE2S[12];
  const int e = blockIdx.x, t = threadIdx.x;
  const int i = t % NP, j = (t / NP) % NP, k = t / NPT;
  if (t < NP) { sLm[t] = P.basis->Lminus[t]; sLh[t] = P.basis->LhatMinus[t]; }
  for (int z = t; z < 12; z += NP3) sE2S[z] = P.e2s[12 * (size_t)e + z];  // NP3 = 8 for N = 1
  double rN[RS];
  {
    const double* Ug = P.U + 5 * ((size_t)e * NP3 + t);
    double u[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) u[v] = Ug[v];
    make_record<VF>(P, u, rN);
  }
  // pair_flux takes half metrics for every flux but the standard DG one (the metric average is a sum)
  constexpr double hm = VF == 0 ? 1.0 : 0.5;
  double m[9];
  {
    const double* M = P.metrics + (size_t)e * 9 * NP3 + t;
#pragma unroll
    for (int c = 0; c < 9; ++c) m[c] = hm * M[c * NP3];
  }
  __syncthreads();
  for (int task = t; task < 6 * NPT; task += NP3) {
    const int s = task / NPT + 1, ab = task - (s - 1) * NPT, a = ab % NP, b = ab / NP;
    const int side = sE2S[2 * (s - 1)], flip = sE2S[2 * (s - 1) + 1], role = flip == 0 ? 0 : 1;
    const int pt = face_point_of(NP, s, flip, a, b);
    double* o = sP + task * FS;
    {
      const double* uf = uface_at(P, NPT, side, role, pt);
      double us[5], r[RS];
#pragma unroll
      for (int v = 0; v < 5; ++v) us[v] = uf[v];
      make_record<VF>(P, us, r);
#pragma unroll
      for (int z = 0; z < NQ; ++z) o[z] = r[z];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) o[NQ + c] = hm * P.surfMet[(((size_t)e * 6 + (s - 1)) * 3 + c) * NPT + pt];
    const double* Fs = P.flux + (size_t)side * 5 * NPT + pt;
#pragma unroll
    for (int v = 0; v < 5; ++v) o[NQ + 3 + v] = Fs[v * NPT];
  }
  double ut[5] = {0., 0., 0., 0., 0.};
  __syncthreads();
#pragma unroll 1
  for (int s = 1; s <= 6; ++s) {
    int l, a, b;
    line_of_node(N, s, i, j, k, l, a, b);
    const int role = sE2S[2 * (s - 1) + 1] == 0 ? 0 : 1;
    const int dir = (s == XI_MINUS || s == XI_PLUS) ? 0 : ((s == ETA_MINUS || s == ETA_PLUS) ? 1 : 2);
    const double sg = (s == ZETA_MINUS || s == ETA_MINUS || s == XI_MINUS) ? -1. : 1.;  // NormalSigns
    const double* o = sP + ((s - 1) * NPT + a + NP * b) * FS;
    double FB[5], mN[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) mN[c] = dir == 0 ? m[c] : (dir == 1 ? m[3 + c] : m[6 + c]);  // registers
    pair_flux<VF>(P, rN, o, mN, o + NQ, FB);
#pragma unroll
    for (int v = 0; v < 5; ++v) sB[v * NP3 + t] = FB[v] * sLm[l];
    __syncthreads();
    double sum[5] = {0., 0., 0., 0., 0.};
    for (int ll = 0; ll < NP; ++ll) {
      const int nd = line_node_of(NP, s, a, b, ll);
#pragma unroll
      for (int v = 0; v < 5; ++v) sum[v] = sum[v] + sB[v * NP3 + nd];
    }
    const double lh = sLh[l];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const double corr = (sum[v] - FB[v]) * sg;
      const double f = o[NQ + 3 + v];
      if (role == 0) ut[v] = ut[v] + (f - corr) * lh;
      else ut[v] = ut[v] - (f + corr) * lh;
    }
    __syncthreads();  // sB is rewritten by the next side
  }
  double* O = P.utsurf + (size_t)e * 5 * NP3 + t;
#pragma unroll
  for (int v = 0; v < 5; ++v) O[v * NP3] = ut[v];
}

}  // namespace gauss
}  // namespace fluxo
