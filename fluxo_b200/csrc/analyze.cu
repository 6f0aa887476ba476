// Device-side analysis of a state: the reference's Analyze path reduced on the GPU.
//   CalcErrorNorms (src/analyze/analyze.f90:557-632): L2 and L_inf errors against an exact function
//     on NAnalyze = 2(N+1) LGL points per direction (U, Elem_xGP and 1/sJ interpolated there), and
//     the L2 error at the collocation points;
//   CalcEntropy (src/equation/navierstokes/analyze_equation.f90:549-599, mhd/analyze_equation.f90:421-470):
//     the total entropy and dS/dU . Ut of the last right-hand side;
//   the Taylor-Green integrands of src/testcase/taylorgreenvortex/testcase_analyze.f90:127-330 (kinetic
//     energy 1/2 rho |v|^2 and enstrophy 1/2 rho |curl v|^2 from the lifted velocity gradients, both
//     divided by the domain volume).
// One block per element writes its partial sums to partial[elem][K]; one block then reduces them in a
// fixed order, so the result does not depend on the launch's scheduling.
#include <cuda_runtime.h>

#include "common.cuh"
#include "launch.h"

namespace fluxo {

namespace {

// ExactFunc of the Euler / Navier-Stokes module (navierstokes/equation.f90:575-811) for the analysis:
// 1 constant reference state, 2 density sine wave, 4 manufactured solution, 7 Taylor-Green vortex,
// 14 soft Sedov-Taylor blast.
__device__ void exact_ns(const AnalyzeArgs& A, double t, const double* x, double* U) {
  double prim[5];
  switch (A.func) {
    case 1:
      for (int v = 0; v < 5; ++v) prim[v] = A.refPrim[v];
      break;
    case 2: {  // equation.f90:632-651
      double s = 0.;
      for (int d = 0; d < 3; ++d) s += A.waveNumber[d] * (x[d] - A.advVel[d] * t);
      prim[0] = 1. * (1. + A.amplitude * sin(M_PI * s));
      for (int d = 0; d < 3; ++d) prim[1 + d] = A.advVel[d];
      prim[4] = 1.;
      break;
    }
    case 4: {  // equation.f90:698-702 (conservative variables directly)
      const double v = 2. + A.amplitude * sin(M_PI * A.frequency * ((x[0] + x[1] + x[2]) - t));
      U[0] = v; U[1] = v; U[2] = v; U[3] = v; U[4] = v * v;
      return;
    }
    case 14: {  // soft Sedov-Taylor blast, equation.f90:906-922
      double nx[3], r2 = 0.;
      for (int d = 0; d < 3; ++d) { nx[d] = x[d] - A.center[d]; r2 += nx[d] * nx[d]; }
      r2 = sqrt(r2);
      prim[0] = 1.; prim[1] = prim[2] = prim[3] = 0.; prim[4] = 1.;
      if (r2 <= 0.5 && r2 != 0.) {
        prim[0] = 1.3416149068323;
        for (int d = 0; d < 3; ++d) prim[1 + d] = 0.361538208967199 * nx[d] / r2;
        prim[4] = 1.51333333333333;
      }
      break;
    }
    default: {  // 7, equation.f90:802-811 (A = 1, Ms = 0.1)
      const double Am = 1., Ms = 0.1;
      prim[0] = 1.;
      prim[1] = Am * sin(x[0]) * cos(x[1]) * cos(x[2]);
      prim[2] = -Am * cos(x[0]) * sin(x[1]) * cos(x[2]);
      prim[3] = 0.;
      prim[4] = Am / Ms * Am / Ms / A.kappa * prim[0];
      prim[4] = prim[4] + 1. / 16. * Am * Am * prim[0] *
                              (cos(2 * x[0]) * cos(2. * x[2]) + 2. * cos(2. * x[1]) + 2. * cos(2. * x[0]) +
                               cos(2 * x[1]) * cos(2. * x[2]));
      break;
    }
  }
  U[0] = prim[0];
  for (int d = 0; d < 3; ++d) U[1 + d] = prim[0] * prim[1 + d];
  U[4] = prim[4] * A.sKappaM1 + 0.5 * prim[0] * (prim[1] * prim[1] + prim[2] * prim[2] + prim[3] * prim[3]);
}

// Deterministic block sum (op 0) or max (op 1) of one value per thread; every thread gets the result.
__device__ double block_reduce(double v, int op, double* red) {
  red[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {  // blockDim is a power of two
    if (threadIdx.x < s) {
      const double o = red[threadIdx.x + s];
      red[threadIdx.x] = op ? fmax(red[threadIdx.x], o) : red[threadIdx.x] + o;
    }
    __syncthreads();
  }
  const double r = red[0];
  __syncthreads();
  return r;
}

__global__ void analyze_elem_kernel(AnalyzeArgs A) {
  extern __shared__ double sm[];
  const int e = blockIdx.x;
  const int NP = A.NP, NP3 = NP * NP * NP, NA1 = A.NA1, NV = A.nVar;
  const int NQ = NV + 4;  // U, x (3), J = 1/sJ
  double* red = sm;                    // [blockDim]
  double* f = red + blockDim.x;        // [NQ][NP^3]
  double* T1 = f + (size_t)NQ * NP3;   // [NQ][NP][NP]
  double* T2 = T1 + (size_t)NQ * NP * NP;  // [NQ][NA1][NP]
  double* out = A.partial + (size_t)e * A.K;

  // node-local integrands with the collocation weights wGPVol/sJ
  double S = 0., dS = 0., Ek = 0., En = 0., Vol = 0., col[9] = {0., 0., 0., 0., 0., 0., 0., 0., 0.};
  for (int n = threadIdx.x; n < NP3; n += blockDim.x) {
    const int i = n % NP, j = (n / NP) % NP, k = n / (NP * NP);
    const size_t o = (size_t)e * NP3 + n;
    const double w = A.wGP[i] * A.wGP[j] * A.wGP[k] / A.sJ[o];
    double U[9], W[9];
    for (int v = 0; v < NV; ++v) U[v] = A.U[NV * o + v];
    const double srho = 1. / U[0];
    const double u = U[1] * srho, vv = U[2] * srho, ww = U[3] * srho;
    const double v2s2 = 0.5 * (u * u + vv * vv + ww * ww);
    double pm = 0.;  // magnetic and psi energy (MHD)
    if (A.mhd) pm = A.s2mu_0 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7] + U[8] * U[8]);
    const double p = A.kappaM1 * (U[4] - U[0] * v2s2 - pm);
    S += -U[0] * (log(p) - A.kappa * log(U[0])) * w;
    // entropy variables (ConsToEntropyVec, equation_vars.f90:397-429; mhd/equation_vars.f90:330-361)
    const double rho_sp = U[0] / p;
    const double s = -(log(rho_sp) + A.kappaM1 * log(U[0]));
    W[0] = (A.kappa - s) * A.sKappaM1 - rho_sp * v2s2;
    W[1] = rho_sp * u; W[2] = rho_sp * vv; W[3] = rho_sp * ww;
    W[4] = -rho_sp;
    for (int v = 5; v < NV; ++v) W[v] = rho_sp * U[v];
    if (A.Ut) {
      double loc = 0.;
      for (int v = 0; v < NV; ++v) loc += W[v] * A.Ut[NV * o + v];
      dS += loc * w;
    }
    Ek += U[0] * v2s2 * w;
    if (A.grad) {  // primitive gradients [elem][node][3][var]: vorticity from the velocity gradients
      const double* g = A.grad + (size_t)3 * NV * o;
      const double wx = g[NV + 3] - g[2 * NV + 2];
      const double wy = g[2 * NV + 1] - g[3];
      const double wz = g[2] - g[NV + 1];
      En += 0.5 * U[0] * (wx * wx + wy * wy + wz * wz) * w;
    }
    Vol += w;
    if (A.func) {
      double ue[5];
      exact_ns(A, A.t, A.xGP + 3 * o, ue);
      for (int v = 0; v < NV; ++v) {
        const double d = U[v] - ue[v];
        col[v] += d * d * w;
      }
    }
  }
  const int base = 3 * NV;
  const double sums[5] = {S, dS, Ek, En, Vol};
  for (int z = 0; z < 5; ++z) {
    const double r = block_reduce(sums[z], 0, red);
    if (threadIdx.x == 0) out[base + z] = r;
  }
  if (!A.func) return;
  for (int v = 0; v < NV; ++v) {
    const double r = block_reduce(col[v], 0, red);
    if (threadIdx.x == 0) out[NV + v] = r;
  }

  // CalcErrorNorms on the NAnalyze grid: sum factorisation plane by plane (c = third index)
  for (int z = threadIdx.x; z < NQ * NP3; z += blockDim.x) {
    const int q = z / NP3, n = z - q * NP3;
    const size_t o = (size_t)e * NP3 + n;
    f[z] = q < NV ? A.U[NV * o + q] : (q < NV + 3 ? A.xGP[3 * o + q - NV] : 1. / A.sJ[o]);
  }
  __syncthreads();
  double l2[9] = {0., 0., 0., 0., 0., 0., 0., 0., 0.}, li[9];
  for (int v = 0; v < 9; ++v) li[v] = -1.e10;
  for (int c = 0; c < NA1; ++c) {
    for (int z = threadIdx.x; z < NQ * NP * NP; z += blockDim.x) {  // T1[q][j][i] = sum_k V(c,k) f[q][k][j][i]
      const int q = z / (NP * NP), ji = z - q * NP * NP;
      double a = 0.;
      for (int k = 0; k < NP; ++k) a += A.V[c * NP + k] * f[(size_t)q * NP3 + k * NP * NP + ji];
      T1[z] = a;
    }
    __syncthreads();
    for (int z = threadIdx.x; z < NQ * NA1 * NP; z += blockDim.x) {  // T2[q][b][i] = sum_j V(b,j) T1[q][j][i]
      const int q = z / (NA1 * NP), r = z - q * NA1 * NP, b = r / NP, i = r - b * NP;
      double a = 0.;
      for (int j = 0; j < NP; ++j) a += A.V[b * NP + j] * T1[(size_t)q * NP * NP + j * NP + i];
      T2[z] = a;
    }
    __syncthreads();
    for (int z = threadIdx.x; z < NA1 * NA1; z += blockDim.x) {  // point (a, b, c)
      const int b = z / NA1, a = z - b * NA1;
      double val[13];
      for (int q = 0; q < NQ; ++q) {
        double s = 0.;
        for (int i = 0; i < NP; ++i) s += A.V[a * NP + i] * T2[((size_t)q * NA1 + b) * NP + i];
        val[q] = s;
      }
      double ue[5];
      exact_ns(A, A.t, val + NV, ue);
      const double wgt = A.wA[a] * A.wA[b] * A.wA[c] * val[NV + 3];
      for (int v = 0; v < NV; ++v) {
        const double d = val[v] - ue[v];
        li[v] = fmax(li[v], fabs(d));
        l2[v] += d * d * wgt;
      }
    }
    __syncthreads();
  }
  for (int v = 0; v < NV; ++v) {
    const double r2 = block_reduce(l2[v], 0, red);
    const double ri = block_reduce(li[v], 1, red);
    if (threadIdx.x == 0) {
      out[v] = r2;
      out[2 * NV + v] = ri;
    }
  }
}

// partial[nElems][K] -> res[K]: sums (max for L_inf) over the elements in a fixed order
__global__ void analyze_reduce_kernel(AnalyzeArgs A, double* res) {
  __shared__ double red[512];
  const int NV = A.nVar;
  for (int z = 0; z < A.K; ++z) {
    const int op = (z >= 2 * NV && z < 3 * NV) ? 1 : 0;
    double a = op ? -1.e10 : 0.;
    for (int e = threadIdx.x; e < A.nElems; e += blockDim.x) {
      const double v = A.partial[(size_t)e * A.K + z];
      a = op ? fmax(a, v) : a + v;
    }
    const double r = block_reduce(a, op, red);
    if (threadIdx.x == 0) res[z] = r;
  }
}

}  // namespace

size_t analyze_smem_bytes(int NP, int nVar, int threads) {
  const int NQ = nVar + 4, NA1 = 2 * NP + 1;
  return sizeof(double) * ((size_t)threads + (size_t)NQ * NP * NP * NP + (size_t)NQ * NP * NP + (size_t)NQ * NA1 * NP);
}

cudaError_t launch_analyze(const AnalyzeArgs& A, double* res, cudaStream_t s) {
  constexpr int kThreads = 256;
  const size_t smem = analyze_smem_bytes(A.NP, A.nVar, kThreads);
  // one limit for every call: the largest case (N+1 = 9, MHD's 9 variables)
  static std::atomic<unsigned long long> attr{0};
  cudaError_t e = smem_attr_once(analyze_elem_kernel, analyze_smem_bytes(FLUXO_NPMAX, 9, kThreads), attr);
  if (e != cudaSuccess) return e;
  if (A.NP > FLUXO_NPMAX || A.nVar > 9) return cudaErrorInvalidValue;
  analyze_elem_kernel<<<A.nElems, kThreads, smem, s>>>(A);
  analyze_reduce_kernel<<<1, 512, 0, s>>>(A, res);
  return cudaGetLastError();
}

}  // namespace fluxo
