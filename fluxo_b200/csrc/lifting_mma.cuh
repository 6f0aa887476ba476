// Lifting + viscous volume kernel for N+1 = 8 with the operator contractions on the FP64 tensor cores.
//
// The same computation as lift_visc_kernel (lifting.cuh), element by element: the derivatives of the
// lifting variable along xi, eta, zeta (br1_volint.f90:45-98: D applied along the lines) and the viscous
// volume integral (volint.f90:228-271: D_hat applied to the contravariant fluxes) are 8x8 operator
// matrices times the 64 lines of each direction, i.e. small dense products.  They run as
// mma.sync.m8n8k4 FP64 tiles: per element 120 tiles for the derivatives (3 directions x 5 variables x
// 8 groups of 8 lines) and 96 for the divergence (3 directions x 4 fluxes x 8), two k-slices each.  The
// operator stays in registers as the A fragment; a tile's B fragment is one double per lane from shared
// memory, against one shared load per multiply-add in the node-centric sums, which bound that kernel
// by the shared-memory pipe.  The node phase between the two products (gradient, face traces,
// fluxes) is lv_node_fluxes, shared with lift_visc_kernel.
//
// Shared layout: every per-node array uses slot(i,j,k) = i + 9 j + 76 k (603 slots).  A tile's 8 columns
// are lines of its direction that differ in k (xi: j fixed, eta: i fixed) or in j (zeta: i fixed); with
// this padding the B loads of all three directions hit distinct banks, and the C stores two-way.
#pragma once
#include "lifting.cuh"

namespace fluxo {

__device__ __forceinline__ int lm_slot(int i, int j, int k) { return i + 9 * j + 76 * k; }
constexpr int kLmStride = 603;  // lm_slot(7, 7, 7) + 1 (slots are distinct: 7 + 9*7 < 76)
constexpr size_t lm_smem_bytes() { return sizeof(double) * (size_t)20 * kLmStride; }

// d += A(8x4) B(4x8) in FP64: a = A[lane/4][lane%4], b = B[lane%4][lane/4],
// d0, d1 = D[lane/4][2 (lane%4)], D[lane/4][2 (lane%4) + 1]
__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// slot of position `pos` on line `c` of tile T of direction DIR
template <int DIR>
__device__ __forceinline__ int lm_tile_slot(int T, int c, int pos) {
  return DIR == 0 ? lm_slot(pos, T, c) : (DIR == 1 ? lm_slot(T, pos, c) : lm_slot(T, c, pos));
}

// One output tile: dst(pos, line) (=, or += with ACC) sum_l Op(pos, l) src(l, line) for the 8 lines of
// tile T; a[kk] = Op[lane/4][4 kk + lane%4] are the operator's two k-slices.
template <int DIR, bool ACC>
__device__ __forceinline__ void lm_tile(const double* a, const double* src, double* dst, int T, int lane) {
  double d0 = 0., d1 = 0.;
  const int l = lane & 3, c = lane >> 2;
  dmma_m8n8k4(d0, d1, a[0], src[lm_tile_slot<DIR>(T, c, l)]);
  dmma_m8n8k4(d0, d1, a[1], src[lm_tile_slot<DIR>(T, c, 4 + l)]);
  const int pos = lane >> 2, c0 = 2 * (lane & 3);
  double* p0 = dst + lm_tile_slot<DIR>(T, c0, pos);
  double* p1 = dst + lm_tile_slot<DIR>(T, c0 + 1, pos);
  if (ACC) {
    *p0 += d0;
    *p1 += d1;
  } else {
    *p0 = d0;
    *p1 = d1;
  }
}

template <int LIFT, int LV>
__global__ void __launch_bounds__(512, lv_minb<8, LIFT>()) lift_visc_mma_kernel(KParams P) {
  if (halted(P)) return;
  constexpr int NP = 8, NP3 = 512, NPT = 64, S = kLmStride;
  extern __shared__ double smem[];
  double* sV = smem;        // [5][S] lifting variable; later the divergence R[4][S]
  double* sW = sV + 5 * S;  // [15][S] derivatives (xi 0-4, eta 5-9, zeta 10-14); later the fluxes [12][S]
  __shared__ int sE2S[12];
  const int t = threadIdx.x, e = blockIdx.x;
  const bool valid = e < P.nElems;  // block-uniform
  const int lane = t & 31, warp = t >> 5;
  const int i = t % NP, j = (t / NP) % NP, k = t / NPT;
  const int slot = lm_slot(i, j, k);
  if (P.pfTiles > 0 && t == 0) {  // the element one wave ahead: its inputs into L2
    const size_t en = (size_t)blockIdx.x + P.pfTiles;
    if (en < (size_t)P.nElems) {
      prefetch_l2_bulk(P.U + 5 * en * NP3, 5 * NP3 * sizeof(double));
      prefetch_l2_bulk(P.metrics + 9 * en * NP3, 9 * NP3 * sizeof(double));
      prefetch_l2_bulk(P.sJ + en * NP3, NP3 * sizeof(double));
    }
  }
  // A fragments (row lane/4, columns 4 kk + lane%4) of D and D_hat, loaded where they are used
  const int ar = (lane >> 2) * NP + (lane & 3);
  const double* Ug = P.U + 5 * ((size_t)e * NP3 + t);
  if (valid) {
    if (t < 12) sE2S[t] = P.e2s[12 * (size_t)e + t];
    double u[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) u[v] = Ug[v];
#pragma unroll
    for (int c = 0; c < 9; ++c) prefetch_l2(P.metrics + (size_t)e * 9 * NP3 + c * NP3 + t);
    prefetch_l2(P.sJ + (size_t)e * NP3 + t);
    double V[5];
    lifting_var_t<LV>(P, u, V);
#pragma unroll
    for (int v = 0; v < 5; ++v) sV[v * S + slot] = V[v];
  }
  __syncthreads();
  // derivatives: 3 directions x 5 variables x 8 tiles, warp-uniform tile loop
  if (valid) {
    const double aD[2] = {P.basis->D[ar], P.basis->D[ar + 4]};
#pragma unroll 1
    for (int w = warp; w < 120; w += 16) {
      const int dir = w / 40, r = w - 40 * dir, v = r >> 3, T = r & 7;
      const double* src = sV + v * S;
      double* dst = sW + (5 * dir + v) * S;
      if (dir == 0) lm_tile<0, false>(aD, src, dst, T, lane);
      else if (dir == 1) lm_tile<1, false>(aD, src, dst, T, lane);
      else lm_tile<2, false>(aD, src, dst, T, lane);
    }
  }
  __syncthreads();
  if (valid) {
    double u[5], dx[5], de[5], dz[5];  // U again from L1/L2 rather than held across the products
#pragma unroll
    for (int v = 0; v < 5; ++v) u[v] = Ug[v];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      dx[v] = sW[v * S + slot];
      de[v] = sW[(5 + v) * S + slot];
      dz[v] = sW[(10 + v) * S + slot];
    }
    // the fluxes overwrite this node's derivative slots only: every other thread reads its own slot
    lv_node_fluxes<NP, LIFT, LV>(P, e, t, i, j, k, u, dx, de, dz, sE2S, sW, S, slot);
  }
  __syncthreads();
  // viscous volume integral: R = D_hat f~ (xi) + D_hat g~ (eta) + D_hat h~ (zeta), one direction per pass
  const double aH[2] = {P.basis->Dhat[ar], P.basis->Dhat[ar + 4]};
  if (valid) {
#pragma unroll 1
    for (int w = warp; w < 32; w += 16) lm_tile<0, false>(aH, sW + (w >> 3) * S, sV + (w >> 3) * S, w & 7, lane);
  }
  __syncthreads();
  if (valid) {
#pragma unroll 1
    for (int w = warp; w < 32; w += 16)
      lm_tile<1, true>(aH, sW + (4 + (w >> 3)) * S, sV + (w >> 3) * S, w & 7, lane);
  }
  __syncthreads();
  if (valid) {
#pragma unroll 1
    for (int w = warp; w < 32; w += 16)
      lm_tile<2, true>(aH, sW + (8 + (w >> 3)) * S, sV + (w >> 3) * S, w & 7, lane);
  }
  __syncthreads();
  if (valid) {
    double* O = P.utvisc + (size_t)e * 4 * NP3 + t;
#pragma unroll
    for (int v = 0; v < 4; ++v) O[v * NP3] = sV[v * S + slot];
  }
}

}  // namespace fluxo
