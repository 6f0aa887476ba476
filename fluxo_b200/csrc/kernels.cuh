// sm_100a FP64 kernels of the DGSEM right-hand side and LSERK stage.
//
// Per RHS evaluation (dg/dg.f90:282-452 on one GPU, all sides inner sides):
//   Euler:          face_flux  ->  volume (split form + surface integral + Jacobian [+ RK stage])
//   Navier-Stokes:  lift_flux  ->  gradient (BR1/BR2 lifting)  ->  face_flux (+ viscous)  ->  volume (+ viscous)
// The element kernels hold one element's state, metrics and per-node auxiliaries in shared
// memory (one thread per volume node); face kernels use one thread per face point.
#pragma once
#include "common.cuh"
#include "physics_ns.cuh"
#include "volume_pairs.cuh"

namespace fluxo {

// Up to three local sides touched by volume node (i,j,k); returns the count.
__device__ __forceinline__ int boundary_sides(int i, int j, int k, int N, int* s) {
  int c = 0;
  if (i == 0) s[c++] = XI_MINUS;
  if (i == N) s[c++] = XI_PLUS;
  if (j == 0) s[c++] = ETA_MINUS;
  if (j == N) s[c++] = ETA_PLUS;
  if (k == 0) s[c++] = ZETA_MINUS;
  if (k == N) s[c++] = ZETA_PLUS;
  return c;
}

// ------------------------------------------------------------------------------------------------
// Face kernel: ProlongToFace (LGL copy) + FillFlux (Riemann, viscous average) + SurfElem scaling.
// prolongtoface.f90:43-132, fillflux.f90:41-110, riemann.f90:104-246.
// ------------------------------------------------------------------------------------------------
template <int RS, bool VISC>
__device__ __forceinline__ void face_flux_body(const KParams& P, int NP) {
  if (halted(P)) return;
  const int npts = NP * NP;
  const int spb = blockDim.x / npts;
  const int ls = threadIdx.x / npts;  // side slot in block
  const int pt = threadIdx.x - ls * npts;
  const int side = blockIdx.x * spb + ls;
  const bool valid = (ls < spb) && (side < P.nSides);
  __shared__ double s_lam[256];
  double L[5], R[5], F[5];
  double nv[3], t1[3], t2[3], se = 0.;
  int eM = 0, eS = 0, nM = 0, nS = 0;
  if (valid) {
    const int* se5 = P.s2e + 5 * side;
    eM = se5[0]; eS = se5[1];
    int lsM = se5[2], lsS = se5[3], fl = se5[4];
    const int p = pt % NP, q = pt / NP;
    nM = side_node(NP - 1, p, q, 0, lsM);
    nS = side_node(NP - 1, p, q, fl, lsS);
    // LGL: the side's volume nodes; Gauss: the interpolated face states of both sides
    const double* UM = P.uface ? P.uface + ((size_t)side * 2 * npts + pt) * 5
                               : P.U + 5 * ((size_t)eM * NP * NP * NP + nM);
    const double* US = P.uface ? P.uface + (((size_t)side * 2 + 1) * npts + pt) * 5
                               : P.U + 5 * ((size_t)eS * NP * NP * NP + nS);
    const double* g = P.facegeo + (size_t)side * 10 * npts + pt;
#pragma unroll
    for (int d = 0; d < 3; ++d) { nv[d] = g[d * npts]; t1[d] = g[(3 + d) * npts]; t2[d] = g[(6 + d) * npts]; }
    se = g[9 * npts];
    double uL[5], uR[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) { uL[v] = UM[v]; uR[v] = US[v]; }
    // RotateState (riemann.f90:218-231)
    L[0] = uL[0]; L[4] = uL[4];
    R[0] = uR[0]; R[4] = uR[4];
    L[1] = uL[1] * nv[0] + uL[2] * nv[1] + uL[3] * nv[2];
    L[2] = uL[1] * t1[0] + uL[2] * t1[1] + uL[3] * t1[2];
    L[3] = uL[1] * t2[0] + uL[2] * t2[1] + uL[3] * t2[2];
    R[1] = uR[1] * nv[0] + uR[2] * nv[1] + uR[3] * nv[2];
    R[2] = uR[1] * t1[0] + uR[2] * t1[1] + uR[3] * t1[2];
    R[3] = uR[1] * t2[0] + uR[2] * t2[1] + uR[3] * t2[2];
  }
  double lmm = 0.;
  if constexpr (riemann_needs_side_max<RS>()) {
    s_lam[threadIdx.x] = valid ? lambda_max_pair(P, L, R) : 0.;
    __syncthreads();
    if (valid) {
      const double* b = s_lam + ls * npts;
      for (int z = 0; z < npts; ++z) lmm = fmax(lmm, b[z]);
    }
  }
  if (!valid) return;
  riemann_rotated<RS>(P, L, R, lmm, F);
  // RotateFluxBack (riemann.f90:235-246)
  double f2 = F[1], f3 = F[2], f4 = F[3];
  F[1] = nv[0] * f2 + t1[0] * f3 + t2[0] * f4;
  F[2] = nv[1] * f2 + t1[1] * f3 + t2[1] * f4;
  F[3] = nv[2] * f2 + t1[2] * f3 + t2[2] * f4;
  if constexpr (VISC) {  // riemann.f90:155-168: + 1/2 (n.F_v(L) + n.F_v(R))
    // each side's n.F_v(U, gradP trace) was formed by the lifting kernel of its element
    const double* tM = P.gtrace + ((size_t)side * 2 + 0) * 4 * npts + pt;
    const double* tS = P.gtrace + ((size_t)side * 2 + 1) * 4 * npts + pt;
#pragma unroll
    for (int v = 1; v < 5; ++v) F[v] = F[v] + 0.5 * (tM[(v - 1) * npts] + tS[(v - 1) * npts]);
  }
  double* out = P.flux + (size_t)side * 5 * npts + pt;
#pragma unroll
  for (int v = 0; v < 5; ++v) out[v * npts] = F[v] * se;
}

// One thread per face point, 128 threads per block; MINB resident blocks per SM bound the registers
// (the memory-bound face pass needs enough warps in flight to cover the DRAM latency).
template <int RS, bool VISC, int MINB = 1>
__global__ void __launch_bounds__(128, MINB) face_flux_kernel(KParams P, int NP) {
  face_flux_body<RS, VISC>(P, NP);
}

// ------------------------------------------------------------------------------------------------
// Lifting surface flux (Lifting_FillFlux br1_fillflux.f90:49-91, EvalLiftingSurfFlux flux.f90:677-716):
// lflux = 1/2 (V_slave - V_master) * SurfElem; the normal components are applied where consumed.
// ------------------------------------------------------------------------------------------------
static __global__ void lift_flux_kernel(KParams P, int NP, double* lf) {
  if (halted(P)) return;
  const int npts = NP * NP;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)P.nSides * npts) return;
  const int side = (int)(idx / npts), pt = (int)(idx - (size_t)side * npts);
  const int* se5 = P.s2e + 5 * side;
  const int p = pt % NP, q = pt / NP;
  const int nM = side_node(NP - 1, p, q, 0, se5[2]);
  const int nS = side_node(NP - 1, p, q, se5[4], se5[3]);
  const double* UM = P.uface ? P.uface + ((size_t)side * 2 * npts + pt) * 5
                             : P.U + 5 * ((size_t)se5[0] * NP * NP * NP + nM);
  const double* US = P.uface ? P.uface + (((size_t)side * 2 + 1) * npts + pt) * 5
                             : P.U + 5 * ((size_t)se5[1] * NP * NP * NP + nS);
  double uM[5], uS[5], VM[5], VS[5];
  for (int v = 0; v < 5; ++v) { uM[v] = UM[v]; uS[v] = US[v]; }
  lifting_var(P, uM, VM);
  lifting_var(P, uS, VS);
  double se = P.facegeo[(size_t)side * 10 * npts + 9 * npts + pt];
  double* o = lf + (size_t)side * 5 * npts + pt;
  for (int v = 0; v < 5; ++v) o[v * npts] = 0.5 * (VS[v] - VM[v]) * se;
}

// ------------------------------------------------------------------------------------------------
// Volume kernel: split-form volume integral (volint.f90:173-218 with EvalAdvFluxAverage3D
// flux_average.f90:198-269), viscous volume integral (volint.f90:228-271), surface integral
// (surfint.f90:177-184, :253-259), Jacobian (dg.f90:446), source (equation.f90:992-1071), and
// optionally the fused LSERK stage (timedisc.f90:452-477).
//
// One thread per volume node, EPB elements per block.  Each node's record (volume_pairs.cuh) and
// the metrics sit in shared memory.  For each direction the threads of one line evaluate every
// pair of the line exactly once (the reference's symmetric reuse, flux_average.f90:232-243):
// in round d thread p takes the pair (p, p+d mod NP); its own contribution stays in registers and
// the partner's share is shuffled to the partner's lane; after the rounds of a direction each node
// adds its sum to its shared accumulator.
//
// The partner's share of each pair flux travels by warp shuffle to the partner's lane, so a line must
// live in one warp.  Launch shape (template parameters, chosen per N by the launcher's autotuner):
// EPB elements per block and the line-to-warp schedule of the pair phase,
//   LPW = 0: thread t of an element takes node t's line position in every direction (lines are
//            contiguous in the thread index; needs NP | 32);
//   LPW > 0: LPW lines per warp, line slot s on lanes [s*G, s*G+NP) with G = 32/LPW, the other lanes
//            idle; the block then has more threads than nodes and the node phases use the first
//            EPB*NP^3 threads.
// Every schedule adds the same terms in the same order; the shapes are separate instantiations,
// though, and the compiler may fuse a different product of an a*b + c*d into a multiply-add in each,
// so shapes agree to roundoff (one process uses one shape per N, flux and viscosity, so batched and
// single solves stay bit-identical).
// ------------------------------------------------------------------------------------------------
template <int NP>
__host__ __device__ constexpr int vol_epb() { return (256 / (NP * NP * NP)) > 0 ? (256 / (NP * NP * NP)) : 1; }

template <int NP, int EPB, int LPW, int MINB_ = 0>
struct VolShape {
  static constexpr int NP3 = NP * NP * NP, NPT = NP * NP;
  static constexpr int WPE = LPW > 0 ? (NPT + LPW - 1) / LPW : 0;  // warps per element (LPW > 0)
  static constexpr int THREADS = LPW > 0 ? EPB * WPE * 32 : EPB * NP3;
  // resident blocks per SM the register allocation must allow
  static constexpr int MINB = MINB_ > 0 ? MINB_ : (THREADS > 512 ? 1 : 2);
};

// Padded slot of node n in the shared record/accumulator arrays: one spare slot every 16 nodes
// spreads the eta- and zeta-lines (node strides NP and NP^2) over the shared-memory banks.
__host__ __device__ constexpr int vol_slot(int n) { return n + (n >> 4); }

// The Euler / Navier-Stokes kernel's node padding per (N+1, lines per warp): chosen with a lane-by-
// lane model of the pair rounds (own and partner records and accumulators of all three directions)
// so that a warp's 8-byte accesses need the minimum number of shared wavefronts (one spare slot
// every 16 nodes needs 1.6-2x as many): N+1 = 8 contiguous, 4 contiguous, 5/6/7 with 4 lines per
// warp and 3 with 8 lines per warp are conflict-free (7: 1.04, 3: 1.08); the other schedules keep
// the 16-node padding.
template <int NP, int LPW = 0>
__host__ __device__ constexpr int vol_pad(int n) {
  return (NP == 8 && LPW == 0)   ? n + 2 * (n >> 4) + 2 * (n >> 6)
         : (NP == 4 && LPW == 0) ? n + 4 * (n >> 4)
         : (NP == 5 && LPW == 4) ? n + n / 5 + 5 * (n / 25)
         : (NP == 6 && LPW == 4) ? n + 2 * (n / 36)
         : (NP == 7 && LPW == 4) ? n + n / 49
         : (NP == 3 && LPW == 8) ? n + 2 * (n >> 4)
                                 : vol_slot(n);
}

template <int NP>
__host__ __device__ constexpr int vol_slots() { return vol_slot(NP * NP * NP - 1) + 1; }
template <int NP, int LPW = 0>
__host__ __device__ constexpr int vol_pad_slots() { return vol_pad<NP, LPW>(NP * NP * NP - 1) + 1; }

template <int NP, int VF, int EPB = vol_epb<NP>(), int LPW = 0>
__host__ __device__ constexpr size_t vol_smem_bytes() {
  return sizeof(double) * (size_t)(2 * NP * NP + EPB * (VolRec<VF>::RS + 5) * vol_pad_slots<NP, LPW>());
}

template <int NP, int VF, bool VISC, int EPB, int LPW, int MINB, int OWNSM>
__global__ void __launch_bounds__(VolShape<NP, EPB, LPW>::THREADS, VolShape<NP, EPB, LPW, MINB>::MINB)
volume_kernel(KParams P) {
  if (halted(P)) return;
  constexpr int NP3 = NP * NP * NP, N = NP - 1, NPT = NP * NP;
  constexpr int RS = VolRec<VF>::RS, NQ = VolRec<VF>::NQ;
  static_assert(LPW > 0 ? (32 / LPW >= NP) : (32 % NP == 0), "a line must fit its lanes of one warp");
  extern __shared__ double smem[];
  double* sDvs = smem;         // Dvolsurf(i,l) at [i*NP+l]
  double* sDhat = sDvs + NPT;  // D_hat(i,l)
  // node phases: thread -> (element slot eb, node t); with PACK the threads past EPB*NP3 idle
  const bool nodeThread = threadIdx.x < EPB * NP3;
  const int eb = nodeThread ? threadIdx.x / NP3 : 0, t = nodeThread ? threadIdx.x - eb * NP3 : 0;
  const int e = blockIdx.x * EPB + eb;
  const bool valid = nodeThread && e < P.nElems;
  constexpr int NS = vol_pad_slots<NP, LPW>();
  double* rec = sDhat + NPT + (size_t)eb * (RS + 5) * NS;  // [slot][RS]
  double* acc = rec + (size_t)RS * NS;                     // [slot][5]
  for (int z = threadIdx.x; z < NPT; z += blockDim.x) {
    sDvs[z] = P.basis->Dvs[z];
    sDhat[z] = P.basis->Dhat[z];
  }
  __shared__ int sE2S[EPB][12];  // the element's ElemToSide (side, flip per local side)
  if (P.pfTiles > 0 && threadIdx.x == 0) {  // the tile one wave ahead: its inputs into L2
    const size_t en = ((size_t)blockIdx.x + P.pfTiles) * EPB;
    if (en < (size_t)P.nElems) {
      const size_t ne = ((size_t)P.nElems - en < (size_t)EPB ? (size_t)P.nElems - en : (size_t)EPB) * NP3;
      prefetch_l2_bulk(P.U + 5 * en * NP3, 5 * ne * sizeof(double));
      prefetch_l2_bulk(P.metrics + 9 * en * NP3, 9 * ne * sizeof(double));
      prefetch_l2_bulk(P.sJ + en * NP3, ne * sizeof(double));
      if (VISC) prefetch_l2_bulk(P.utvisc + 4 * en * NP3, 4 * ne * sizeof(double));
      if (P.stage > 1) prefetch_l2_bulk(P.UtTmp + 5 * en * NP3, 5 * ne * sizeof(double));
    }
  }
  double u[5];
  if (valid) {
    for (int z = t; z < 12; z += NP3) sE2S[eb][z] = P.e2s[12 * (size_t)e + z];  // NP3 = 8 for N = 1
    const double* Ug = P.U + 5 * ((size_t)e * NP3 + t);
#pragma unroll
    for (int v = 0; v < 5; ++v) u[v] = Ug[v];
    // the epilogue's operands are needed only after the pair loops: start their way to L2 now
    prefetch_l2(P.sJ + (size_t)e * NP3 + t);
    if (P.stage > 1) prefetch_l2(P.UtTmp + 5 * ((size_t)e * NP3 + t));
    if constexpr (VISC) {
#pragma unroll
      for (int v = 0; v < 4; ++v) prefetch_l2(P.utvisc + (size_t)e * 4 * NP3 + v * NP3 + t);
    }
    double* r = rec + vol_pad<NP, LPW>(t) * RS;
    make_record<VF>(P, u, r);
    const double* Mg = P.metrics + (size_t)e * 9 * NP3 + t;
#pragma unroll
    for (int c = 0; c < 9; ++c) r[VolRec<VF>::MO + c] = (VF == 0 ? 1.0 : 0.5) * Mg[c * NP3];  // half metrics
#pragma unroll
    for (int v = 0; v < 5; ++v) acc[vol_pad<NP, LPW>(t) * 5 + v] = 0.;
  }
  __syncthreads();
  // split-form volume integral, line by line
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
    double* prec = sDhat + NPT + (size_t)pe * (RS + 5) * NS;
    double* pacc = prec + (size_t)RS * NS;
#pragma unroll 1
    for (int dir = 0; dir < 3; ++dir) {
      const int stride = dir == 0 ? 1 : (dir == 1 ? NP : NPT);
      const int base = dir == 0 ? NP * (la + NP * lb) : (dir == 1 ? la + NPT * lb : la + NP * lb);
      const int own = base + p * stride, os = vol_pad<NP, LPW>(own);
      // own record: held in registers for all rounds, or (OWNSM) read from shared memory in every
      // round, which frees 2*(NQ+3) registers
      double ro[NQ], mo[3], racc[5] = {0., 0., 0., 0., 0.};
      if (!OWNSM && lv) {
        load_rec<VF>(prec + os * RS, ro);
        load_metric<VF>(prec + os * RS, dir, mo);
      }
      const double* rOwn = OWNSM ? prec + os * RS : ro;
      const double* mOwn = OWNSM ? prec + os * RS + VolRec<VF>::MO + 3 * dir : mo;
#pragma unroll
      for (int d = 1; d <= NP / 2; ++d) {
        const bool active = lv && (2 * d < NP || p < d);
        int q = p + d;
        if (q >= NP) q -= NP;
        double F[5] = {0., 0., 0., 0., 0.};
        if (active) {
          // the partner's record is read in place (the log-mean logarithms only when needed)
          const double* rq = prec + vol_pad<NP, LPW>(base + q * stride) * RS;
          pair_flux<VF>(P, rOwn, rq, mOwn, rq + VolRec<VF>::MO + 3 * dir, F);
        }
        const double dOwn = sDvs[p * NP + q], dPart = sDvs[q * NP + p];
        int src = p - d;
        if (src < 0) src += NP;
        // An inactive lane has F = 0, so its own share and the share it sends are zeros; a lane that
        // receives nothing in the last round (2d = NP, p < d) gets the zero of an inactive sender.
        // Hence no selects: the sums are the same (up to the sign of an exact zero).
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          racc[v] = fma(dOwn, F[v], racc[v]);
          racc[v] += __shfl_sync(0xffffffffu, dPart * F[v], (lbase + src) & 31);
        }
      }
      if (lv) {
#pragma unroll
        for (int v = 0; v < 5; ++v) pacc[os * 5 + v] += racc[v];
      }
      __syncthreads();
    }
  }
  double ut[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) ut[v] = valid ? acc[vol_pad<NP, LPW>(t) * 5 + v] : 0.;
  if (!valid) return;
  if (P.nfvse) {  // VolInt_NFVSE (nfvse.f90:475-565): blend with alpha * F_FV of the subcell FV kernel
    const double a = P.alpha[e];
    const double* FV = P.fv + (size_t)e * 5 * NP3 + t;
    if (P.nfvseCorr) {  // F_FV of every element; FFV_m_FDG = (F_FV - Ut) (-sJ) for the correction
      const double sjn = P.sJ[(size_t)e * NP3 + t];
      double* FF = P.ffvmfdg + 5 * ((size_t)e * NP3 + t);
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        const double f = FV[v * NP3];
        FF[v] = (f - ut[v]) * (-sjn);
        ut[v] = (1. - a) * ut[v] + a * f;
      }
    } else if (a > 4.440892098500626e-16) {
#pragma unroll
      for (int v = 0; v < 5; ++v) ut[v] = (1. - a) * ut[v] + FV[v * NP3];
    }
  }
  if constexpr (VISC) {  // viscous volume integral (volint.f90:228-271), computed by the lifting kernel
    const double* V = P.utvisc + (size_t)e * 4 * NP3 + t;
#pragma unroll
    for (int v = 0; v < 4; ++v) ut[1 + v] += V[v * NP3];
  }
  if (P.utsurf) {  // Gauss nodes: the surface integral of every node, formed by the surface kernel
    const double* S = P.utsurf + (size_t)e * 5 * NP3 + t;
#pragma unroll
    for (int v = 0; v < 5; ++v) ut[v] += S[v * NP3];
  } else {  // surface integral at the boundary nodes (LGL)
    const int i = t % NP, j = (t / NP) % NP, k = t / NPT;
    int sides[3];
    const int ns = boundary_sides(i, j, k, N, sides);
    const double lh = P.basis->LhatM0;
    for (int z = 0; z < ns; ++z) {
      const int s = sides[z], side = sE2S[eb][2 * (s - 1)], flip = sE2S[eb][2 * (s - 1) + 1];
      const int pt = node_side_point(N, s, flip, i, j, k);
      const double* F = P.flux + (size_t)side * 5 * NPT + pt;
      const double sg = (flip == 0) ? lh : -lh;
#pragma unroll
      for (int v = 0; v < 5; ++v) ut[v] += sg * F[v * NPT];
    }
  }
  // Ut = -Ut*sJ  (+ source)
  const double sj = P.sJ[(size_t)e * NP3 + t];
  const double tStage = P.dtDev ? (P.dtDev[1] + P.rkC * P.dtDev[0]) : P.t;
#pragma unroll
  for (int v = 0; v < 5; ++v) ut[v] = ut[v] * (-sj);
  if (P.source) {  // CalcSource CASE(4), equation.f90:1000-1024
    const double* x = P.xGP + 3 * ((size_t)e * NP3 + t);
    double arg = P.srcOmega * (x[0] + x[1] + x[2] - tStage);
    double c = cos(arg), sn = sin(arg), s2 = 2. * sn * c;
    ut[0] += P.srcTmp[0] * c;
    double mm = P.srcTmp[1] * c + P.srcTmp[2] * s2;
    ut[1] += mm; ut[2] += mm; ut[3] += mm;
    ut[4] += P.srcTmp[3] * c + P.srcTmp[4] * s2 + P.srcTmp[5] * sn;
  }
  const size_t o = 5 * ((size_t)e * NP3 + t);
  if (P.stage == 0) {
#pragma unroll
    for (int v = 0; v < 5; ++v) P.Ut[o + v] = ut[v];
  } else {
    // LSERK-2reg stage: Ut_tmp = Ut - A*Ut_tmp (stage 1: Ut_tmp = Ut); U = U + b*dt*Ut_tmp
    const double dt = stage_dt(P, e);
    const double bdt = P.rkB * dt;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      double tmp = (P.stage == 1) ? ut[v] : ut[v] - P.UtTmp[o + v] * P.rkA;
      P.UtTmp[o + v] = tmp;
      P.U[o + v] = u[v] + tmp * bdt;
    }
  }
}

// ------------------------------------------------------------------------------------------------
// CALCTIMESTEP (navierstokes/calctimestep.f90:39-170): per-element max eigenvalues, global min dt,
// error code of the first bad element (last bad node in it).  dtBits holds the double bits of
// the minimum (atomicMin on the bit pattern of non-negative doubles); errKey = elem*8 + errType.
// ------------------------------------------------------------------------------------------------
template <int NP, bool VISC>
__global__ void __launch_bounds__(512) timestep_kernel(KParams P, unsigned long long* dtBits, int* errKey) {
  if (halted(P)) return;
  constexpr int NP3 = NP * NP * NP;
  constexpr int EPB = (256 / NP3) > 0 ? (256 / NP3) : 1;
  constexpr int RSTART = (NP3 > 256) ? 256 : (NP3 > 128) ? 128 : (NP3 > 64) ? 64 : (NP3 > 32) ? 32 : (NP3 > 16) ? 16 : (NP3 > 8) ? 8 : 4;
  __shared__ double s_l[EPB][6][NP3 % 32 == 0 ? 1 : NP3];
  __shared__ int s_err[EPB];
  const int eb = threadIdx.x / NP3, n = threadIdx.x - eb * NP3;
  const int e = blockIdx.x * EPB + eb;
  const bool valid = e < P.nElems;
  if (n == 0) s_err[eb] = -1;
  __syncthreads();
  double lam[6] = {1e-12, 1e-12, 1e-12, 1e-12, 1e-12, 1e-12};
  int code = 0;
  if (valid) {
    const double* U = P.U + 5 * ((size_t)e * NP3 + n);
    double u[5];
    for (int v = 0; v < 5; ++v) u[v] = U[v];
    if (isnan(u[0])) code = 1;
    double sRho = 1. / u[0];
    double vv[3] = {u[1] * sRho, u[2] * sRho, u[3] * sRho};
    double p = P.kappaM1 * (u[4] - 0.5 * u[0] * (vv[0] * vv[0] + vv[1] * vv[1] + vv[2] * vv[2]));
    if (p <= 0.) code = 2;
    double c = sqrt(P.kappa * p * sRho);
    const double* M = P.metrics + (size_t)e * 9 * NP3 + n;
    const double sj = P.sJ[(size_t)e * NP3 + n];
    double mu = 0.;
    if (VISC) mu = sRho * P.KappasPrMax * visc_mu(P, p, sRho);
    for (int d = 0; d < 3; ++d) {
      double m0 = M[(3 * d + 0) * NP3], m1 = M[(3 * d + 1) * NP3], m2 = M[(3 * d + 2) * NP3];
      lam[d] = sj * (fabs(m0 * vv[0] + m1 * vv[1] + m2 * vv[2]) + c * sqrt(m0 * m0 + m1 * m1 + m2 * m2));
      if (VISC) {
        double a = m0 * sj, b = m1 * sj, cc = m2 * sj;
        lam[3 + d] = mu * (a * a + b * b + cc * cc);
      }
    }
  }
  // per-element max (fmax is exact, so the order of the reduction does not change the result)
  if (code != 0) atomicMax(&s_err[eb], n * 8 + code);
  if constexpr (NP3 % 32 == 0) {  // whole warps per element: shuffles, then one value per warp
    constexpr int WPE = NP3 / 32;
    __shared__ double s_w[EPB * WPE][6];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int d = 0; d < 6; ++d) lam[d] = fmax(lam[d], __shfl_xor_sync(0xffffffffu, lam[d], o));
    if ((threadIdx.x & 31) == 0)
#pragma unroll
      for (int d = 0; d < 6; ++d) s_w[threadIdx.x >> 5][d] = lam[d];
    __syncthreads();
    if (n == 0)
      for (int w = 1; w < WPE; ++w)
#pragma unroll
        for (int d = 0; d < 6; ++d) lam[d] = fmax(lam[d], s_w[eb * WPE + w][d]);
  } else {  // tree reduction in shared memory
    for (int d = 0; d < 6; ++d) s_l[eb][d][n] = lam[d];
    __syncthreads();
    for (int stride = RSTART; stride > 0; stride >>= 1) {
      if (n < stride && n + stride < NP3)
        for (int d = 0; d < 6; ++d) s_l[eb][d][n] = fmax(s_l[eb][d][n], s_l[eb][d][n + stride]);
      __syncthreads();
    }
    for (int d = 0; d < 6; ++d) lam[d] = s_l[eb][d][0];
  }
  if (n != 0 || !valid) return;
  int err = (s_err[eb] >= 0) ? (s_err[eb] & 7) : 0;
  double dtE = P.CFLScale * 2. / (lam[0] + lam[1] + lam[2]);
  if (isnan(dtE)) err = 3;
  if (VISC) {
    double dtV = P.DFLScale * 4. / (lam[3] + lam[4] + lam[5]);
    if (isnan(dtV)) err = 4;
    dtE = fmin(dtE, dtV);
  }
  reduce_timestep(P, e, dtE, err, dtBits, errKey);
}

}  // namespace fluxo
