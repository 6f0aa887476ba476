// Shared definitions of the sm_100a FP64 DGSEM kernels.
//
// Device layouts (per handle, all FP64 unless noted):
//   U, Ut, UtTmp   [elem][node][var]            var fastest = the reference's U(nVar,i,j,k,iElem)
//   metrics        [elem][9][node]              Ja^1 (x,y,z), Ja^2 (x,y,z), Ja^3 (x,y,z), node fastest
//   sJ             [elem][node]
//   facegeo        [side][10][pt]               nx,ny,nz, t1x..t1z, t2x..t2z, SurfElem; pt = p + (N+1)*q
//   flux           [side][var][pt]              Flux_master*SurfElem (slave flux is the same value)
//   lflux          [side][var][pt]              lifting surface flux 0.5*(V_slave-V_master)*SurfElem
//   grad           [elem][node][3][var]         primitive gradients (x,y,z) of Navier-Stokes
//   s2e            [side][5]                    SideToElem, 0-based elements (-1 none)
//   e2s            [elem][6][2]                 ElemToSide, 0-based side ids
// node = i + (N+1)*(j + (N+1)*k).
#pragma once
#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

#include "side_index.h"

#define FLUXO_NPMAX 9  // N <= 8

namespace fluxo {

// local side ids of the reference (src/defines.h:67-72)
enum { ZETA_MINUS = 1, ETA_MINUS = 2, XI_PLUS = 3, ETA_PLUS = 4, XI_MINUS = 5, ZETA_PLUS = 6 };

// Per-N operator tables, filled on the host from the LGL basis (dg/dg.f90:181-252).
struct BasisTables {
  double Dvs[FLUXO_NPMAX * FLUXO_NPMAX];   // Dvolsurf(i,l) at [i*NP+l], diagonal forced to 0
  double Dhat[FLUXO_NPMAX * FLUXO_NPMAX];  // D_hat(i,l) at [i*NP+l]
  double D[FLUXO_NPMAX * FLUXO_NPMAX];     // D(i,l) at [i*NP+l]
  double LhatM0;                           // L_HatMinus(0)
  double wGP[FLUXO_NPMAX];
  double xGP[FLUXO_NPMAX];                 // LGL (or Gauss) nodes
  // Gauss nodes (PP_NodeType = 1): the face interpolation L_Minus(l) and L_HatMinus(l) = L_Minus(l)/w(l),
  // l counted from the side (prolongtoface.f90:103-132, surfint.f90:118-175); zero for LGL
  double Lminus[FLUXO_NPMAX];
  double LhatMinus[FLUXO_NPMAX];
  int gauss;
};

// Everything a kernel needs, passed by value.
struct KParams {
  int nElems, nSides;
  // state
  double* U;
  double* Ut;
  double* UtTmp;
  double* grad;           // volume gradients [elem][node][3][var], written only when non-null
  double* utvisc;         // viscous volume integral [elem][4][node] (momentum and energy)
  // geometry
  const double* metrics;
  const double* sJ;
  const double* facegeo;
  const double* xGP;      // Elem_xGP [elem][node][3] or null
  const int* s2e;
  const int* e2s;
  // face buffers
  double* flux;
  double* lflux;
  double* gtrace;         // face traces of the viscous flux: n.F_v(U, gradP trace) of the master / slave
                          // side [side][master|slave][4 (Navier-Stokes) or 7 (MHD)][pt]
  const BasisTables* basis;
  // physics constants (navierstokes/equation.f90:162-260)
  double kappa, kappaM1, sKappaM1, kappaP1, sKappa, R, s23, KappasPr, mu0, Ts, sTref, ExpoSuth, cSuth, ExpoPow;
  double etaBR2;
  int visc, lifting_var, lifting;
  int volumeFlux;         // VolumeFlux id (the Roe solver's baseline flux depends on it)
  // source term (IniExactFunc 4)
  int source;
  double srcOmega, srcTmp[6];
  // time stepping
  double t;               // stage time (host value) ...
  const double* dtDev;    // ... or device dt (time_disc loop): dtDev[0]=dt, dtDev[1]=t
  double dt;
  double rkA, rkB, rkC;   // A_s, b_s, c_s of the current stage
  int stage;              // 1-based stage; 0 = plain DGTimeDerivative (write Ut)
  const int* haltFlag;    // device flag: nonzero -> kernels return at once
  double CFLScale, DFLScale, KappasPrMax;
  // MHD with GLM (equation/mhd/equation.f90:134-285); the state has 9 variables
  double smu_0, s2mu_0, kappaM2, etasmu_0, muMHD, glmScr;
  int noncons;            // NONCONS: 0 off, 1 Powell, 2 Brackbill, 3 Janhunen
  int ncGLM;              // PP_NC_GLM
  int parabolic;          // resistive / viscous MHD (lifting + viscous fluxes)
  double glmCh;           // GLM_ch of this RHS (host value) ...
  const double* chDev;    // ... or from device memory (time_disc loop)
  // NFVSE shock capturing (shockcapturing/nfvse.f90): blending of the volume integral with the
  // first-order subcell finite-volume one on the elements whose alpha > 2*EPSILON
  int nfvse;
  double* alpha;          // [elem] blending coefficient after propagation (kept for TimeRelFactor)
  double* alphaRaw;       // [elem] before propagation
  int* blendList;         // [elem] blended elements of this RHS, count in *blendCount
  int* blendCount;
  double* fv;             // [elem][var][node] alpha * F_FV of the blended elements
  const double* sVdm;     // nodal -> modal Legendre coefficients [m][i]
  int computeAlpha, indicatorQuantity, propSweeps;
  int subFV, reconsBoundaries;       // SubFVMethod (1 first order, 2 TVD, 3 TVD-ES, 4 TVD-Fjordholm),
                                     // ReconsBoundaries (1..3)
  double threshold, sharpness, alphaMax, alphaMin, propFactor, timeRelFactor, shockBlendCoef;
  // NFVSE_CORR (Apply_NFVSE_Correction, nfvse.f90:1688-1883): F_FV of every element, and
  // FFV_m_FDG = (F_FV - Ut_DG) (-sJ) [elem][node][var] written by the volume kernel
  int nfvseCorr;
  double* ffvmfdg;
  double positCorrFactor;
  int positMaxIter;
  // element kernels: blocks resident at once on the device (0: no prefetch); block b prefetches the
  // tile of block b + pfTiles into L2
  int pfTiles;
  // Gauss nodes: face states of ProlongToFace_U [side][master|slave][pt][5], the surface integral with
  // the split-form correction [elem][5][node] (added by the volume kernel instead of the LGL surface
  // terms), SurfMetrics [elem][6][3][pt] (mesh_vars.f90:67-70); all null for LGL
  double* uface;
  double* utsurf;
  const double* surfMet;
  // batched solves: the elements of many independent instances in one launch; each instance has
  // its own time step (null for a single solve)
  const int* elemInst;               // [elem] index of the element's instance in the arrays below
  const double* instDt;              // [instance] dt of the current step (0 once finished)
  unsigned long long* instDtBits;    // [instance] CALCTIMESTEP minimum (bits of a double)
  int* instErrKey;                   // [instance] elem*8+errType of the first bad element
};

__device__ __forceinline__ bool halted(const KParams& P) { return P.haltFlag && *P.haltFlag != 0; }

// dt of the LSERK stage update of element e (host value, device time loop, or per instance)
__device__ __forceinline__ double stage_dt(const KParams& P, int e) {
  if (P.elemInst) return P.instDt[P.elemInst[e]];
  return P.dtDev ? P.dtDev[0] : P.dt;
}

// global minimum of CALCTIMESTEP (one solve) or the minimum of the element's instance (batch)
__device__ __forceinline__ void reduce_timestep(const KParams& P, int e, double dtE, int err,
                                                unsigned long long* dtBits, int* errKey) {
  if (P.elemInst) {
    const int inst = P.elemInst[e];
    dtBits = P.instDtBits + inst;
    errKey = P.instErrKey + inst;
  }
  if (err != 0) atomicMin(errKey, e * 8 + err);
  else atomicMin(dtBits, (unsigned long long)__double_as_longlong(dtE));
}
__device__ __forceinline__ double glm_ch(const KParams& P) { return P.chDev ? *P.chDev : P.glmCh; }

// Asks the memory system to bring the line holding p into L2 (no register result, no fault on the
// caller's side: only addresses inside live allocations are passed).
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// One bulk prefetch of the 16-byte-aligned interior of [p, p + bytes) into L2 (a TMA-unit request of
// up to 4 GB; nothing is read into registers).  The element kernels issue it for the element one wave
// ahead, so that element's prologue reads L2 instead of DRAM.
__device__ __forceinline__ void prefetch_l2_bulk(const void* p, size_t bytes) {
  uintptr_t a = (uintptr_t)p, b = a + bytes;
  a = (a + 15) & ~(uintptr_t)15;
  b &= ~(uintptr_t)15;
  if (b > a) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((unsigned)(b - a)) : "memory");
}

// Raises kernel k's dynamic shared-memory limit to `bytes` on the current device.  The attribute
// belongs to (kernel, device), so `done` keeps one bit per device ordinal < 64 (a launcher passes a
// function-local static per kernel instantiation); concurrent first calls from several host threads
// both set the attribute, which is harmless.  Ordinals >= 64 set it on every call.
template <class K>
inline cudaError_t smem_attr_once(K* k, size_t bytes, std::atomic<unsigned long long>& done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = (dev >= 0 && dev < 64) ? (1ull << dev) : 0ull;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_acq_rel);
  return e;
}

// Blocks of kernel k (threads, dynamic shared memory) resident on the current device at once: the
// stride of the element kernels' one-wave-ahead prefetch.  Cached per device ordinal < 64 in
// `cache` (0: not known yet); 0 when the query fails, which turns the prefetch off.
template <class K>
inline int resident_blocks(K* k, int threads, size_t smem, std::atomic<int>* cache) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (dev >= 0 && dev < 64) {
    const int c = cache[dev].load(std::memory_order_relaxed);
    if (c > 0) return c;
  }
  int perSM = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k, threads, smem) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  const int r = perSM * sms;
  if (dev >= 0 && dev < 64 && r > 0) cache[dev].store(r, std::memory_order_relaxed);
  return r;
}

}  // namespace fluxo
