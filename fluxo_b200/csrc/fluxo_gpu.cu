// C ABI of the B200 DGSEM right-hand side / LSERK step (include/fluxo_gpu.h).
// Host orchestration only: buffers, geometry repacking, kernel sequencing per RHS and per RK stage,
// and the device-resident TimeDisc loop.  No numerical work happens on the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/fluxo_gpu.h"
#include "common.cuh"
#include "host_basis.h"
#include "host_setup.h"
#include "host_copy.h"
#include "launch.h"
#include "time_disc.h"
#include "vol_shapes.h"

using namespace fluxo;

namespace {

// State of the device-resident time loop (one per handle, in device memory).
struct TDState {
  double dt;                   // current step size (dtDev[0])
  double t;                    // time at the start of the current step (dtDev[1])
  double tEnd;
  unsigned long long dtBits;   // CALCTIMESTEP result (bits of a non-negative double)
  int errKey;                  // elem*8+errType of the first bad element, INT_MAX if none
  int iter, maxIter, last, done, err;
  int halt;                    // kernels return at once when nonzero
  int glm;                     // MHD: GLM_ch follows every CALCTIMESTEP
  double ch, glmScale, glmDtch1;  // GLM_ch of the current step, GLM_scale, GLM_dtch1
};

__global__ void td_glm_kernel(TDState* s, int glm, double ch, double scale, double dtch1) {
  s->glm = glm; s->ch = ch; s->glmScale = scale; s->glmDtch1 = dtch1;
}

__global__ void td_begin_kernel(TDState* s, double t, double tEnd, int maxIter) {
  s->t = t; s->tEnd = tEnd; s->dt = 0.; s->iter = 0; s->maxIter = maxIter;
  s->last = 0; s->done = 0; s->err = 0;
  s->halt = (t >= tEnd || maxIter == 0) ? 1 : 0;
  if (s->halt) s->done = 1;
  s->dtBits = 0x7FF0000000000000ull;
  s->errKey = INT_MAX;
}

// after CALCTIMESTEP: error check and dt clipping to tEnd (timedisc.f90:289-317)
__global__ void td_finalize_kernel(TDState* s) {
  if (s->halt) return;
  if (s->errKey != INT_MAX) { s->err = s->errKey & 7; s->halt = 1; return; }
  double dt = __longlong_as_double((long long)s->dtBits);
  if (s->glm) s->ch = s->glmScale * (s->glmDtch1 / dt);  // mhd/calctimestep.f90:176, before clipping
  s->last = 0;
  if (s->tEnd - s->t <= dt * (1. + 1.e-4)) { dt = s->tEnd - s->t; s->last = 1; }
  s->dt = dt;
}

// after the stages: t += dt, iteration count, termination (timedisc.f90:329-359)
__global__ void td_advance_kernel(TDState* s) {
  if (s->halt) return;
  if (s->errKey != INT_MAX) { s->err = s->errKey & 7; s->halt = 1; return; }  // NFVSE_CORR during the step
  s->t = s->t + s->dt;
  s->iter += 1;
  if (s->last || (s->maxIter > 0 && s->iter >= s->maxIter)) { s->done = 1; s->halt = 1; }
  s->dtBits = 0x7FF0000000000000ull;
  s->errKey = INT_MAX;
}

__global__ void dt_reset_kernel(unsigned long long* bits, int* key) {
  *bits = 0x7FF0000000000000ull;
  *key = INT_MAX;
}

// Stage updates of the Runge-Kutta schemes that are not fused into the volume kernel (their registers
// and combinations differ from LSERKW2's); the right-hand side of the stage was written to Ut.
//   LSERKK3 (timedisc.f90:489-542): R1 = S2, R2 = Uprev;  SSPRK2 (ssprk4-5, :560-640): R1 = r0, R2 = r1;
//   SSPRK33 (:647-687): R1 = Ut_temp.  Each line keeps the reference's operations and their order.
struct RKStageArgs {
  int type, stage, nStages;
  size_t n;
  double* U;
  const double* Ut;
  double *R1, *R2;
  double b, g1, g2, g3, delta, a, d, e;
  const double* dtDev;  // device time loop: dt in dtDev[0] ...
  double dt;            // ... or the host value
  const int* halt;
  int part;             // SSPRK2 with NFVSE_CORR: 1 the U update only, 2 the r1 update only (after the
                        // correction of U and Ut); 0 both
};

// before the first stage's right-hand side: LSERKK3 Uprev = S2 = U, SSPRK2 r0 = U
__global__ void rk_begin_kernel(RKStageArgs A) {
  if (A.halt && *A.halt) return;
  for (size_t z = (size_t)blockIdx.x * blockDim.x + threadIdx.x; z < A.n; z += (size_t)gridDim.x * blockDim.x) {
    const double u = A.U[z];
    A.R1[z] = u;
    if (A.type == RK_LSERKK3) A.R2[z] = u;
  }
}

__global__ void rk_stage_kernel(RKStageArgs A) {
  if (A.halt && *A.halt) return;
  const double dt = A.dtDev ? A.dtDev[0] : A.dt;
  const double bdt = A.b * dt;
  const int st = A.stage;
  for (size_t z = (size_t)blockIdx.x * blockDim.x + threadIdx.x; z < A.n; z += (size_t)gridDim.x * blockDim.x) {
    double u = A.U[z];
    const double ut = A.Ut[z];
    if (A.type == RK_LSERKK3) {
      if (st == 1) {
        u = u + ut * bdt;
      } else {
        const double s2 = A.R1[z] + u * A.delta;  // S2 = S2 + U*RKdelta
        A.R1[z] = s2;
        u = u * A.g1 + s2 * A.g2;                 // U = RKg1*U + RKg2*S2
        u = u + A.R2[z] * A.g3;                   // U = U + RKg3*Uprev
        u = u + ut * bdt;                         // U = U + Ut*b_dt
      }
    } else if (A.type == RK_SSPRK2) {
      if (A.part == 2) {  // r1 from the corrected U and Ut (timedisc.f90:600-604)
        if (st == 2) A.R2[z] = u * A.e;
        else if (st == 3) A.R2[z] = A.R2[z] + u * A.e;
        else if (st == 4) A.R2[z] = A.R2[z] + dt * ut * A.e;
        continue;
      }
      if (st == 1) {
        u = u + ut * bdt;
      } else if (st < A.nStages) {
        u = u * A.d + A.R1[z] * A.a + ut * bdt;
        if (A.part == 0) {
          if (st == 2) A.R2[z] = u * A.e;
          else if (st == 3) A.R2[z] = A.R2[z] + u * A.e;
          else if (st == 4) A.R2[z] = A.R2[z] + dt * ut * A.e;
        }
      } else {
        u = u * A.d + A.R1[z] * A.a + ut * bdt + A.R2[z];
      }
    } else {  // SSPRK33, cc = (-3/4, 1/4, -1/12, 2/3) times dt
      if (st == 1) {
        A.R1[z] = ut;
        u = u + ut * dt;
      } else if (st == 2) {
        const double tmp = A.R1[z];
        u = u + tmp * (-0.75 * dt) + ut * (0.25 * dt);
        A.R1[z] = tmp + ut;
      } else {
        u = u + A.R1[z] * (-1. / 12. * dt) + ut * (2. / 3. * dt);
      }
    }
    A.U[z] = u;
  }
}

}  // namespace

struct fluxo_handle {
  fluxo_cfg cfg{};
  int N = 0, NP = 0, nElems = 0, nSides = 0;
  // a partition of one solve over several handles: the first nOwn elements are this handle's, the
  // others ghost copies of the neighbours that the exchange callback refreshes
  int nOwn = 0;
  fluxo_exchange_fn xfn = nullptr;
  void* xctx = nullptr;
  int nVar = 5;                     // 5 (Euler / Navier-Stokes), 9 (MHD + GLM)
  bool mhd = false;
  double glmCh = 0., glmDtch1 = 0.;  // MHD: GLM_ch, GLM_dtch1 (from the metrics at set_mesh)
  // NFVSE: blending coefficients, list of blended elements, alpha * F_FV, modal transform
  double *dAlpha = nullptr, *dAlphaRaw = nullptr, *dAlphaTmp = nullptr, *dFV = nullptr, *dSVdm = nullptr;
  double* dFFV = nullptr;  // NFVSE_CORR: FFV_m_FDG [elem][node][var]
  // Gauss nodes: face states, surface integral, SurfMetrics (set by fluxo_gpu_set_surf_metrics)
  bool gauss = false, surfMetSet = false;
  double *dUface = nullptr, *dUtSurf = nullptr, *dSurfMet = nullptr;
  int *dBlendList = nullptr, *dBlendCount = nullptr;
  int nSMs = 148;
  bool visc = false, meshSet = false, stateSet = false, haveXGP = false;
  cudaStream_t stream = nullptr;
  BasisTables hb{};
  BasisTables* dBasis = nullptr;
  double *dU = nullptr, *dUt = nullptr, *dUtTmp = nullptr, *dGrad = nullptr, *dUtVisc = nullptr;
  double* dUReg2 = nullptr;  // second extra register of LSERKK3 / SSPRK2
  double *dMetrics = nullptr, *dsJ = nullptr, *dFaceGeo = nullptr, *dXGP = nullptr;
  double *dFlux = nullptr, *dLFlux = nullptr, *dGTrace = nullptr;
  int *dS2E = nullptr, *dE2S = nullptr;
  TDState* dTD = nullptr;
  unsigned long long* dDtBits = nullptr;
  int* dErrKey = nullptr;
  // analysis (fluxo_gpu_analyze): per-element partial sums, results, interpolation tables
  double *dAnaPartial = nullptr, *dAnaRes = nullptr, *dAnaTables = nullptr;
  int nStages = 0;
  double RKA[24]{}, RKb[24]{}, RKc[24]{};
  const RKTable* rk = nullptr;  // the scheme's table (type and the other coefficients)
  double CFLScale = 0., DFLScale = 0.;
  uint64_t launches = 0;
  std::string lastError;
  bool profiling = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof[6];
};

namespace {

// SplitMix64 (Steele, Lea, Flood 2014): the next uniform double in [0,1) of the stream `state`
double splitmix64_unit(uint64_t& state) {
  uint64_t z = (state += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  z ^= z >> 31;
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

std::mutex g_err_mutex;
std::string g_create_error;

int fail(fluxo_handle* h, int code, const std::string& msg) {
  if (h) h->lastError = msg;
  else {
    std::lock_guard<std::mutex> lk(g_err_mutex);
    g_create_error = msg;
  }
  return code;
}

int cuda_fail(fluxo_handle* h, cudaError_t e, const char* where) {
  return fail(h, FLUXO_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define FLUXO_CUDA(h, call)                                  \
  do {                                                       \
    cudaError_t _e = (call);                                 \
    if (_e != cudaSuccess) return cuda_fail((h), _e, #call); \
  } while (0)

template <class T>
int dalloc(fluxo_handle* h, T** p, size_t n) {
  if (*p) cudaFree(*p);
  *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(h, FLUXO_ENOMEM_HBM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  return FLUXO_OK;
}

// Gauss nodes (InitDGbasis with NodeType 'GAUSS', dg.f90:181-252)
void build_gauss_basis_tables(int N, BasisTables& B) {
  host::GaussBasis b(N);
  const int NP = N + 1;
  std::memset(&B, 0, sizeof(B));
  for (int i = 0; i < NP; ++i)
    for (int l = 0; l < NP; ++l) {
      B.Dvs[i * NP + l] = (i == l) ? 0. : b.Dvs[(size_t)i * NP + l];  // skew-symmetric: zero diagonal
      B.Dhat[i * NP + l] = b.Dhat[(size_t)i * NP + l];
      B.D[i * NP + l] = b.D[(size_t)i * NP + l];
    }
  B.LhatM0 = b.LhatMinus[0];
  for (int i = 0; i < NP; ++i) {
    B.wGP[i] = b.w[i]; B.xGP[i] = b.x[i];
    B.Lminus[i] = b.Lminus[i]; B.LhatMinus[i] = b.LhatMinus[i];
  }
  B.gauss = 1;
}

void build_basis_tables(int N, BasisTables& B) {
  host::LGLBasis b(N);
  const int NP = N + 1;
  std::memset(&B, 0, sizeof(B));
  for (int i = 0; i < NP; ++i)
    for (int l = 0; l < NP; ++l) {
      B.Dvs[i * NP + l] = (i == l) ? 0. : b.Dvs[(size_t)i * NP + l];  // diagonal is zero (dg.f90:232-240)
      B.Dhat[i * NP + l] = b.Dhat[(size_t)i * NP + l];
      B.D[i * NP + l] = b.D[(size_t)i * NP + l];
    }
  B.LhatM0 = b.LhatM0;
  for (int i = 0; i < NP; ++i) { B.wGP[i] = b.w[i]; B.xGP[i] = b.x[i]; }
}

KParams base_params(fluxo_handle* h) {
  KParams P{};
  const fluxo_cfg& c = h->cfg;
  P.nElems = h->nOwn; P.nSides = h->nSides;
  P.U = h->dU; P.Ut = h->dUt; P.UtTmp = h->dUtTmp; P.grad = nullptr; P.utvisc = h->dUtVisc;
  P.metrics = h->dMetrics; P.sJ = h->dsJ; P.facegeo = h->dFaceGeo; P.xGP = h->dXGP;
  P.s2e = h->dS2E; P.e2s = h->dE2S;
  P.flux = h->dFlux; P.lflux = h->dLFlux; P.gtrace = h->dGTrace;
  P.basis = h->dBasis;
  if (h->gauss) { P.uface = h->dUface; P.utsurf = h->dUtSurf; P.surfMet = h->dSurfMet; }
  fill_ns_physics(P, c);
  P.source = (c.ini_exact_func == 4 && h->haveXGP) ? 1 : 0;
  if (P.source) {  // CalcSource CASE(4) constants, equation.f90:1000-1012
    double Omega = M_PI * c.ini_frequency, A = c.ini_amplitude, km1 = c.kappa - 1.;
    double tmp[6] = {2., 2. + 2.5 * km1, A * km1, 0.5 * (9. + c.kappa * 15.) - 4., A * (3. * c.kappa - 1.),
                     h->visc ? 3. * c.mu0 * c.kappa * Omega / c.Pr : 0.};
    P.srcOmega = Omega;
    for (int z = 0; z < 6; ++z) P.srcTmp[z] = tmp[z] * A * Omega;
  }
  P.CFLScale = h->CFLScale; P.DFLScale = h->DFLScale;
  if (h->mhd) {  // mhd/equation.f90:170-209; calctimestep.f90:81-84
    P.kappaM2 = c.kappa - 2.;
    P.smu_0 = 1. / c.mu_0; P.s2mu_0 = 0.5 * P.smu_0;
    P.etasmu_0 = h->visc ? c.eta * P.smu_0 : 0.;
    P.muMHD = h->visc ? c.mu0 : 0.;
    P.KappasPrMax = P.muMHD * std::max(4. / 3., P.KappasPr);
    P.glmScr = c.glm_scr;
    P.source = (std::fabs(c.glm_scr) > 0.) ? 1 : 0;  // GLM damping in the volume kernel
    P.glmCh = h->glmCh; P.chDev = nullptr;
    P.noncons = c.noncons; P.ncGLM = c.nc_glm; P.parabolic = h->visc ? 1 : 0;
    P.mu0 = 0.; P.visc = 0;
  }
  if (c.nfvse) {  // InitNFVSE, nfvse.f90:106-260; sharpness nfvse_vars.f90:74
    P.nfvse = 1;
    P.alpha = h->dAlpha; P.alphaRaw = h->dAlphaRaw; P.blendList = h->dBlendList; P.blendCount = h->dBlendCount;
    P.fv = h->dFV; P.sVdm = h->dSVdm;
    P.computeAlpha = c.compute_alpha; P.indicatorQuantity = c.indicator_quantity; P.propSweeps = c.space_prop_sweeps;
    P.subFV = c.sub_fv_method; P.reconsBoundaries = c.recons_boundaries;
    P.threshold = (c.modal_threshold == 2) ? 0.5 * std::pow(10.0, -1.8 * std::pow((double)h->N, 0.25))
                                           : 0.5 * std::pow(10.0, -1.8 * std::pow(h->N + 1., 0.25));
    P.sharpness = std::log((1.0 - 1.e-4) / 1.e-4);
    P.alphaMax = c.alpha_max; P.alphaMin = c.alpha_min; P.propFactor = c.space_prop_factor;
    P.timeRelFactor = c.time_rel_factor; P.shockBlendCoef = c.shock_blend_coef;
    P.nfvseCorr = c.nfvse_corr ? 1 : 0; P.ffvmfdg = h->dFFV;
    P.positCorrFactor = c.posit_corr_factor; P.positMaxIter = c.posit_max_iter;
  }
  return P;
}

// Brackets one launch with CUDA events when profiling is on.
struct ProfScope {
  fluxo_handle* h;
  int kind;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(fluxo_handle* h_, int k) : h(h_), kind(k) {
    if (h->profiling) {
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      cudaEventRecord(a, h->stream);
    }
  }
  ~ProfScope() {
    if (h->profiling) {
      cudaEventRecord(b, h->stream);
      h->prof[kind].emplace_back(a, b);
    }
  }
};

// The exchange callback of a partitioned solve (a no-op without one); a failure ends the call.
int exchange(fluxo_handle* h, int what, void* a, void* b) {
  if (!h->xfn) return FLUXO_OK;
  const int r = h->xfn(h->xctx, what, (void*)h->stream, a, b);
  if (r != 0) return fail(h, FLUXO_EXCHANGE, "exchange callback failed (what = " + std::to_string(what) + ")");
  return FLUXO_OK;
}

// CalcBlendingCoefficient with PropagateBlendingCoeff (nfvse.f90:1537-1620, nfvse_mpi.f90:62-131); a
// partitioned solve exchanges the ghost elements' coefficients before every propagation sweep
int nfvse_alpha(fluxo_handle* h, const KParams& P, cudaStream_t s) {
  if (!h->xfn) {
    FLUXO_CUDA(h, launch_nfvse_alpha(h->NP, h->mhd, h->nOwn, s, P, h->dAlphaTmp));
    return FLUXO_OK;
  }
  FLUXO_CUDA(h, launch_nfvse_indicator(h->NP, h->mhd, h->nOwn, s, P));
  if (P.propSweeps <= 0) {
    FLUXO_CUDA(h, launch_nfvse_list(h->nOwn, s, P));
    return FLUXO_OK;
  }
  if (int r = exchange(h, FLUXO_XCHG_ALPHA, h->dAlphaRaw, nullptr)) return r;
  for (int sw = 1; sw <= P.propSweeps; ++sw) {
    const double* src = P.alphaRaw;
    if (sw > 1) {
      if (int r = exchange(h, FLUXO_XCHG_ALPHA, h->dAlpha, nullptr)) return r;
      FLUXO_CUDA(h, cudaMemcpyAsync(h->dAlphaTmp, h->dAlpha, sizeof(double) * h->nElems, cudaMemcpyDeviceToDevice, s));
      src = h->dAlphaTmp;
    }
    FLUXO_CUDA(h, launch_nfvse_sweep(h->nOwn, s, P, src, sw == P.propSweeps));
  }
  return FLUXO_OK;
}

// One DGTimeDerivative; stage 0 writes Ut, stage >= 1 applies the fused LSERK stage update.
int rhs(fluxo_handle* h, KParams P) {
  cudaStream_t s = h->stream;
  // a partitioned solve: the ghost elements' state from their owners (StartReceiveMPIData /
  // StartSendMPIData of U_slave, dg.f90:342-356, here whole ghost elements)
  if (int r = exchange(h, FLUXO_XCHG_STATE, h->dU, nullptr)) return r;
  if (h->mhd) {
    if (h->cfg.nfvse) {  // CalcBlendingCoefficient (dg.f90:358-361) and VolInt_NFVSE's FV part (:380-383)
      ProfScope ps(h, 5);
      if (int r = nfvse_alpha(h, P, s)) return r;
      FLUXO_CUDA(h, launch_nfvse_fv(h->cfg.riemann, h->NP, h->nOwn, h->nSMs, s, P));
      h->launches += 3 + (h->cfg.space_prop_sweeps > 1 ? 2 * (h->cfg.space_prop_sweeps - 1) : 0);
    }
    if (h->gauss) {  // ProlongToFace_U (dg.f90:458-511), entropy-projected for Derigs / FloGor (10, 12)
      if (!h->surfMetSet) return fail(h, FLUXO_ENOTREADY, "Gauss nodes: SurfMetrics not set");
      const int vf = h->cfg.volume_flux;
      ProfScope ps(h, 2);
      FLUXO_CUDA(h, launch_gauss_prolong(h->NP, vf == 10 || vf == 12, true, h->nOwn, s, P));
      h->launches += 1;
    }
    if (h->visc) {
      {
        ProfScope ps(h, 0);
        FLUXO_CUDA(h, launch_mhd_lift_flux(h->NP, h->nSides, s, P));
      }
      {
        ProfScope ps(h, 1);
        if (h->gauss) FLUXO_CUDA(h, launch_gauss_mhd_lift_visc(h->NP, h->cfg.lifting, h->nOwn, s, P));
        else FLUXO_CUDA(h, launch_mhd_lift_visc(h->NP, h->cfg.lifting, h->nOwn, s, P));
      }
      h->launches += 2;
      if (int r = exchange(h, FLUXO_XCHG_GTRACE, h->dGTrace, nullptr)) return r;  // the ghost sides' shares
    }
    {
      ProfScope ps(h, 2);
      FLUXO_CUDA(h, launch_mhd_face(h->cfg.riemann, h->visc, h->NP, h->nSides, s, P));
    }
    if (h->gauss) {  // SurfInt with the split-form correction and the non-conservative terms
      ProfScope ps(h, 2);
      FLUXO_CUDA(h, launch_gauss_surf_mhd(h->NP, h->cfg.volume_flux, h->nOwn, s, P));
      h->launches += 1;
    }
    {
      ProfScope ps(h, 3);
      const int vf = h->cfg.volume_flux;
      FLUXO_CUDA(h, (vf == 10 || vf == 12) ? launch_mhd_volume_ec(h->NP, vf, h->nOwn, s, P)
                                           : launch_mhd_volume_std(h->NP, vf, h->nOwn, s, P));
    }
    h->launches += 2;
    return FLUXO_OK;
  }
  if (h->cfg.nfvse) {  // CalcBlendingCoefficient (dg.f90:358-361) and VolInt_NFVSE's FV part (:380-383)
    ProfScope ps(h, 5);
    if (int r = nfvse_alpha(h, P, s)) return r;
    FLUXO_CUDA(h, launch_nfvse_fv_ns(h->cfg.riemann, h->NP, h->nOwn, h->nSMs, s, P));
    h->launches += 3 + (h->cfg.space_prop_sweeps > 1 ? 2 * (h->cfg.space_prop_sweeps - 1) : 0);
  }
  if (h->gauss) {  // ProlongToFace_U (dg.f90:458-511): interpolated (entropy-projected) face states
    if (!h->surfMetSet) return fail(h, FLUXO_ENOTREADY, "Gauss nodes: SurfMetrics not set");
    const int vf = h->cfg.volume_flux;
    const bool ent = vf == 5 || vf == 6 || vf == 7 || vf == 10 || vf == 32;  // equation.f90:413-455
    ProfScope ps(h, 2);
    FLUXO_CUDA(h, launch_gauss_prolong(h->NP, ent, false, h->nOwn, s, P));
    h->launches += 1;
  }
  if (h->visc) {
    {
      ProfScope ps(h, 0);
      FLUXO_CUDA(h, launch_lift_flux(h->NP, h->nSides, s, P));
    }
    {
      ProfScope ps(h, 1);
      if (h->gauss) FLUXO_CUDA(h, launch_gauss_lift_visc(h->NP, h->cfg.lifting, h->cfg.lifting_var, h->nOwn, s, P));
      else FLUXO_CUDA(h, launch_gradient(h->NP, h->nOwn, s, P));
    }
    h->launches += 2;
    // the ghost sides' shares n.F_v of the viscous face flux (the gradient traces of br1.f90:154-364)
    if (int r = exchange(h, FLUXO_XCHG_GTRACE, h->dGTrace, nullptr)) return r;
  }
  {
    ProfScope ps(h, 2);
    FLUXO_CUDA(h, launch_face_flux(h->cfg.riemann, h->visc, h->NP, h->nSides, s, P));
  }
  if (h->gauss) {  // SurfInt with the split-form correction (surfint.f90:118-175)
    ProfScope ps(h, 2);
    FLUXO_CUDA(h, launch_gauss_surf(h->NP, h->cfg.volume_flux, h->nOwn, s, P));
    h->launches += 1;
  }
  if (volume_shape(h->NP, h->cfg.volume_flux, h->visc) < 0) {  // first RHS of this (N, flux, visc)
    FLUXO_CUDA(h, tune_volume(h->NP, h->cfg.volume_flux, h->visc, h->nOwn, s, P));
    if (volume_shape_count(h->NP) > 1) h->launches += 4 * volume_shape_count(h->NP);
  }
  {
    ProfScope ps(h, 3);
    FLUXO_CUDA(h, launch_volume(h->NP, h->cfg.volume_flux, h->visc, h->nOwn, s, P));
  }
  h->launches += 2;
  return FLUXO_OK;
}

// FP64 roofline denominator: 8 independent DFMA chains per thread, all in registers.
__global__ void fp64_fma_kernel(double* out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-3 + k;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
  }
  double s = 0.;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == 1234.5678) out[threadIdx.x] = s;  // keeps the chains alive
}

// One LSERK-2reg step (timedisc.f90:424-480): host dt (dtDev == null) or device dt.
int rk_step(fluxo_handle* h, double t, double dt, const double* dtDev, const int* halt,
            const double* chDev = nullptr, int* errKey = nullptr) {
  KParams P = base_params(h);
  P.dtDev = dtDev; P.haltFlag = halt; P.dt = dt;
  P.chDev = chDev;
  // NFVSE_CORR: Apply_NFVSE_Correction after each stage update (timedisc.f90:457-473, 583-621); not
  // for SSPRK33, which the reference steps without it
  const bool corr = h->cfg.nfvse && h->cfg.nfvse_corr && h->rk->type != RK_SSPRK33;
  if (!errKey) errKey = h->dErrKey;
  if (h->rk->type != RK_LSERKW2) {  // right-hand side into Ut, then the scheme's own stage update
    RKStageArgs A{};
    A.type = h->rk->type; A.nStages = h->nStages;
    A.n = (size_t)h->nVar * h->NP * h->NP * h->NP * h->nOwn;
    A.U = h->dU; A.Ut = h->dUt; A.R1 = h->dUtTmp; A.R2 = h->dUReg2;
    A.dtDev = dtDev; A.dt = dt; A.halt = halt;
    const int grid = h->nSMs * 8;
    if (A.type != RK_SSPRK33) {
      rk_begin_kernel<<<grid, 256, 0, h->stream>>>(A);
      FLUXO_CUDA(h, cudaGetLastError());
      h->launches += 1;
    }
    for (int st = 1; st <= h->nStages; ++st) {
      P.stage = 0;
      P.rkC = h->RKc[st];
      P.t = t + dt * h->RKc[st];
      int r = rhs(h, P);
      if (r) return r;
      A.stage = st;
      A.b = h->rk->b[st];
      A.g1 = h->rk->g1[st]; A.g2 = h->rk->g2[st]; A.g3 = h->rk->g3[st]; A.delta = h->rk->delta[st];
      A.a = h->rk->A[st]; A.d = h->rk->d[st]; A.e = h->rk->e[st];
      A.part = corr ? 1 : 0;
      rk_stage_kernel<<<grid, 256, 0, h->stream>>>(A);
      FLUXO_CUDA(h, cudaGetLastError());
      h->launches += 1;
      if (corr) {
        FLUXO_CUDA(h, launch_nfvse_corr(h->NP, h->mhd, h->nOwn, h->stream, P, h->dUt, h->rk->b[st], errKey));
        h->launches += 1;
        if (st >= 2 && st <= 4 && st < h->nStages) {
          A.part = 2;
          rk_stage_kernel<<<grid, 256, 0, h->stream>>>(A);
          FLUXO_CUDA(h, cudaGetLastError());
          h->launches += 1;
        }
      }
    }
    return FLUXO_OK;
  }
  for (int st = 1; st <= h->nStages; ++st) {
    P.stage = st;
    P.rkA = h->RKA[st]; P.rkB = h->RKb[st]; P.rkC = h->RKc[st];
    P.t = t + dt * h->RKc[st];
    int r = rhs(h, P);
    if (r) return r;
    if (corr) {  // Ut is not kept by the fused stage update (the next stage recomputes it)
      FLUXO_CUDA(h, launch_nfvse_corr(h->NP, h->mhd, h->nOwn, h->stream, P, nullptr, h->RKb[st], errKey));
      h->launches += 1;
    }
  }
  return FLUXO_OK;
}

int check_ready(fluxo_handle* h) {
  if (!h) return FLUXO_EINVAL_CFG;
  if (!h->meshSet) return fail(h, FLUXO_ENOTREADY, "mesh not set");
  if (!h->stateSet) return fail(h, FLUXO_ENOTREADY, "state not set");
  FLUXO_CUDA(h, cudaSetDevice(h->cfg.device));
  return FLUXO_OK;
}

}  // namespace

namespace fluxo {
void basis_tables_for(int N, BasisTables& B) { build_basis_tables(N, B); }

// Equation constants of the Euler / Navier-Stokes kernels (navierstokes/equation.f90:162-260)
void fill_ns_physics(KParams& P, const fluxo_cfg& c) {
  P.kappa = c.kappa; P.kappaM1 = c.kappa - 1.; P.sKappaM1 = 1. / (c.kappa - 1.); P.kappaP1 = c.kappa + 1.;
  P.sKappa = 1. / c.kappa; P.volumeFlux = c.volume_flux;
  P.R = c.R; P.s23 = 2. / 3.; P.KappasPr = c.kappa / c.Pr; P.mu0 = c.mu0;
  P.visc = c.visc; P.lifting_var = c.lifting_var; P.lifting = c.lifting; P.etaBR2 = c.etaBR2;
  if (c.visc == 1) {  // equation.f90:226-233 (Sutherland constants)
    P.sTref = 1. / c.Tref; P.ExpoSuth = c.ExpoSuth; P.Ts = c.Ts * P.sTref;
    P.cSuth = std::pow(P.Ts, P.ExpoSuth) * (1 + P.Ts) / (2 * P.Ts * P.Ts);
  } else if (c.visc == 2) {  // equation.f90:236-241 (power law)
    P.ExpoPow = c.ExpoPow; P.mu0 = c.mu0 / std::pow(c.Tref, c.ExpoPow);
  }
  P.KappasPrMax = std::max(4. / 3., P.KappasPr);
}

// Runge-Kutta coefficients (index 1..nStages: RKA, RKb and RKc of the table) and the scaled CFL/DFL
// numbers of a configuration (timedisc_vars.f90:94-726, FillCFL_DFL timedisc.f90:697-741); false for an
// unknown time_disc
bool time_disc_setup(const fluxo_cfg& c, double* RKA, double* RKb, double* RKc, int* nStages, double* CFLScale,
                     double* DFLScale) {
  if (c.time_disc < 0 || c.time_disc >= kRKTableCount) return false;
  const RKTable& T = kRKTables[c.time_disc];
  *nStages = T.nStages;
  for (int k = 0; k <= T.nStages; ++k) { RKA[k] = T.A[k]; RKb[k] = T.b[k]; RKc[k] = T.c[k]; }
  const int N = c.N;
  const bool gauss = c.node_type == 1;
  const double dflLGL[10] = {4.50, 1.95, 1.18, 0.79, 0.56, 0.42, 0.32, 0.25, 0.20, 0.17};
  const double* dflAlpha = gauss ? kGaussDflAlpha : dflLGL;
  const double* cflAlpha = gauss ? kGaussCflAlpha[c.time_disc] : T.cflAlpha;
  *CFLScale = c.cfl_scale * cflAlpha[std::min(15, N) - 1] / (2. * N + 1.);
  *DFLScale = c.dfl_scale * dflAlpha[std::min(10, N) - 1] * T.relativeDFL / ((2. * N + 1.) * (2. * N + 1.));
  return true;
}

int record_unbound_error(int code, const std::string& msg) { return fail(nullptr, code, msg); }
}  // namespace fluxo

extern "C" {

int fluxo_gpu_create(const fluxo_cfg* cfg, fluxo_handle** out) {
  if (!cfg || !out) return fail(nullptr, FLUXO_EINVAL_CFG, "null argument");
  *out = nullptr;
  if (cfg->struct_size != (int)sizeof(fluxo_cfg)) return fail(nullptr, FLUXO_EINVAL_CFG, "fluxo_cfg size mismatch");
  if (cfg->N < 1 || cfg->N > 7) return fail(nullptr, FLUXO_EINVAL_CFG, "N must be in 1..7");
  if (cfg->eqn < FLUXO_EQN_EULER || cfg->eqn > FLUXO_EQN_MHD_PARABOLIC)
    return fail(nullptr, FLUXO_EINVAL_CFG, "unknown equation system");
  const bool mhd = (cfg->eqn == FLUXO_EQN_MHD || cfg->eqn == FLUXO_EQN_MHD_PARABOLIC);
  const bool parabolic = (cfg->eqn == FLUXO_EQN_NAVIERSTOKES || cfg->eqn == FLUXO_EQN_MHD_PARABOLIC);
  if (mhd) {
    if (!mhd_riemann_supported(cfg->riemann)) return fail(nullptr, FLUXO_EINVAL_CFG, "MHD Riemann solver not implemented");
    if (cfg->riemann == 5 && std::fabs(cfg->mu_0 - 1.) > 1.0e-12)  // mhd/equation.f90:343-346
      return fail(nullptr, FLUXO_EINVAL_CFG, "HLLD solver only for mu_0=1 implemented");
    if (!mhd_volume_flux_supported(cfg->volume_flux))
      return fail(nullptr, FLUXO_EINVAL_CFG, "MHD volume flux not implemented");
    if (cfg->noncons < 0 || cfg->noncons > 3) return fail(nullptr, FLUXO_EINVAL_CFG, "noncons must be 0..3");
    if (!(cfg->mu_0 > 0.)) return fail(nullptr, FLUXO_EINVAL_CFG, "mu_0 must be > 0");
    if (cfg->ini_exact_func == 4) return fail(nullptr, FLUXO_EINVAL_CFG, "MHD source terms are not implemented");
  } else {
    if (!riemann_supported(cfg->riemann)) return fail(nullptr, FLUXO_EINVAL_CFG, "Riemann solver not implemented");
    if (!volume_flux_supported(cfg->volume_flux))
      return fail(nullptr, FLUXO_EINVAL_CFG, "volume flux not implemented");
  }
  if (cfg->nfvse) {  // InitShockCapturing / InitNFVSE checks (shockcapturing.f90:82-112, nfvse.f90:120-170)
    if (cfg->N < 2) return fail(nullptr, FLUXO_EINVAL_CFG, "NFVSE needs N >= 2");
    if (cfg->compute_alpha != 1 && cfg->compute_alpha != 3 && cfg->compute_alpha != 20)
      return fail(nullptr, FLUXO_EINVAL_CFG, "ComputeAlpha must be 1 (indicator), 3 (fixed) or 20 (random, kept)");
    if (cfg->indicator_quantity < 1 || cfg->indicator_quantity > 4)
      return fail(nullptr, FLUXO_EINVAL_CFG, "ShockIndicatorQuantity must be 1..4");
    if (cfg->space_prop_sweeps < 0) return fail(nullptr, FLUXO_EINVAL_CFG, "SpacePropSweeps must be >= 0");
    if (cfg->sub_fv_method < 1 || cfg->sub_fv_method > 4) return fail(nullptr, FLUXO_EINVAL_CFG, "SubFVMethod not implemented");
    if (cfg->sub_fv_method >= 2 && (cfg->recons_boundaries < 1 || cfg->recons_boundaries > 3))
      return fail(nullptr, FLUXO_EINVAL_CFG, "ReconsBoundaries must be 1..3");
    const int rs = cfg->riemann;
    const bool matrices = mhd ? (rs == 14 || rs == 15) : (rs == 4 || rs == 44 || rs == 33);
    if (cfg->sub_fv_method >= 3 && !matrices)  // nfvse.f90:174-187
      return fail(nullptr, FLUXO_EINVAL_CFG, "SubFVMethod 3/4 need a Riemann solver with RiemannVolFluxAndDissipMatrices");
    if (cfg->nfvse_corr) {
      if (cfg->time_disc == 6 || cfg->time_disc == 7)  // timedisc_vars.f90:111-114
        return fail(nullptr, FLUXO_EINVAL_CFG, "NFVSE correction is only implemented for LSERKW2 methods and ssprk4-5");
      if (cfg->posit_max_iter < 0) return fail(nullptr, FLUXO_EINVAL_CFG, "PositMaxIter must be >= 0");
    }
  } else if (cfg->nfvse_corr) {
    return fail(nullptr, FLUXO_EINVAL_CFG, "nfvse_corr needs nfvse = 1");
  }
  if (parabolic) {
    if (cfg->lifting != 1 && cfg->lifting != 2) return fail(nullptr, FLUXO_EINVAL_CFG, "lifting must be BR1 or BR2");
    if (cfg->lifting_var < 1 || cfg->lifting_var > 3) return fail(nullptr, FLUXO_EINVAL_CFG, "lifting_var must be 1..3");
    if (cfg->visc < 0 || cfg->visc > 2) return fail(nullptr, FLUXO_EINVAL_CFG, "visc must be 0..2");
  }
  if (!(cfg->kappa > 1.)) return fail(nullptr, FLUXO_EINVAL_CFG, "kappa must be > 1");
  if (cfg->node_type != 0 && cfg->node_type != 1 && cfg->node_type != 2)
    return fail(nullptr, FLUXO_EINVAL_CFG, "node_type must be 1 (Gauss) or 2 (Gauss-Lobatto)");
  if (cfg->node_type == 1) {  // the Gauss path of this library: every equation system, no NFVSE
    if (cfg->nfvse) return fail(nullptr, FLUXO_EINVAL_CFG, "Gauss nodes: NFVSE needs the LGL subcells");
  }
  fluxo_handle* h = new fluxo_handle();
  h->cfg = *cfg;
  h->N = cfg->N; h->NP = cfg->N + 1;
  h->visc = parabolic;
  h->mhd = mhd;
  h->nVar = mhd ? 9 : 5;
  h->gauss = cfg->node_type == 1;
  if (!time_disc_setup(*cfg, h->RKA, h->RKb, h->RKc, &h->nStages, &h->CFLScale, &h->DFLScale)) {
    delete h;
    return fail(nullptr, FLUXO_EINVAL_CFG, "time_disc must be 0..9 (the TimeDiscMethod list of fluxo_cfg)");
  }
  h->rk = &kRKTables[cfg->time_disc];
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    std::string m = std::string("CUDA init: ") + cudaGetErrorString(e);
    delete h;
    return fail(nullptr, FLUXO_ECUDA, m);
  }
  if (h->gauss) build_gauss_basis_tables(h->N, h->hb);
  else build_basis_tables(h->N, h->hb);
  cudaDeviceGetAttribute(&h->nSMs, cudaDevAttrMultiProcessorCount, cfg->device);
  if (dalloc(h, &h->dBasis, 1) || dalloc(h, &h->dTD, 1) || dalloc(h, &h->dDtBits, 1) || dalloc(h, &h->dErrKey, 1) ||
      (cfg->nfvse && (dalloc(h, &h->dSVdm, (size_t)h->NP * h->NP) || dalloc(h, &h->dBlendCount, 1)))) {
    std::string m = h->lastError;
    fluxo_gpu_destroy(h);
    return fail(nullptr, FLUXO_ENOMEM_HBM, m);
  }
  if (cfg->nfvse) {  // sVdm_Leg of BuildLegendreVdm (basis.f90:196-251), indicators.f90:176-197
    std::vector<double> sv = host::legendre_modal(h->N);
    e = cudaMemcpy(h->dSVdm, sv.data(), sv.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      fluxo_gpu_destroy(h);
      return fail(nullptr, FLUXO_ECUDA, cudaGetErrorString(e));
    }
  }
  e = cudaMemcpy(h->dBasis, &h->hb, sizeof(BasisTables), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    fluxo_gpu_destroy(h);
    return fail(nullptr, FLUXO_ECUDA, cudaGetErrorString(e));
  }
  *out = h;
  return FLUXO_OK;
}

int fluxo_gpu_set_mesh(fluxo_handle* h, int nElems, int nSides, const int* S2E, const int* E2S, const double* Mf,
                       const double* Mg, const double* Mh, const double* sJ, const double* NormVec,
                       const double* TangVec1, const double* TangVec2, const double* SurfElem,
                       const double* Elem_xGP) {
  if (!h) return FLUXO_EINVAL_CFG;
  if (nElems < 1 || nSides < 1 || !S2E || !E2S || !Mf || !Mg || !Mh || !sJ || !NormVec || !TangVec1 || !TangVec2 ||
      !SurfElem)
    return fail(h, FLUXO_EINVAL_CFG, "set_mesh: missing array");
  if (h->cfg.ini_exact_func == 4 && !Elem_xGP) return fail(h, FLUXO_EINVAL_CFG, "source term needs Elem_xGP");
  FLUXO_CUDA(h, cudaSetDevice(h->cfg.device));
  const int NP = h->NP, NP3 = NP * NP * NP, NPT = NP * NP;
  // connectivity 1-based -> 0-based (checked), metrics [elem][9][node], face geometry [side][10][pt]
  std::vector<int> s2e, e2s;
  std::vector<double> met, geo;
  std::string rerr;
  if (!host::repack_mesh(h->N, nElems, nSides, S2E, E2S, Mf, Mg, Mh, NormVec, TangVec1, TangVec2, SurfElem, s2e, e2s,
                         met, geo, rerr))
    return fail(h, FLUXO_EINVAL_CFG, "set_mesh: " + rerr);
  h->nElems = nElems; h->nSides = nSides;
  h->nOwn = nElems;
  h->xfn = nullptr;
  h->xctx = nullptr;
  if (h->dAnaPartial) {  // sized by nElems at the next analysis
    cudaFree(h->dAnaPartial);
    h->dAnaPartial = nullptr;
  }
  const int NV = h->nVar;
  const size_t nU = (size_t)NV * NP3 * nElems, nF = (size_t)NV * NPT * nSides;
  const size_t nFlux = (size_t)(h->mhd ? 13 : 5) * NPT * nSides;  // MHD: + non-conservative weights
  int r = FLUXO_OK;
  if ((r = dalloc(h, &h->dU, nU)) || (r = dalloc(h, &h->dUt, nU)) || (r = dalloc(h, &h->dUtTmp, nU)) ||
      (r = dalloc(h, &h->dMetrics, met.size())) || (r = dalloc(h, &h->dsJ, (size_t)NP3 * nElems)) ||
      (r = dalloc(h, &h->dFaceGeo, geo.size())) || (r = dalloc(h, &h->dFlux, nFlux)) ||
      (r = dalloc(h, &h->dS2E, s2e.size())) || (r = dalloc(h, &h->dE2S, e2s.size())))
    return r;
  if ((h->rk->type == RK_LSERKK3 || h->rk->type == RK_SSPRK2) && (r = dalloc(h, &h->dUReg2, nU))) return r;
  if (h->visc) {
    if ((r = dalloc(h, &h->dGrad, 3 * nU)) || (r = dalloc(h, &h->dLFlux, nF)) ||
        (r = dalloc(h, &h->dUtVisc, (size_t)(h->mhd ? 7 : 4) * NP3 * nElems)) ||
        // face traces per side and point: n.F_v of both sides (MHD 7 components, Navier-Stokes 4)
        (r = dalloc(h, &h->dGTrace, (size_t)2 * (h->mhd ? 7 : 4) * NPT * nSides)))
      return r;
  }
  if (h->gauss) {
    const size_t nv = (size_t)h->nVar;
    if ((r = dalloc(h, &h->dUface, 2 * nv * NPT * nSides)) || (r = dalloc(h, &h->dUtSurf, nv * NP3 * nElems)) ||
        (r = dalloc(h, &h->dSurfMet, (size_t)18 * NPT * nElems)))
      return r;
    h->surfMetSet = false;
  }
  if (h->mhd) {  // InitTimeStep_GLM, mhd/calctimestep.f90:187-223
    double dtch1 = 1.7976931348623157e308;
    for (int e = 0; e < nElems; ++e) {
      double ml[3] = {0., 0., 0.};
      for (int n = 0; n < NP3; ++n) {
        const size_t o = (size_t)e * NP3 + n;
        const double* M[3] = {Mf + 3 * o, Mg + 3 * o, Mh + 3 * o};
        for (int d = 0; d < 3; ++d)
          ml[d] = std::max(ml[d], sJ[o] * std::sqrt(M[d][0] * M[d][0] + M[d][1] * M[d][1] + M[d][2] * M[d][2]));
      }
      dtch1 = std::min(dtch1, h->CFLScale * 2. / (ml[0] + ml[1] + ml[2]));
    }
    h->glmDtch1 = dtch1;
  }
  if (h->cfg.nfvse) {
    if ((r = dalloc(h, &h->dAlpha, (size_t)nElems)) || (r = dalloc(h, &h->dAlphaRaw, (size_t)nElems)) ||
        (r = dalloc(h, &h->dAlphaTmp, (size_t)nElems)) || (r = dalloc(h, &h->dBlendList, (size_t)nElems)) ||
        (r = dalloc(h, &h->dFV, nU)) || (h->cfg.nfvse_corr && (r = dalloc(h, &h->dFFV, nU))))
      return r;
    if (h->cfg.compute_alpha == 20) {
      // ComputeAlpha 20 (nfvse.f90:1591-1596): alpha = RANDOM_NUMBER * alpha_max once, then kept.  The
      // reference's stream is compiler-specific; this one is SplitMix64 from state 0, one draw per
      // element in element order (fluxo_gpu_set_alpha replaces it).
      std::vector<double> a((size_t)nElems);
      uint64_t state = 0;
      for (int e = 0; e < nElems; ++e) a[e] = splitmix64_unit(state) * h->cfg.alpha_max;
      FLUXO_CUDA(h, cudaMemcpy(h->dAlpha, a.data(), a.size() * sizeof(double), cudaMemcpyHostToDevice));
    } else {
      FLUXO_CUDA(h, cudaMemsetAsync(h->dAlpha, 0, (size_t)nElems * sizeof(double), h->stream));
    }
    if (h->cfg.nfvse_corr) FLUXO_CUDA(h, cudaMemsetAsync(h->dFFV, 0, nU * sizeof(double), h->stream));
  }
  cudaStream_t s = h->stream;
  FLUXO_CUDA(h, copy_h2d(h->dMetrics, met.data(), met.size() * 8, s));
  FLUXO_CUDA(h, copy_h2d(h->dsJ, sJ, (size_t)NP3 * nElems * 8, s));
  FLUXO_CUDA(h, copy_h2d(h->dFaceGeo, geo.data(), geo.size() * 8, s));
  FLUXO_CUDA(h, cudaMemcpyAsync(h->dS2E, s2e.data(), s2e.size() * 4, cudaMemcpyHostToDevice, s));
  FLUXO_CUDA(h, cudaMemcpyAsync(h->dE2S, e2s.data(), e2s.size() * 4, cudaMemcpyHostToDevice, s));
  FLUXO_CUDA(h, cudaMemsetAsync(h->dUtTmp, 0, nU * 8, s));
  FLUXO_CUDA(h, cudaMemsetAsync(h->dUt, 0, nU * 8, s));
  if (Elem_xGP) {
    if ((r = dalloc(h, &h->dXGP, (size_t)3 * NP3 * nElems))) return r;
    FLUXO_CUDA(h, cudaMemcpyAsync(h->dXGP, Elem_xGP, (size_t)3 * NP3 * nElems * 8, cudaMemcpyHostToDevice, s));
    h->haveXGP = true;
  }
  FLUXO_CUDA(h, cudaStreamSynchronize(s));
  h->meshSet = true;
  h->stateSet = false;
  return FLUXO_OK;
}

int fluxo_gpu_set_surf_metrics(fluxo_handle* h, const double* SM) {
  if (!h || !SM) return fail(h, FLUXO_EINVAL_CFG, "set_surf_metrics: null argument");
  if (!h->gauss) return fail(h, FLUXO_EINVAL_CFG, "set_surf_metrics: only for Gauss nodes (node_type = 1)");
  if (!h->meshSet) return fail(h, FLUXO_ENOTREADY, "set_surf_metrics: mesh not set");
  FLUXO_CUDA(h, cudaSetDevice(h->cfg.device));
  // SurfMetrics(3,0:N,0:N,6,nElems) -> [elem][side][3][pt]
  const int NP = h->NP, NPT = NP * NP;
  std::vector<double> d((size_t)18 * NPT * h->nElems);
  for (int e = 0; e < h->nElems; ++e)
    for (int s = 0; s < 6; ++s)
      for (int pt = 0; pt < NPT; ++pt)
        for (int c = 0; c < 3; ++c)
          d[(((size_t)e * 6 + s) * 3 + c) * NPT + pt] = SM[c + 3 * (pt + (size_t)NPT * (s + 6 * (size_t)e))];
  FLUXO_CUDA(h, cudaMemcpyAsync(h->dSurfMet, d.data(), d.size() * 8, cudaMemcpyHostToDevice, h->stream));
  FLUXO_CUDA(h, cudaStreamSynchronize(h->stream));
  h->surfMetSet = true;
  return FLUXO_OK;
}

int fluxo_gpu_set_state(fluxo_handle* h, const double* U) {
  if (!h || !U) return FLUXO_EINVAL_CFG;
  if (!h->meshSet) return fail(h, FLUXO_ENOTREADY, "mesh not set");
  FLUXO_CUDA(h, cudaSetDevice(h->cfg.device));
  const size_t nU = (size_t)h->nVar * h->NP * h->NP * h->NP * h->nElems;
  FLUXO_CUDA(h, copy_h2d(h->dU, U, nU * 8, h->stream));
  FLUXO_CUDA(h, cudaStreamSynchronize(h->stream));
  h->stateSet = true;
  return FLUXO_OK;
}

int fluxo_gpu_get_state(fluxo_handle* h, double* U) {
  int r = check_ready(h);
  if (r) return r;
  const size_t nU = (size_t)h->nVar * h->NP * h->NP * h->NP * h->nElems;
  FLUXO_CUDA(h, copy_d2h(U, h->dU, nU * 8, h->stream));
  FLUXO_CUDA(h, cudaStreamSynchronize(h->stream));
  return FLUXO_OK;
}

int fluxo_gpu_get_ut(fluxo_handle* h, double* Ut) {
  int r = check_ready(h);
  if (r) return r;
  const size_t nU = (size_t)h->nVar * h->NP * h->NP * h->NP * h->nElems;
  FLUXO_CUDA(h, copy_d2h(Ut, h->dUt, nU * 8, h->stream));
  FLUXO_CUDA(h, cudaStreamSynchronize(h->stream));
  return FLUXO_OK;
}

int fluxo_gpu_get_gradients(fluxo_handle* h, double* gx, double* gy, double* gz) {
  int r = check_ready(h);
  if (r) return r;
  if (!h->visc) return fail(h, FLUXO_EINVAL_CFG, "gradients exist for the parabolic equations only");
  const size_t nD = (size_t)h->NP * h->NP * h->NP * h->nElems;
  const int NV = h->nVar;
  std::vector<double> g(3 * NV * nD);
  FLUXO_CUDA(h, cudaMemcpyAsync(g.data(), h->dGrad, g.size() * 8, cudaMemcpyDeviceToHost, h->stream));
  FLUXO_CUDA(h, cudaStreamSynchronize(h->stream));
  for (size_t z = 0; z < nD; ++z)
    for (int v = 0; v < NV; ++v) {
      if (gx) gx[NV * z + v] = g[3 * NV * z + v];
      if (gy) gy[NV * z + v] = g[3 * NV * z + NV + v];
      if (gz) gz[NV * z + v] = g[3 * NV * z + 2 * NV + v];
    }
  return FLUXO_OK;
}

int fluxo_gpu_dg_time_derivative(fluxo_handle* h, double t) {
  int r = check_ready(h);
  if (r) return r;
  KParams P = base_params(h);
  P.stage = 0;
  P.t = t;
  P.grad = h->dGrad;  // keep the volume gradients of this RHS for fluxo_gpu_get_gradients
  if ((r = rhs(h, P))) return r;
  FLUXO_CUDA(h, cudaStreamSynchronize(h->stream));
  FLUXO_CUDA(h, cudaGetLastError());
  return FLUXO_OK;
}

int fluxo_gpu_calc_timestep(fluxo_handle* h, double* dt, int* errType) {
  int r = check_ready(h);
  if (r) return r;
  KParams P = base_params(h);
  dt_reset_kernel<<<1, 1, 0, h->stream>>>(h->dDtBits, h->dErrKey);
  FLUXO_CUDA(h, cudaGetLastError());
  if (h->mhd) FLUXO_CUDA(h, launch_mhd_timestep(h->NP, h->visc, h->nOwn, h->stream, P, h->dDtBits, h->dErrKey));
  else FLUXO_CUDA(h, launch_timestep(h->NP, h->visc, h->nOwn, h->stream, P, h->dDtBits, h->dErrKey));
  h->launches += 2;
  if ((r = exchange(h, FLUXO_XCHG_DT, h->dDtBits, h->dErrKey))) return r;  // MPI_ALLREDUCE(MIN), calctimestep.f90:159-167
  unsigned long long bits = 0;
  int key = 0;
  FLUXO_CUDA(h, cudaMemcpyAsync(&bits, h->dDtBits, 8, cudaMemcpyDeviceToHost, h->stream));
  FLUXO_CUDA(h, cudaMemcpyAsync(&key, h->dErrKey, 4, cudaMemcpyDeviceToHost, h->stream));
  FLUXO_CUDA(h, cudaStreamSynchronize(h->stream));
  double d;
  std::memcpy(&d, &bits, 8);
  if (dt) *dt = d;
  if (h->mhd && key == INT_MAX) h->glmCh = h->cfg.glm_scale * (h->glmDtch1 / d);  // mhd/calctimestep.f90:176
  int err = (key == INT_MAX) ? 0 : (key & 7);
  if (errType) *errType = err;
  return err ? FLUXO_ENAN_STATE : FLUXO_OK;
}

int fluxo_gpu_timestep(fluxo_handle* h, double t, double dt) {
  int r = check_ready(h);
  if (r) return r;
  const bool corr = h->cfg.nfvse && h->cfg.nfvse_corr;
  if (corr) {
    dt_reset_kernel<<<1, 1, 0, h->stream>>>(h->dDtBits, h->dErrKey);
    FLUXO_CUDA(h, cudaGetLastError());
  }
  if ((r = rk_step(h, t, dt, nullptr, nullptr))) return r;
  if (corr) {  // Apply_NFVSE_Correction stops the reference when a safe state is not admissible
    int key = INT_MAX;
    FLUXO_CUDA(h, cudaMemcpyAsync(&key, h->dErrKey, 4, cudaMemcpyDeviceToHost, h->stream));
    FLUXO_CUDA(h, cudaStreamSynchronize(h->stream));
    if (key != INT_MAX)
      return fail(h, FLUXO_ENAN_STATE, "NFVSE correction: safe state not admissible in element " +
                                           std::to_string(key / 8 + 1));
    return FLUXO_OK;
  }
  FLUXO_CUDA(h, cudaStreamSynchronize(h->stream));
  return FLUXO_OK;
}

int fluxo_gpu_time_disc(fluxo_handle* h, double t, double tEnd, int maxIter, double* tOut, int* nIter,
                        int* errType) {
  int r = check_ready(h);
  if (r) return r;
  cudaStream_t s = h->stream;
  TDState* td = h->dTD;
  td_begin_kernel<<<1, 1, 0, s>>>(td, t, tEnd, maxIter);
  td_glm_kernel<<<1, 1, 0, s>>>(td, h->mhd ? 1 : 0, h->glmCh, h->cfg.glm_scale, h->glmDtch1);
  FLUXO_CUDA(h, cudaGetLastError());
  h->launches += 2;
  // steps are enqueued in chunks between halt checks; with maxIter > 0 no more than maxIter steps
  // are enqueued in all (steps after a halt return at once but still count as launches)
  const int chunk = 16;
  int enqueued = 0;
  for (;;) {
    for (int c = 0; c < chunk; ++c) {
      KParams P = base_params(h);
      P.haltFlag = &td->halt;
      {
        ProfScope ps(h, 4);
        if (h->mhd) FLUXO_CUDA(h, launch_mhd_timestep(h->NP, h->visc, h->nOwn, s, P, &td->dtBits, &td->errKey));
        else FLUXO_CUDA(h, launch_timestep(h->NP, h->visc, h->nOwn, s, P, &td->dtBits, &td->errKey));
      }
      if ((r = exchange(h, FLUXO_XCHG_DT, &td->dtBits, &td->errKey))) return r;
      td_finalize_kernel<<<1, 1, 0, s>>>(td);
      FLUXO_CUDA(h, cudaGetLastError());
      if ((r = rk_step(h, 0., 0., &td->dt, &td->halt, h->mhd ? &td->ch : nullptr, &td->errKey))) return r;
      td_advance_kernel<<<1, 1, 0, s>>>(td);
      FLUXO_CUDA(h, cudaGetLastError());
      h->launches += 3;
      if (maxIter > 0 && ++enqueued >= maxIter) break;
    }
    TDState hs;
    FLUXO_CUDA(h, cudaMemcpyAsync(&hs, td, sizeof(TDState), cudaMemcpyDeviceToHost, s));
    FLUXO_CUDA(h, cudaStreamSynchronize(s));
    if (hs.halt) {
      if (h->mhd) h->glmCh = hs.ch;
      if (tOut) *tOut = hs.t;
      if (nIter) *nIter = hs.iter;
      if (errType) *errType = hs.err;
      return hs.err ? FLUXO_ENAN_STATE : FLUXO_OK;
    }
  }
}

int fluxo_gpu_analyze(fluxo_handle* h, double t, const fluxo_exact* ex, double* L2, double* Linf, double* L2colloc,
                      double* scalars) {
  int r = check_ready(h);
  if (r) return r;
  if (h->nOwn != h->nElems) return fail(h, FLUXO_EINVAL_CFG, "analyze: not on a partitioned handle");
  const int func = ex ? ex->func : 0;
  if (func != 0) {
    if (h->mhd) return fail(h, FLUXO_EINVAL_CFG, "analyze: error norms need an Euler / Navier-Stokes exact function");
    if (func != 1 && func != 2 && func != 4 && func != 7 && func != 14)
      return fail(h, FLUXO_EINVAL_CFG, "analyze: exact function must be 1, 2, 4, 7 or 14");
    if (!h->haveXGP) return fail(h, FLUXO_EINVAL_CFG, "analyze: error norms need Elem_xGP at set_mesh");
  }
  // DGTimeDerivative(t) before Analyze (timedisc.f90:387): Ut and the gradients of the current U
  KParams P = base_params(h);
  P.stage = 0;
  P.t = t;
  P.grad = h->dGrad;
  if ((r = rhs(h, P))) return r;
  const int NP = h->NP, NA1 = 2 * NP + 1, NV = h->nVar, K = 3 * NV + 5;
  if (!h->dAnaTables) {  // LGL weights (NP), interpolation N -> NAnalyze [NA1][NP], NAnalyze weights (NA1)
    std::vector<double> xa, wa;
    host::lgl(2 * NP, xa, wa);  // NAnalyze = 2(N+1), InitAnalyzeBasis (analyze.f90)
    std::vector<double> xg(h->hb.xGP, h->hb.xGP + NP), V = host::interp_matrix(xg, xa);
    std::vector<double> tab;
    tab.insert(tab.end(), h->hb.wGP, h->hb.wGP + NP);
    tab.insert(tab.end(), V.begin(), V.end());
    tab.insert(tab.end(), wa.begin(), wa.end());
    if ((r = dalloc(h, &h->dAnaTables, tab.size())) || (r = dalloc(h, &h->dAnaRes, (size_t)K))) return r;
    FLUXO_CUDA(h, cudaMemcpyAsync(h->dAnaTables, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice, h->stream));
    FLUXO_CUDA(h, cudaStreamSynchronize(h->stream));  // tab is a host temporary
  }
  if (!h->dAnaPartial && (r = dalloc(h, &h->dAnaPartial, (size_t)h->nElems * K))) return r;
  AnalyzeArgs A{};
  A.nElems = h->nElems; A.NP = NP; A.NA1 = NA1; A.nVar = NV; A.K = K;
  A.mhd = h->mhd ? 1 : 0;
  A.func = func;
  A.t = t;
  A.U = h->dU; A.Ut = h->dUt; A.sJ = h->dsJ; A.xGP = h->dXGP;
  A.grad = (h->visc && !h->mhd) ? h->dGrad : nullptr;
  A.wGP = h->dAnaTables; A.V = A.wGP + NP; A.wA = A.V + (size_t)NA1 * NP;
  A.kappa = h->cfg.kappa; A.kappaM1 = h->cfg.kappa - 1.; A.sKappaM1 = 1. / (h->cfg.kappa - 1.);
  A.s2mu_0 = h->mhd ? 0.5 / h->cfg.mu_0 : 0.;
  if (ex) {
    for (int v = 0; v < 5; ++v) A.refPrim[v] = ex->ref_state_prim[v];
    for (int d = 0; d < 3; ++d) {
      A.advVel[d] = ex->adv_vel[d]; A.waveNumber[d] = ex->ini_wavenumber[d]; A.center[d] = ex->ini_center[d];
    }
    A.amplitude = ex->ini_amplitude; A.frequency = ex->ini_frequency;
  }
  A.partial = h->dAnaPartial;
  FLUXO_CUDA(h, launch_analyze(A, h->dAnaRes, h->stream));
  h->launches += 2;
  std::vector<double> res(K);
  FLUXO_CUDA(h, cudaMemcpyAsync(res.data(), h->dAnaRes, K * 8, cudaMemcpyDeviceToHost, h->stream));
  FLUXO_CUDA(h, cudaStreamSynchronize(h->stream));
  const double Vol = res[3 * NV + 4];
  for (int v = 0; v < NV; ++v) {  // analyze.f90:627-629: L2 = sqrt(sum / Vol)
    if (L2) L2[v] = func ? std::sqrt(res[v] / Vol) : 0.;
    if (L2colloc) L2colloc[v] = func ? std::sqrt(res[NV + v] / Vol) : 0.;
    if (Linf) Linf[v] = func ? res[2 * NV + v] : 0.;
  }
  if (scalars) {
    scalars[0] = res[3 * NV] * A.sKappaM1;
    scalars[1] = res[3 * NV + 1];
    scalars[2] = res[3 * NV + 2] / Vol;
    scalars[3] = res[3 * NV + 3] / Vol;
    scalars[4] = Vol;
  }
  return FLUXO_OK;
}

int fluxo_gpu_set_glm_ch(fluxo_handle* h, double ch) {
  if (!h) return FLUXO_EINVAL_CFG;
  if (!h->mhd) return fail(h, FLUXO_EINVAL_CFG, "GLM_ch exists for MHD only");
  h->glmCh = ch;
  return FLUXO_OK;
}

int fluxo_gpu_get_glm_ch(fluxo_handle* h, double* ch) {
  if (!h || !ch) return FLUXO_EINVAL_CFG;
  if (!h->mhd) return fail(h, FLUXO_EINVAL_CFG, "GLM_ch exists for MHD only");
  *ch = h->glmCh;
  return FLUXO_OK;
}

int fluxo_gpu_set_partition(fluxo_handle* h, int nOwned, fluxo_exchange_fn fn, void* ctx) {
  if (!h) return FLUXO_EINVAL_CFG;
  if (!h->meshSet) return fail(h, FLUXO_ENOTREADY, "set_partition: mesh not set");
  if (nOwned < 1 || nOwned > h->nElems) return fail(h, FLUXO_EINVAL_CFG, "set_partition: nOwned out of range");
  if (h->gauss) return fail(h, FLUXO_EINVAL_CFG, "set_partition: LGL nodes only");
  h->nOwn = nOwned;
  h->xfn = fn;
  h->xctx = ctx;
  if (h->mhd) {  // GLM_dtch1 of the whole mesh: MIN over the handles (InitTimeStep_GLM's MPI_ALLREDUCE)
    unsigned long long bits;
    const int none = INT_MAX;
    std::memcpy(&bits, &h->glmDtch1, 8);
    FLUXO_CUDA(h, cudaMemcpyAsync(h->dDtBits, &bits, 8, cudaMemcpyHostToDevice, h->stream));
    FLUXO_CUDA(h, cudaMemcpyAsync(h->dErrKey, &none, 4, cudaMemcpyHostToDevice, h->stream));
    if (int r = exchange(h, FLUXO_XCHG_DT, h->dDtBits, h->dErrKey)) return r;
    FLUXO_CUDA(h, cudaMemcpyAsync(&bits, h->dDtBits, 8, cudaMemcpyDeviceToHost, h->stream));
    FLUXO_CUDA(h, cudaStreamSynchronize(h->stream));
    std::memcpy(&h->glmDtch1, &bits, 8);
  }
  return FLUXO_OK;
}

int fluxo_gpu_exchange_buffers(fluxo_handle* h, double** gtrace) {
  if (!h || !gtrace) return FLUXO_EINVAL_CFG;
  if (!h->meshSet) return fail(h, FLUXO_ENOTREADY, "exchange_buffers: mesh not set");
  *gtrace = h->dGTrace;
  return FLUXO_OK;
}

int fluxo_gpu_set_alpha(fluxo_handle* h, const double* alpha) {
  int r = check_ready(h);
  if (r) return r;
  if (!alpha) return FLUXO_EINVAL_CFG;
  if (!h->cfg.nfvse) return fail(h, FLUXO_EINVAL_CFG, "NFVSE is off");
  FLUXO_CUDA(h, cudaMemcpyAsync(h->dAlpha, alpha, (size_t)h->nElems * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  FLUXO_CUDA(h, cudaStreamSynchronize(h->stream));
  return FLUXO_OK;
}

int fluxo_gpu_get_alpha(fluxo_handle* h, double* alpha) {
  int r = check_ready(h);
  if (r) return r;
  if (!alpha) return FLUXO_EINVAL_CFG;
  if (!h->cfg.nfvse) return fail(h, FLUXO_EINVAL_CFG, "NFVSE is off");
  FLUXO_CUDA(h, cudaMemcpyAsync(alpha, h->dAlpha, (size_t)h->nElems * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  FLUXO_CUDA(h, cudaStreamSynchronize(h->stream));
  return FLUXO_OK;
}

int fluxo_gpu_device_buffers(fluxo_handle* h, double** dU, double** dUt, void** stream) {
  if (!h) return FLUXO_EINVAL_CFG;
  if (dU) *dU = h->dU;
  if (dUt) *dUt = h->dUt;
  if (stream) *stream = (void*)h->stream;
  if (h->meshSet && dU) h->stateSet = true;  // caller may fill U directly on the device
  return FLUXO_OK;
}

int fluxo_gpu_launch_count(fluxo_handle* h, uint64_t* n) {
  if (!h || !n) return FLUXO_EINVAL_CFG;
  *n = h->launches;
  return FLUXO_OK;
}

int fluxo_gpu_set_profiling(fluxo_handle* h, int enable) {
  if (!h) return FLUXO_EINVAL_CFG;
  h->profiling = enable != 0;
  return FLUXO_OK;
}

int fluxo_gpu_get_profile(fluxo_handle* h, int kind, double* total_ms, uint64_t* count) {
  if (!h || kind < 0 || kind > 5) return FLUXO_EINVAL_CFG;
  FLUXO_CUDA(h, cudaStreamSynchronize(h->stream));
  double tot = 0.;
  for (auto& pr : h->prof[kind]) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, pr.first, pr.second);
    tot += ms;
    cudaEventDestroy(pr.first);
    cudaEventDestroy(pr.second);
  }
  if (total_ms) *total_ms = tot;
  if (count) *count = h->prof[kind].size();
  h->prof[kind].clear();
  return FLUXO_OK;
}

int fluxo_gpu_volume_shape(int N, int volume_flux, int visc, int* count, int* index, int* epb, int* lpw) {
  const int NP = N + 1;
  if (N < 1 || N > 8 || !volume_flux_supported(volume_flux))
    return fail(nullptr, FLUXO_EINVAL_CFG, "volume_shape: unsupported N or volume flux");
  const int c = volume_shape_count(NP), i = volume_shape(NP, volume_flux, visc != 0);
  if (count) *count = c;
  if (index) *index = i;
  const int k = i < 0 ? 0 : i;
  if (epb) *epb = kVolShapes[NP][k].epb;
  if (lpw) *lpw = kVolShapes[NP][k].lpw;
  return FLUXO_OK;
}

int fluxo_gpu_set_volume_shape(int N, int volume_flux, int visc, int index) {
  if (N < 1 || N > 8 || !volume_flux_supported(volume_flux) || !pin_volume_shape(N + 1, volume_flux, visc != 0, index))
    return fail(nullptr, FLUXO_EINVAL_CFG, "set_volume_shape: unsupported N, volume flux or shape index");
  return FLUXO_OK;
}

int fluxo_gpu_fp64_peak(int device, double* tflops) {
  if (!tflops) return FLUXO_EINVAL_CFG;
  if (cudaSetDevice(device) != cudaSuccess) return FLUXO_ECUDA;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  double* out = nullptr;
  if (cudaMalloc(&out, 1024 * sizeof(double)) != cudaSuccess) return FLUXO_ENOMEM_HBM;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const int threads = 512, blocks = sms * 4, iters = 4096;
  fp64_fma_kernel<<<blocks, threads>>>(out, 64, 1.0000001, 1e-9);  // warm-up
  double best = 0.;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(a);
    fp64_fma_kernel<<<blocks, threads>>>(out, iters, 1.0000001, 1e-9);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    const double fl = 2.0 * 8.0 * iters * (double)threads * blocks;
    best = std::max(best, fl / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return FLUXO_ECUDA;
  *tflops = best;
  return FLUXO_OK;
}

int fluxo_gpu_destroy(fluxo_handle* h) {
  if (!h) return FLUXO_OK;
  for (int k = 0; k < 6; ++k) {
    for (auto& pr : h->prof[k]) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
    h->prof[k].clear();
  }
  cudaSetDevice(h->cfg.device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  void* ptrs[] = {h->dBasis, h->dU, h->dUt, h->dUtTmp, h->dGrad, h->dUtVisc, h->dMetrics, h->dsJ, h->dFaceGeo, h->dXGP,
                  h->dFlux, h->dLFlux, h->dGTrace, h->dS2E, h->dE2S, h->dTD, h->dDtBits, h->dErrKey,
                  h->dAlpha, h->dAlphaRaw, h->dAlphaTmp, h->dFV, h->dFFV, h->dSVdm, h->dBlendList, h->dBlendCount,
                  h->dAnaPartial, h->dAnaRes, h->dAnaTables, h->dUReg2, h->dUface, h->dUtSurf, h->dSurfMet};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return FLUXO_OK;
}

int fluxo_gpu_last_error(fluxo_handle* h, char* buf, size_t len) {
  if (!buf || len == 0) return FLUXO_EINVAL_CFG;
  std::string m;
  if (h) m = h->lastError;
  else {
    std::lock_guard<std::mutex> lk(g_err_mutex);
    m = g_create_error;
  }
  std::snprintf(buf, len, "%s", m.c_str());
  return FLUXO_OK;
}

}  // extern "C"
