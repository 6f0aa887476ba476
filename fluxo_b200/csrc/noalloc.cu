// fluxo_gpu_dg_time_derivative_noalloc: the Euler right-hand side on caller-owned device arrays,
// with its one scratch buffer (the face fluxes, plus the operator tables) in a file-scope device
// array instead of device memory obtained at run time.
//
// Who needs it: callers that own all device memory themselves and must not allocate while they
// run, e.g. a host code that reserves one arena of HBM at start-up and places its state, residual
// and geometry arrays in it (a Jacobian-free Newton-Krylov or embedded-error integrator evaluating
// the right-hand side on many of its own vectors).  Such callers cannot create a fluxo_handle
// (fluxo_gpu_create and fluxo_gpu_set_mesh allocate), and an allocation inside the call would
// fail once the arena holds the memory, or stall the device: cudaFree synchronises every stream.
//
// The kernels are the same face-flux and volume kernels as fluxo_gpu_dg_time_derivative; only the
// face-flux buffer and the operator tables live in g_noalloc_scratch.  Every call on a device
// shares that array, so calls whose GPU work overlaps (different streams, different host threads)
// race on it; the call synchronises its stream before it returns, so calls from one host thread
// never overlap.  No byte of the scratch has to start at zero: the operator tables are written by
// the first call at each N (a call at another N overwrites them) and every call writes every face
// flux before the volume kernel reads it.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/fluxo_gpu.h"
#include "common.cuh"
#include "launch.h"

using namespace fluxo;

// The scratch shared by all calls on a device (allocated with the module, not by any call).
static __device__ __align__(256) unsigned char g_noalloc_scratch[FLUXO_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
constexpr size_t kTablesBytes = (sizeof(BasisTables) + 255) / 256 * 256;  // face fluxes start 256-aligned
static_assert(kTablesBytes == 2304, "the scratch size formula in fluxo_gpu.h states 2304 bytes of tables");

std::mutex g_mutex;
void* g_scratch[kMaxDevices];       // device address of g_noalloc_scratch, looked up once per device
int g_scratch_N[kMaxDevices];       // N whose operator tables the device's scratch holds (0: none yet)
BasisTables g_tables[8];            // host copies of the operator tables per N (static storage)
bool g_tables_built[8];

int bad(int code, const std::string& msg) {
  return record_unbound_error(code, "fluxo_gpu_dg_time_derivative_noalloc: " + msg);
}

// True if p is device (or managed) memory of `device`; queries only, no allocation.
bool on_device(const void* p, int device) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == device;
}

// Restores the caller's current device on every return path.
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" int fluxo_gpu_dg_time_derivative_noalloc(const fluxo_cfg* cfg, int nElems, int nSides, const double* dU,
                                                    double* dUt, const double* dMetrics, const double* dsJ,
                                                    const double* dFaceGeo, const int* dS2E, const int* dE2S,
                                                    void* stream) {
  // argument checks first: nothing below touches the device before they pass
  if (!cfg) return bad(FLUXO_EINVAL_CFG, "null cfg");
  if (cfg->struct_size != (int)sizeof(fluxo_cfg)) return bad(FLUXO_EINVAL_CFG, "fluxo_cfg size mismatch");
  if (cfg->N < 1 || cfg->N > 7) return bad(FLUXO_EINVAL_CFG, "N must be in 1..7");
  if (cfg->eqn != FLUXO_EQN_EULER) return bad(FLUXO_EINVAL_CFG, "only the Euler equations (eqn 0) are supported");
  if (cfg->ini_exact_func == 4) return bad(FLUXO_EINVAL_CFG, "the source term (IniExactFunc 4) is not supported");
  if (cfg->nfvse != 0) return bad(FLUXO_EINVAL_CFG, "NFVSE shock capturing (nfvse = 1) is not supported");
  if (cfg->node_type == 1) return bad(FLUXO_EINVAL_CFG, "Gauss nodes (node_type = 1) are not supported");
  if (!riemann_supported(cfg->riemann)) return bad(FLUXO_EINVAL_CFG, "Riemann solver not implemented");
  if (!volume_flux_supported(cfg->volume_flux)) return bad(FLUXO_EINVAL_CFG, "volume flux not implemented");
  if (!(cfg->kappa > 1.)) return bad(FLUXO_EINVAL_CFG, "kappa must be > 1");
  if (nElems < 1 || nSides < 1) return bad(FLUXO_EINVAL_CFG, "nElems and nSides must be >= 1");
  if (!dU || !dUt || !dMetrics || !dsJ || !dFaceGeo || !dS2E || !dE2S) return bad(FLUXO_EINVAL_CFG, "null array");
  const int NP = cfg->N + 1;
  const size_t need = kTablesBytes + (size_t)nSides * 5 * NP * NP * sizeof(double);
  if (need > (size_t)FLUXO_NOALLOC_SCRATCH_BYTES) {
    char msg[256];
    std::snprintf(msg, sizeof msg,
                  "N=%d with %d sides needs %zu bytes of scratch; the maximum is %zu (FLUXO_NOALLOC_SCRATCH_BYTES)",
                  cfg->N, nSides, need, (size_t)FLUXO_NOALLOC_SCRATCH_BYTES);
    return bad(FLUXO_EINVAL_CFG, msg);
  }
  if (cfg->device < 0 || cfg->device >= kMaxDevices) return bad(FLUXO_EINVAL_CFG, "device ordinal out of range");

  DeviceGuard guard;
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e != cudaSuccess) return bad(FLUXO_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  const void* arrays[] = {dU, dUt, dMetrics, dsJ, dFaceGeo, dS2E, dE2S};
  for (const void* p : arrays)
    if (!on_device(p, cfg->device)) return bad(FLUXO_EINVAL_CFG, "an array is not device memory of cfg->device");

  void* scratch = nullptr;
  const BasisTables* tables = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mutex);
    if (!g_scratch[cfg->device]) {  // set-up, once per device, with that device current
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return bad(FLUXO_ECUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
      g_scratch[cfg->device] = p;
    }
    scratch = g_scratch[cfg->device];
    if (!g_tables_built[cfg->N]) {
      basis_tables_for(cfg->N, g_tables[cfg->N]);
      g_tables_built[cfg->N] = true;
    }
    // the tables go up only when the device's scratch holds another N's (a copy from pageable host
    // memory is staged by the runtime, a fixed cost a caller evaluating many right-hand sides on one
    // mesh would otherwise pay on every call)
    if (g_scratch_N[cfg->device] != cfg->N) {
      tables = &g_tables[cfg->N];
      g_scratch_N[cfg->device] = cfg->N;
    }
  }

  cudaStream_t s = (cudaStream_t)stream;
  BasisTables* dTables = (BasisTables*)scratch;
  double* dFlux = (double*)((unsigned char*)scratch + kTablesBytes);
  if (tables) {
    e = cudaMemcpyAsync(dTables, tables, sizeof(BasisTables), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
      std::lock_guard<std::mutex> lk(g_mutex);
      g_scratch_N[cfg->device] = 0;
      return bad(FLUXO_ECUDA, std::string("tables copy: ") + cudaGetErrorString(e));
    }
  }

  KParams P{};
  P.nElems = nElems; P.nSides = nSides;
  P.U = const_cast<double*>(dU); P.Ut = dUt;
  P.metrics = dMetrics; P.sJ = dsJ; P.facegeo = dFaceGeo; P.s2e = dS2E; P.e2s = dE2S;
  P.flux = dFlux;
  P.basis = dTables;
  P.kappa = cfg->kappa; P.kappaM1 = cfg->kappa - 1.; P.sKappaM1 = 1. / (cfg->kappa - 1.);
  P.kappaP1 = cfg->kappa + 1.; P.R = cfg->R;
  P.stage = 0;  // plain DGTimeDerivative: the volume kernel writes Ut

  if ((e = launch_face_flux(cfg->riemann, false, NP, nSides, s, P)) != cudaSuccess ||
      (e = launch_volume(NP, cfg->volume_flux, false, nElems, s, P)) != cudaSuccess)
    return bad(FLUXO_ECUDA, std::string("launch: ") + cudaGetErrorString(e));
  e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return bad(FLUXO_ECUDA, std::string("kernels: ") + cudaGetErrorString(e));
  return FLUXO_OK;
}
