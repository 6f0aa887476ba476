// Launchers of the face, lifting and time-step kernels, the volume-flux dispatcher and the volume
// kernel's launch-shape autotuner.
#include <mutex>

#include "kernels.cuh"
#include "launch.h"
#include "vol_shapes.h"

namespace fluxo {

cudaError_t launch_volume_shape(int NP, int VF, bool visc, int shape, int nElems, cudaStream_t s,
                                const KParams& P) {
  switch (VF) {
    case 0: return launch_volume_vf0(NP, visc, shape, nElems, s, P);
    case 1: return launch_volume_vf1(NP, visc, shape, nElems, s, P);
    case 2: return launch_volume_vf2(NP, visc, shape, nElems, s, P);
    case 3: return launch_volume_vf3(NP, visc, shape, nElems, s, P);
    case 4: return launch_volume_vf4(NP, visc, shape, nElems, s, P);
    case 5: return launch_volume_vf5(NP, visc, shape, nElems, s, P);
    case 6: return launch_volume_vf6(NP, visc, shape, nElems, s, P);
    case 7: return launch_volume_vf7(NP, visc, shape, nElems, s, P);
    case 8: return launch_volume_vf8(NP, visc, shape, nElems, s, P);
    case 9: return launch_volume_vf9(NP, visc, shape, nElems, s, P);
    case 10: return launch_volume_vf10(NP, visc, shape, nElems, s, P);
    case 32: return launch_volume_vf32(NP, visc, shape, nElems, s, P);
    default: return cudaErrorInvalidValue;
  }
}

namespace {
// chosen launch shape per (NP, VF, visc); -1 = not tuned
std::mutex g_shape_mutex;
int g_shape[10][33][2];
bool g_shape_init = false;

int* shape_slot(int NP, int VF, bool visc) {
  if (NP < 2 || NP > 9 || VF < 0 || VF > 32) return nullptr;
  if (!g_shape_init) {
    for (auto& a : g_shape)
      for (auto& b : a) b[0] = b[1] = -1;
    g_shape_init = true;
  }
  return &g_shape[NP][VF][visc ? 1 : 0];
}
}  // namespace

int volume_shape_count(int NP) { return vol_shape_count(NP); }

int volume_shape(int NP, int VF, bool visc) {
  std::lock_guard<std::mutex> lk(g_shape_mutex);
  int* p = shape_slot(NP, VF, visc);
  return p ? *p : -1;
}

bool pin_volume_shape(int NP, int VF, bool visc, int shape) {
  std::lock_guard<std::mutex> lk(g_shape_mutex);
  int* p = shape_slot(NP, VF, visc);
  if (!p || shape >= vol_shape_count(NP)) return false;
  *p = shape < 0 ? -1 : shape;
  return true;
}

cudaError_t launch_volume(int NP, int VF, bool visc, int nElems, cudaStream_t s, const KParams& P) {
  const int sh = volume_shape(NP, VF, visc);
  return launch_volume_shape(NP, VF, visc, sh < 0 ? 0 : sh, nElems, s, P);
}

cudaError_t tune_volume(int NP, int VF, bool visc, int nElems, cudaStream_t s, const KParams& P) {
  const int C = vol_shape_count(NP);
  if (volume_shape(NP, VF, visc) >= 0) return cudaSuccess;
  if (C <= 1) {
    pin_volume_shape(NP, VF, visc, 0);
    return cudaSuccess;
  }
  KParams Q = P;
  Q.stage = 0;           // writes Ut only: the state and the RK register stay untouched
  Q.haltFlag = nullptr;  // every launch does its full work
  Q.grad = nullptr;
  cudaEvent_t a, b;
  cudaError_t e;
  if ((e = cudaEventCreate(&a)) != cudaSuccess) return e;
  if ((e = cudaEventCreate(&b)) != cudaSuccess) { cudaEventDestroy(a); return e; }
  int best = 0;
  float bestMs = 0.f;
  for (int i = 0; i < C && e == cudaSuccess; ++i) {
    if ((e = launch_volume_shape(NP, VF, visc, i, nElems, s, Q)) != cudaSuccess) break;  // warm-up
    if ((e = cudaEventRecord(a, s)) != cudaSuccess) break;
    for (int r = 0; r < 3 && e == cudaSuccess; ++r) e = launch_volume_shape(NP, VF, visc, i, nElems, s, Q);
    if (e != cudaSuccess) break;
    if ((e = cudaEventRecord(b, s)) != cudaSuccess || (e = cudaEventSynchronize(b)) != cudaSuccess) break;
    float ms = 0.f;
    if ((e = cudaEventElapsedTime(&ms, a, b)) != cudaSuccess) break;
    if (i == 0 || ms < bestMs) { bestMs = ms; best = i; }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (e == cudaSuccess) pin_volume_shape(NP, VF, visc, best);
  return e;
}

bool volume_flux_supported(int VF) {
  return (VF >= 0 && VF <= 10) || VF == 32;
}

bool riemann_supported(int RS) {
  switch (RS) {
    case 0: case 1: case 2: case 3: case 4: case 5: case 6: case 7: case 8: case 9: case 10: case 11: case 12:
    case 13: case 14: case 15: case 16: case 17: case 18: case 19: case 20: case 21: case 22: case 23: case 24:
    case 32: case 33: case 44:
      return true;
    default:
      return false;
  }
}

template <int RS, bool VISC>
static cudaError_t face_t(int NP, int nSides, cudaStream_t s, const KParams& P) {
  const int npts = NP * NP;
  const int spb = (128 / npts) > 0 ? (128 / npts) : 1;
  const int grid = (nSides + spb - 1) / spb;
  // 8 resident blocks of 128 threads per SM (64 registers): the face pass is DRAM-latency bound, and
  // the extra warps in flight outweigh the spills of the heavier Riemann solvers (measured at N=7 with
  // the matrix-dissipation solver: 4.2 TB/s against 3.5 TB/s at the unbounded 114 registers)
  face_flux_kernel<RS, VISC, 8><<<grid, spb * npts, 0, s>>>(P, NP);
  return cudaGetLastError();
}

cudaError_t launch_face_flux(int RS, bool visc, int NP, int nSides, cudaStream_t s, const KParams& P) {
#define FLUXO_RS_CASE(K) \
  case K: return visc ? face_t<K, true>(NP, nSides, s, P) : face_t<K, false>(NP, nSides, s, P);
  switch (RS) {
    FLUXO_RS_CASE(0) FLUXO_RS_CASE(1) FLUXO_RS_CASE(2) FLUXO_RS_CASE(3) FLUXO_RS_CASE(4) FLUXO_RS_CASE(5)
    FLUXO_RS_CASE(6) FLUXO_RS_CASE(7) FLUXO_RS_CASE(8) FLUXO_RS_CASE(9) FLUXO_RS_CASE(10) FLUXO_RS_CASE(11)
    FLUXO_RS_CASE(12) FLUXO_RS_CASE(13) FLUXO_RS_CASE(14) FLUXO_RS_CASE(15) FLUXO_RS_CASE(16) FLUXO_RS_CASE(17)
    FLUXO_RS_CASE(18) FLUXO_RS_CASE(19) FLUXO_RS_CASE(20) FLUXO_RS_CASE(21) FLUXO_RS_CASE(22) FLUXO_RS_CASE(23)
    FLUXO_RS_CASE(24) FLUXO_RS_CASE(32) FLUXO_RS_CASE(33) FLUXO_RS_CASE(44)
    default: return cudaErrorInvalidValue;
  }
#undef FLUXO_RS_CASE
}

cudaError_t launch_lift_flux(int NP, int nSides, cudaStream_t s, const KParams& P) {
  const size_t n = (size_t)nSides * NP * NP;
  const int grid = (int)((n + 255) / 256);
  lift_flux_kernel<<<grid, 256, 0, s>>>(P, NP, P.lflux);
  return cudaGetLastError();
}

cudaError_t launch_gradient(int NP, int nElems, cudaStream_t s, const KParams& P) {
  return launch_lift_visc(NP, P.lifting, P.lifting_var, nElems, s, P);
}

template <int NP, bool VISC>
static cudaError_t dt_t(int nElems, cudaStream_t s, const KParams& P, unsigned long long* dtBits, int* errKey) {
  constexpr int NP3 = NP * NP * NP;
  constexpr int EPB = (256 / NP3) > 0 ? (256 / NP3) : 1;
  timestep_kernel<NP, VISC><<<(nElems + EPB - 1) / EPB, EPB * NP3, 0, s>>>(P, dtBits, errKey);
  return cudaGetLastError();
}

cudaError_t launch_timestep(int NP, bool visc, int nElems, cudaStream_t s, const KParams& P,
                            unsigned long long* dtBits, int* errKey) {
#define FLUXO_DT_CASE(K) \
  case K: return visc ? dt_t<K, true>(nElems, s, P, dtBits, errKey) : dt_t<K, false>(nElems, s, P, dtBits, errKey);
  switch (NP) {
    FLUXO_DT_CASE(2) FLUXO_DT_CASE(3) FLUXO_DT_CASE(4) FLUXO_DT_CASE(5)
    FLUXO_DT_CASE(6) FLUXO_DT_CASE(7) FLUXO_DT_CASE(8) FLUXO_DT_CASE(9)
    default: return cudaErrorInvalidValue;
  }
#undef FLUXO_DT_CASE
}

}  // namespace fluxo
