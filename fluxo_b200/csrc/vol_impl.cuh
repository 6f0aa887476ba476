// Instantiates the volume kernel for one volume flux family (VF_ID), N = 1..8 and every candidate
// launch shape of vol_shapes.h.
#include <utility>
#include "kernels.cuh"
#include "launch.h"
#include "vol_shapes.h"

#define FLUXO_CAT2(a, b) a##b
#define FLUXO_CAT(a, b) FLUXO_CAT2(a, b)

namespace fluxo {

template <int NP, bool VISC, int I>
static cudaError_t vol_shape_launch(int nElems, cudaStream_t s, const KParams& P) {
  constexpr VolShapeId sh = kVolShapes[NP][I];
  constexpr int EPB = sh.epb, LPW = sh.lpw, MINB = sh.minb, OWNSM = sh.ownsm;
  constexpr size_t smem = vol_smem_bytes<NP, VF_ID, EPB, LPW>();
  static std::atomic<unsigned long long> attr{0};
  static std::atomic<int> resident[64];
  auto k = volume_kernel<NP, VF_ID, VISC, EPB, LPW, MINB, OWNSM>;
  cudaError_t e = smem_attr_once(k, smem, attr);
  if (e != cudaSuccess) return e;
  const int grid = (nElems + EPB - 1) / EPB;
  KParams Q = P;
  Q.pfTiles = resident_blocks(k, VolShape<NP, EPB, LPW>::THREADS, smem, resident);
  k<<<grid, VolShape<NP, EPB, LPW>::THREADS, smem, s>>>(Q);
  return cudaGetLastError();
}

template <int NP, bool VISC>
static cudaError_t vol_np(int shape, int nElems, cudaStream_t s, const KParams& P) {
  constexpr int C = vol_shape_count(NP);
  if (shape == 0) return vol_shape_launch<NP, VISC, 0>(nElems, s, P);
  if constexpr (C > 1) {
    if (shape == 1) return vol_shape_launch<NP, VISC, 1>(nElems, s, P);
  }
  if constexpr (C > 2) {
    if (shape == 2) return vol_shape_launch<NP, VISC, 2>(nElems, s, P);
  }
  return cudaErrorInvalidValue;
}

cudaError_t FLUXO_CAT(launch_volume_vf, VF_ID)(int NP, bool visc, int shape, int nElems, cudaStream_t s,
                                              const KParams& P) {
#define FLUXO_NP_CASE(K) \
  case K: return visc ? vol_np<K, true>(shape, nElems, s, P) : vol_np<K, false>(shape, nElems, s, P);
  switch (NP) {
    FLUXO_NP_CASE(2) FLUXO_NP_CASE(3) FLUXO_NP_CASE(4) FLUXO_NP_CASE(5)
    FLUXO_NP_CASE(6) FLUXO_NP_CASE(7) FLUXO_NP_CASE(8) FLUXO_NP_CASE(9)
    default: return cudaErrorInvalidValue;
  }
#undef FLUXO_NP_CASE
}

}  // namespace fluxo
