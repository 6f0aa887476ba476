// Instantiates the volume kernel for one volume flux family (VF_ID) and N = 1..8.
#include <utility>
#include "kernels.cuh"
#include "launch.h"

#define FLUXO_CAT2(a, b) a##b
#define FLUXO_CAT(a, b) FLUXO_CAT2(a, b)

namespace fluxo {

template <int NP, bool VISC>
static cudaError_t vol_launch_t(int nElems, cudaStream_t s, const KParams& P) {
  constexpr int EPB = vol_epb<NP>();
  constexpr size_t smem = vol_smem_bytes<NP, VF_ID>();
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(volume_kernel<NP, VF_ID, VISC>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int grid = (nElems + EPB - 1) / EPB;
  volume_kernel<NP, VF_ID, VISC><<<grid, EPB * NP * NP * NP, smem, s>>>(P);
  return cudaGetLastError();
}

cudaError_t FLUXO_CAT(launch_volume_vf, VF_ID)(int NP, bool visc, int nElems, cudaStream_t s, const KParams& P) {
#define FLUXO_NP_CASE(K) \
  case K: return visc ? vol_launch_t<K, true>(nElems, s, P) : vol_launch_t<K, false>(nElems, s, P);
  switch (NP) {
    FLUXO_NP_CASE(2) FLUXO_NP_CASE(3) FLUXO_NP_CASE(4) FLUXO_NP_CASE(5)
    FLUXO_NP_CASE(6) FLUXO_NP_CASE(7) FLUXO_NP_CASE(8) FLUXO_NP_CASE(9)
    default: return cudaErrorInvalidValue;
  }
#undef FLUXO_NP_CASE
}

}  // namespace fluxo
