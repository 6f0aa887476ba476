// Instantiations of the lifting + viscous volume kernel: N = 1..7, BR1/BR2, three lifting variables.
#include "kernels.cuh"
#include "launch.h"
#include "lifting.cuh"

namespace fluxo {

template <int NP, int LIFT, int LV>
static cudaError_t lv_t(int nElems, cudaStream_t s, const KParams& P) {
  constexpr int EPB = lv_epb<NP>();
  constexpr size_t smem = lv_smem_bytes<NP>();
  static std::atomic<unsigned long long> attr{0};
  cudaError_t e = smem_attr_once(lift_visc_kernel<NP, LIFT, LV>, smem, attr);
  if (e != cudaSuccess) return e;
  lift_visc_kernel<NP, LIFT, LV><<<(nElems + EPB - 1) / EPB, EPB * NP * NP * NP, smem, s>>>(P);
  return cudaGetLastError();
}

template <int NP>
static cudaError_t lv_np(int lift, int lv, int nElems, cudaStream_t s, const KParams& P) {
  if (lift == 1) {
    if (lv == 1) return lv_t<NP, 1, 1>(nElems, s, P);
    if (lv == 2) return lv_t<NP, 1, 2>(nElems, s, P);
    if (lv == 3) return lv_t<NP, 1, 3>(nElems, s, P);
  } else if (lift == 2) {
    if (lv == 1) return lv_t<NP, 2, 1>(nElems, s, P);
    if (lv == 2) return lv_t<NP, 2, 2>(nElems, s, P);
    if (lv == 3) return lv_t<NP, 2, 3>(nElems, s, P);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_lift_visc(int NP, int lift, int lv, int nElems, cudaStream_t s, const KParams& P) {
  switch (NP) {
    case 2: return lv_np<2>(lift, lv, nElems, s, P);
    case 3: return lv_np<3>(lift, lv, nElems, s, P);
    case 4: return lv_np<4>(lift, lv, nElems, s, P);
    case 5: return lv_np<5>(lift, lv, nElems, s, P);
    case 6: return lv_np<6>(lift, lv, nElems, s, P);
    case 7: return lv_np<7>(lift, lv, nElems, s, P);
    case 8: return lv_np<8>(lift, lv, nElems, s, P);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fluxo
