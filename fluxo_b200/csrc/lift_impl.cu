// Instantiations of the lifting + viscous volume kernel: N = 1..7, BR1/BR2, three lifting variables.
#include "kernels.cuh"
#include "launch.h"
#include "lifting.cuh"
#include "lifting_mma.cuh"

namespace fluxo {

template <int NP, int LIFT, int LV>
static cudaError_t lv_t(int nElems, cudaStream_t s, const KParams& P) {
  constexpr int EPB = lv_epb<NP>();
  constexpr size_t smem = lv_smem_bytes<NP>();
  static std::atomic<unsigned long long> attr{0};
  static std::atomic<int> resident[64];
  auto k = lift_visc_kernel<NP, LIFT, LV>;
  cudaError_t e = smem_attr_once(k, smem, attr);
  if (e != cudaSuccess) return e;
  KParams Q = P;
  Q.pfTiles = resident_blocks(k, EPB * NP * NP * NP, smem, resident);
  k<<<(nElems + EPB - 1) / EPB, EPB * NP * NP * NP, smem, s>>>(Q);
  return cudaGetLastError();
}

// N+1 = 8: the operator contractions on the FP64 tensor cores (lifting_mma.cuh), one element per block
template <int LIFT, int LV>
static cudaError_t lv_mma_t(int nElems, cudaStream_t s, const KParams& P) {
  constexpr size_t smem = lm_smem_bytes();
  static std::atomic<unsigned long long> attr{0};
  static std::atomic<int> resident[64];
  auto k = lift_visc_mma_kernel<LIFT, LV>;
  cudaError_t e = smem_attr_once(k, smem, attr);
  if (e != cudaSuccess) return e;
  KParams Q = P;
  Q.pfTiles = resident_blocks(k, 512, smem, resident);
  k<<<nElems, 512, smem, s>>>(Q);
  return cudaGetLastError();
}

template <int NP, int LIFT, int LV>
static cudaError_t lv_pick(int nElems, cudaStream_t s, const KParams& P) {
  if constexpr (NP == 8) return lv_mma_t<LIFT, LV>(nElems, s, P);
  else return lv_t<NP, LIFT, LV>(nElems, s, P);
}

template <int NP>
static cudaError_t lv_np(int lift, int lv, int nElems, cudaStream_t s, const KParams& P) {
  if (lift == 1) {
    if (lv == 1) return lv_pick<NP, 1, 1>(nElems, s, P);
    if (lv == 2) return lv_pick<NP, 1, 2>(nElems, s, P);
    if (lv == 3) return lv_pick<NP, 1, 3>(nElems, s, P);
  } else if (lift == 2) {
    if (lv == 1) return lv_pick<NP, 2, 1>(nElems, s, P);
    if (lv == 2) return lv_pick<NP, 2, 2>(nElems, s, P);
    if (lv == 3) return lv_pick<NP, 2, 3>(nElems, s, P);
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
