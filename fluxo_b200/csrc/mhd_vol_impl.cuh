// Instantiation helper of the MHD volume kernel for one volume flux (one translation unit each).
#pragma once
#include "launch.h"
#include "mhd_kernels.cuh"

namespace fluxo {
namespace mhd_detail {

template <int NP, int VF>
cudaError_t volume_np(int nElems, cudaStream_t s, const KParams& P) {
  constexpr int EPB = mhd::epb<NP>();
  constexpr size_t smem = mhd::vol_smem_bytes<NP, VF>();
  auto k = mhd::volume_kernel<NP, VF>;
  static std::atomic<unsigned long long> attr{0};
  cudaError_t e = smem_attr_once(k, smem, attr);
  if (e != cudaSuccess) return e;
  k<<<(nElems + EPB - 1) / EPB, mhd::vol_threads<NP>(), smem, s>>>(P);
  return cudaGetLastError();
}

template <int VF>
cudaError_t volume_vf(int NP, int nElems, cudaStream_t s, const KParams& P) {
  switch (NP) {
    case 2: return volume_np<2, VF>(nElems, s, P);
    case 3: return volume_np<3, VF>(nElems, s, P);
    case 4: return volume_np<4, VF>(nElems, s, P);
    case 5: return volume_np<5, VF>(nElems, s, P);
    case 6: return volume_np<6, VF>(nElems, s, P);
    case 7: return volume_np<7, VF>(nElems, s, P);
    case 8: return volume_np<8, VF>(nElems, s, P);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace mhd_detail
}  // namespace fluxo
