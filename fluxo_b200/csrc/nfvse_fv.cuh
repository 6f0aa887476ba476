// Launch templates of the NFVSE subcell FV kernel (shared by the MHD and Euler / Navier-Stokes
// launchers, which instantiate them in separate translation units).
#pragma once
#include "nfvse.cuh"

namespace fluxo {
namespace nfvse {

template <bool MHD, int NP, int RS>
cudaError_t fv_np(int grid, cudaStream_t s, const KParams& P) {
  constexpr size_t smem = fv_smem_bytes<NP>();
  auto k = fv_kernel<NP, RS, MHD>;
  static std::atomic<unsigned long long> attr{0};
  cudaError_t e = smem_attr_once(k, smem, attr);
  if (e != cudaSuccess) return e;
  k<<<grid, NP * NP * NP, smem, s>>>(P);
  return cudaGetLastError();
}

template <bool MHD, int RS>
cudaError_t fv_rs(int NP, int grid, cudaStream_t s, const KParams& P) {
  switch (NP) {
    case 3: return fv_np<MHD, 3, RS>(grid, s, P);
    case 4: return fv_np<MHD, 4, RS>(grid, s, P);
    case 5: return fv_np<MHD, 5, RS>(grid, s, P);
    case 6: return fv_np<MHD, 6, RS>(grid, s, P);
    case 7: return fv_np<MHD, 7, RS>(grid, s, P);
    case 8: return fv_np<MHD, 8, RS>(grid, s, P);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace nfvse
}  // namespace fluxo
