// Launch templates of the NFVSE subcell FV kernel and of the NFVSE_CORR correction kernel (shared by the
// MHD and Euler / Navier-Stokes launchers, which instantiate them in separate translation units).
#pragma once
#include "nfvse.cuh"

namespace fluxo {
namespace nfvse {

template <bool MHD, int NP, int RS, int ES>
cudaError_t fv_np(int grid, cudaStream_t s, const KParams& P) {
  constexpr size_t smem = fv_smem_bytes<NP, ES>();
  auto k = fv_kernel<NP, RS, MHD, ES>;
  static std::atomic<unsigned long long> attr{0};
  cudaError_t e = smem_attr_once(k, smem, attr);
  if (e != cudaSuccess) return e;
  k<<<grid, NP * NP * NP, smem, s>>>(P);
  return cudaGetLastError();
}

// SubFVMethod 3 / 4 exist only for the solvers with dissipation matrices (checked at create)
template <bool MHD, int NP, int RS>
cudaError_t fv_es(int grid, cudaStream_t s, const KParams& P) {
  if constexpr (has_dissip_matrices<MHD, RS>()) {
    if (P.subFV == 3) return fv_np<MHD, NP, RS, 3>(grid, s, P);
    if (P.subFV == 4) return fv_np<MHD, NP, RS, 4>(grid, s, P);
  }
  if (P.subFV > 2) return cudaErrorInvalidValue;
  return fv_np<MHD, NP, RS, 0>(grid, s, P);
}

template <bool MHD, int RS>
cudaError_t fv_rs(int NP, int grid, cudaStream_t s, const KParams& P) {
  switch (NP) {
    case 3: return fv_es<MHD, 3, RS>(grid, s, P);
    case 4: return fv_es<MHD, 4, RS>(grid, s, P);
    case 5: return fv_es<MHD, 5, RS>(grid, s, P);
    case 6: return fv_es<MHD, 6, RS>(grid, s, P);
    case 7: return fv_es<MHD, 7, RS>(grid, s, P);
    case 8: return fv_es<MHD, 8, RS>(grid, s, P);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace nfvse
}  // namespace fluxo
