// Host launchers of the Gauss-node MHD kernels (gauss_mhd.cuh): the surface integral for the volume
// fluxes 0, 1, 10, 12 and the BR1 / BR2 lifting with the viscous / resistive terms, N = 1..7.
#include "gauss_mhd.cuh"
#include "launch.h"

namespace fluxo {

namespace {
template <int NP, int VF>
cudaError_t surf_mhd_t(int nElems, cudaStream_t s, const KParams& P) {
  constexpr size_t smem = gauss::surf_mhd_smem_bytes<NP, VF>();
  static std::atomic<unsigned long long> attr{0};
  auto k = gauss::surf_mhd_kernel<NP, VF>;
  cudaError_t e = smem_attr_once(k, smem, attr);
  if (e != cudaSuccess) return e;
  k<<<nElems, NP * NP * NP, smem, s>>>(P);
  return cudaGetLastError();
}

template <int NP>
cudaError_t surf_mhd_np(int vf, int nElems, cudaStream_t s, const KParams& P) {
  switch (vf) {
    case 0: return surf_mhd_t<NP, 0>(nElems, s, P);
    case 1: return surf_mhd_t<NP, 1>(nElems, s, P);
    case 10: return surf_mhd_t<NP, 10>(nElems, s, P);
    case 12: return surf_mhd_t<NP, 12>(nElems, s, P);
    default: return cudaErrorInvalidValue;
  }
}
template <int NP, int LIFT>
cudaError_t lift_mhd_t(int nElems, cudaStream_t s, const KParams& P) {
  constexpr size_t smem = gauss::mlift_smem_bytes<NP>();
  static std::atomic<unsigned long long> attr{0};
  auto k = gauss::mhd_lift_visc_kernel<NP, LIFT>;
  cudaError_t e = smem_attr_once(k, smem, attr);
  if (e != cudaSuccess) return e;
  k<<<nElems, NP * NP * NP, smem, s>>>(P);
  return cudaGetLastError();
}

template <int NP>
cudaError_t lift_mhd_np(int lift, int nElems, cudaStream_t s, const KParams& P) {
  if (lift == 1) return lift_mhd_t<NP, 1>(nElems, s, P);
  if (lift == 2) return lift_mhd_t<NP, 2>(nElems, s, P);
  return cudaErrorInvalidValue;
}
}  // namespace

cudaError_t launch_gauss_mhd_lift_visc(int NP, int lift, int nElems, cudaStream_t s, const KParams& P) {
  switch (NP) {
    case 2: return lift_mhd_np<2>(lift, nElems, s, P);
    case 3: return lift_mhd_np<3>(lift, nElems, s, P);
    case 4: return lift_mhd_np<4>(lift, nElems, s, P);
    case 5: return lift_mhd_np<5>(lift, nElems, s, P);
    case 6: return lift_mhd_np<6>(lift, nElems, s, P);
    case 7: return lift_mhd_np<7>(lift, nElems, s, P);
    case 8: return lift_mhd_np<8>(lift, nElems, s, P);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_gauss_surf_mhd(int NP, int vf, int nElems, cudaStream_t s, const KParams& P) {
  switch (NP) {
    case 2: return surf_mhd_np<2>(vf, nElems, s, P);
    case 3: return surf_mhd_np<3>(vf, nElems, s, P);
    case 4: return surf_mhd_np<4>(vf, nElems, s, P);
    case 5: return surf_mhd_np<5>(vf, nElems, s, P);
    case 6: return surf_mhd_np<6>(vf, nElems, s, P);
    case 7: return surf_mhd_np<7>(vf, nElems, s, P);
    case 8: return surf_mhd_np<8>(vf, nElems, s, P);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fluxo
