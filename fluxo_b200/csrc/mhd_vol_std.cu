// MHD volume kernel instantiations: standard DG volume fluxes (0, 1).
#include "mhd_vol_impl.cuh"

namespace fluxo {
cudaError_t launch_mhd_volume_std(int NP, int VF, int nElems, cudaStream_t s, const KParams& P) {
  if (VF == 0) return mhd_detail::volume_vf<0>(NP, nElems, s, P);
  if (VF == 1) return mhd_detail::volume_vf<1>(NP, nElems, s, P);
  return cudaErrorInvalidValue;
}
}  // namespace fluxo
