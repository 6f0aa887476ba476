// MHD volume kernel instantiations: entropy-conserving volume fluxes (Derigs 10, FloGor 12).
#include "mhd_vol_impl.cuh"

namespace fluxo {
cudaError_t launch_mhd_volume_ec(int NP, int VF, int nElems, cudaStream_t s, const KParams& P) {
  if (VF == 10) return mhd_detail::volume_vf<10>(NP, nElems, s, P);
  if (VF == 12) return mhd_detail::volume_vf<12>(NP, nElems, s, P);
  return cudaErrorInvalidValue;
}
}  // namespace fluxo
