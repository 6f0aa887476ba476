// Host launcher of the Gauss-node surface integral with the split-form correction (gauss.cuh):
// every volume flux of the split form, N = 1..7.
#include "gauss.cuh"
#include "launch.h"

namespace fluxo {

namespace {
template <int NP, int VF>
cudaError_t surf_t(int nElems, cudaStream_t s, const KParams& P) {
  constexpr size_t smem = gauss::surf_smem_bytes<NP, VF>();
  static std::atomic<unsigned long long> attr{0};
  auto k = gauss::surf_kernel<NP, VF>;
  cudaError_t e = smem_attr_once(k, smem, attr);
  if (e != cudaSuccess) return e;
  k<<<nElems, NP * NP * NP, smem, s>>>(P);
  return cudaGetLastError();
}

template <int NP>
cudaError_t surf_np(int vf, int nElems, cudaStream_t s, const KParams& P) {
#define FLUXO_GS_VF(V) \
  case V: return surf_t<NP, V>(nElems, s, P);
  switch (vf) {
    FLUXO_GS_VF(0) FLUXO_GS_VF(1) FLUXO_GS_VF(2) FLUXO_GS_VF(3) FLUXO_GS_VF(4) FLUXO_GS_VF(5)
    FLUXO_GS_VF(6) FLUXO_GS_VF(7) FLUXO_GS_VF(8) FLUXO_GS_VF(9) FLUXO_GS_VF(10) FLUXO_GS_VF(32)
    default: return cudaErrorInvalidValue;
  }
#undef FLUXO_GS_VF
}
}  // namespace

cudaError_t launch_gauss_surf(int NP, int vf, int nElems, cudaStream_t s, const KParams& P) {
  switch (NP) {
    case 2: return surf_np<2>(vf, nElems, s, P);
    case 3: return surf_np<3>(vf, nElems, s, P);
    case 4: return surf_np<4>(vf, nElems, s, P);
    case 5: return surf_np<5>(vf, nElems, s, P);
    case 6: return surf_np<6>(vf, nElems, s, P);
    case 7: return surf_np<7>(vf, nElems, s, P);
    case 8: return surf_np<8>(vf, nElems, s, P);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fluxo
