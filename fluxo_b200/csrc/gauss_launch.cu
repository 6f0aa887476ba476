// Host launchers of the Gauss-node prolongation and lifting kernels (gauss.cuh), N = 1..7.
#include "gauss.cuh"
#include "launch.h"

namespace fluxo {

namespace {
template <int NP>
cudaError_t prolong_np(bool ent, bool mhd, int nElems, cudaStream_t s, const KParams& P) {
  if (mhd) {
    if (ent) gauss::prolong_kernel<NP, true, 9><<<nElems, NP * NP * NP, 0, s>>>(P);
    else gauss::prolong_kernel<NP, false, 9><<<nElems, NP * NP * NP, 0, s>>>(P);
  } else {
    if (ent) gauss::prolong_kernel<NP, true, 5><<<nElems, NP * NP * NP, 0, s>>>(P);
    else gauss::prolong_kernel<NP, false, 5><<<nElems, NP * NP * NP, 0, s>>>(P);
  }
  return cudaGetLastError();
}

template <int NP, int LIFT, int LV>
cudaError_t lift_t(int nElems, cudaStream_t s, const KParams& P) {
  constexpr size_t smem = gauss::lift_smem_bytes<NP>();
  static std::atomic<unsigned long long> attr{0};
  auto k = gauss::lift_visc_kernel<NP, LIFT, LV>;
  cudaError_t e = smem_attr_once(k, smem, attr);
  if (e != cudaSuccess) return e;
  k<<<nElems, NP * NP * NP, smem, s>>>(P);
  return cudaGetLastError();
}

template <int NP>
cudaError_t lift_np(int lift, int lv, int nElems, cudaStream_t s, const KParams& P) {
  if (lift == 1) {
    if (lv == 1) return lift_t<NP, 1, 1>(nElems, s, P);
    if (lv == 2) return lift_t<NP, 1, 2>(nElems, s, P);
    if (lv == 3) return lift_t<NP, 1, 3>(nElems, s, P);
  } else if (lift == 2) {
    if (lv == 1) return lift_t<NP, 2, 1>(nElems, s, P);
    if (lv == 2) return lift_t<NP, 2, 2>(nElems, s, P);
    if (lv == 3) return lift_t<NP, 2, 3>(nElems, s, P);
  }
  return cudaErrorInvalidValue;
}
}  // namespace

cudaError_t launch_gauss_prolong(int NP, bool ent, bool mhd, int nElems, cudaStream_t s, const KParams& P) {
  switch (NP) {
    case 2: return prolong_np<2>(ent, mhd, nElems, s, P);
    case 3: return prolong_np<3>(ent, mhd, nElems, s, P);
    case 4: return prolong_np<4>(ent, mhd, nElems, s, P);
    case 5: return prolong_np<5>(ent, mhd, nElems, s, P);
    case 6: return prolong_np<6>(ent, mhd, nElems, s, P);
    case 7: return prolong_np<7>(ent, mhd, nElems, s, P);
    case 8: return prolong_np<8>(ent, mhd, nElems, s, P);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_gauss_lift_visc(int NP, int lift, int lv, int nElems, cudaStream_t s, const KParams& P) {
  switch (NP) {
    case 2: return lift_np<2>(lift, lv, nElems, s, P);
    case 3: return lift_np<3>(lift, lv, nElems, s, P);
    case 4: return lift_np<4>(lift, lv, nElems, s, P);
    case 5: return lift_np<5>(lift, lv, nElems, s, P);
    case 6: return lift_np<6>(lift, lv, nElems, s, P);
    case 7: return lift_np<7>(lift, lv, nElems, s, P);
    case 8: return lift_np<8>(lift, lv, nElems, s, P);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fluxo
