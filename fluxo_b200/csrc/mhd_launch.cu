// Host launchers of the MHD face, lifting-flux, lifting + viscous and time-step kernels.
#include "launch.h"
#include "mhd_lifting.cuh"

namespace fluxo {

bool mhd_riemann_supported(int RS) {
  return (RS >= 0 && RS <= 5) || (RS >= 10 && RS <= 15);
}
bool mhd_volume_flux_supported(int VF) { return VF == 0 || VF == 1 || VF == 10 || VF == 12; }

namespace {
template <int RS>
cudaError_t face_rs(bool visc, int NP, int nSides, cudaStream_t s, const KParams& P) {
  const size_t n = (size_t)nSides * NP * NP;
  const int bs = 128;
  const unsigned grid = (unsigned)((n + bs - 1) / bs);
  if (visc) mhd::face_kernel<RS, true><<<grid, bs, 0, s>>>(P, NP);
  else mhd::face_kernel<RS, false><<<grid, bs, 0, s>>>(P, NP);
  return cudaGetLastError();
}

template <int NP, int LIFT>
cudaError_t lift_visc_np(int nElems, cudaStream_t s, const KParams& P) {
  constexpr int EPB = mhd::epb<NP>();
  constexpr size_t smem = mhd::lv_smem_bytes<NP>();
  auto k = mhd::lift_visc_kernel<NP, LIFT>;
  static std::atomic<unsigned long long> attr{0};
  cudaError_t e = smem_attr_once(k, smem, attr);
  if (e != cudaSuccess) return e;
  k<<<(nElems + EPB - 1) / EPB, EPB * NP * NP * NP, smem, s>>>(P);
  return cudaGetLastError();
}

template <int NP>
cudaError_t timestep_np(bool visc, int nElems, cudaStream_t s, const KParams& P, unsigned long long* dtBits,
                        int* errKey) {
  constexpr int EPB = (256 / (NP * NP * NP)) > 0 ? (256 / (NP * NP * NP)) : 1;
  const unsigned grid = (unsigned)((nElems + EPB - 1) / EPB);
  if (visc) mhd::timestep_kernel<NP, true><<<grid, EPB * NP * NP * NP, 0, s>>>(P, dtBits, errKey);
  else mhd::timestep_kernel<NP, false><<<grid, EPB * NP * NP * NP, 0, s>>>(P, dtBits, errKey);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_mhd_face(int RS, bool visc, int NP, int nSides, cudaStream_t s, const KParams& P) {
  switch (RS) {
    case 0: return face_rs<0>(visc, NP, nSides, s, P);
    case 1: return face_rs<1>(visc, NP, nSides, s, P);
    case 2: return face_rs<2>(visc, NP, nSides, s, P);
    case 3: return face_rs<3>(visc, NP, nSides, s, P);
    case 4: return face_rs<4>(visc, NP, nSides, s, P);
    case 5: return face_rs<5>(visc, NP, nSides, s, P);
    case 10: return face_rs<10>(visc, NP, nSides, s, P);
    case 11: return face_rs<11>(visc, NP, nSides, s, P);
    case 12: return face_rs<12>(visc, NP, nSides, s, P);
    case 13: return face_rs<13>(visc, NP, nSides, s, P);
    case 14: return face_rs<14>(visc, NP, nSides, s, P);
    case 15: return face_rs<15>(visc, NP, nSides, s, P);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_mhd_lift_flux(int NP, int nSides, cudaStream_t s, const KParams& P) {
  const size_t n = (size_t)nSides * NP * NP;
  const int bs = 128;
  const unsigned grid = (unsigned)((n + bs - 1) / bs);
  switch (P.lifting_var) {
    case 1: mhd::lift_flux_kernel<1><<<grid, bs, 0, s>>>(P, NP); break;
    case 2: mhd::lift_flux_kernel<2><<<grid, bs, 0, s>>>(P, NP); break;
    default: mhd::lift_flux_kernel<3><<<grid, bs, 0, s>>>(P, NP); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_mhd_lift_visc(int NP, int lift, int nElems, cudaStream_t s, const KParams& P) {
#define FLUXO_MHD_LV(np)                                                   \
  case np:                                                                 \
    return lift == 2 ? lift_visc_np<np, 2>(nElems, s, P) : lift_visc_np<np, 1>(nElems, s, P);
  switch (NP) {
    FLUXO_MHD_LV(2) FLUXO_MHD_LV(3) FLUXO_MHD_LV(4) FLUXO_MHD_LV(5) FLUXO_MHD_LV(6) FLUXO_MHD_LV(7) FLUXO_MHD_LV(8)
    default: return cudaErrorInvalidValue;
  }
#undef FLUXO_MHD_LV
}

cudaError_t launch_mhd_timestep(int NP, bool visc, int nElems, cudaStream_t s, const KParams& P,
                                unsigned long long* dtBits, int* errKey) {
  switch (NP) {
    case 2: return timestep_np<2>(visc, nElems, s, P, dtBits, errKey);
    case 3: return timestep_np<3>(visc, nElems, s, P, dtBits, errKey);
    case 4: return timestep_np<4>(visc, nElems, s, P, dtBits, errKey);
    case 5: return timestep_np<5>(visc, nElems, s, P, dtBits, errKey);
    case 6: return timestep_np<6>(visc, nElems, s, P, dtBits, errKey);
    case 7: return timestep_np<7>(visc, nElems, s, P, dtBits, errKey);
    case 8: return timestep_np<8>(visc, nElems, s, P, dtBits, errKey);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fluxo
