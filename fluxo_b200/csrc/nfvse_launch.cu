// Host launchers of the NFVSE kernels (indicator, propagation, subcell FV of MHD).
#include <algorithm>

#include "launch.h"
#include "nfvse.cuh"

namespace fluxo {

namespace {
template <int NP, int NV>
cudaError_t alpha_np(int nElems, cudaStream_t s, const KParams& P) {
  constexpr int NP3 = NP * NP * NP, EPB = (256 / NP3) > 0 ? (256 / NP3) : 1;
  nfvse::alpha_kernel<NP, NV><<<(nElems + EPB - 1) / EPB, EPB * NP3, 0, s>>>(P);
  return cudaGetLastError();
}

template <int NP, int RS>
cudaError_t fv_np(int grid, cudaStream_t s, const KParams& P) {
  constexpr size_t smem = nfvse::fv_smem_bytes<NP>();
  auto k = nfvse::fv_kernel_mhd<NP, RS>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k<<<grid, NP * NP * NP, smem, s>>>(P);
  return cudaGetLastError();
}

template <int RS>
cudaError_t fv_rs(int NP, int grid, cudaStream_t s, const KParams& P) {
  switch (NP) {
    case 3: return fv_np<3, RS>(grid, s, P);
    case 4: return fv_np<4, RS>(grid, s, P);
    case 5: return fv_np<5, RS>(grid, s, P);
    case 6: return fv_np<6, RS>(grid, s, P);
    case 7: return fv_np<7, RS>(grid, s, P);
    case 8: return fv_np<8, RS>(grid, s, P);
    default: return cudaErrorInvalidValue;
  }
}
}  // namespace

cudaError_t launch_nfvse_alpha(int NP, bool mhd, int nElems, cudaStream_t s, const KParams& P, double* scratch) {
  cudaError_t e;
#define FLUXO_NF_A(np) \
  case np: e = mhd ? alpha_np<np, 9>(nElems, s, P) : alpha_np<np, 5>(nElems, s, P); break;
  switch (NP) {
    FLUXO_NF_A(3) FLUXO_NF_A(4) FLUXO_NF_A(5) FLUXO_NF_A(6) FLUXO_NF_A(7) FLUXO_NF_A(8)
    default: return cudaErrorInvalidValue;
  }
#undef FLUXO_NF_A
  if (e != cudaSuccess) return e;
  const int bs = 256, grid = (nElems + bs - 1) / bs;
  if (P.propSweeps <= 0) {
    nfvse::list_kernel<<<grid, bs, 0, s>>>(P);
    return cudaGetLastError();
  }
  // sweep 1 reads the raw values; later sweeps read the previous sweep's result (copied to scratch)
  for (int sw = 1; sw <= P.propSweeps; ++sw) {
    const double* src = P.alphaRaw;
    if (sw > 1) {
      e = cudaMemcpyAsync(scratch, P.alpha, sizeof(double) * nElems, cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return e;
      src = scratch;
    }
    nfvse::propagate_kernel<<<grid, bs, 0, s>>>(P, src, sw == P.propSweeps);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_nfvse_fv(int RS, int NP, int nElems, int nSMs, cudaStream_t s, const KParams& P) {
  const int grid = std::min(nElems, 8 * nSMs);
  switch (RS) {
    case 0: return fv_rs<0>(NP, grid, s, P);
    case 1: return fv_rs<1>(NP, grid, s, P);
    case 2: return fv_rs<2>(NP, grid, s, P);
    case 3: return fv_rs<3>(NP, grid, s, P);
    case 4: return fv_rs<4>(NP, grid, s, P);
    case 5: return fv_rs<5>(NP, grid, s, P);
    case 10: return fv_rs<10>(NP, grid, s, P);
    case 11: return fv_rs<11>(NP, grid, s, P);
    case 12: return fv_rs<12>(NP, grid, s, P);
    case 13: return fv_rs<13>(NP, grid, s, P);
    case 14: return fv_rs<14>(NP, grid, s, P);
    case 15: return fv_rs<15>(NP, grid, s, P);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fluxo
