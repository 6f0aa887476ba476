// Host launchers of the NFVSE kernels (indicator, propagation, subcell FV of MHD; the Euler /
// Navier-Stokes subcell FV launcher is in nfvse_ns.cu).
#include <algorithm>

#include "launch.h"
#include "nfvse_fv.cuh"

namespace fluxo {

namespace {
template <int NP, int NV>
cudaError_t alpha_np(int nElems, cudaStream_t s, const KParams& P) {
  constexpr int NP3 = NP * NP * NP, EPB = (256 / NP3) > 0 ? (256 / NP3) : 1;
  nfvse::alpha_kernel<NP, NV><<<(nElems + EPB - 1) / EPB, EPB * NP3, 0, s>>>(P);
  return cudaGetLastError();
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

// The steps of launch_nfvse_alpha one by one, for a partitioned solve that exchanges the ghost elements'
// coefficients between them: the indicator (alphaRaw), one propagation sweep from src (the last one
// also lists the blended elements), or the list without propagation.
cudaError_t launch_nfvse_indicator(int NP, bool mhd, int nElems, cudaStream_t s, const KParams& P) {
#define FLUXO_NF_I(np) \
  case np: return mhd ? alpha_np<np, 9>(nElems, s, P) : alpha_np<np, 5>(nElems, s, P);
  switch (NP) {
    FLUXO_NF_I(3) FLUXO_NF_I(4) FLUXO_NF_I(5) FLUXO_NF_I(6) FLUXO_NF_I(7) FLUXO_NF_I(8)
    default: return cudaErrorInvalidValue;
  }
#undef FLUXO_NF_I
}

cudaError_t launch_nfvse_sweep(int nElems, cudaStream_t s, const KParams& P, const double* src, bool last) {
  const int bs = 256, grid = (nElems + bs - 1) / bs;
  nfvse::propagate_kernel<<<grid, bs, 0, s>>>(P, src, last);
  return cudaGetLastError();
}

cudaError_t launch_nfvse_list(int nElems, cudaStream_t s, const KParams& P) {
  const int bs = 256, grid = (nElems + bs - 1) / bs;
  nfvse::list_kernel<<<grid, bs, 0, s>>>(P);
  return cudaGetLastError();
}

cudaError_t launch_nfvse_corr(int NP, bool mhd, int nElems, cudaStream_t s, const KParams& P, double* ut, double b,
                              int* errKey) {
#define FLUXO_NF_C(np)                                                                                        \
  case np:                                                                                                    \
    if (mhd) nfvse::corr_kernel<np, 9><<<nElems, np * np * np, 0, s>>>(P, ut, b, errKey);                      \
    else nfvse::corr_kernel<np, 5><<<nElems, np * np * np, 0, s>>>(P, ut, b, errKey);                          \
    break;
  switch (NP) {
    FLUXO_NF_C(3) FLUXO_NF_C(4) FLUXO_NF_C(5) FLUXO_NF_C(6) FLUXO_NF_C(7) FLUXO_NF_C(8)
    default: return cudaErrorInvalidValue;
  }
#undef FLUXO_NF_C
  return cudaGetLastError();
}

cudaError_t launch_nfvse_fv(int RS, int NP, int nElems, int nSMs, cudaStream_t s, const KParams& P) {
  const int grid = std::min(nElems, 8 * nSMs);
  switch (RS) {
    case 0: return nfvse::fv_rs<true, 0>(NP, grid, s, P);
    case 1: return nfvse::fv_rs<true, 1>(NP, grid, s, P);
    case 2: return nfvse::fv_rs<true, 2>(NP, grid, s, P);
    case 3: return nfvse::fv_rs<true, 3>(NP, grid, s, P);
    case 4: return nfvse::fv_rs<true, 4>(NP, grid, s, P);
    case 5: return nfvse::fv_rs<true, 5>(NP, grid, s, P);
    case 10: return nfvse::fv_rs<true, 10>(NP, grid, s, P);
    case 11: return nfvse::fv_rs<true, 11>(NP, grid, s, P);
    case 12: return nfvse::fv_rs<true, 12>(NP, grid, s, P);
    case 13: return nfvse::fv_rs<true, 13>(NP, grid, s, P);
    case 14: return nfvse::fv_rs<true, 14>(NP, grid, s, P);
    case 15: return nfvse::fv_rs<true, 15>(NP, grid, s, P);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fluxo
