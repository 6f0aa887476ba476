// Launcher of the Euler / Navier-Stokes NFVSE subcell FV kernel: every Riemann solver of the
// navierstokes module (the LLF-dissipation variants with the wave-speed maximum over each subcell
// face plane), N+1 = 3..8.
#include "launch.h"
#include "nfvse_fv.cuh"

namespace fluxo {

cudaError_t launch_nfvse_fv_ns(int RS, int NP, int nElems, int nSMs, cudaStream_t s, const KParams& P) {
  const int grid = nElems < 8 * nSMs ? nElems : 8 * nSMs;
#define FLUXO_NFV_CASE(K) \
  case K: return nfvse::fv_rs<false, K>(NP, grid, s, P);
  switch (RS) {
    FLUXO_NFV_CASE(0) FLUXO_NFV_CASE(1) FLUXO_NFV_CASE(2) FLUXO_NFV_CASE(3) FLUXO_NFV_CASE(4) FLUXO_NFV_CASE(5)
    FLUXO_NFV_CASE(6) FLUXO_NFV_CASE(7) FLUXO_NFV_CASE(8) FLUXO_NFV_CASE(9) FLUXO_NFV_CASE(10) FLUXO_NFV_CASE(11)
    FLUXO_NFV_CASE(12) FLUXO_NFV_CASE(13) FLUXO_NFV_CASE(14) FLUXO_NFV_CASE(15) FLUXO_NFV_CASE(16) FLUXO_NFV_CASE(17)
    FLUXO_NFV_CASE(18) FLUXO_NFV_CASE(19) FLUXO_NFV_CASE(20) FLUXO_NFV_CASE(21) FLUXO_NFV_CASE(22) FLUXO_NFV_CASE(23)
    FLUXO_NFV_CASE(24) FLUXO_NFV_CASE(32) FLUXO_NFV_CASE(33) FLUXO_NFV_CASE(44)
    default: return cudaErrorInvalidValue;
  }
#undef FLUXO_NFV_CASE
}

}  // namespace fluxo
