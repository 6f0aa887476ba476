// Host-side launchers of the templated kernels (one translation unit per volume flux
// family so that the instantiations compile in parallel).
#pragma once
#include <cstddef>
#include <string>
#include <cuda_runtime.h>
#include "common.cuh"

struct fluxo_cfg;  // include/fluxo_gpu.h

namespace fluxo {

struct LaunchError {
  cudaError_t err;
};

// Volume kernel: NP in 2..9, VF in {0,1,2,5,10,32}, in the launch shape the autotuner chose for
// (NP, VF, visc) (vol_shapes.h; shape 0 until tuned or pinned).  Returns cudaErrorInvalidValue for
// unsupported combinations.
cudaError_t launch_volume(int NP, int VF, bool visc, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_volume_shape(int NP, int VF, bool visc, int shape, int nElems, cudaStream_t s,
                                const KParams& P);
cudaError_t launch_volume_vf0(int NP, bool visc, int shape, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_volume_vf1(int NP, bool visc, int shape, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_volume_vf2(int NP, bool visc, int shape, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_volume_vf3(int NP, bool visc, int shape, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_volume_vf4(int NP, bool visc, int shape, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_volume_vf5(int NP, bool visc, int shape, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_volume_vf6(int NP, bool visc, int shape, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_volume_vf7(int NP, bool visc, int shape, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_volume_vf8(int NP, bool visc, int shape, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_volume_vf9(int NP, bool visc, int shape, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_volume_vf10(int NP, bool visc, int shape, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_volume_vf32(int NP, bool visc, int shape, int nElems, cudaStream_t s, const KParams& P);
// Autotuner of the volume kernel's launch shape: times every candidate shape of (NP, VF, visc) on the
// given data (stage-0 launches, which write only Ut) and keeps the fastest for the process; a no-op
// once (NP, VF, visc) is tuned or pinned, or when it has one candidate.  Not callable during stream
// capture (it synchronises the stream).
cudaError_t tune_volume(int NP, int VF, bool visc, int nElems, cudaStream_t s, const KParams& P);
// Chosen shape (-1: not tuned), pin (shape < 0: back to untuned), candidate count.
int volume_shape(int NP, int VF, bool visc);
bool pin_volume_shape(int NP, int VF, bool visc, int shape);
int volume_shape_count(int NP);

cudaError_t launch_face_flux(int RS, bool visc, int NP, int nSides, cudaStream_t s, const KParams& P);
cudaError_t launch_lift_flux(int NP, int nSides, cudaStream_t s, const KParams& P);
cudaError_t launch_gradient(int NP, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_lift_visc(int NP, int lift, int lv, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_timestep(int NP, bool visc, int nElems, cudaStream_t s, const KParams& P,
                            unsigned long long* dtBits, int* errKey);
bool riemann_supported(int RS);
bool volume_flux_supported(int VF);

// MHD + GLM (9 variables): face (Riemann 0,1,4,10-15), lifting flux, lifting + viscous, volume
// (VF 0,1 standard; 10,12 entropy conserving), time step.  Non-conservative terms and the
// parabolic part are runtime flags of KParams.
bool mhd_riemann_supported(int RS);
bool mhd_volume_flux_supported(int VF);
cudaError_t launch_mhd_face(int RS, bool visc, int NP, int nSides, cudaStream_t s, const KParams& P);
cudaError_t launch_mhd_lift_flux(int NP, int nSides, cudaStream_t s, const KParams& P);
cudaError_t launch_mhd_lift_visc(int NP, int lift, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_mhd_volume_ec(int NP, int VF, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_mhd_volume_std(int NP, int VF, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_mhd_timestep(int NP, bool visc, int nElems, cudaStream_t s, const KParams& P,
                                unsigned long long* dtBits, int* errKey);

// NFVSE shock capturing: blending coefficient (indicator + propagation + list of blended elements;
// `scratch` holds nElems doubles for sweeps > 1) and the subcell FV volume integral of MHD.
// Gauss nodes (gauss.cuh): face states (ent: entropy-projected), lifting + viscous volume integral, and
// the surface integral with the split-form correction
cudaError_t launch_gauss_prolong(int NP, bool ent, bool mhd, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_gauss_lift_visc(int NP, int lift, int lv, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_gauss_surf(int NP, int vf, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_gauss_surf_mhd(int NP, int vf, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_gauss_mhd_lift_visc(int NP, int lift, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_nfvse_alpha(int NP, bool mhd, int nElems, cudaStream_t s, const KParams& P, double* scratch);
cudaError_t launch_nfvse_indicator(int NP, bool mhd, int nElems, cudaStream_t s, const KParams& P);
cudaError_t launch_nfvse_sweep(int nElems, cudaStream_t s, const KParams& P, const double* src, bool last);
cudaError_t launch_nfvse_list(int nElems, cudaStream_t s, const KParams& P);
// NFVSE_CORR: Apply_NFVSE_Correction of every element after a stage update with step b * dt (ut: the
// stage's Ut to correct as well, or null); errKey records elem*8 + 5 for a safe state that is not admissible
cudaError_t launch_nfvse_corr(int NP, bool mhd, int nElems, cudaStream_t s, const KParams& P, double* ut, double b,
                              int* errKey);
cudaError_t launch_nfvse_fv(int RS, int NP, int nElems, int nSMs, cudaStream_t s, const KParams& P);
cudaError_t launch_nfvse_fv_ns(int RS, int NP, int nElems, int nSMs, cudaStream_t s, const KParams& P);

// Analysis of a state (analyze.cu): per-element partial sums partial[nElems][K] with
// K = 3*nVar + 5: L2 error (nVar), collocation L2 error (nVar), L_inf error (nVar), entropy, dS/dU.Ut,
// kinetic energy, enstrophy, volume (unnormalised); res[K] receives their sums / maxima.
struct AnalyzeArgs {
  int nElems, NP, NA1, nVar, K;
  int mhd;
  int func;                          // exact function of the error norms (0: none)
  double t;
  const double *U, *Ut, *sJ, *xGP, *grad;  // Ut, xGP, grad may be null
  const double *wGP, *V, *wA;        // LGL weights, N -> NAnalyze interpolation [NA1][NP], NAnalyze weights
  double kappa, kappaM1, sKappaM1, s2mu_0;
  double refPrim[5], advVel[3], waveNumber[3], center[3], amplitude, frequency;
  double* partial;
};
size_t analyze_smem_bytes(int NP, int nVar, int threads);
cudaError_t launch_analyze(const AnalyzeArgs& A, double* res, cudaStream_t s);

// Host helpers of fluxo_gpu.cu for entry points without a handle: the per-N operator tables, and
// the message that fluxo_gpu_last_error(NULL, ...) returns (returns `code`).
void basis_tables_for(int N, BasisTables& B);
int record_unbound_error(int code, const std::string& msg);
// Equation constants of the Euler / Navier-Stokes kernels, and the LSERK tables with the scaled
// CFL / DFL numbers of a configuration (false for an unknown time_disc).
void fill_ns_physics(KParams& P, const fluxo_cfg& c);
bool time_disc_setup(const fluxo_cfg& c, double* RKA, double* RKb, double* RKc, int* nStages, double* CFLScale,
                     double* DFLScale);

}  // namespace fluxo
