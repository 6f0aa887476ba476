// Oracle test infrastructure (CPU only, never on the product path).
//
// C interface of the CPU restatement of the reference DGSEM right-hand side
// and LSERK time step (FLUXO, Fortran).  Only tests/, __graft_entry__.smoke()
// and the cpu_baseline leg of bench.py load this library, as the checker.
//
// Arrays use the reference's Fortran layouts (first index fastest):
//   U, Ut          (nVar,0:N,0:N,0:N,nElems)          dg/dg_vars.f90:75-80
//   Metrics_*Tilde (3,0:N,0:N,0:N,nElems), sJ (0:N,0:N,0:N,nElems)
//   NormVec, TangVec1, TangVec2 (3,0:N,0:N,nSides), SurfElem (0:N,0:N,nSides)
//   SideToElem (5,nSides), ElemToSide (2,6,nElems); element/side ids 1-based,
//   -1 for "none", exactly as mesh/mesh_vars.f90 and mesh/prepare_mesh.f90.
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_params {
  int N;                  /* polynomial degree (parameter.ini: N) */
  int nElems[3];          /* periodic box, elements per direction */
  double xmin[3], xmax[3];
  int NGeo;               /* geometry degree of the node coordinates */
  double deform_amp;      /* X_d += amp*prod_e sin(2*pi*(x_e-c_e)/L_e) */
  int eqn;                /* 0 Euler (PARABOLIC=0), 1 Navier-Stokes, 2 ideal MHD + GLM, 3 MHD + GLM with PARABOLIC */
  int lifting;            /* 1 BR1, 2 BR2 */
  int lifting_var;        /* 1 cons_var, 2 prim_var, 3 entropy_var */
  int visc;               /* PP_VISC: 0 constant, 1 Sutherland, 2 power law */
  int riemann;            /* parameter.ini: Riemann */
  int volume_flux;        /* parameter.ini: VolumeFlux */
  double kappa, R, Pr, mu0, Ts, Tref, ExpoSuth, ExpoPow, etaBR2;
  int ini_exact_func;     /* parameter.ini: IniExactFunc */
  double adv_vel[3];      /* AdvVel */
  double ini_amplitude;   /* IniAmplitude */
  double ini_wavenumber[3]; /* IniWaveNumber */
  double ini_frequency;   /* IniFrequency */
  double ref_state[5];    /* RefState (primitive) used by IniExactFunc=1 */
  double cfl_scale, dfl_scale;  /* CFLScale, DFLScale (unscaled input values) */
  int time_disc;          /* 0 carpenterrk4-5, 1 standardrk3-3, 2 niegemannrk4-14, 3 toulorgerk4-8c,
                             4 toulorgerk3-7c, 5 toulorgerk4-8f, 6 ketchesonrk4-20, 7 ketchesonrk4-18,
                             8 ssprk4-5, 9 ssprk3-3 */
  /* MHD (eqn 2: ideal, eqn 3: with eta / mu, PARABOLIC), equation/mhd/equation.f90:134-285 */
  double mu_0;            /* mu_0 (magnetic permeability) */
  double eta;             /* eta (resistivity); the viscosity mu is mu0 above */
  double glm_scale, glm_scr;  /* GLM_scale, GLM_scr */
  double glm_ch;          /* GLM_ch before the first CALCTIMESTEP */
  int noncons;            /* NONCONS: 0 off, 1 Powell, 2 Brackbill, 3 Janhunen */
  int nc_glm;             /* PP_NC_GLM */
  double mhd_ref_state[2][8];  /* RefState 1 and 2 (rho,u,v,w,p,B1,B2,B3) */
  double ini_center[3];   /* IniCenter */
  double ini_halfwidth;   /* IniHalfwidth */
  /* NFVSE shock capturing (shockcapturing/nfvse.f90:63-260), SubFVMethod = 1..4 */
  int nfvse;              /* SHOCK_NFVSE on/off */
  int compute_alpha;      /* ComputeAlpha: 1 Persson-Peraire indicator, 3 fixed ShockBlendCoef,
                             20 random values drawn once and kept */
  double shock_blend_coef;
  int modal_threshold;    /* ModalThreshold 1 or 2 */
  double alpha_max, alpha_min, space_prop_factor;
  int space_prop_sweeps;
  double time_rel_factor;
  int indicator_quantity; /* ShockIndicatorQuantity: 1 Density, 2 Pressure, 3 DensityTimesPressure, 4 KinEnergy */
  int sub_fv_method;      /* SubFVMethod: 1 first order, 2 TVD (minmod reconstruction of primitive variables),
                             3 TVD-ES (TVD states, entropy-stable switch), 4 TVD-Fjordholm (reconstruction of
                             the scaled entropy variables) */
  int recons_boundaries;  /* ReconsBoundaries (SubFVMethod 2-4): 1 none, 2 central, 3 neighbour element */
  int nfvse_corr;         /* NFVSE_CORR (CMake FLUXO_SHOCK_NFVSE_CORR): positivity correction after each stage */
  double posit_corr_factor;  /* PositCorrFactor */
  int posit_max_iter;     /* PositMaxIter */
  int node_type;          /* PP_NodeType (CMake FLUXO_DISC_NODETYPE): 1 Gauss, 2 (or 0) Gauss-Lobatto */
} orc_params;

void* orc_create(const orc_params* p);
/* The same case on a HOPR mesh given by the arrays of its file (mesh/mesh_readin.f90:168-716):
   ElemInfo(6,nElems), SideInfo(5,nSideInfo), BCType(4,nBCs), NodeCoords(3,(NGeo+1)^3*nElems) on
   equidistant (nodesGL=0) or Gauss-Lobatto (nodesGL=1) points; p->nElems, xmin, xmax, NGeo and
   deform_amp are ignored.  Conforming meshes whose boundaries are all periodic. */
void* orc_create_hopr(const orc_params* p, int nElems, const int* ElemInfo, int nSideInfo, const int* SideInfo,
                      int nBCs, const int* BCType, int NGeo, int nodesGL, const double* NodeCoords,
                      double meshScale, int useCurveds);
void orc_destroy(void* h);
void orc_sizes(void* h, int* nElems, int* nSides, int* nVar, int* N);
/* Mesh arrays in the reference layout (any pointer may be NULL). */
void orc_get_mesh(void* h, int* SideToElem, int* ElemToSide, double* Mf, double* Mg,
                  double* Mh, double* sJ, double* NormVec, double* TangVec1,
                  double* TangVec2, double* SurfElem, double* Elem_xGP);
/* Replace the geometry (e.g. to feed externally built metrics). */
void orc_set_metrics(void* h, const double* Mf, const double* Mg, const double* Mh,
                     const double* sJ, const double* NormVec, const double* TangVec1,
                     const double* TangVec2, const double* SurfElem);
void orc_get_U(void* h, double* U);
void orc_set_U(void* h, const double* U);
/* DGTimeDerivative_weakForm(t): U -> Ut (returns Ut copy) */
void orc_dg_time_derivative(void* h, double t, double* Ut);
/* Volume gradients of the primitive variables after the last RHS (NS only). */
void orc_get_gradients(void* h, double* gx, double* gy, double* gz);
double orc_calc_timestep(void* h, int* errType);
void orc_timestep(void* h, double t, double dt);
/* Runs the TimeDisc loop for n steps (dt from CALCTIMESTEP each step,
   clipped to tEnd), returns the final time. */
double orc_run(void* h, double t, double tEnd, int maxIter, int* nSteps);
/* Analysis at time t: L2/Linf error vs IniExactFunc (nVar each, NULL ok),
   entropy, dS/dU*Ut, kinetic energy, enstrophy (volume averaged). */
void orc_analyze(void* h, double t, double* L2, double* Linf, double* entropy,
                 double* dSdU_Ut, double* ekin, double* enstrophy);
/* Exact function at points: x(3,n) -> U(nVar,n). */
void orc_exact_func(void* h, int func, double t, int n, const double* x, double* U);
/* 1D operators: xGP,wGP (N+1), D, Dvolsurf, D_hat (N+1)^2 column-major. */
void orc_basis(int N, double* xGP, double* wGP, double* wBary, double* D,
               double* Dvolsurf, double* Dhat, double* Lminus, double* Lplus);
/* Operation counter (only meaningful in the counting build). */
uint64_t orc_flops(void);
/* Per-phase counts: 0 split-form volume, 1 lifting, 2 viscous volume, 3 face fluxes,
   4 surface integral, 5 Jacobian + source. */
uint64_t orc_phase_flops(int phase);
void orc_reset_flops(void);
/* Two-point volume flux and Riemann solver at single points (unit tests). */
void orc_volume_flux(void* h, const double* UL, const double* UR, const double* mL,
                     const double* mR, double* F);
void orc_riemann_point(void* h, const double* UL, const double* UR, const double* nv,
                       const double* t1, const double* t2, double* F);
double orc_ln_mean(double aL, double aR);
/* NFVSE: blending coefficient alpha(nElems) of the last right-hand side. */
void orc_get_alpha(void* h, double* alpha);
/* NFVSE: alpha(nElems) that the next right-hand side starts from (ComputeAlpha 20 keeps it). */
void orc_set_alpha(void* h, const double* alpha);
/* Gauss nodes: SurfMetrics(3,0:N,0:N,6,nElems) of mesh/metrics.f90:420-427 (NULL-safe; LGL: zeros). */
void orc_get_surf_metrics(void* h, double* SurfMetrics);
/* NFVSE_CORR: element + 1 whose safe state had negative density or pressure (0: none). */
int orc_corr_error(void* h);
/* MHD: the GLM cleaning speed GLM_ch (set by CALCTIMESTEP, or explicitly). */
void orc_set_glm_ch(void* h, double ch);
double orc_get_glm_ch(void* h);

#ifdef __cplusplus
}
#endif
