/*
 * fluxo_gpu.h — C ABI of the B200 (sm_100a, FP64) DGSEM right-hand side and
 * LSERK time step.  It is the drop-in boundary for the reference's
 * DGTimeDerivative / TimeStep / CALCTIMESTEP path: a Fortran host binds these
 * entry points with ISO_C_BINDING (a TYPE, BIND(C) that mirrors fluxo_cfg field
 * for field, and one INTERFACE block per entry point) and keeps its own
 * parameter.ini parsing, mesh reading, analysis and output.
 *
 * Conventions
 *  - Every entry point returns an int status: FLUXO_OK (0) or a negative
 *    FLUXO_E* code.  The library never calls exit(); fluxo_gpu_last_error()
 *    returns the message of the last failure on a handle.
 *  - Host arrays use the reference's Fortran layouts, first index fastest:
 *      U, Ut          (nVar,0:N,0:N,0:N,nElems)      src/dg/dg_vars.f90:75-80
 *      Metrics_fTilde (3,0:N,0:N,0:N,nElems) (also g,h)  src/mesh/mesh.f90:251-256
 *      sJ             (0:N,0:N,0:N,nElems)
 *      NormVec, TangVec1, TangVec2 (3,0:N,0:N,1:nSides); SurfElem (0:N,0:N,1:nSides)
 *      SideToElem     (5,1:nSides)  ElemToSide (2,6,nElems)   1-based ids, -1 = none
 *  - Only conforming meshes whose sides are all inner sides (periodic boxes):
 *    nBCSides = 0, no mortars, no MPI sides (the same single-process side
 *    ranges as src/mesh/mesh.f90:171-183 with firstInnerSide = 1).
 *  - One handle owns one CUDA stream; calls on a handle must be serialised by
 *    the caller.  Distinct handles may be used from distinct host threads.
 */
#ifndef FLUXO_GPU_H
#define FLUXO_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  FLUXO_OK = 0,
  FLUXO_EINVAL_CFG = -1,  /* unsupported or inconsistent configuration / arguments */
  FLUXO_ENOMEM_HBM = -2,  /* device allocation failed (or HBM budget refused) */
  FLUXO_ECUDA = -3,       /* CUDA runtime error (message in last_error) */
  FLUXO_ENAN_STATE = -4,  /* CALCTIMESTEP found an invalid state, see errType */
  FLUXO_ETIMEOUT = -5,    /* a bounded device wait expired */
  FLUXO_ENOTREADY = -6,   /* mesh or state not set */
  FLUXO_EXCHANGE = -7     /* the exchange callback of a partitioned solve reported a failure */
};

enum { FLUXO_EQN_EULER = 0, FLUXO_EQN_NAVIERSTOKES = 1, FLUXO_EQN_MHD = 2, FLUXO_EQN_MHD_PARABOLIC = 3 };

/* Runtime configuration: the parameter.ini keys of the reference's hot path
 * (src/equation/navierstokes/equation.f90:162-470, src/timedisc/timedisc.f90:74-137,
 * src/dg/br2/br2.f90:91-149) plus the compile-time switches the reference fixes
 * with CMake (PARABOLIC, PP_Lifting, PP_Lifting_Var, PP_VISC, PP_NodeType), which are runtime
 * choices here.  The split (flux-differencing) form is fixed. */
typedef struct fluxo_cfg {
  int struct_size;   /* sizeof(fluxo_cfg) */
  int N;             /* N: polynomial degree, 1..7 (one thread per volume node) */
  int eqn;           /* FLUXO_EQN_EULER (PARABOLIC=0) or FLUXO_EQN_NAVIERSTOKES */
  int riemann;       /* Riemann: 0-24, 32, 33, 44 */
  int volume_flux;   /* VolumeFlux: 0-10, 32 */
  int lifting;       /* 1 = BR1 (br1.f90), 2 = BR2 (br2.f90) */
  int lifting_var;   /* PP_Lifting_Var: 1 cons_var, 2 prim_var, 3 entropy_var */
  int visc;          /* PP_VISC: 0 constant mu0, 1 Sutherland, 2 power law */
  double kappa, R, Pr, mu0, Ts, Tref, ExpoSuth, ExpoPow, etaBR2;
  int time_disc;     /* TimeDiscMethod (timedisc_vars.f90:94-726): 0 carpenterrk4-5, 1 standardrk3-3,
                        2 niegemannrk4-14, 3 toulorgerk4-8c, 4 toulorgerk3-7c, 5 toulorgerk4-8f (two-register
                        LSERKW2, fused into the volume kernel), 6 ketchesonrk4-20, 7 ketchesonrk4-18 (LSERKK3),
                        8 ssprk4-5, 9 ssprk3-3 (batched solves: 0..5) */
  double cfl_scale;  /* CFLScale (unscaled, as read from parameter.ini) */
  double dfl_scale;  /* DFLScale (unscaled) */
  int ini_exact_func;   /* IniExactFunc: only 4 adds a source term (CalcSource) */
  double ini_frequency, ini_amplitude;
  int device;        /* CUDA device ordinal */
  /* MHD with GLM cleaning, eqn = FLUXO_EQN_MHD / FLUXO_EQN_MHD_PARABOLIC
   * (src/equation/mhd/equation.f90:134-285; nVar = 9: rho, rho*v, E, B, psi).  The MHD viscosity
   * mu is mu0 above (constant); riemann 0-5 (5 = HLLD needs mu_0 = 1), 10-15; volume_flux 0,1,10,12. */
  double mu_0;       /* mu_0, magnetic permeability */
  double eta;        /* eta, resistivity (PARABOLIC) */
  double glm_scale;  /* GLM_scale: GLM_ch = GLM_scale * GLM_dtch1 / dt (calctimestep.f90:176) */
  double glm_scr;    /* GLM_scr: damping Ut(9) -= GLM_scr*GLM_ch*U(9) (equation.f90:1698-1706) */
  int noncons;       /* NONCONS: 0 off, 1 Powell, 2 Brackbill, 3 Janhunen (CMake FLUXO_EQN_NONCONS_TYPE) */
  int nc_glm;        /* PP_NC_GLM: non-conservative GLM terms (CMake FLUXO_EQN_NONCONS_GLM) */
  /* NFVSE shock capturing (CMake FLUXO_SHOCKCAP_NFVSE; src/shockcapturing/nfvse.f90:63-260), Euler,
   * Navier-Stokes and MHD, N >= 2, SubFVMethod = 1 (first-order subcell finite volumes), 2 (TVD),
   * 3 (TVD-ES) or 4 (TVD-Fjordholm); 3 and 4 need a Riemann solver with dissipation matrices
   * (Navier-Stokes 4, 44, 33; MHD 14, 15). */
  int nfvse;               /* 0 off, 1 on */
  int compute_alpha;       /* ComputeAlpha: 1 Persson-Peraire indicator, 3 fixed ShockBlendCoef,
                              20 random values drawn once and kept (see fluxo_gpu_set_alpha) */
  double shock_blend_coef; /* ShockBlendCoef */
  int modal_threshold;     /* ModalThreshold: 1 T = 0.5*10^(-1.8 (N+1)^0.25), 2 T = 0.5*10^(-1.8 N^0.25) */
  double alpha_max, alpha_min, space_prop_factor; /* alpha_max, alpha_min, SpacePropFactor */
  int space_prop_sweeps;   /* SpacePropSweeps */
  double time_rel_factor;  /* TimeRelFactor */
  int indicator_quantity;  /* ShockIndicatorQuantity: 1 Density, 2 Pressure, 3 DensityTimesPressure,
                              4 KinPlusMagEnergy */
  int sub_fv_method;       /* SubFVMethod: 1 first-order subcell FV, 2 TVD (minmod reconstruction of the
                              primitive variables, nfvse.f90:674-815, 1448-1529), 3 TVD-ES (TVD states with
                              an entropy-stability switch, :826-1090), 4 TVD-Fjordholm (reconstruction of the
                              scaled entropy variables, :1101-1386) */
  int recons_boundaries;   /* ReconsBoundaries (SubFVMethod 2-4): 1 none, 2 central, 3 neighbour element */
  /* NFVSE_CORR (CMake FLUXO_SHOCK_NFVSE_CORR; Apply_NFVSE_Correction nfvse.f90:1688-1883): after every
   * stage update the blending coefficient of each element is raised as far as needed to keep density and
   * pressure at PositCorrFactor of their values under the pure subcell FV update.  Only with the
   * LSERKW2 schemes (time_disc 0..5) and ssprk4-5 (8); ssprk3-3 (9) runs without the correction as in
   * the reference.  A safe state with negative density or pressure ends the step with
   * FLUXO_ENAN_STATE, errType 5 (the reference stops). */
  int nfvse_corr;          /* 0 off, 1 on (needs nfvse = 1) */
  double posit_corr_factor; /* PositCorrFactor (reference default 0.1) */
  int posit_max_iter;      /* PositMaxIter (reference default 10) */
  /* PP_NodeType (CMake FLUXO_DISC_NODETYPE): 2 (or 0) Gauss-Lobatto, 1 Gauss.  Gauss nodes run the
   * entropy-stable Gauss collocation of the split form (interpolated face states, entropy-projected for
   * the EC volume fluxes 5, 6, 7, 10, 32; surface correction with SurfMetrics, which the caller supplies
   * with fluxo_gpu_set_surf_metrics after fluxo_gpu_set_mesh); Euler / Navier-Stokes only, without
   * NFVSE, batches or the allocation-free entry point. */
  int node_type;
} fluxo_cfg;

typedef struct fluxo_handle fluxo_handle;

/* Exchange points of a partitioned solve (fluxo_gpu_set_partition).  The callback runs on the calling
 * host thread and enqueues its work on `stream` (the handle's CUDA stream), in stream order with the
 * handle's kernels; it returns 0, or nonzero to make the call fail with FLUXO_EXCHANGE.  Every handle of
 * the solve reaches the same exchange points in the same order.
 *   FLUXO_XCHG_STATE   a = U (device, [elem][node][var]): before each right-hand side, the ghost
 *                      elements' U from their owners (dg.f90:342-356 exchanges U_slave of MPI sides;
 *                      here whole ghost elements);
 *   FLUXO_XCHG_GTRACE  a = the viscous face shares [side][master|slave][nv][pt] (nv = 4 Navier-Stokes,
 *                      7 MHD): after the lifting kernel, the ghost side's share of every partition side
 *                      (the gradient traces of br1.f90:154-364);
 *   FLUXO_XCHG_DT      a = dt bits (uint64, the IEEE bits of a non-negative double), b = error key
 *                      (int32, INT_MAX = none): after CALCTIMESTEP, both reduced with MIN over the
 *                      handles (MPI_ALLREDUCE, calctimestep.f90:159-167); for MHD also once inside
 *                      fluxo_gpu_set_partition, with a = the bits of GLM_dtch1;
 *   FLUXO_XCHG_ALPHA   a = NFVSE blending coefficients (double per element): the ghost elements' values
 *                      before every propagation sweep (ProlongBlendingCoeffToFaces, nfvse_mpi.f90:31-58). */
enum { FLUXO_XCHG_STATE = 1, FLUXO_XCHG_GTRACE = 2, FLUXO_XCHG_DT = 3, FLUXO_XCHG_ALPHA = 4 };
typedef int (*fluxo_exchange_fn)(void* ctx, int what, void* stream, void* a, void* b);

/* InitEquation + InitDGbasis + InitTimeDisc equivalent.
 * Replaces: src/equation/navierstokes/equation.f90:162 InitEquation,
 *           src/dg/dg.f90:61 InitDG / :181 InitDGbasis,
 *           src/timedisc/timedisc.f90:74 InitTimeDisc (coefficients, FillCFL_DFL :697). */
int fluxo_gpu_create(const fluxo_cfg* cfg, fluxo_handle** out);

/* Copies the geometry of InitMesh/CalcMetrics to the device.
 * Replaces the module state read by the RHS: src/mesh/mesh_vars.f90:40-104
 * (SideToElem, ElemToSide, Metrics_*Tilde, sJ, NormVec, TangVec1/2, SurfElem,
 * Elem_xGP).  Elem_xGP may be NULL unless a source term is active. */
int fluxo_gpu_set_mesh(fluxo_handle* h, int nElems, int nSides, const int* SideToElem,
                       const int* ElemToSide, const double* Metrics_fTilde,
                       const double* Metrics_gTilde, const double* Metrics_hTilde,
                       const double* sJ, const double* NormVec, const double* TangVec1,
                       const double* TangVec2, const double* SurfElem, const double* Elem_xGP);

/* Gauss nodes: SurfMetrics(3,0:N,0:N,6,nElems), the normal metric term of every element side at the
 * side's points in the master side's point order (src/mesh/metrics.f90:420-427, mesh_vars.f90:67-70).
 * Required before the first right-hand side of a handle with node_type = 1; FLUXO_EINVAL_CFG for LGL. */
int fluxo_gpu_set_surf_metrics(fluxo_handle* h, const double* SurfMetrics);

/* MOD_DG_Vars::U host <-> device (src/dg/dg_vars.f90:75).  The device copy is
 * authoritative between set_state and get_state. */
int fluxo_gpu_set_state(fluxo_handle* h, const double* U);
int fluxo_gpu_get_state(fluxo_handle* h, double* U);
/* MOD_DG_Vars::Ut after the last fluxo_gpu_dg_time_derivative (dg_vars.f90:80). */
int fluxo_gpu_get_ut(fluxo_handle* h, double* Ut);
/* Primitive-variable gradients gradPx/y/z (nVar,0:N,0:N,0:N,nElems) of the last RHS
 * (src/dg/br1/br1_vars.f90 gradPx..); Navier-Stokes only. */
int fluxo_gpu_get_gradients(fluxo_handle* h, double* gradPx, double* gradPy, double* gradPz);

/* DGTimeDerivative_weakForm(tIn): device U -> device Ut.
 * Replaces: src/dg/dg.f90:282-452. */
int fluxo_gpu_dg_time_derivative(fluxo_handle* h, double t);

/* CALCTIMESTEP(errType): minimum over elements of the convective (and viscous)
 * time step; errType 1 NaN density, 2 p<=0, 3 NaN dt_conv, 4 NaN dt_visc (5: NFVSE_CORR safe state
 * not admissible, from fluxo_gpu_timestep / fluxo_gpu_time_disc).
 * Replaces: src/equation/navierstokes/calctimestep.f90:39-170. */
int fluxo_gpu_calc_timestep(fluxo_handle* h, double* dt, int* errType);

/* One full Runge-Kutta step from t with step dt (U updated in place), the scheme of cfg->time_disc.
 * Replaces the TimeStep pointer: src/timedisc/timedisc.f90:424-480 TimeStepByLSERKW2,
 * :489-542 TimeStepByLSERKK3, :560-640 TimeStepBySSPRK2, :647-687 TimeStepBySSPRK33. */
int fluxo_gpu_timestep(fluxo_handle* h, double t, double dt);

/* The TimeDisc loop (src/timedisc/timedisc.f90:274-359) without output: per step
 * CALCTIMESTEP on the device, dt clipped to tEnd, one LSERK step, until
 * t >= tEnd or maxIter steps (maxIter < 0: no limit).  The host does not
 * synchronise between steps.  Returns the final time, the steps taken and the
 * errType that stopped the loop (0 = none). */
int fluxo_gpu_time_disc(fluxo_handle* h, double t, double tEnd, int maxIter, double* tOut,
                        int* nIter, int* errType);

/* MHD: MOD_Equation_Vars::GLM_ch, the GLM cleaning speed used by the RHS.  CALCTIMESTEP
 * (fluxo_gpu_calc_timestep, and every step of fluxo_gpu_time_disc) sets it to
 * GLM_scale*GLM_dtch1/dt (src/equation/mhd/calctimestep.f90:175-177, InitTimeStep_GLM :187-223). */
int fluxo_gpu_set_glm_ch(fluxo_handle* h, double ch);
int fluxo_gpu_get_glm_ch(fluxo_handle* h, double* ch);

/* One solve over several handles (one per GPU, or several on one GPU): this handle's mesh holds its
 * nOwned elements first and then ghost copies of the neighbouring elements of other handles, its sides
 * are every side of an owned element (both elements of each present), and the element kernels,
 * CALCTIMESTEP and the stage updates run over the owned elements only.  Both handles of a partition
 * side compute its flux from the same two states, so fluxes need no exchange.  `fn(ctx, ...)` is called
 * at the exchange points above; the caller moves the data (NCCL, peer copies).  LGL nodes (Euler,
 * Navier-Stokes, MHD, NFVSE; for MHD this call is itself collective: it reduces GLM_dtch1; ComputeAlpha
 * 20 draws per handle);
 * fluxo_gpu_analyze and the batch entry points are not available on a partitioned handle.  A later
 * fluxo_gpu_set_mesh removes the partition.
 * Replaces the single-process part of the reference's MPI decomposition (mesh_readin.f90:246-292
 * offsetElemMPI, prepare_mesh.f90 MPI sides, dg.f90:342-442 the exchanges). */
int fluxo_gpu_set_partition(fluxo_handle* h, int nOwned, fluxo_exchange_fn fn, void* ctx);
/* Device buffer of the FLUXO_XCHG_GTRACE exchange (NULL without parabolic terms). */
int fluxo_gpu_exchange_buffers(fluxo_handle* h, double** gtrace);

/* NFVSE: MOD_NFVSE_Vars::alpha(nElems), the blending coefficients of the last right-hand side
 * (src/shockcapturing/nfvse_vars.f90). */
int fluxo_gpu_get_alpha(fluxo_handle* h, double* alpha);
/* Sets alpha(nElems) before the next right-hand side: the values that ComputeAlpha 20 keeps (the
 * reference draws them once with RANDOM_NUMBER * alpha_max, src/shockcapturing/nfvse.f90:1591-1596;
 * fluxo_gpu_set_mesh draws them from a SplitMix64 stream), or the previous alpha that TimeRelFactor
 * weighs for ComputeAlpha 1.  No counterpart call in the reference (there alpha is module data). */
int fluxo_gpu_set_alpha(fluxo_handle* h, const double* alpha);

/* Exact function of the error norms (the reference's AnalyzeExactFunc with the IniExactFunc
 * parameters, src/equation/navierstokes/equation.f90:575-811): func 0 none, 1 constant reference
 * state (ref_state_prim: rho, u, v, w, p), 2 density sine wave (adv_vel, ini_wavenumber,
 * ini_amplitude), 4 manufactured solution (ini_amplitude, ini_frequency), 7 Taylor-Green vortex,
 * 14 soft Sedov-Taylor blast (ini_center). */
typedef struct fluxo_exact {
  int func;
  double adv_vel[3];
  double ini_wavenumber[3];
  double ini_amplitude, ini_frequency;
  double ref_state_prim[5];
  double ini_center[3];
} fluxo_exact;

/* Analysis of the device state at time t, reduced on the device.  Like the reference's TimeDisc at an
 * analyze point (src/timedisc/timedisc.f90:387-404: DGTimeDerivative(t), then Analyze), it first
 * evaluates the right-hand side at t (Ut and, for Navier-Stokes, the gradients are then those of the
 * current U), then reduces:
 *   L2, Linf, L2colloc (nVar each; ex->func != 0, Euler / Navier-Stokes, needs Elem_xGP at set_mesh):
 *     CalcErrorNorms (src/analyze/analyze.f90:557-632) on NAnalyze = 2(N+1) LGL points per direction
 *     and at the collocation points;
 *   scalars[0] entropy: sum of -rho (log p - kappa log rho)/(kappa-1) * wGPVol/sJ (CalcEntropy,
 *     navierstokes/analyze_equation.f90:549-599; MHD: mhd/analyze_equation.f90:421-470);
 *   scalars[1] dS/dU . Ut: the entropy production of the right-hand side, sum of W(U).Ut wGPVol/sJ;
 *   scalars[2] kinetic energy 1/Vol sum 1/2 rho |v|^2, scalars[3] enstrophy 1/Vol sum 1/2 rho |curl v|^2
 *     (Navier-Stokes, from the lifted velocity gradients; 0 otherwise): the Taylor-Green integrands of
 *     src/testcase/taylorgreenvortex/testcase_analyze.f90:127-330;
 *   scalars[4] the domain volume Vol.
 * Any output may be NULL.  The reductions run in a fixed order (the result is reproducible). */
int fluxo_gpu_analyze(fluxo_handle* h, double t, const fluxo_exact* ex, double* L2, double* Linf, double* L2colloc,
                      double* scalars);

/* Device pointers and stream for zero-copy callers (e.g. torch tensors):
 * U, Ut are device buffers of nVar*(N+1)^3*nElems doubles in the host layout. */
int fluxo_gpu_device_buffers(fluxo_handle* h, double** dU, double** dUt, void** stream);
/* Number of kernels this handle launched so far. */
int fluxo_gpu_launch_count(fluxo_handle* h, uint64_t* n);

/* Per-kernel timing with CUDA events on the handle's stream (off by default).
 * kind: 0 lifting surface flux, 1 gradient, 2 face flux, 3 volume, 4 time step, 5 NFVSE
 * (indicator, propagation and subcell finite volumes).
 * fluxo_gpu_get_profile synchronises, returns the summed milliseconds and launch count of
 * that kind since profiling was enabled, and resets them. */
int fluxo_gpu_set_profiling(fluxo_handle* h, int enable);
int fluxo_gpu_get_profile(fluxo_handle* h, int kind, double* total_ms, uint64_t* count);

/* Launch shape of the Euler / Navier-Stokes volume kernel (no counterpart in the reference): for each
 * (N, volume_flux, visc) a few candidate shapes (elements per block, lines per warp; 0 = lines
 * contiguous in the thread index) give identical results; the first right-hand side of a handle, or
 * the first run of a batch group, times them on its own data and keeps the fastest for the process.
 * fluxo_gpu_volume_shape reports the candidates, the chosen index (-1: not tuned yet) and its shape;
 * fluxo_gpu_set_volume_shape pins one (index < 0: tune again at the next use). */
int fluxo_gpu_volume_shape(int N, int volume_flux, int visc, int* count, int* index, int* epb, int* lpw);
int fluxo_gpu_set_volume_shape(int N, int volume_flux, int visc, int index);

/* FP64 FMA throughput of the device (a register-resident DFMA loop over all SMs), in TFLOP/s
 * counting an FMA as 2 flops: the denominator of the FP64 roofline. */
int fluxo_gpu_fp64_peak(int device, double* tflops);

/* Euler DGTimeDerivative (stage 0: Ut written) on caller-owned device arrays, allocating nothing.
 * No counterpart in the reference: it is for callers that own all device memory and must not
 * allocate while they run (e.g. a host code that reserves one arena of HBM at start-up and
 * evaluates the right-hand side on its own vectors), which therefore cannot create a handle;
 * cudaMalloc would fail once the arena holds the memory, and cudaFree synchronises the device.
 * Same kernels and results as fluxo_gpu_dg_time_derivative for eqn = FLUXO_EQN_EULER without a
 * source term and without NFVSE (ini_exact_func = 4 or nfvse = 1 return FLUXO_EINVAL_CFG).
 * Arrays are device memory of cfg->device in the device layouts of fluxo_gpu_set_mesh:
 *   dU, dUt  (nVar,0:N,0:N,0:N,nElems) as U;  dsJ (0:N,0:N,0:N,nElems)
 *   dMetrics [elem][9][node]: Metrics_f/g/hTilde (x,y,z) each, node = i+(N+1)(j+(N+1)k) fastest
 *   dFaceGeo [side][10][pt]: NormVec, TangVec1, TangVec2 (x,y,z), SurfElem; pt = p+(N+1)q fastest
 *   dS2E [side][5]: SideToElem with 0-based element ids;  dE2S [elem][6][2]: 0-based side id, flip.
 * The connectivity is not checked (it is device memory): it must be a mesh that fluxo_gpu_set_mesh
 * accepts, with element ids in [0,nElems), side ids in [0,nSides), local sides 1..6 and flips 0..4;
 * other ids make the kernels read and write outside the arrays.
 * The face fluxes and operator tables live in one static device array of
 * FLUXO_NOALLOC_SCRATCH_BYTES shared by all calls on a device: it needs
 * 2304 + nSides*5*(N+1)^2*8 bytes (N=7: about 3270 sides; N=3: about 13100 sides), larger
 * meshes return FLUXO_EINVAL_CFG.  Calls whose GPU work overlaps (other streams or host threads)
 * race on that array; the call runs on `stream` (NULL: the legacy default stream) and
 * synchronises it before returning.  The first call on a device looks up the array's device
 * address, and the first call at each N copies that N's operator tables into it.
 * Errors: fluxo_gpu_last_error(NULL, ...). */
#define FLUXO_NOALLOC_SCRATCH_BYTES (8u * 1024u * 1024u)
int fluxo_gpu_dg_time_derivative_noalloc(const fluxo_cfg* cfg, int nElems, int nSides, const double* dU,
                                         double* dUt, const double* dMetrics, const double* dsJ,
                                         const double* dFaceGeo, const int* dS2E, const int* dE2S,
                                         void* stream);

int fluxo_gpu_destroy(fluxo_handle* h);
/* Copies the last error message of the handle (or of the last failed create if h is NULL). */
int fluxo_gpu_last_error(fluxo_handle* h, char* buf, size_t len);

/* ------------------------------------------------------------------------------------------
 * Batched solves.  No counterpart in the reference, which runs one mesh per program
 * (src/fluxo.f90: InitMesh .. TimeDisc): many independent Euler / Navier-Stokes instances
 * (own mesh, N, fluxes, end time) advance together, each exactly as fluxo_gpu_time_disc would
 * advance it alone (same kernels, same per-instance CALCTIMESTEP and dt clipping).
 * Instances with the same kernel configuration (everything in fluxo_cfg except ini_* and device)
 * share one launch per kernel; one step of all instances is one CUDA graph replay.
 *   add:       takes the arrays of fluxo_gpu_set_mesh (no Elem_xGP: no source terms) and the
 *              initial U; the instance joins at the next run.  maxIter < 0: no limit.
 *   run:       up to nSteps steps of every unfinished instance; returns how many are unfinished.
 *   status:    time, steps taken, finished flag and errType (as fluxo_gpu_time_disc).
 *   get_state: the instance's U (host layout of fluxo_gpu_get_state); set_state overwrites it.
 *   remove:    frees the instance's slot at the next run.
 * ------------------------------------------------------------------------------------------ */
typedef struct fluxo_batch fluxo_batch;
int fluxo_batch_create(int device, fluxo_batch** out);
int fluxo_batch_add(fluxo_batch* b, const fluxo_cfg* cfg, int nElems, int nSides, const int* SideToElem,
                    const int* ElemToSide, const double* Metrics_fTilde, const double* Metrics_gTilde,
                    const double* Metrics_hTilde, const double* sJ, const double* NormVec,
                    const double* TangVec1, const double* TangVec2, const double* SurfElem, const double* U,
                    double t, double tEnd, int maxIter, int* id);
/* The same admission in two parts, so that its host work can run ahead of it: fluxo_batch_prepare
 * checks the configuration and repacks the mesh arrays and U on the host into an opaque object (it
 * touches no batch and no GPU, and any host thread may call it while a batch runs);
 * fluxo_batch_add_prepared hands that object to a batch (it takes ownership; nothing is copied) and
 * returns the instance id; fluxo_batch_prepared_free drops one that is not added.  Errors of prepare:
 * fluxo_gpu_last_error(NULL, ...). */
typedef struct fluxo_batch_prepared fluxo_batch_prepared;
int fluxo_batch_prepare(const fluxo_cfg* cfg, int nElems, int nSides, const int* SideToElem, const int* ElemToSide,
                        const double* Metrics_fTilde, const double* Metrics_gTilde, const double* Metrics_hTilde,
                        const double* sJ, const double* NormVec, const double* TangVec1, const double* TangVec2,
                        const double* SurfElem, const double* U, double t, double tEnd, int maxIter,
                        fluxo_batch_prepared** out);
int fluxo_batch_add_prepared(fluxo_batch* b, fluxo_batch_prepared* p, int* id);
int fluxo_batch_prepared_free(fluxo_batch_prepared* p);
int fluxo_batch_run(fluxo_batch* b, int nSteps, int* nRunning);
int fluxo_batch_status(fluxo_batch* b, int id, double* t, int* nIter, int* done, int* errType);
int fluxo_batch_get_state(fluxo_batch* b, int id, double* U);
/* Overwrites the instance's U (its time and step count stay). */
int fluxo_batch_set_state(fluxo_batch* b, int id, const double* U);
int fluxo_batch_remove(fluxo_batch* b, int id);
/* Groups with elements, placed instances and the device bytes they occupy. */
int fluxo_batch_info(fluxo_batch* b, int* nGroups, int* nInstances, size_t* deviceBytes);
/* The stream all of the batch's GPU work runs on (for events around fluxo_batch_run). */
int fluxo_batch_stream(fluxo_batch* b, void** stream);
/* Device bytes one instance of this configuration and mesh size occupies (admission control). */
int fluxo_batch_instance_bytes(const fluxo_cfg* cfg, int nElems, int nSides, size_t* bytes);
int fluxo_batch_last_error(fluxo_batch* b, char* buf, size_t len);
int fluxo_batch_destroy(fluxo_batch* b);

/* Device-resident request loop (no counterpart in the reference).  A server calls loop_start and goes
 * on with host work (admitting, preparing and reading back requests); the GPU repeats the time step of
 * all instances, one conditional while-node of a CUDA graph, without returning to the host until
 *   FLUXO_LOOP_FINISHED    an instance finished (reached its end time or maxIter, or CALCTIMESTEP
 *                          stopped it),
 *   FLUXO_LOOP_WOKEN       the host called fluxo_batch_loop_wake (e.g. a request can be admitted:
 *                          fluxo_batch_add is host-only and may be called while the loop runs; the
 *                          instance joins at the next loop_start or run),
 *   FLUXO_LOOP_STEP_LIMIT  maxSteps steps ran (every loop ends),
 *   FLUXO_LOOP_IDLE        nothing was running (no step ran).
 * The wake word is a store into mapped pinned host memory that the loop reads once per step.
 * loop_poll returns at once (*finished 0 while the loop runs); loop_wait waits for the end; both
 * then update every instance's status and give the steps run, the reason and the instances still
 * running.  Each instance advances exactly as under fluxo_batch_run (the same step graph).  While a
 * loop runs, run, get_state, set_state and loop_start return FLUXO_ENOTREADY; fluxo_batch_destroy wakes
 * a running loop and waits for its end. */
enum { FLUXO_LOOP_IDLE = 0, FLUXO_LOOP_FINISHED = 1, FLUXO_LOOP_WOKEN = 2, FLUXO_LOOP_STEP_LIMIT = 3 };
int fluxo_batch_loop_start(fluxo_batch* b, int maxSteps);
int fluxo_batch_loop_wake(fluxo_batch* b);
int fluxo_batch_loop_poll(fluxo_batch* b, int* finished, int* steps, int* reason, int* nRunning);
int fluxo_batch_loop_wait(fluxo_batch* b, int* steps, int* reason, int* nRunning);

/* ------------------------------------------------------------------------------------------
 * Host-side setup (no GPU needed).  The reference builds these arrays in InitMesh /
 * CalcMetrics from an HDF5 (HOPR) mesh; here they are generated for a periodic box
 * of nx*ny*nz hexahedra whose NGeo node coordinates are deformed by
 * X_d += amp * prod_e sin(2*pi*(x_e-c_e)/L_e).  Outputs use the layouts above.
 * Replaces: src/mesh/mesh.f90:89-296 InitMesh (with meshdeform :238-245),
 *           src/mesh/metrics.f90:78-484 CalcMetrics / CalcSurfMetrics (curl form).
 * ------------------------------------------------------------------------------------------ */
int fluxo_host_box_sizes(const int* nElemsXYZ, int* nElems, int* nSides);
int fluxo_host_box_mesh(int N, const int* nElemsXYZ, const double* xmin, const double* xmax, int NGeo,
                        double deform_amp, int* SideToElem, int* ElemToSide, double* Metrics_fTilde,
                        double* Metrics_gTilde, double* Metrics_hTilde, double* sJ, double* NormVec,
                        double* TangVec1, double* TangVec2, double* SurfElem, double* Elem_xGP);
/* The same periodic box for Gauss nodes (node_type = 1): metric terms and Jacobian at the Gauss nodes,
 * side quantities at the sides' Gauss points, and SurfMetrics(3,0:N,0:N,6,nElems) for
 * fluxo_gpu_set_surf_metrics.  Replaces the NodeType 'GAUSS' branch of src/mesh/metrics.f90:78-440. */
int fluxo_host_box_mesh_gauss(int N, const int* nElemsXYZ, const double* xmin, const double* xmax, int NGeo,
                              double deform_amp, int* SideToElem, int* ElemToSide, double* Metrics_fTilde,
                              double* Metrics_gTilde, double* Metrics_hTilde, double* sJ, double* NormVec,
                              double* TangVec1, double* TangVec2, double* SurfElem, double* Elem_xGP,
                              double* SurfMetrics);
/* A HOPR mesh from the arrays of its HDF5 file: ElemInfo(6,nElems), SideInfo(5,nSideInfo),
 * BCType(4,nBCs) and NodeCoords(3,(NGeo+1)^3*nElems) as the file stores them (first index fastest),
 * the node coordinates on equidistant (mesh_nodes_gl = 0, OutputNodeType 'EQUIDISTANT') or
 * Gauss-Lobatto points (1); use_curveds = 0 keeps the element corners (NGeo = 1); mesh_scale
 * multiplies the coordinates (parameter.ini: useCurveds, meshScale).  Conforming meshes whose
 * boundaries are all periodic (BCType 1): every side is an inner side, nSides = 3*nElems, and
 * mortar or other boundary sides return FLUXO_EINVAL_CFG with the reason in
 * fluxo_gpu_last_error(NULL, ...).  node_type 2 (LGL) fills the outputs of fluxo_host_box_mesh,
 * node_type 1 (Gauss) also SurfMetrics.  Side ids, flips and SideToElem follow the reference for
 * a single process.
 * Replaces: src/mesh/mesh_readin.f90:168-511 ReadMesh (connectivity and node coordinates),
 *           src/mesh/prepare_mesh.f90:59-215 setLocalSideIDs, :662-710 fillMeshInfo,
 *           src/mesh/mesh.f90:141-245 (useCurveds, meshScale), src/mesh/metrics.f90:78-484. */
int fluxo_host_hopr_mesh(int N, int node_type, int nElems, const int* ElemInfo, int nSideInfo,
                         const int* SideInfo, int nBCs, const int* BCType, int NGeo, int mesh_nodes_gl,
                         const double* NodeCoords, double mesh_scale, int use_curveds, int* SideToElem,
                         int* ElemToSide, double* Metrics_fTilde, double* Metrics_gTilde, double* Metrics_hTilde,
                         double* sJ, double* NormVec, double* TangVec1, double* TangVec2, double* SurfElem,
                         double* Elem_xGP, double* SurfMetrics);
/* The 1D nodes and weights of degree N: node_type 1 Gauss (LegendreGaussNodesAndWeights), 2 Gauss-Lobatto
 * (LegGaussLobNodesAndWeights), src/interpolation/basis.f90:430-608; w may be NULL. */
int fluxo_host_nodes(int N, int node_type, double* x, double* w);
/* FillIni(IniExactFunc, U) on the given node coordinates (src/equation/navierstokes/equation.f90:575-950):
 * IniExactFunc 1 (constant refstate, prim given), 2 (density sine wave), 4 (manufactured), 7 (Taylor-Green),
 * 14 (soft Sedov-Taylor blast around IniCenter = 0). */
int fluxo_host_exact_func(int func, double t, size_t nPoints, const double* x, double kappa,
                          const double* adv_vel, double ini_amplitude, const double* ini_wavenumber,
                          double ini_frequency, const double* ref_state_prim, double* U);

#ifdef __cplusplus
}
#endif
#endif /* FLUXO_GPU_H */
