/*
 * theseus_b200.h -- C ABI of the B200-native DGSEM right-hand-side evaluation.
 *
 * The library evaluates dU/dt = L(U) for the compressible Euler and
 * Navier-Stokes equations discretised with DGSEM on Legendre-Gauss-Lobatto
 * nodes, exactly the operator that Theseus exposes as
 *   RHSOperator<PhysicsT>::Mult(const mfem::Vector &u, mfem::Vector &dudt)
 *   (include/RHSOperator.hpp:100,172; include/RHSOperator_impl.hpp:719-793)
 * with the flow-specific body EulerOperator::FlowMult
 *   (include/EulerOperator_impl.hpp:396-421) or NSOperator::FlowMult
 *   (include/NSOperator_impl.hpp:161-192).
 *
 * Conventions shared by every entry point:
 *  - State vectors are the MFEM "byNODES" L-vector of an L2 DG space whose
 *    element DOFs are lexicographic (x fastest):  u[eq][elem][node], with
 *    eq in [rho, rho*u_0 .. rho*u_{dim-1}, rho*E] (include/GasState.hpp:16-26,
 *    69-92) and node = i + Np*(j + Np*k).
 *  - Device pointers are caller-owned CUDA global-memory pointers; the library
 *    never frees them.  Host pointers are only read during the call.
 *  - Every call returns a thx_status; no C++ exception crosses the ABI.
 *  - One handle is bound to one CUDA device (the current device at
 *    thx_create).  Calls on one handle must not overlap: the handle owns its
 *    scratch buffers, like the reference's mutable operator caches
 *    (include/RHSOperator.hpp:129-130).  Distinct handles are independent.
 *  - thx_rhs and thx_rk3_steps only enqueue work on the given stream (no host
 *    synchronisation inside).
 */
#ifndef THESEUS_B200_H
#define THESEUS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  THX_OK = 0,
  THX_ERR_INVALID_ARGUMENT = 1,   /* bad size, null pointer, unknown selector */
  THX_ERR_UNSUPPORTED = 2,        /* valid but not built (order, dim, combination) */
  THX_ERR_CUDA = 3,               /* a CUDA runtime call failed */
  THX_ERR_NO_DEVICE = 4,          /* no CUDA device visible: there is no CPU fallback */
  THX_ERR_OUT_OF_MEMORY = 5,
  THX_ERR_NUMERICS = 6,           /* device-side status flag set (non-positive state, Newton failure) */
  THX_ERR_BUSY = 7,               /* batch engine: the case does not fit the memory budget now */
  THX_ERR_IO = 8                  /* checkpoint file could not be created, opened, read or written */
} thx_status;

/* Two-point volume fluxes and surface (Riemann) fluxes.  The numbering is the
 * reference's selection list (include/SimFactory_impl.hpp:75-128).  Volume and
 * surface fluxes are selected independently; for the central fluxes
 * (HLL/LLF/Roe) the volume flux is the arithmetic average of the physical
 * fluxes, as in include/HLLFlux.hpp:21-51 and include/RoeFlux.hpp:12-37. */
typedef enum {
  THX_FLUX_CHANDRASHEKAR = 0, /* include/ChandrashekarFlux.hpp:20-89, face: +scalar dissipation :91-155 */
  THX_FLUX_RANOCHA = 1,       /* include/RanochaFlux.hpp:20-79, face: +Roe dissipation :81-134 */
  THX_FLUX_PIROZZOLI = 2,     /* include/PirozzoliFlux.hpp:19-71, face: +Roe dissipation :73-120 */
  THX_FLUX_HLL = 3,           /* include/HLLFlux.hpp:53-116 */
  THX_FLUX_LLF = 4,           /* include/LaxFriedrichsFlux.hpp:54-77 */
  THX_FLUX_ROE = 5,           /* include/RoeFlux.hpp:42-149 */
  THX_FLUX_LTEEC = 6,         /* include/LTEECFlux.hpp:11-99 (LTE Helmholtz gas only) */
  THX_FLUX_COUNT = 7
} thx_flux;

typedef enum {
  THX_FLOW_EULER = 0,           /* EulerOperator */
  THX_FLOW_NAVIER_STOKES = 1    /* NSOperator, BR1 gradients of entropy variables */
} thx_flow_model;

typedef enum {
  THX_PRECISION_FP64 = 0,       /* every operation in double */
  THX_PRECISION_FP32_MIXED = 1  /* flux arithmetic in float, FP64 log-mean series and RK accumulation */
} thx_precision;

/* Physics and discretisation switches.  Defaults mirror the reference's
 * runtime JSON defaults (include/SimFactory_impl.hpp:131-135) and
 * include/Physics.hpp (mu_bulk = 2/3). */
typedef struct {
  int32_t flow_model;        /* thx_flow_model */
  int32_t volume_flux;       /* thx_flux */
  int32_t surface_flux;      /* thx_flux */
  int32_t fv_flux;           /* thx_flux used on subcell faces when blending */
  int32_t blending;          /* 1 = Persson-Peraire indicator + subcell FV blending */
  int32_t precision;         /* thx_precision */
  int32_t sutherland;        /* 1 = Sutherland viscosity (reference compile flag SUTHERLAND) */
  int32_t geometry_layout;   /* 0: store geometric factors once where they are exactly
                                constant over nodes/elements/faces; 1: full per-node arrays */
  double gamma;              /* 1.4 */
  double Pr;                 /* 0.72 */
  double R_gas;              /* 287.05 */
  double mu;                 /* 0.02 */
  double mu0;                /* 1.716e-5 (Sutherland) */
  double mu_bulk;            /* 2/3 */
  double T0;                 /* 273.15 */
  double Ts;                 /* 110.4 */
  double alpha_max;          /* 0.5  (src/Simulation.cpp:482-489) */
  double alpha_min;          /* 0.001 */
  double sharpness;          /* 9.21024 (include/RHSOperator.hpp:33) */
  double modal_threshold;    /* <= 0: 0.5*10^(-1.8 p^0.25) (include/RHSOperator.hpp:64) */
  double state_offset[5];    /* FP32-mixed only: constant reference state u_ref (rho, rho*u_0..,
                                rho*E) subtracted from the FP32 working copy; pressure enters
                                the momentum fluxes as p - p(u_ref).  Zeros: plain FP32 copy. */
  int32_t volume_staging;    /* 0: the volume kernel loads each element block's state itself;
                                1: persistent CTAs stage the next block's state by bulk copy
                                (cp.async.bulk, mbarrier completion) while evaluating the
                                current one (not with blending or the LTE gas: falls back to 0) */
  int32_t mixed_blended_fp32; /* FP32-mixed Euler with blending: 0 (default) evaluates every
                                block of elements holding a blended element, and its faces, in
                                FP64 from the FP64 stage state ("FP64 islands"); 1 keeps them
                                in FP32 */
  int32_t mixed_flux_no_perturbation; /* FP32-mixed with the Chandrashekar volume flux and an
                                HLL/LLF/Roe surface flux about a physical offset state: 0
                                (default) evaluates the fluxes in perturbation form, F - F(offset),
                                from the state's deviations (the constant cancels in the
                                right-hand side); 1 evaluates F itself */
} thx_config;

/* Mesh and geometric factors, in the layout of the reference's device cache
 * DGSEMDeviceCacheT (include/dgsem_cache.hpp:173-241), on the host.
 *
 *  jac[e][node]                        Tr.Weight() at each LGL node
 *  metric[e][node][dir][phys]          adjugate Jacobian, row dir
 *                                      (include/dgsem_cache_utilities.hpp:503-511)
 *  face_elem[f][2], face_lface[f][2]   minus/plus element of interior face f and
 *                                      the local face index in that element
 *                                      (0:x-, 1:x+, 2:y-, 3:y+, 4:z-, 5:z+)
 *  face_normal[f][fp][dim]             MFEM CalcOrtho normal of side 0, scaled by
 *                                      the face Jacobian (:601-605)
 *  face_wminus[f][fp], face_wplus[f][fp]  1/(w0*J) lift weights (:555,609-611)
 *
 * Face point fp enumerates the trace nodes of both sides in the same
 * lexicographic order of the two (one) tangential reference coordinates,
 * i.e. faces are conforming and aligned.  This replaces MFEM's interior face
 * restriction (include/dgsem_cache_utilities.hpp:67-79).
 *
 * Boundary faces (all zero/NULL for a periodic mesh), in the layout of the
 * reference's boundary cache (include/dgsem_cache_utilities.hpp:355-440):
 *  bdr_elem[b], bdr_lface[b]           the element and local face of boundary face b
 *  bdr_normal[b][fp][dim]              outward CalcOrtho normal (face Jacobian scaled)
 *  bdr_weight[b][fp]                   1/(w0*J) of the element at the trace
 *  bdr_bc[b]                           index into bcs[] (the face's boundary marker)
 *  bcs[i]                              condition type and offset of its payload in
 *                                      bc_data (src/Simulation.cpp:540-860)
 * Boundary face points use the same lexicographic face-point order.  A node's
 * boundary-face lifts are summed in boundary-face order and added after the
 * interior faces' (include/EulerOperator_impl.hpp:292-392). */

/* Boundary condition types: the reference's BCType numbering
 * (include/bc_cache_utilities.hpp:11-23).  Payloads in bc_data:
 * SUPERSONIC_INFLOW / PRESCRIBED_STATE: the exterior conserved state (dim+2);
 * NOSLIP_ADIABATIC: wall velocity (dim), wall heat flux; NOSLIP_ISOTHERMAL:
 * wall velocity (dim), wall temperature. */
enum {
  THX_BC_SLIP_WALL = 0,
  THX_BC_SUPERSONIC_INFLOW = 1,
  THX_BC_SUPERSONIC_OUTFLOW = 2,
  THX_BC_PRESCRIBED_STATE = 3,
  THX_BC_SYMMETRY = 4,
  THX_BC_AXIS = 5,               /* axisymmetric builds only: not supported */
  THX_BC_NOSLIP_ADIABATIC = 6,
  THX_BC_NOSLIP_ISOTHERMAL = 7
};

typedef struct {               /* BCDescriptor (include/bc_cache_utilities.hpp:36-44) */
  int32_t type;
  int32_t data_index;          /* offset of the payload in bc_data */
} thx_bc;

typedef struct {
  int32_t dim;               /* 2 or 3 */
  int32_t order;             /* polynomial order p (Np = p+1 nodes per direction) */
  int32_t num_elements;
  int32_t num_faces;         /* interior faces (periodic wrap faces included) */
  const double *jac;
  const double *metric;
  const int32_t *face_elem;
  const int32_t *face_lface;
  const double *face_normal;
  const double *face_wminus;
  const double *face_wplus;
  /* boundary faces (see above) */
  int32_t num_bdr_faces;
  const int32_t *bdr_elem;
  const int32_t *bdr_lface;
  const double *bdr_normal;
  const double *bdr_weight;
  const int32_t *bdr_bc;
  int32_t num_bcs;
  const thx_bc *bcs;
  int32_t bc_data_len;
  const double *bc_data;
} thx_geometry;

/* LTE Helmholtz gas table in the reference's six-plane layout
 * (include/LTEHelmholtzTable.hpp:13-35, include/LTETable.hpp:56-71), host
 * pointers: planes[p][j][i] with p = H, H_rho, H_T, H_rhoT, mu, lambda (physical
 * derivatives), i the density and j the temperature sample; inverse[j][i] is the
 * temperature guess at (rho_grid[i], e_grid[j]). */
typedef struct {
  int32_t nx;                /* density samples */
  int32_t ny;                /* temperature (and energy) samples */
  const double *rho_grid;    /* [nx], increasing */
  const double *T_grid;      /* [ny], increasing */
  const double *e_grid;      /* [ny], increasing */
  const double *planes;      /* [6][ny][nx] */
  const double *inverse;     /* [ny][nx] */
} thx_lte_table;

/* Synthetic ideal-dissociating gas (Lighthill): molecular gas constant R,
 * characteristic density rho_d, dissociation temperature theta_d; transport
 * mu = mu0 (T/T0)^0.7, lambda = mu 4R(1+alpha)/Pr. */
typedef struct {
  double R, rho_d, theta_d, mu0, T0, Pr;
} thx_idg_params;

typedef struct thx_operator_s *thx_handle;

/* ---- version and status ------------------------------------------------- */
const char *thx_version(void);
const char *thx_status_string(int status);
/* The CUDA runtime call that last failed inside the library on the calling
 * thread, with the runtime's error name ("" if none has).  Diagnostic only;
 * no counterpart in the reference. */
const char *thx_last_cuda_failure(void);
/* Default configuration (CPG air, Chandrashekar volume / Chandrashekar surface,
 * blending off, FP64). */
void thx_config_default(thx_config *cfg);

/* ---- host-side set-up (no device work) ---------------------------------- */
/* Number of LGL nodes per element (Np^dim), face points (Np^(dim-1)),
 * conserved variables (dim+2). */
int thx_sizes(int dim, int order, int32_t *nodes_per_element,
              int32_t *points_per_face, int32_t *num_equations);

/* Periodic axis-aligned box [lo,hi] split into n[0] x n[1] (x n[2]) equal
 * elements, numbered x fastest like mfem::Mesh::MakeCartesian2D/3D.  Fills
 * caller-allocated geometry arrays sized by thx_box_counts.  Stands in for
 * MFEM's mesh + FiniteElementSpace + geometric-factor set-up
 * (include/dgsem_cache_utilities.hpp:83-215, 516-639) for this mesh family. */
int thx_box_counts(int dim, const int32_t *n, int32_t *num_elements,
                   int32_t *num_faces);
int thx_box_geometry(int dim, int order, const int32_t *n, const double *lo,
                     const double *hi, double *jac, double *metric,
                     int32_t *face_elem, int32_t *face_lface,
                     double *face_normal, double *face_wminus,
                     double *face_wplus, double *node_coords /* [dim][e][node] or NULL */);

/* LGL nodes and weights on [0,1] (MFEM's GaussLobatto rule on the segment). */
int thx_lgl(int np, double *x, double *w);

/* ---- operator ------------------------------------------------------------ */
/* Builds the operator on the current CUDA device: uploads geometry, derives
 * D, D-hat, D-hat2 (include/dgsem_cache_utilities.hpp:123-181), subcell
 * metrics (:641-763) and the Persson modal transform (:867-943).
 * Replaces RHSOperator::Finalize (include/RHSOperator_impl.hpp:273-314) and
 * MakeRHSOperator (include/SimFactory_impl.hpp:63-488). */
int thx_create(const thx_geometry *geom, const thx_config *cfg,
               thx_handle *out);

/* The same operator on the LTE Helmholtz gas (include/LTEGasModel.hpp:339
 * LTEHelmholtzGas, include/LTEHelmholtzGasEOS.hpp:10-172) with the LTEEC flux
 * on volume and faces (cfg->volume_flux == cfg->surface_flux == THX_FLUX_LTEEC),
 * FP64, no blending; Euler or Navier-Stokes (transport from the table's mu and
 * lambda planes, include/LTETransport.hpp:19-66).  The table (host pointers)
 * is copied to the device.  Every right-hand side recovers T(rho, e) once per
 * node by the reference's Newton iteration (include/LTEHelmholtzEOS.hpp:158-223);
 * a failed recovery sets THX_STATUS_EOS.  Replaces MakeRHSOperator with the
 * LTE gas selected (include/SimFactory_impl.hpp:63-488). */
int thx_create_lte(const thx_geometry *geom, const thx_config *cfg,
                   const thx_lte_table *table, thx_handle *out);

/* Energy grid and inverse table of a forward Helmholtz table: e_grid[ny]
 * uniform over [e_min - pad, e_max + pad], inverse[j][i] = T(rho_i, e_j) by
 * bisection -- the part of HelmholtzTable::Build that does not need PLATO
 * (include/LTEHelmholtzTableBuilder.hpp:131-218).  Host arrays. */
int thx_lte_inverse_table(int nx, int ny, const double *rho_grid, const double *T_grid,
                          const double *planes, double *e_grid, double *inverse);

/* Forward planes of the synthetic ideal-dissociating-gas table on log-spaced
 * grids (include/LTETable.hpp:95-103): rho_grid[nx] over 10^[lr0, lr1],
 * T_grid[ny] over 10^[lt0, lt1], planes[6][ny][nx].  Host arrays. */
int thx_lte_idg_table(const thx_idg_params *gas, int nx, int ny, double lr0, double lr1,
                      double lt0, double lt1, double *rho_grid, double *T_grid, double *planes);

int thx_destroy(thx_handle h);

/* dudt = L(u).  u and dudt are device FP64 L-vectors (byNODES) in both
 * precisions; in THX_PRECISION_FP32_MIXED the state is narrowed to the FP32
 * working copy (u - state_offset), the right-hand side is evaluated in FP32 and
 * widened back.  Replaces RHSOperator<PhysicsT>::Mult
 * (include/RHSOperator_impl.hpp:719-793). */
int thx_rhs(thx_handle h, const void *u, void *dudt, void *stream);

/* Allocation-free Euler right-hand side (no counterpart in the reference).
 * For hosts that cannot let a library call cudaMalloc -- a solver whose
 * device memory belongs to its own pool or caching allocator, or a time loop
 * that must not absorb cudaMalloc's device-wide synchronisation.  Needs no
 * handle: geom holds DEVICE pointers in the thx_geometry layout (full per-node
 * arrays), u and dudt are device FP64 L-vectors.  Euler flow, FP64, no
 * blending (else THX_ERR_UNSUPPORTED).  Its scratch (face fluxes, element-to-face
 * table, checked copies of the face tables, operators) is one static 8 MiB
 * device array per GPU, kept until the process exits: meshes needing more
 * return THX_ERR_INVALID_ARGUMENT.  The first call on a device looks the array
 * up (make it before any stream capture); every call rewrites what it reads,
 * and calls that overlap on the GPU race on the shared array.
 * status (may be NULL): a caller-owned word in device or page-locked host
 * memory that receives, stream-ordered, this call's THX_STATUS_* bits --
 * THX_STATUS_NONPOSITIVE for a non-positive density or pressure,
 * THX_STATUS_LAUNCH when the volume kernel could not run,
 * THX_STATUS_FACE_TABLE when a face_elem/face_lface entry is out of range
 * (that face's fluxes are NaN and nothing outside the arrays is touched).
 * Read it after the stream has synchronised. */
int thx_rhs_euler_noalloc(const thx_geometry *geom_dev, const thx_config *cfg,
                          const double *u, double *dudt, unsigned int *status, void *stream);

/* FP64 fused-multiply-add throughput of the current device (no counterpart in
 * the reference): eight independent FMA chains per thread on eight 256-thread
 * CTAs per SM, `iters` rounds of 64 FMAs each, the best of `repeats` timed
 * launches after one warm-up, CUDA events on `stream`.  *flops_per_s counts an
 * FMA as two operations.  The denominator of the FP64-pipe roofline of the
 * flux-differencing kernels. */
int thx_measure_fp64_fma_peak(int iters, int repeats, double *flops_per_s, void *stream);

/* Tensor-core trial of the gradient's element-local derivative contraction
 * (no counterpart in the reference): for every element of a 3-D p=4 mesh, the
 * LGL derivative matrix D_host (N*N, row-major) applied along every tensor
 * line of the NEQ fields `fields` (device, [NEQ][elements][nodes], FP64 for
 * THX_PRECISION_FP64, FP32 for THX_PRECISION_FP32_MIXED), reduced per node
 * to out[elements][nodes] = sum over (direction d, field k) of
 * (1 + (d*NEQ + k)/8) dS_k/dxi_d.  form 0: SIMT FMA, one thread per node;
 * FP64 form 1: mma.sync m8n8k4 FP64 tensor-core tiles; FP32 form 1:
 * mma.sync m16n8k8 TF32 (one product), form 2: TF32 split into high and low
 * parts (three products).  *ms: mean device time of `reps` launches after one
 * warm-up (CUDA events on `stream`). */
int thx_trial_contraction(int dim, int order, int num_elements, int precision, int form,
                          const void *fields, const double *D_host, void *out, int reps,
                          double *ms, void *stream);

/* Right-hand sides of n states held in HOST memory: dudt_host[i] = L(u_host[i])
 * (FP64 L-vectors; in FP32-mixed mode each state is evaluated as thx_rhs does).
 * The library copies state i+1 in and rate i-1 out while it evaluates state
 * i (two device buffers, a copy-in and a copy-out stream); with page-locked
 * host buffers the transfers in both directions overlap the kernels.  The
 * calls are stream-ordered on `stream`: work queued there before the call
 * runs first, and work queued after it waits for the last copy-out.  Host
 * buffers must stay valid until then. */
int thx_rhs_host(thx_handle h, int n, const double *const *u_host, double *const *dudt_host, void *stream);

/* nsteps SSP-RK3 steps (Shu-Osher form, as mfem::RK3SSPSolver::Step driven at
 * src/Simulation.cpp:1255) on a device FP64 state u, in place, with fixed dt.
 * In FP32-mixed mode the FP64 master state is accumulated in double and each
 * RHS is evaluated on a float working copy. */
int thx_rk3_steps(thx_handle h, double *u, double dt, int nsteps, void *stream);
/* nsteps SSP-RK3 steps with dt = cfl / (max(advective, surface) + diffusive
 * rate) of each step's initial state (src/Simulation.cpp:1150-1160), computed
 * on the device: the loop never waits for the host, so it can be captured in
 * a CUDA graph.  Unlike the reference's loop it applies no growth limit and
 * lands on no events; thx_rk3_time_loop runs that loop.  dt_history (device, may be NULL) receives each step's dt.  A
 * non-positive rate sets the numerics status flag and dt = 0. */
int thx_rk3_steps_cfl(thx_handle h, double *u, double cfl, int nsteps, double *dt_history,
                      void *stream);

/* State of the reference's clocked time loop (src/Simulation.cpp:1150-1335
 * with include/TimeStepControl.hpp and include/RunControl.hpp): the nominal
 * step, the final time and the time-based output and checkpoint events the
 * step is shortened to land on.  thx_time_loop_defaults fills the reference's
 * runTime defaults. */
typedef struct thx_time_loop {
  double t;                 /* simulation time */
  double dt;                /* nominal step (Simulation::dt); with cfl > 0 a value <= 0
                               takes cfl / TotalRate of the current state first */
  double t_final;           /* runTime.final_time */
  double max_dt_growth;     /* runTime.max_dt_growth (1.2) */
  double next_output;       /* next_save_t; INFINITY: no output events */
  double output_dt;         /* runTime.initial_save_dt (0.01) */
  double refined_output_dt; /* runTime.refined_save_dt (initial_save_dt) */
  double refine_time;       /* runTime.refined_trigger (2.0) */
  double next_checkpoint;   /* next_checkpoint_t; INFINITY: no checkpoint events */
  double checkpoint_dt;     /* runTime.checkpoint_dt (0.01) */
  double last_dt;           /* the step the last cycle took (dt_real) */
  int64_t cycle;            /* ti */
  int64_t max_cycles;       /* runTime.nsteps_max; <= 0: no limit */
  int64_t output_cycles;    /* runTime.vis_steps (100) */
  int64_t outputs;          /* output events so far */
  int64_t checkpoints;      /* checkpoint events so far */
  int32_t done;             /* the loop has ended; further cycles leave the state alone */
  int32_t reserved;
} thx_time_loop;

void thx_time_loop_defaults(thx_time_loop *loop);
/* TimeEventReached (include/TimeStepControl.hpp:21-25). */
int thx_time_event_reached(double t, double event_time);
/* LimitTimeStepToEvents over n event times (include/TimeStepControl.hpp:42-49). */
double thx_limit_time_step_to_events(double step, double t, const double *events, int n);
/* StepLimitReached (include/RunControl.hpp:11-14). */
int thx_step_limit_reached(int64_t cycle, int64_t max_cycles);
/* One cycle of the loop's bookkeeping on a HOST record, the code the device
 * loop runs: begin returns the step to take (0 once done); end advances the
 * time and cycle, updates the nominal step from total_rate when cfl > 0
 * (total_rate = max(advective, surface) + diffusive rate of the new state),
 * decides done and counts the output and checkpoint events. */
double thx_time_loop_begin(thx_time_loop *loop);
void thx_time_loop_end(thx_time_loop *loop, double dt_taken, double total_rate, double cfl);

/* Face table of conforming straight-sided cells (host; the face maps of
 * include/dgsem_cache_utilities.hpp:516-639 for meshes whose cells are
 * oriented along the mesh axes).  vertex_ids: int64[ne][2^dim], each cell's
 * vertex ids in lexicographic order of its reference coordinates (x fastest);
 * shared ids make a face interior (give periodic partners one id; faces are
 * told apart by their vertex ids, so a periodic direction needs at least
 * three cells).  An
 * interior face's minus side is the cell whose + face it is; faces are
 * ordered by (direction, minus cell), boundary faces by (direction, cell,
 * local face).  Capacities: face arrays ne*dim entries (pairs), boundary
 * arrays 2*dim*ne; any output pointer may be NULL to count only.
 * THX_ERR_INVALID_ARGUMENT for faces that are not aligned or shared by more
 * than two cells. */
int thx_cell_faces(int dim, int ne, const int64_t *vertex_ids, int32_t *face_elem, int32_t *face_lface,
                   int32_t *num_faces, int32_t *bdr_elem, int32_t *bdr_lface, int32_t *num_bdr_faces);
/* Geometric factors of straight-sided (bi/trilinear) cells computed on the
 * DEVICE (replaces SetupGeometricTerms / AssembleElementVolumeGeometricTerms /
 * AssembleInteriorFaceGeometryTerms, include/dgsem_cache_utilities.hpp:83-215,
 * 470-639): per LGL node the Jacobian determinant and the adjugate rows,
 * per face point the minus cell's outward face-Jacobian-scaled normal and
 * the lift weights 1/(w0 J) of both sides, per boundary face point the
 * normal and weight; optionally the node coordinates [dim][ne][nodes].
 * Every pointer is DEVICE memory: corners double[ne][2^dim][dim]
 * (lexicographic vertices), the face tables of thx_cell_faces, the outputs in
 * the thx_geometry layout.  Allocates nothing and waits for nothing
 * (stream-ordered).  A face entry naming no cell or local face of the mesh
 * yields NaN normals and weights for that face. */
int thx_cell_geometry(int dim, int order, int ne, const double *corners, int nf, const int32_t *face_elem,
                      const int32_t *face_lface, int nbf, const int32_t *bdr_elem, const int32_t *bdr_lface,
                      double *jac, double *metric, double *face_normal, double *face_wminus,
                      double *face_wplus, double *bdr_normal, double *bdr_weight, double *node_coords,
                      void *stream);

/* ncycles cycles of the reference's clocked SSP-RK3 loop on a device FP64
 * state u, in place: each cycle takes the nominal step shortened to the next
 * event (final time, output, checkpoint), then, with cfl > 0, sets the next
 * nominal step to min(cfl / TotalRate, max_dt_growth * dt) from the new
 * state's stability rates (cfl <= 0: fixed step).  loop points to a
 * thx_time_loop in DEVICE memory, read and advanced on the device; once it is
 * done the remaining cycles leave u unchanged.  Nothing waits for the host,
 * so the call can be captured in a CUDA graph.  dt_history (device, may be
 * NULL) receives each cycle's step. */
int thx_rk3_time_loop(thx_handle h, double *u, double cfl, int ncycles, thx_time_loop *loop,
                      double *dt_history, void *stream);

/* Per-element blending coefficient alpha of the last RHS (device, double[E])
 * and the Persson smoothness eta (double[E]); either pointer may be NULL.
 * Mirrors ComputeBlendingCoefficient / CheckIndicatorSmoothness
 * (include/RHSOperator_impl.hpp:411-527). */
int thx_blending_coefficients(thx_handle h, double *alpha_dev, double *eta_dev,
                              void *stream);

/* Stable time step estimate: sigma = max(adv, surface) + diffusive rate and
 * dt = cfl/sigma (include/RHSOperator_impl.hpp:10-270,
 * include/StabilityEstimate.hpp:12-92).  u is a device FP64 state.  Blocks
 * until the reduction is finished (it returns a host value). */
int thx_estimate_dt(thx_handle h, const double *u, double cfl, double *dt_out,
                    double *rates_out /* [3]: advective, surface, diffusive */);

/* Integral measures of a device FP64 state u (IntegralMeasures,
 * include/RHSOperator_impl.hpp:530-717): out[9] = integrals of rho, of the
 * kinetic energy density |m|^2/(2 rho) and of rho E (node quadrature, J times
 * the LGL weights), then min/max pressure, min/max temperature, min/max density.
 * Per-element sums in node order, combined on the host in element order.
 * Blocks until done (it returns host values). */
int thx_integral_measures(thx_handle h, const double *u, double *out);

/* Device status word of the evaluations since the last read, a bitwise OR of
 * THX_STATUS_* flags.  Reading it synchronises the stream and clears it. */
#define THX_STATUS_NONPOSITIVE 1u  /* non-positive density or pressure seen */
#define THX_STATUS_NONFINITE 2u    /* non-finite value seen */
#define THX_STATUS_LAUNCH 4u       /* a kernel got too little shared memory and did nothing */
#define THX_STATUS_EOS 8u          /* LTE temperature recovery failed or left the table */
#define THX_STATUS_FACE_TABLE 16u  /* a face table entry was out of range (thx_rhs_euler_noalloc) */
#define THX_STATUS_TIMEOUT 32u     /* a bulk copy into shared memory did not land within 1 s */
int thx_read_status(thx_handle h, uint32_t *flags, void *stream);

/* ---- batch engine (no counterpart in the reference) -----------------------
 * Many independent cases -- each its own periodic mesh, polynomial order and
 * flow model -- advanced together: cases with the same (dimension, order,
 * flow model) form a group whose SSP-RK3 stages run as persistent kernels
 * over one device work list, launched from a CUDA graph of `steps_per_launch`
 * steps that stays valid while cases join and leave.  The reference's
 * Simulation (src/Simulation.cpp:43-47) runs one case per process; the engine
 * replaces a loop of RHSOperator::Mult-driven solves.
 *
 * cfg fixes the flux selection, precision and gas constants of every case;
 * each case brings its geometry (host pointers), flow model, step count, dt,
 * viscosity and FP32 working-copy offset.  States stay on the device from
 * admission to fetch.  Results are bit-identical to the same case run alone
 * through thx_rk3_steps with the same configuration. */
typedef struct thx_engine_s *thx_engine;

typedef struct {
  int32_t flow_model;        /* THX_FLOW_EULER or THX_FLOW_NAVIER_STOKES */
  int32_t nsteps;            /* SSP-RK3 steps */
  double dt;                 /* fixed step */
  double mu, Pr;             /* transport (Navier-Stokes) */
  double state_offset[5];    /* FP32 working-copy offset (FP32-mixed engines) */
  int64_t geometry_key;      /* 0: the case's geometry is uploaded for it alone; otherwise cases
                                with the same key share one device copy of the geometry (built from
                                the first such case's mesh and kept until the engine is destroyed;
                                the caller guarantees the key names one mesh -- a later case with a
                                different element/face count under the key is refused) */
} thx_case;

typedef struct {
  int32_t active_cases;      /* admitted and not yet fetched */
  int32_t groups;            /* (dimension, order, flow) groups seen */
  int64_t bytes_in_use;      /* footprint of the active cases */
  int64_t launches;          /* graph launches so far */
  int64_t cases_done;        /* cases fetched */
  double admit_lock_s;       /* host seconds admissions waited for the engine lock */
  double admit_setup_s;      /* host seconds in case set-up (packing, allocations) */
  double admit_copy_s;       /* host seconds issuing the initial-state upload */
  double advance_s;          /* host seconds inside advance (lock held) */
  double fetch_copy_s;       /* host seconds copying results to the host */
  int64_t pool_reserved_bytes;  /* device memory the engine's pool holds */
  int64_t pool_used_bytes;      /* of which allocated to cases */
  int64_t advance_calls;        /* calls of thx_engine_advance */
  double advance_tables_s;      /* of advance_s: rewriting and uploading group tables */
  double advance_launch_s;      /* of advance_s: graph captures and launches */
  int64_t table_bytes;          /* bytes of group tables uploaded */
  double ring_wait_s;           /* host seconds uploads waited for pinned staging space */
  double ring_copy_s;           /* host seconds copying uploads into pinned staging */
} thx_engine_stats;

/* Device bytes one case needs (state, stage copies, scratch, geometry). */
int thx_case_footprint(const thx_geometry *geom, const thx_config *cfg, int flow_model,
                       size_t *bytes);
/* hbm_budget: bytes the engine may hold for cases; steps_per_launch: SSP-RK3
 * steps per graph launch (cases whose step count is not a multiple finish
 * their last steps one launch at a time). */
int thx_engine_create(const thx_config *cfg, size_t hbm_budget, int steps_per_launch,
                      thx_engine *out);
int thx_engine_destroy(thx_engine e);
/* Admit a case with initial state u0 (host FP64 L-vector); THX_ERR_BUSY if its
 * footprint does not fit the budget now.  Set-up runs on the engine's own
 * stream and overlaps with the running groups. */
int thx_engine_admit(thx_engine e, const thx_geometry *geom, const thx_case *c,
                     const double *u0, int64_t *id);
/* Launch the next `steps_per_launch` steps of every group with active cases
 * (asynchronous; returns immediately). */
int thx_engine_advance(thx_engine e);
/* Ids of cases whose steps are complete on the device (up to cap). */
int thx_engine_poll(thx_engine e, int64_t *ids, int cap, int *count);
/* Copy a finished case's state to the host and release it. */
int thx_engine_fetch(thx_engine e, int64_t id, double *u_host);
int thx_engine_get_stats(thx_engine e, thx_engine_stats *out);

/* One batch group of the engine (cases of the same dimension, order and
 * flow model share persistent batched kernels and one CUDA graph).  The
 * engine tunes those kernels online by coordinate search: the elements per
 * CTA of the volume and gradient kernels (as many as fit 256 threads, or
 * half as many), then the volume grid over {1,2,4} x SMs, the face grid over
 * {4,8,16} x SMs and (Navier-Stokes) the gradient grid over {1,2,4} x SMs,
 * each candidate timed with CUDA events around two launches that advance real
 * cases (the better one counts); cost = device milliseconds per (solution
 * node x step). */
typedef struct {
  int32_t dim, order, navier_stokes;
  int32_t active_cases;
  int32_t tuned;          /* 1 once every axis has been searched */
  int32_t volume_grid, face_grid, gradient_grid;  /* the best so far */
  int32_t elements_per_block;  /* of the best configuration */
  double best_cost_ms;    /* cost of the best grids on the axis being searched
                             (-1 before its first timing) */
} thx_engine_group;
/* Up to cap groups in key order; *count = the number of groups. */
int thx_engine_groups(thx_engine e, thx_engine_group *out, int cap, int *count);

/* Diagnostics of the configured kernels (for roofline bookkeeping). */
int thx_describe(thx_handle h, char *buf, size_t len);

/* One right-hand side like thx_rhs, with CUDA events between its kernels;
 * synchronises the stream and returns the device time of each phase in
 * milliseconds: ms[0] indicator, ms[1] gradient, ms[2] face fluxes,
 * ms[3] volume + lift (0 for phases the configuration does not run). */
int thx_rhs_profile(thx_handle h, const void *u, void *dudt, void *stream, double *ms);

/* ---- checkpoint interchange (host only) ---------------------------------
 * The reference's restart format (src/Simulation.cpp:1477-1603,
 * include/CheckpointConfig.hpp): per rank
 *   <dir>/Cycle<c>/checkpoint_cycle_<c>.<rank:08d>.chk =
 *     "THESEUS_CHECKPOINT_RAW_V1\n", uint64 count, count doubles (the state
 *     L-vector, native byte order)
 * and once per cycle <dir>/Cycle<c>/checkpoint_cycle_<c>.json with the
 * compatibility record below (format_version 2).  `dir` is the run's
 * checkpoints folder (runTime.checkpoints_folder under the output directory).
 * Failure reasons are written to msg (may be NULL) with the reference's
 * wording. */
typedef struct {               /* CheckpointCompatibility (CheckpointConfig.hpp:19-29) */
  int32_t mpi_ranks;
  int32_t order;
  int32_t dimension;
  int32_t num_equations;
  int32_t real_bytes;          /* 8: FP64 states */
  int32_t axisymmetric;
  int64_t global_elements;
  int64_t global_dofs;         /* the global state-vector length (num_equations x nodes) */
} thx_checkpoint_compat;

/* The metadata JSON text of a cycle (CheckpointConfig::Metadata). */
int thx_checkpoint_metadata(double time, int cycle, const thx_checkpoint_compat *c, char *buf,
                            size_t len);
/* CheckpointConfig::ValidateMetadata: THX_OK with *current_format = 1, or 0
 * for legacy metadata (time and cycle only); THX_ERR_INVALID_ARGUMENT when
 * incompatible. */
int thx_checkpoint_validate(const char *json, const thx_checkpoint_compat *expected,
                            int *current_format, char *msg, size_t msg_len);
/* Simulation::SaveCheckpoint for one rank: the state file, and the metadata
 * when write_metadata != 0 (rank 0 in the reference, after every rank's
 * state is complete). */
int thx_checkpoint_save(const char *dir, int cycle, int rank, double time,
                        const thx_checkpoint_compat *compat, const double *state, int64_t count,
                        int write_metadata, char *msg, size_t msg_len);
/* Simulation::LoadCheckpoint for one rank: checks the cycle, the time entry
 * and the compatibility record, then reads `count` doubles into state (host)
 * and the simulation time.  Legacy (MFEM grid-function) states return
 * THX_ERR_UNSUPPORTED. */
int thx_checkpoint_load(const char *dir, int cycle, int rank, const thx_checkpoint_compat *expected,
                        double *time, double *state, int64_t count, char *msg, size_t msg_len);

#ifdef __cplusplus
}
#endif
#endif /* THESEUS_B200_H */
