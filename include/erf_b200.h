/*
 * erf_b200.h -- C-ABI of the B200-native multirate RK3 dycore.
 *
 * The reference (ERF) exposes this hot path as free functions on AMReX
 * MultiFab/Array4 objects, wired into MRISplitIntegrator through std::function
 * hooks (Source/TimeIntegration/ERF_MRI.H:137-180, installed by
 * Source/TimeIntegration/ERF_advance_dycore.cpp:285-302).  This header replaces
 * those signatures with plain pointers, sizes and POD structs so that an
 * AMReX-based caller can hand over fab.dataPtr() plus the box and strides
 * zero-copy, and any other host language can bind it through its FFI.
 *
 * Conventions
 *   - Every array is an erf_b200_fab: a device pointer to FP64 data in Array4
 *     order (i fastest), the index box [lo, hi] the pointer covers (valid
 *     region plus whatever ghost cells the caller allocated), and strides.
 *     p[(i-lo.x) + (j-lo.y)*jstride + (k-lo.z)*kstride + n*nstride].
 *   - Cell-centred data use cell indices 0..n-1; x-face data use face indices
 *     0..nx (nodal in x), and likewise for y and z.
 *   - All calls are asynchronous on the stream given to erf_b200_create (or
 *     the stream passed per call where a call takes one).  Only
 *     erf_b200_get_status synchronises.
 *   - Every function returns an int status: ERF_B200_OK (0) or one of the
 *     ERF_B200_E* codes below.  Nothing in the library aborts or exits.
 */
#ifndef ERF_B200_H
#define ERF_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------------------------------------
 * Status codes
 * ------------------------------------------------------------------------- */
#define ERF_B200_OK               0
#define ERF_B200_EINVAL           1   /* bad argument / unsupported option      */
#define ERF_B200_ECUDA            2   /* a CUDA runtime call failed             */
#define ERF_B200_ENOMEM           3   /* device allocation failed               */
#define ERF_B200_EBADSTATE        4   /* non-positive rho*theta or rho seen     */
#define ERF_B200_ENAN             5   /* NaN/Inf detected in the state          */
#define ERF_B200_EPIVOT           6   /* vertical tridiagonal pivot ~ 0         */
#define ERF_B200_ETIMEOUT         7   /* a bounded device wait ran out          */
#define ERF_B200_ECONFIG          8   /* configuration rejected                 */
#define ERF_B200_EABORTED         9   /* an ensemble run was stopped by its abort word */
#define ERF_B200_EBOUNDS         10   /* bounds-checked build (liberf_b200_bounds.so):
                                         a kernel formed an index outside its array */

/* ----------------------------------------------------------------------------
 * Enumerations: numeric values match the reference's enums so that a caller
 * can pass its own SolverChoice fields straight through.
 * ------------------------------------------------------------------------- */
/* AdvType (Source/ERF_IndexDefines.H): Centered_2nd=101 ... */
#define ERF_ADV_CENTERED_2ND 101
#define ERF_ADV_UPWIND_3RD   102
#define ERF_ADV_CENTERED_4TH 103
#define ERF_ADV_UPWIND_5TH   104
#define ERF_ADV_CENTERED_6TH 105
#define ERF_ADV_WENO_3       106
#define ERF_ADV_WENO_3Z      107
#define ERF_ADV_WENO_5       108
#define ERF_ADV_WENO_5Z      109
#define ERF_ADV_WENO_3MZQ    110
#define ERF_ADV_WENO_7       111
#define ERF_ADV_WENO_7Z      112

/* LESType (Source/DataStructs/ERF_TurbStruct.H) */
#define ERF_LES_NONE         0
#define ERF_LES_SMAGORINSKY  1
#define ERF_LES_DEARDORFF    2
/* Learned closure (no reference counterpart): the erf_b200_mlp network of
 * erf_b200_set_closure, with Smagorinsky outside its training envelope. */
#define ERF_LES_MLP          3

/* MolecDiffType (Source/DataStructs/ERF_DiffStruct.H) */
#define ERF_MOLEC_NONE           0
#define ERF_MOLEC_CONSTANT       1
#define ERF_MOLEC_CONSTANT_ALPHA 2

/* MoistureType subset */
#define ERF_MOIST_NONE            0
#define ERF_MOIST_KESSLER         1
#define ERF_MOIST_KESSLER_NORAIN  2

/* ERF_BC (Source/ERF_IndexDefines.H): vertical boundary kinds supported */
#define ERF_BC_NO_SLIP_WALL  5
#define ERF_BC_SLIP_WALL     6
#define ERF_BC_PERIODIC      7
#define ERF_BC_MOST          8   /* Monin-Obukhov surface layer (ground only) */

/* Arithmetic of the bulk dycore */
#define ERF_PREC_FP64        0   /* plain FP64 form                          */
#define ERF_PREC_MIXED       1   /* FP32 bulk on perturbations, FP64 state   */

/* Cell-centred component layout (Source/ERF_IndexDefines.H:36-48) */
#define ERF_RHO_COMP        0
#define ERF_RHOTHETA_COMP   1
#define ERF_RHOKE_COMP      2
#define ERF_RHOQKE_COMP     3
#define ERF_RHOSCALAR_COMP  4
#define ERF_RHOQ1_COMP      5

/* ----------------------------------------------------------------------------
 * Array4-style view
 * ------------------------------------------------------------------------- */
typedef struct erf_b200_fab {
    double*  p;        /* device pointer to element (lo.x, lo.y, lo.z, 0)    */
    int      lo[3];    /* inclusive index bounds covered by p               */
    int      hi[3];
    int64_t  jstride;  /* elements between j and j+1                        */
    int64_t  kstride;  /* elements between k and k+1                        */
    int64_t  nstride;  /* elements between components                       */
    int      ncomp;
} erf_b200_fab;

/* ----------------------------------------------------------------------------
 * Configuration: the SolverChoice / AdvChoice / DiffChoice / TurbChoice keys
 * that the hot path reads (Source/DataStructs/ERF_DataStruct.H:80-580,
 * ERF_AdvStruct.H:26-186, ERF_TurbStruct.H:29-210, ERF_DiffStruct.H:26-32),
 * plus the grid and the fixed time step.  POD, passed by pointer.
 * ------------------------------------------------------------------------- */
/* Substepping types (SubsteppingType, DataStructs/ERF_DataStruct.H) */
#define ERF_SUBSTEP_IMPLICIT 0
#define ERF_SUBSTEP_NONE     1

/* terrain_type */
#define ERF_TERRAIN_STATIC 0
#define ERF_TERRAIN_MOVING 1

typedef struct erf_b200_config {
    /* grid: one box covering the domain, periodic in x and y */
    int    nx, ny, nz;
    double dx, dy, dz;
    int    zlo_bc, zhi_bc;            /* ERF_BC_NO_SLIP_WALL / _SLIP_WALL (/ _MOST below) */

    /* time stepping: fixed_dt, fixed_mri_dt_ratio, force_stage1_single_substep */
    double dt;
    int    mri_ratio;                 /* even, >= 2                          */
    int    force_stage1_single_substep;

    /* state layout: NDRY(4) + NSCALARS(1) + n_qstate */
    int    ncomp;
    int    moisture;                  /* ERF_MOIST_*                         */

    /* advection (AdvChoice) */
    int    dycore_horiz_adv, dycore_vert_adv;
    int    dryscal_horiz_adv, dryscal_vert_adv;
    int    moistscal_horiz_adv, moistscal_vert_adv;
    double dycore_horiz_upw_frac, dycore_vert_upw_frac;
    double dryscal_horiz_upw_frac, dryscal_vert_upw_frac;
    double moistscal_horiz_upw_frac, moistscal_vert_upw_frac;

    /* diffusion (DiffChoice) and LES closure (TurbChoice) */
    int    molec_diff_type;
    double alpha_T, alpha_C, dynamic_viscosity, rho0_trans;
    int    les_type;
    double Cs, Pr_t, Sc_t, Ck, Ce, Ce_wall, sigma_k, theta_ref;

    /* forcing */
    double gravity;                   /* 9.81 with use_gravity, else 0       */
    double c_p;                       /* 1004.5 default                      */
    int    buoyancy_type;             /* 1 dry rho', 2 T'-based (moist)      */
    int    use_coriolis;
    double coriolis_factor, sinphi, cosphi;
    double abl_geo_forcing[3];

    /* arithmetic of the bulk (ERF_PREC_*) */
    int    precision;
    /* static terrain-following grid (SolverChoice::use_terrain with
     * terrain_type Static): z_phys_nd installed by erf_b200_set_terrain */
    int    use_terrain;
    /* SolverChoice::substepping_type: ERF_SUBSTEP_IMPLICIT (acoustic
     * substepping, the default) or ERF_SUBSTEP_NONE (one update per RK stage
     * with the whole slow right-hand side, MRISplitIntegrator::set_no_substep,
     * TimeIntegration/ERF_MRI.H:177-180, 255-324; mri_ratio is then unused) */
    int    substepping_type;
    /* SolverChoice::terrain_type with use_terrain: ERF_TERRAIN_STATIC
     * (z_phys_nd installed by erf_b200_set_terrain) or ERF_TERRAIN_MOVING:
     * the library regenerates the grid at every geometry time from the
     * travelling surface wave h(x, t) = mt_ampl sin(k x - omega t),
     * k = 2 pi / mt_wavelength, omega = sqrt(g k) (the surface of
     * Exec/DevTests/MovingTerrain/ERF_prob.cpp:147-200) smoothed upward with
     * Sullivan's factor (1 - z/z_top)^3 (terrain_smoothing = 2,
     * Utils/ERF_TerrainMetrics.cpp:501-536) over the uniform levels k dz;
     * with or without acoustic substepping (erf_fast_rhs_MT) */
    int    terrain_type;
    /* SolverChoice::use_lagged_delta_rt = false (1 here; 0 keeps the
     * reference default, true): the acoustic substeps over moving terrain
     * then extrapolate d(rho theta) without the lagged correction
     * (ERF_fast_rhs_MT.cpp:197-210); the reference allows it for moving
     * terrain only (ERF_DataStruct.H:389) */
    int    no_lagged_delta_rt;
    int    reserved[3];
    /* MOST surface layer for zlo_bc ERF_BC_MOST (ABLMost, erf.most.*): the
     * roughness length z0 and the reference height zref (moved to the
     * centre of the cell level that contains it, as MOSTAverage does); Moeng
     * stress, adiabatic surface, plane averages */
    double most_z0, most_zref;
    /* moving terrain (terrain_type ERF_TERRAIN_MOVING): wave amplitude and
     * wavelength in metres (prob.Ampl; the wavelength is 100 m upstream) */
    double mt_ampl, mt_wavelength;
} erf_b200_config;

/* Opaque context: owns all integrator scratch (S_sum, S_scratch, F_slow,
 * primitive variables, fast coefficients, eddy viscosity, stress, ...). */
typedef struct erf_b200_ctx erf_b200_ctx;

/* ----------------------------------------------------------------------------
 * Life cycle
 * ------------------------------------------------------------------------- */

/* Fill *cfg with the reference defaults (SolverChoice defaults; dycore and dry
 * scalars Upwind_3rd, moist scalars WENO3, Implicit substepping, c_p 1004.5). */
int erf_b200_config_defaults(erf_b200_config* cfg);

/* Create a context on the current CUDA device; all scratch is allocated here
 * and never inside a step.  `stream` is a cudaStream_t (NULL = legacy default). */
int erf_b200_create(erf_b200_ctx** ctx, const erf_b200_config* cfg, void* stream);
int erf_b200_destroy(erf_b200_ctx* ctx);
int erf_b200_set_stream(erf_b200_ctx* ctx, void* stream);

/* Synchronise the context's stream and return (and clear) the sticky device
 * status word: ERF_B200_OK, ERF_B200_EBADSTATE, ERF_B200_ENAN, ... */
int erf_b200_get_status(erf_b200_ctx* ctx);

/* Bytes of device memory the context holds (scratch only). */
int erf_b200_scratch_bytes(const erf_b200_ctx* ctx, size_t* bytes);

/* ----------------------------------------------------------------------------
 * Base state (BaseState::r0_comp, p0_comp, pi0_comp, th0_comp)
 * ------------------------------------------------------------------------- */

/* Hydrostatic base state from a sounding, computed on the GPU in FP64.
 * Replaces InputSoundingData::calc_rho_p (DataStructs/ERF_InputSoundingData.H:176-256,
 * Newton iterations of Utils/ERF_HSE_utils.H:34-72) followed by
 * ERF::erf_enforce_hse (Initialization/ERF_init1d.cpp:152-260).
 * theta_cc/qv_cc: nz device values at cell centres; theta_sfc/qv_sfc/p_sfc at z=0.
 * Writes rho0, p0, pi0, th0 (nz+2 device values each, index k+1 for cell k,
 * so the k=-1 and k=nz ghosts are included). */
int erf_b200_make_base_state(erf_b200_ctx* ctx,
                             const double* theta_cc, const double* qv_cc,
                             double theta_sfc, double qv_sfc, double p_sfc,
                             double* rho0, double* p0, double* pi0, double* th0);

/* Install the base state the dycore uses (same nz+2 layout as above; with
 * terrain, nz+2 planes of nx*ny). */
int erf_b200_set_base_state(erf_b200_ctx* ctx, const double* rho0,
                            const double* p0, const double* pi0, const double* th0);

/* ----------------------------------------------------------------------------
 * Static terrain (contexts created with use_terrain = 1)
 * ------------------------------------------------------------------------- */

/* Install the terrain-following grid: z_phys_nd at the (nx+1)(ny+1)(nz+1)
 * nodes of the valid box, i fastest (host or device pointer), as built by
 * init_terrain_grid (Source/Utils/ERF_TerrainMetrics.cpp:88-335).  The
 * terrain must be periodic (node nx equal to node 0 and node ny to node 0).
 * Ghost levels and the metrics detJ / z_cc (make_J, make_zcc,
 * ERF_TerrainMetrics.cpp:583-715) are formed here.  EINVAL for a
 * non-periodic or folded grid. */
int erf_b200_set_terrain(erf_b200_ctx* ctx, const double* z_nd);

/* Hydrostatic base state over the terrain (device pointers): theta3 / qv3 at
 * the cell centres, nz planes of nx*ny; rho0, p0, pi0, th0 receive nz+2
 * planes (plane k+1 for level k), the layout erf_b200_set_base_state expects
 * with terrain.  Replaces calc_rho_p + ERF::erf_enforce_hse with terrain
 * (Initialization/ERF_init1d.cpp:152-241). */
/* Moving terrain (terrain_type ERF_TERRAIN_MOVING).  The grid is not
 * installed but generated by every step at the geometry times the
 * reference's moving-terrain path asks for (slow_rhs_fun_pre,
 * TimeIntegration/ERF_TI_slow_rhs_fun.H:55-107: the step's old time and each
 * RK stage's source and new times), from a device clock that each step
 * advances by dt (post_timestep, ERF.cpp:547-559).  The base state set by
 * erf_b200_set_base_state is the initial one and evolves with the grid.
 *   erf_b200_set_time: the clock (the old time of the next step; 0 after
 *     create);
 *   erf_b200_moving_terrain_state: the clock, the grid at that time
 *     ((nz+1)(ny+1)(nx+1) nodes, i fastest; node nx / ny repeat node 0) and
 *     the evolved base density and pressure ((nz+2) planes of nx*ny, plane
 *     k+1 for level k) into host memory; NULL skips an output.
 * Both return ERF_B200_EINVAL for a context without moving terrain. */
int erf_b200_set_time(erf_b200_ctx* ctx, double time);

/* Step diagnostics of the latest state (the resident one after
 * erf_b200_load_state / erf_b200_advance_resident, or the one the last
 * erf_b200_advance returned): out[0] the mass, the integral of rho over the
 * physical volume (dx dy dz detJ per cell: ERF's sum_interval mass check,
 * sum_integrated_quantities / volWgtSumMF, IO/ERF_WriteScalarProfiles.cpp:
 * 14-60, 378-420), out[1] the integral of rho theta, out[2] max |w|.  A
 * fixed-order reduction on the device; synchronises the stream. */
int erf_b200_diagnostics(erf_b200_ctx* ctx, double* out);
int erf_b200_moving_terrain_state(erf_b200_ctx* ctx, double* time, double* z_nd, double* rho0, double* p0);

int erf_b200_make_base_state_terrain(erf_b200_ctx* ctx, const double* theta3, const double* qv3,
                                     double theta_sfc, double qv_sfc, double p_sfc,
                                     double* rho0, double* p0, double* pi0, double* th0);

/* ----------------------------------------------------------------------------
 * Full step: replaces ERF::advance_dycore + MRISplitIntegrator::advance +
 * ERF::advance_microphysics (TimeIntegration/ERF_Advance.cpp:165-174,
 * ERF_advance_dycore.cpp:37-305, ERF_MRI.H:187-369, ERF_advance_microphysics.cpp).
 * cons (ncomp comps), xvel, yvel, zvel are read at the start and overwritten
 * with the state after `nsteps` steps; ghost cells of the caller's fabs are
 * filled (periodic laterally, wall conditions vertically) on return.  The step
 * sequence is captured once into a CUDA graph and replayed.
 * ------------------------------------------------------------------------- */
int erf_b200_advance(erf_b200_ctx* ctx,
                     const erf_b200_fab* cons, const erf_b200_fab* xvel,
                     const erf_b200_fab* yvel, const erf_b200_fab* zvel,
                     int nsteps);

/* Same as erf_b200_advance with host buffers: copies in, advances, copies out.
 * Host arrays are dense valid-region arrays (no ghosts), i fastest:
 * cons[ncomp][nz][ny][nx], u[nz][ny][nx+1], v[nz][ny+1][nx], w[nz+1][ny][nx].
 * Components the step neither reads nor changes (rho*QKE, and rho*KE unless
 * les_type is ERF_LES_DEARDORFF) are left in place on the host, uncopied. */
int erf_b200_advance_host(erf_b200_ctx* ctx, double* cons, double* u,
                          double* v, double* w, int nsteps);

/* ----------------------------------------------------------------------------
 * Instrumentation (no counterpart in the reference, which only has TinyProfiler
 * regions, Source/TimeIntegration/ERF_MRI.H:189): erf_b200_advance without the
 * CUDA graph, with a CUDA event pair around every kernel launch.  kernel_ms /
 * kernel_launches (nslots >= ERF_B200_NUM_KERNEL_SLOTS) receive the summed
 * device time and launch count per kernel slot:
 *   0 step_begin, 1 stress, 2 slow_cell, 3 plane_avg, 4 slow_mom,
 *   5 fast_horizontal, 6 fast_column, 7 slow_post, 8 kessler, 9 fast_coeffs,
 *   10 no_substep (the stage update without acoustic substepping).
 * ------------------------------------------------------------------------- */
#define ERF_B200_NUM_KERNEL_SLOTS 11
int erf_b200_advance_profiled(erf_b200_ctx* ctx,
                              const erf_b200_fab* cons, const erf_b200_fab* xvel,
                              const erf_b200_fab* yvel, const erf_b200_fab* zvel,
                              int nsteps, double* kernel_ms, int* kernel_launches,
                              int nslots);

/* Number of kernel launches one step issues (the CUDA graph's node count). */
int erf_b200_kernels_per_step(const erf_b200_ctx* ctx, int* launches);

/* ----------------------------------------------------------------------------
 * Per-pass entry points with the roles and argument order of the reference
 * functions, for callers that keep their own integrator.  State vectors are
 * passed as arrays of 4 fabs {cons, xmom, ymom, zmom} (IntVars order).
 * ------------------------------------------------------------------------- */

/* ComputeStrain_N + ComputeTurbulentViscosityLES (Smagorinsky / Deardorff):
 * Diffusion/ERF_ComputeStrain_N.cpp:28-229,
 * Diffusion/ERF_ComputeTurbulentViscosity.cpp:32-433.  Reads velocities and
 * cons, writes the eddy viscosity held in the context. */
int erf_b200_turbulent_viscosity(erf_b200_ctx* ctx, const erf_b200_fab* xvel,
                                 const erf_b200_fab* yvel, const erf_b200_fab* zvel,
                                 const erf_b200_fab* cons);

/* ABLMost::update_fluxes (BoundaryConditions/ERF_ABLMost.cpp:11-142) for a
 * context with a MOST ground (zlo_bc ERF_BC_MOST; ERF_B200_ECONFIG
 * otherwise): the plane means of u, v and the horizontal speed at the
 * reference level and the friction velocity, from the step's old velocities
 * (ERF_Advance.cpp:62-86 calls it once per step, before the step's boundary
 * fills).  erf_b200_slow_rhs_pre then evaluates the MOST ghost velocities of
 * the stage fills (ABLMost::impose_most_bcs, ERF_ABLMost.cpp:289-489) from
 * them; it returns ERF_B200_EBADSTATE over a MOST ground until this has been
 * called once.  erf_b200_advance makes them itself each step. */
int erf_b200_most_update_fluxes(erf_b200_ctx* ctx, const erf_b200_fab* xvel,
                                const erf_b200_fab* yvel);

/* erf_slow_rhs_pre (TimeIntegration/ERF_slow_rhs_pre.cpp:67-774, declared in
 * ERF_TI_slow_headers.H:54-110) including make_mom_sources/make_buoyancy and
 * erf_make_tau_terms.  S_rhs[4] out; S_data[4] stage state in; S_scratch[4]
 * receives the stage mass fluxes as average momenta; xvel/yvel/zvel the stage
 * velocities. */
int erf_b200_slow_rhs_pre(erf_b200_ctx* ctx, int nrk, double slow_dt,
                          const erf_b200_fab* S_rhs, const erf_b200_fab* S_data,
                          const erf_b200_fab* S_scratch,
                          const erf_b200_fab* xvel, const erf_b200_fab* yvel,
                          const erf_b200_fab* zvel);

/* make_fast_coeffs (TimeIntegration/ERF_make_fast_coeffs.cpp:27-294):
 * fast_coeffs has 5 comps on z-faces: A, 1/B', C, P, Q. */
int erf_b200_make_fast_coeffs(erf_b200_ctx* ctx, const erf_b200_fab* fast_coeffs,
                              const erf_b200_fab* S_stage, double dtau);

/* erf_fast_rhs_N (TimeIntegration/ERF_fast_rhs_N.cpp:36-614): one acoustic
 * substep.  S_prev is S_old at step 0 and S_data afterwards (may alias). */
int erf_b200_fast_rhs_N(erf_b200_ctx* ctx, int step, int nrk,
                        const erf_b200_fab* S_slow_rhs, const erf_b200_fab* S_prev,
                        const erf_b200_fab* S_stage, const erf_b200_fab* S_data,
                        const erf_b200_fab* S_scratch,
                        double dtau, double facinv);

/* erf_fast_rhs_T (TimeIntegration/ERF_fast_rhs_T.cpp:39-704, declared in
 * ERF_TI_fast_headers.H:47-75): the same substep over static terrain, for a
 * context created with use_terrain; S_scratch's z-momentum is the average
 * contravariant momentum (Omega).  The other per-pass entries (turbulent
 * viscosity, slow_rhs_pre / post, make_fast_coeffs) take the terrain branch
 * themselves in such a context, as their reference counterparts do;
 * erf_b200_fast_rhs_N returns ERF_B200_ECONFIG there. */
int erf_b200_fast_rhs_T(erf_b200_ctx* ctx, int step, int nrk,
                        const erf_b200_fab* S_slow_rhs, const erf_b200_fab* S_prev,
                        const erf_b200_fab* S_stage, const erf_b200_fab* S_data,
                        const erf_b200_fab* S_scratch,
                        double dtau, double facinv);

/* The no_substep hook of MRISplitIntegrator (set_no_substep,
 * TimeIntegration/ERF_MRI.H:177-180, called at :320; the lambda of
 * ERF_TI_no_substep_fun.H:6-150) for substepping_type ERF_SUBSTEP_NONE:
 * S_sum's rho, rho*theta and momenta = S_old + slow_dt * F_slow, then the
 * boundary fill of S_sum.  nrk is the RK stage (0..2). */
int erf_b200_no_substep(erf_b200_ctx* ctx, const erf_b200_fab* S_sum,
                        const erf_b200_fab* S_old, const erf_b200_fab* F_slow,
                        double slow_dt, int nrk);

/* erf_slow_rhs_post (TimeIntegration/ERF_slow_rhs_post.cpp:49-559). */
int erf_b200_slow_rhs_post(erf_b200_ctx* ctx, int nrk, double slow_dt,
                           const erf_b200_fab* S_rhs, const erf_b200_fab* S_old,
                           const erf_b200_fab* S_new, const erf_b200_fab* S_data,
                           const erf_b200_fab* S_scratch);

/* Kessler::AdvanceKessler with Copy_State_to_Micro / Copy_Micro_to_State
 * (Microphysics/Kessler/ERF_Kessler.cpp:11-185, ERF_Init_Kessler.cpp:64-99,
 * ERF_Update_Kessler.cpp:14-40), in place on cons. */
int erf_b200_kessler_advance(erf_b200_ctx* ctx, const erf_b200_fab* cons, double dt);

/* ----------------------------------------------------------------------------
 * Allocation-free Kessler step.  No counterpart in the reference: it is the
 * same computation as erf_b200_kessler_advance for callers that cannot
 * allocate device memory -- a host code whose device memory is all reserved
 * up front by its own pool (an AMReX arena, say) and which must not see a
 * second allocator beside it.  It takes no context.  Its scratch is one
 * library-owned device array of ERF_B200_NOALLOC_MAX_DOUBLES doubles
 * (16 MiB), present on every GPU that loads the library until the process
 * exits; requests with ncomp*nx*ny*nz > ERF_B200_NOALLOC_MAX_DOUBLES, or
 * with more than 65535 levels in the valid region or the view, are rejected
 * with ERF_B200_EINVAL, and configurations erf_b200_create rejects (Kessler
 * over terrain among them) with ERF_B200_ECONFIG.  The first call in a
 * device's context looks up the array's device address
 * (cudaGetSymbolAddress) with that device current, so make that first call
 * before any stream capture; after cudaDeviceReset the next call looks it up
 * again in the new context.  All calls share the one array: calls that
 * overlap on the GPU (different streams, or different host threads on the
 * same device) race, so serialise them.  If a CUDA error from earlier work
 * is pending on the calling thread, the call launches nothing, leaves that
 * error in place and returns ERF_B200_ECUDA.  Asynchronous on `stream`
 * (a cudaStream_t; NULL = legacy default stream).
 * ------------------------------------------------------------------------- */
#define ERF_B200_NOALLOC_MAX_DOUBLES 2097152
int erf_b200_kessler_advance_noalloc(const erf_b200_config* cfg,
                                     const erf_b200_fab* cons, double dt,
                                     void* stream);

/* ------------------------------------------------------------------------
 * Learned subgrid closure (no reference counterpart; ERF's closures are
 * ComputeTurbulentViscosity.cpp's Smagorinsky / Deardorff).  A 13-64-64-64-9
 * GELU network in BF16 on the tcgen05 tensor cores (FP32 accumulation) maps
 * the 9 resolved velocity-gradient components (du/dx du/dy du/dz dv/dx ...
 * dw/dz), the 3 potential-temperature gradient components and the filter
 * width to the 6 kinematic subgrid stresses (11 22 33 12 13 23) and the 3
 * subgrid heat fluxes (x y z).  Parameters are NPAR FP32 values in the padded
 * layout W1[64][16] W2[64][64] W3[64][64] W4[16][64] b1 b2 b3 b4[16].
 * Training and inference arrays are device pointers, row-major.
 * ------------------------------------------------------------------------ */
typedef struct erf_b200_mlp erf_b200_mlp;

int erf_b200_mlp_num_params(void);
int erf_b200_mlp_create(erf_b200_mlp** out, void* stream);
int erf_b200_mlp_destroy(erf_b200_mlp* m);
/* host_params: NPAR floats; resets the optimiser state. */
int erf_b200_mlp_set_params(erf_b200_mlp* m, const float* host_params);
int erf_b200_mlp_get_params(erf_b200_mlp* m, float* host_params);
/* Feature / target normalisation (host arrays: 13, 13, 9, 9) and the
 * training envelope of the raw features (13 + 13, may be NULL). */
int erf_b200_mlp_set_normalization(erf_b200_mlp* m, const float* in_mean, const float* in_std,
                                   const float* out_mean, const float* out_std,
                                   const float* in_lo, const float* in_hi);
/* Loss sum((y-t)^2)/(9n) and its gradient (NPAR floats to host_grad) for
 * normalised inputs xn[n][13] and targets tn[n][9]. */
int erf_b200_mlp_gradient(erf_b200_mlp* m, const float* xn, const float* tn, int n,
                          float* host_grad, float* host_loss);
/* iters Adam steps (lr) over consecutive minibatches of `batch` rows. */
int erf_b200_mlp_train(erf_b200_mlp* m, const float* xn, const float* tn, int n, int batch,
                       int iters, float lr, float* host_loss);
/* y[n][9] (raw units) from x[n][13] (raw units). */
int erf_b200_mlp_infer(erf_b200_mlp* m, const float* x, int n, float* y);

/* Name of the CUDA error behind the last ERF_B200_ECUDA / ERF_B200_ENOMEM
 * returned on this host thread. */
const char* erf_b200_last_cuda_error(void);

/* Failure-detection self-test of the current device: one kernel waits on an
 * mbarrier phase that can never complete, with the bounded poll the
 * tensor-core kernels use (at most `limit` polls).  *timed_out is 1 when the
 * bound ended the wait, as it must (the library's kernels then raise
 * ERF_B200_ETIMEOUT and return instead of hanging).  Synchronous. */
int erf_b200_selftest_bounded_wait(int limit, int* timed_out);

/* Write an AMReX plotfile (single level, one grid) of a host state, as
 * ERF::WritePlotFile does (Source/IO/ERF_Plotfile.cpp:186-1500): directory
 * `dir` gets Header, Level_0/Cell_H and Level_0/Cell_D_00000.  Arrays are in
 * the erf_b200_advance_host layout.  Variables: density, x/y/z_velocity
 * (cell-centred), temp, theta, KE (Deardorff only), scalar, pres_hse and
 * dens_hse (when rho0 and p0 are given: the base state as passed to
 * erf_b200_set_base_state), pressure, qv / qc / qrain (moist), z_phys and detJ
 * (when z_nd, the node heights given to erf_b200_set_terrain, is given with
 * use_terrain; the nodal Level_0/Nu_nd is written then too).  Host-only: no
 * context or device is needed.  Returns ERF_B200_EINVAL on a bad argument or
 * a failed file write. */
int erf_b200_write_plotfile(const erf_b200_config* cfg, const char* dir, const double* cons, const double* u,
                            const double* v, const double* w, const double* rho0, const double* p0,
                            const double* z_nd, double time, int step);

/* Checkpoint / restart in ERF's native checkpoint layout
 * (ERF::WriteCheckpointFile / ReadCheckpointFile, Source/IO/
 * ERF_Checkpoint.cpp:25-470), single level: Header (istep, dt, t_new, the
 * BoxArray), Level_0/Cell, XFace, YFace, ZFace, BaseState (r0, p0, pi0, th0,
 * 3 ghost cells), Z_Phys_nd (terrain) and MapFactor_m/_u/_v (all 1).  Arrays
 * are host arrays in the erf_b200_advance_host layout; the base state is laid
 * out as for erf_b200_set_base_state; z_nd as for erf_b200_set_terrain
 * (required with use_terrain, ignored otherwise).  Host-only.
 *
 * The reader accepts checkpoints with any number of grids and ghost widths
 * (the reference's own included) whose Header matches cfg: one level, ncomp
 * conserved components.  The base-state pointers may all be NULL (not read),
 * as may z_nd and the step / dt / time outputs.  Returns ERF_B200_EINVAL on a
 * missing or malformed file or a shape mismatch. */
int erf_b200_write_checkpoint(const erf_b200_config* cfg, const char* dir, const double* cons, const double* u,
                              const double* v, const double* w, const double* r0, const double* p0,
                              const double* pi0, const double* th0, const double* z_nd, int step, double dt,
                              double time);
int erf_b200_read_checkpoint(const erf_b200_config* cfg, const char* dir, double* cons, double* u, double* v,
                             double* w, double* r0, double* p0, double* pi0, double* th0, double* z_nd, int* step,
                             double* dt, double* time);

/* ------------------------------------------------------------------------
 * Resident state, autotuning and ensembles (no reference counterpart).
 * ------------------------------------------------------------------------ */
/* Load a state into the context; it stays on the device between calls. */
int erf_b200_load_state(erf_b200_ctx* ctx, const erf_b200_fab* cons, const erf_b200_fab* xvel,
                        const erf_b200_fab* yvel, const erf_b200_fab* zvel);
/* Copy the resident state out. */
int erf_b200_store_state(erf_b200_ctx* ctx, const erf_b200_fab* cons, const erf_b200_fab* xvel,
                         const erf_b200_fab* yvel, const erf_b200_fab* zvel);
/* Advance the resident state nsteps steps (one graph launch per step). */
int erf_b200_advance_resident(erf_b200_ctx* ctx, int nsteps);
/* Pick the context's launch shapes by timing candidates on the resident
 * state (which is left unchanged); best_ms receives the tuned step time. */
int erf_b200_autotune(erf_b200_ctx* ctx, int reps, double* best_ms);

typedef struct erf_b200_ensemble erf_b200_ensemble;
/* An ensemble of contexts holding resident states (any sizes, all at the
 * same state slot).  erf_b200_ensemble_advance runs nsteps steps of every
 * member in one graph launch: a device-side loop (a conditional WHILE graph
 * node) whose body holds two steps of every member's step graph, members
 * concurrently, and a one-thread kernel that counts the steps and polls the
 * host's abort word in mapped pinned memory; an odd last step runs in a
 * second launch behind the same check.  The members' state slots are
 * settled by erf_b200_ensemble_sync, which must come before any other call
 * on a member (they return ERF_B200_EBADSTATE until then). */
int erf_b200_ensemble_create(erf_b200_ensemble** out, erf_b200_ctx* const* members, int n, void* stream);
int erf_b200_ensemble_advance(erf_b200_ensemble* e, int nsteps);
/* Set (flag != 0) or clear the abort word.  The loop reads it between
 * steps: once set, no further step starts, every member keeps the state of
 * its last whole step, and sync returns ERF_B200_EABORTED.  Clearing waits
 * for the ensemble's stream and re-arms the loop. */
int erf_b200_ensemble_abort(erf_b200_ensemble* e, int flag);
/* Wait for the ensemble's work and settle the members' state slots;
 * ERF_B200_EABORTED if an abort stopped it. */
int erf_b200_ensemble_sync(erf_b200_ensemble* e);
/* Steps every member has run since the ensemble was made (as of the last
 * sync). */
int erf_b200_ensemble_steps(const erf_b200_ensemble* e, int* steps);
int erf_b200_ensemble_destroy(erf_b200_ensemble* e);

/* Attach a trained network to a context created with les_type ERF_LES_MLP
 * (the step graphs are built here; advancing before it returns
 * ERF_B200_EBADSTATE).  The network must outlive the context's use of it. */
int erf_b200_set_closure(erf_b200_ctx* ctx, const erf_b200_mlp* m);
/* Cells that fell back to Smagorinsky since the last call (reset on read). */
int erf_b200_closure_fallbacks(erf_b200_ctx* ctx, unsigned long long* count);
/* The 13 closure features of every cell (cell order i fastest) of a state
 * given as host arrays in the erf_b200_advance_host layout; features is a
 * host array of 13*nx*ny*nz floats. */
int erf_b200_closure_features_host(erf_b200_ctx* ctx, const double* cons, const double* u, const double* v,
                                   const double* w, float* features);

#ifdef __cplusplus
}
#endif

#endif /* ERF_B200_H */
