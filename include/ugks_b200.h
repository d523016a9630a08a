/*
 * ugks_b200.h -- C ABI of the B200 (sm_100a, FP64) UGKS2D kinetic hot path.
 *
 * The reference (Sherlmess/UGKS2D_high_order, Fortran 2008 + MPI) drives its hot path through
 * argument-less subroutines that act on module globals, called from Solve_UGKS
 * (src/mod_Solve.f90:84-186).  Each entry point below replaces one of them; the citation on each
 * declaration names the routine it stands in for.  Plain pointers and sizes only: a Fortran
 * `bind(C)` interface or ctypes can call every function.
 *
 * Host arrays use the reference's backing-store layout with the halo stripped:
 *   h, b : [ny][nx][nvel]  (Fortran cell_h_store(Nvel, 1:nx, 1:ny), velocity fastest)
 *   W    : [ny][nx][4]     (ctr%conVars packed)
 * The library owns the device mirrors for the context lifetime; state stays resident in HBM
 * between calls and crosses PCIe only in upload/download.
 *
 * Every function returns UGKS_OK (0) or a positive status.  Numerical failures detected on the
 * device are reported with the reference's own MPI_Abort codes (ugks_status_reference_code).
 * Nothing traps on the device; a failing call leaves the context usable.
 * One context is not thread-safe: all its work is serialised on one CUDA stream.
 */
#ifndef UGKS_B200_H
#define UGKS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UGKS_OK 0
#define UGKS_EINVAL 1        /* bad argument */
#define UGKS_ECUDA 2         /* CUDA runtime error */
#define UGKS_ENUMERIC 3      /* device-side numerical gate failed (see ugks_last_status) */
#define UGKS_ETIMEOUT 4      /* a bounded device-side wait expired */
#define UGKS_ENOMEM 5
#define UGKS_EUNSUPPORTED 6

#define UGKS_METHOD_EXPLICIT 0
#define UGKS_METHOD_IMPLICIT_STEADY 1
#define UGKS_METHOD_HIGH_ORDER_IMPLICIT 2   /* S2 evolution + the implicit PR(2)/LU-SGS update */
#define UGKS_METHOD_S2CN2 3                 /* explicit high-order step: S2 evolution + CN collision */

/* Subset of the reference's &config_para / &boundary_para that the hot path reads
 * (src/mod_ImportPara.f90:141-173, set_const_para :911-930). */
typedef struct ugks_params {
    int nx, ny;              /* Nx_all, Ny_all (one domain; the reference's NP_X x NP_Y blocking collapses) */
    int nvel;                /* Nu*Nv */
    double dx, dy;           /* uniform cell lengths of Mesh2d.dat */
    int ck;                  /* internal degrees of freedom */
    double pr;               /* Prandtl number (Shakhov) */
    double omega;            /* power-law viscosity exponent */
    double mu_ref;           /* CouetteMuRef */
    double cfl;              /* CFL */
    double wall_ux[2];       /* WallUx(3), WallUx(4): bottom and top wall speed */
    double wall_tnative[2];  /* wall temperature (native scale, Tw) bottom/top */
    double fixed_dt;         /* > 0: Time_global_fixed with this dt; <= 0: global CFL dt */
    int method;              /* UGKS_METHOD_* */
    /* ImplicitSteady controls (mod_SteadyImplicit.f90, mod_ImplicitMacro.f90, mod_ImplicitMicro.f90) */
    double ncfl;             /* Implicit_nCFL */
    int nslab;               /* NP_Y of the reference blocking: LU-SGS/PR2 seams are block-Jacobi per slab */
    int mass_rescale;        /* ClosedCouetteMassRescale */
    int macro_sweeps;        /* Implicit_MacroSweeps */
    double residual_tol;     /* Implicit_ResidualTol */
    double moment_tol;       /* Implicit_MomentTol */
    double min_alpha;        /* Implicit_MinAlpha */
    /* The research S2 wall variants (mod_ImportPara.f90:88-93, checked as :455-471 and :516-533 check
     * them); all zero is the delivered configuration, FluxWall_type = 1 (the multiscale wall).  The
     * kinetic wall on S2CN2 and HighOrderImplicit contexts, the other three on S2CN2 contexts;
     * ugks_ctx_create returns UGKS_EINVAL for a combination the reference rejects. */
    int s2_kinetic_wall;     /* FluxWall_type = 0: the free-streaming diffuse wall (s2w1_wall_node) */
    int s2_time_centered;    /* S2W1_time_centered = 1: W1T, the walls re-evaluated at a predicted
                                midpoint state (needs s2_kinetic_wall) */
    int s2_face_time;        /* S2W1D_face_time_consistent = 1: W1D, the interior faces' leading flux
                                moved to that midpoint too (needs s2_time_centered) */
    int s2_shared_predictor; /* S2W2R_shared_predictor = 1: W2R, every face corrected at a shared
                                predictor (multiscale wall, ck = 1, Pr = 1) */
} ugks_params;

typedef struct ugks_ctx ugks_ctx;

/* Create a context on CUDA device `device` with the velocity table (u, v, w of nvel entries,
 * k = i + (j-1)*Nu as in InitVelocityFromStructuredFile, src/mod_InitializeFlow.f90:480-509). */
int ugks_ctx_create(const ugks_params* params, const double* u, const double* v, const double* w, int device,
                    ugks_ctx** out);
int ugks_ctx_destroy(ugks_ctx* ctx);

/* Copy state host <-> device (the only PCIe crossings). */
int ugks_upload_state(ugks_ctx* ctx, const double* h, const double* b, const double* W);
int ugks_download_state(ugks_ctx* ctx, double* h, double* b, double* W);
/* The same with h and b in the reference's own backing stores, halo included: cell_h_store(Nvel,
 * 1-LAP:nx+LAP, 1-LAP:ny+LAP) and cell_b_store (src/mod_InitializeFlow.f90:109-110), that is host arrays
 * [ny + 2 lap][nx + 2 lap][nvel] with the interior at (lap, lap); W as above (ctr%conVars packed).  Only
 * the interior is read or written, so the Fortran driver passes its stores as they are (lap = LAP = 2,
 * src/mod_Globaldata.f90:95) and keeps filling its halo itself. */
int ugks_upload_state_halo(ugks_ctx* ctx, const double* h, const double* b, const double* W, int lap);
int ugks_download_state_halo(ugks_ctx* ctx, double* h, double* b, double* W, int lap);

/* InitFlow_Freestream + cold-start EnforceAcceptedMomentCompatibility
 * (src/mod_InitializeFlow.f90:826-856; src/mod_SteadyImplicit.f90:28-42). */
int ugks_init_freestream(ugks_ctx* ctx, double rho, double U, double V, double tnative);

/* TimeStep (src/mod_Solve.f90:373-421): computes dt_global on the device; *dt_out optional. */
int ugks_timestep(ugks_ctx* ctx, double* dt_out);

/* Interpolation() + Evolution() (src/mod_Interpolation.f90:26, src/mod_Evolution.f90:35-41), which
 * dispatches on the method as the reference does: Explicit / ImplicitSteady run EvolutionNative, the
 * Van-Leer slopes fused into the UGKS face fluxes (interior faces and W2B moving walls); S2CN2 and
 * HighOrderImplicit run S2NativeEvolution (src/mod_S2NativeAdapter.f90:469-490), as ugks_evolution_s2
 * with the reference's target rule: HighOrderImplicit rebuilds the volume targets every time, S2CN2
 * keeps those of the accepted state (UGKS_EINVAL before ugks_s2cn2_init or ugks_init_freestream). */
int ugks_evolution(ugks_ctx* ctx);

/* S2NativeEvolution (src/mod_S2NativeAdapter.f90:469-599 -> CartesianEvolution
 * src/mod_S2CartesianMPI.f90:182-234 -> compute_flux src/mod_S2D1.f90:632-959) on an S2CN2 or
 * HighOrderImplicit context: the WENO-AO face and wall fluxes of the current state into the face arrays
 * (ugks_copy_array "fxh", "fyw", ...) and the wall aerodynamics.  rebuild_targets nonzero rebuilds the
 * volume targets of the current W first (build_targets, src/mod_S2D1.f90:1246-1300; always on
 * HighOrderImplicit, whose targets the reference invalidates at every evaluation, :479); zero keeps the
 * S2CN2 targets of the accepted state.  On S2CN2 this starts a per-operator step: ugks_timestep,
 * ugks_evolution (or this), ugks_compute_residual, ugks_apply_explicit_update advance the state exactly
 * as one step of ugks_s2cn2_steps.  UGKS_EUNSUPPORTED on a second-order context. */
int ugks_evolution_s2(ugks_ctx* ctx, int rebuild_targets);

/* ComputeResidual() (src/mod_Residual.f90:17-132) with the unified streaming-moment projection;
 * with_collision also forms the physical equilibrium/collision used by the implicit paths.
 * S2CN2 (after the evolution of the step): the residual, the stream state, the S2 physical collision
 * and its moment gate (S2NativePhysicalCollision, src/mod_S2NativeAdapter.f90:735-759) and the
 * Crank-Nicolson right-hand side of advance_step (src/mod_S2D1.f90:1376-1390); UGKS_EINVAL out of that
 * order.  HighOrderImplicit: UGKS_EUNSUPPORTED, its residual runs inside ugks_implicit_steps. */
int ugks_compute_residual(ugks_ctx* ctx, int with_collision);

/* ApplyExplicitUpdate() (src/mod_TimeIntegrator.f90:16-134): macro update, CN Shakhov
 * collision with variable tau, residual norms; res_out[4] optional = the reference `res`.
 * S2CN2 (after ugks_compute_residual): S2NativeApplyUpdate (src/mod_S2NativeAdapter.f90:867-940), the
 * targets of the stream state, the CN collision, the cnres / mmerr / conservation gates and the
 * acceptance; a rejected step keeps the accepted state and returns UGKS_ENUMERIC (reference code 203);
 * res_out is not written (ugks_s2cn2_report gives the step's report).  HighOrderImplicit:
 * UGKS_EUNSUPPORTED (ugks_implicit_steps). */
int ugks_apply_explicit_update(ugks_ctx* ctx, double* res_out);

/* nsteps full Explicit steps (TimeStep, Interpolation, Evolution, ComputeResidual,
 * ApplyExplicitUpdate; src/mod_Solve.f90:84-186) fused into two kernels per step and replayed
 * from a CUDA graph.  dt_out / res_out (optional) report the last step. */
int ugks_step_explicit(ugks_ctx* ctx, int nsteps, double* dt_out, double* res_out);

/* The Explicit step of ugks_step_explicit for callers that cannot allocate device memory.  No
 * counterpart in the reference (its Fortran solver owns module globals); added for host codes
 * that manage every byte of device memory themselves (their own pre-sized pool, or a hard memory
 * cap) and for latency-critical loops where cudaMalloc/cudaFree would synchronise the device.
 * It creates no context and allocates nothing: u, v, w (nvel each), h, b ([ny][nx][nvel]) and W
 * ([ny][nx][4]) are the caller's DEVICE arrays, updated in place by nsteps steps on `stream`
 * (a cudaStream_t; NULL = legacy default stream); dt_out / res_out are optional host outputs as in
 * ugks_step_explicit.  Working arrays live in one fixed 36 MiB __device__ array inside the library:
 * a call whose working set (about 8*nx*ny*nvel + 2*nx*nvel + 22*nx*ny doubles; 33.8 MB for
 * 8x64 cells x 32x32 velocities) does not fit returns UGKS_EINVAL before any GPU work.  The array is
 * loaded on a device, and its 36 MiB taken there, at the first call on that device (CUDA loads modules
 * lazily), so callers that size their own device pool or run under a memory cap make one call per
 * device before they do; the array then stays until the process exits.  Each call synchronises
 * `stream` twice (it reads the velocity table's extent, which sets dt, and then the status), so it
 * cannot be captured in a CUDA graph.  All calls on one device share the array: calls that overlap on
 * that GPU (other streams, other host threads) race and must be serialised by the caller; host threads
 * driving different devices share nothing. */
int ugks_step_explicit_noalloc(const ugks_params* params, const double* u, const double* v, const double* w,
                               double* h, double* b, double* W, int nsteps, void* stream, double* dt_out,
                               double* res_out);

/* ImplicitSteady / HighOrderImplicit with the closed-Couette mass rescale (methods
 * UGKS_METHOD_IMPLICIT_STEADY, UGKS_METHOD_HIGH_ORDER_IMPLICIT; the latter evaluates the S2
 * high-order residual, src/mod_S2NativeAdapter.f90:469-759, and adds the high-order collision
 * correction to the micro right-hand side, src/mod_ImplicitMicro.f90:66-79,467-470).
 * ugks_implicit_init: InitializeClosedMass (src/mod_ClosedCouetteMass.f90:212-241) -- the persistent
 * M0 from the current state and a fresh residual-reference epoch; call after the state is set.
 * ugks_implicit_steps: up to max_steps pseudo-steps of Solve_UGKS (src/mod_Solve.f90:84-293), each
 * TimeStep, Interpolation + Evolution, ComputeResidual, ApplySteadyImplicitUpdate (PR(2) + one
 * LU-SGS sweep pair with the reference's nslab block-Jacobi seams, src/mod_SteadyImplicit.f90:379-462),
 * RescaleClosedMass and the accepted-state re-evaluation with the five-state gate
 * (src/mod_R5Observe.f90:287-320); stops early when the gate has passed 5 states in a row.
 * On the second-order path whole batches of 8 steps run on the device under one graph launch (a
 * conditional WHILE node bounded by max_steps / 8 batches), and the host waits once per call.
 * report[80] (optional) = the last accepted state's sparse_residual.csv row: [0] gate pass,
 * [1] moment, [2] M_W, [3] M_h, [4..11] R1..R8, [12..33] science_1..22, [34..49] flux_1..16,
 * [50..51] reference_h/b, [52] c_minus_1, [53] alpha, [54] macro alpha, [55] dt, [56] streak,
 * [57..78] science of the pre-update evaluation. */
int ugks_implicit_init(ugks_ctx* ctx);
/* Resume from a restart (InitFlow_Restart + ReadMassRestart, src/mod_ClosedCouetteMass.f90:352-393, and
 * the residual-reference inheritance of src/mod_R5Observe.f90:176-186): like ugks_implicit_init but
 * with the persistent M0 read from closed_mass_rank*.bin instead of the current mass, and, when
 * have_reference is nonzero, the residual references (reference_h, reference_b) of
 * residual_reference.in instead of those of the first evaluation.  UGKS_EINVAL if M0 is not finite
 * and positive or an inherited reference is not finite.  Call after the state is uploaded. */
int ugks_implicit_restore(ugks_ctx* ctx, double m0, double reference_h, double reference_b, int have_reference);
int ugks_implicit_steps(ugks_ctx* ctx, int max_steps, int* steps_done, int* converged, double* report);
/* state[16]: M0, reference_h, reference_b, reference set, mass_scale, streak, stop, steps, alpha,
 * macro alpha, moment error, converged (see ugks_implicit.cuh); report[80] as above. */
int ugks_implicit_state(ugks_ctx* ctx, double* state, double* report);

/* S2CN2, the explicit high-order method (TimeIntegration_method='S2CN2', consistency/high_explicit).
 * ugks_s2cn2_init: the ledger of S2NativeInitializeState (src/mod_S2NativeAdapter.f90:323-349;
 * total0 = sum of W over the cells, empty wall balance) and the volume targets of the current state
 * (build_targets, src/mod_S2D1.f90:1246-1300).  ugks_init_freestream does this itself after the S2
 * cold start; call it after ugks_upload_state.
 * ugks_s2cn2_steps: up to nsteps steps of Solve_UGKS (src/mod_Solve.f90:84-165), each TimeStep,
 * S2NativeEvolution with the targets kept between steps (src/mod_S2NativeAdapter.f90:469-490),
 * ComputeResidual, and S2NativeApplyUpdate (:867-940) whose advance_step
 * (src/mod_S2D1.f90:1302-1435) rebuilds the targets of the stream state and applies the
 * Crank-Nicolson collision, gated by cnres / mmerr <= 2e-12 and the global conservation drift
 * against the wall ledger.  A rejected step (the reference aborts with 203) ends the sequence: the
 * state stays the last accepted one, *steps_done counts the accepted steps and the call returns
 * UGKS_ENUMERIC with ugks_status_reference_code 203.  report[24] (optional) = the last step:
 * [0] dt, [1] cnres, [2] mmerr, [3] max 2 beta, [4] transport CFL, [5..8] min/max of h and b,
 * [9] drift, [10..13] bottom and [14..17] top wall macro flux / dy, [18..21] wall balance,
 * [22] accepted, [23] accepted steps of this call. */
int ugks_s2cn2_init(ugks_ctx* ctx);
int ugks_s2cn2_steps(ugks_ctx* ctx, int nsteps, int* steps_done, double* report);
/* The reference's test hooks for a rejected S2CN2 step (S2D3_TEST_GLOBAL_REJECT,
 * src/mod_S2NativeAdapter.f90:433-435,926; S2E3_TEST_REJECT_STEP, src/mod_S2CartesianMPI.f90:254-264):
 * the conservation drift of step `step` (1-based) of the next ugks_s2cn2_steps call is forced above
 * the gate, so that step is rejected.  One-shot; 0 clears it.  Host-side, numerical only. */
int ugks_s2cn2_test_reject(ugks_ctx* ctx, int step);
/* report[24] of the last S2CN2 step (layout of ugks_s2cn2_steps), whether it ran through
 * ugks_s2cn2_steps or the per-operator calls. */
int ugks_s2cn2_report(ugks_ctx* ctx, double* report);

/* Gradients of the S2CN2 wall outputs by the discrete adjoint of the step (no counterpart routine in the
 * reference, which has no derivatives; the gradient of its S2CN2 trajectory, mod_S2D1.f90:1302-1435 with
 * compute_flux :632-959 and the walls of mod_S2MultiscaleWall.f90:45-184).  The outputs are the wall
 * aerodynamics of the last step's evaluation averaged over each wall (PublishWallDiagnostics,
 * src/mod_S2NativeAdapter.f90:1075-1097): out[4] = bottom shear (pnt), bottom heat flux (qn), top shear,
 * top heat flux.  The parameters are grad[5] = d/d(mu_ref, wall_ux[0], wall_ux[1], wall_tnative[0],
 * wall_tnative[1]) of the seeded output combination sum_i seed[i] out[i].
 * ugks_s2cn2_forward_checkpointed: nsteps accepted S2CN2 steps from the current state (as
 *   ugks_s2cn2_steps), storing the state and the conservation ledger every `every` steps in device memory
 *   the context keeps (about (nsteps / every) x 16 doubles per cell-velocity); out[4] optional.  A rejected step returns UGKS_ENUMERIC (reference code 203) and leaves no trajectory.
 * ugks_s2cn2_backward: the reverse sweep over that trajectory: each segment's states are recomputed from
 *   its checkpoint, then every step is re-run for its evaluation scratch and transposed.  Its work memory
 *   (`every` states with their targets, about 64 doubles per cell-velocity more) is reserved by the first
 *   backward and kept with the context.  grad[5]
 *   optional; gh0, gb0 [ny][nx][nvel] and gW0 [ny][nx][4] (optional) receive the cotangent of the initial
 *   state (its targets' dependence on W included).  The adjoint holds the time step fixed: it returns
 *   UGKS_ENUMERIC with ugks_last_status bit 0x400 if a state's dt is set by |U| + c instead of the
 *   velocity table's extent.  The context's state (the last forward state) is not changed.
 * ugks_s2cn2_step_vjp: the vector-Jacobian product of one step at the current state (not advanced): the
 *   cotangents gh, gb [ny][nx][nvel], gW [ny][nx][4] of the step's outputs (NULL = zero) and seed[4] of
 *   the step's wall outputs (NULL = zero) give the input cotangents gh_in, gb_in, gW_in (optional) and
 *   grad[5] (optional). */
int ugks_s2cn2_forward_checkpointed(ugks_ctx* ctx, int nsteps, int every, double* out);
int ugks_s2cn2_backward(ugks_ctx* ctx, const double* seed, double* grad, double* gh0, double* gb0, double* gW0);
int ugks_s2cn2_step_vjp(ugks_ctx* ctx, const double* gh, const double* gb, const double* gW, const double* seed,
                        double* gh_in, double* gb_in, double* gW_in, double* grad);

/* Batched S2CN2: many independent Couette instances of uneven grid and velocity-set sizes advanced
 * together (a parameter sweep of the Couette case run as one job; no counterpart routine in the
 * reference, whose runs are one case per job).  Each instance is described by ugks_params (method UGKS_METHOD_S2CN2) and its velocity
 * table.  Instances own their persistent state (two state sets, two target sets, ledger: about 16
 * doubles per cell-velocity); the per-step scratch lives in up to max_streams slots sized for the
 * largest instance, instances being assigned to slots largest-first.  One CUDA graph launch advances
 * every instance by two steps, the slots running concurrently.
 * ugks_batch_init_freestream: InitFlow_Freestream + the S2 cold start + the ledger of every instance.
 * ugks_batch_run: nsteps steps of every instance; steps_done[n] / status[n] (optional) per instance;
 *   an instance whose step is rejected stops at its last accepted state (status bit of reference
 *   code 203 or the gate's own code), the others continue; returns UGKS_ENUMERIC if any stopped.
 * ugks_batch_tune: times `steps` steps at 1, 2, 4, ... max_streams slots on the live batch (the
 *   instances advance) and keeps the fastest; *chosen and *ms_per_step report it.
 * ugks_batch_upload / download / report / wall_aero: per-instance state, last-step report[24] (as
 *   ugks_s2cn2_steps) and wall (pnn, pnt, qn). */
typedef struct ugks_instance_desc {
    ugks_params params;
    const double *u, *v, *w;   /* host velocity table, params.nvel entries */
} ugks_instance_desc;
typedef struct ugks_batch ugks_batch;
int ugks_batch_create(int n, const ugks_instance_desc* desc, int device, int max_streams, ugks_batch** out);
int ugks_batch_destroy(ugks_batch* batch);
int ugks_batch_init_freestream(ugks_batch* batch, double rho, double U, double V, double tnative);
int ugks_batch_run(ugks_batch* batch, int nsteps, int* steps_done, unsigned* status);
int ugks_batch_tune(ugks_batch* batch, int steps, int* chosen, double* ms_per_step);
int ugks_batch_set_streams(ugks_batch* batch, int streams);
int ugks_batch_upload(ugks_batch* batch, int i, const double* h, const double* b, const double* W);
int ugks_batch_download(ugks_batch* batch, int i, double* h, double* b, double* W);
int ugks_batch_report(ugks_batch* batch, int i, double* report);
int ugks_batch_wall_aero(ugks_batch* batch, int i, double* out);
long long ugks_batch_launch_count(const ugks_batch* batch);
void* ugks_batch_stream(ugks_batch* batch);

/* Steady output fields of every cell, as Output writes them (src/mod_Output.f90:102-116):
 * out[nc][10] = r, u, v, T (= 1/lambda), p (= r T / 2), sxx, sxy, syy (Get_Stress_Vec,
 * src/mod_Tools.f90:409-432), qx, qy (GetHeatFlux_Vec, src/mod_Tools.f90:355-373). */
int ugks_macro_fields(ugks_ctx* ctx, double* out);

/* Wall Aerodynamics of the last Evolution: out[2][nx][3] = (pnn, pnt, qn) per bottom/top wall face.
 * Second-order methods: the local frame of W2BMultiscaleFluxBoundary (src/mod_Evolution.f90:2402-2409);
 * high-order methods: the native frame n = +y, t = -x of PublishWallDiagnostics
 * (src/mod_S2NativeAdapter.f90:1075-1097), qn net of the moving wall's work. */
int ugks_wall_aero(ugks_ctx* ctx, double* out);

/* Copy a named device work array to the host (diagnostics / parity tests).  Names:
 * "res_w" [nc][4], "res_h", "res_b" [nc][nvel], "fxh", "fxb" [ny][nx][nvel], "fyh", "fyb"
 * [ny+1][nx][nvel], "fxw" [ny][nx][4], "fyw" [ny+1][nx][4], "pcol_h", "pcol_b", "peq_h",
 * "peq_b" [nc][nvel], "dt" [1]. n = number of doubles the caller's buffer holds. */
int ugks_copy_array(ugks_ctx* ctx, const char* name, double* host, size_t n);

/* Device status word of the last synchronising call and the reference abort code it maps to
 * (101-106 GetPrimary/GetTau, 444/446 projections, 13-16 non-finite flux, 4/17 state). */
unsigned ugks_last_status(const ugks_ctx* ctx);
int ugks_status_reference_code(unsigned status);
const char* ugks_error_string(int code);

/* The context's CUDA stream (cudaStream_t) for event timing by the caller, and a blocking sync. */
void* ugks_stream(ugks_ctx* ctx);
int ugks_synchronize(ugks_ctx* ctx);

/* Kernel-level timing: when enabled, ugks_step_explicit records CUDA events around each kernel
 * launch (graph replay off) and accumulates per-kernel milliseconds and launch counts.
 * names: "slopes", "faces", "walls", "cells".  ugks_implicit_steps times its pseudo-step stages
 * (names: the stage names of the implicit report, "timestep" ... "post_residual"): enable = 1 runs the
 * steps one by one with an event after every stage; enable = 2 runs them in batch graphs of 8 with the
 * stage events captured into the graph, timing each batch's last pseudo-step as the graphs run it
 * (the launches counted are then the sampled pseudo-steps). */
int ugks_profile_enable(ugks_ctx* ctx, int enable);
int ugks_profile_read(ugks_ctx* ctx, const char* kernel, double* total_ms, long long* launches);

/* Number of kernels this library launched on the context since creation (evidence counter). */
long long ugks_launch_count(const ugks_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif
