/*
 * ugks_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-threaded CPU restatement of the reference UGKS2D Fortran hot path
 * (Sherlmess/UGKS2D_high_order, Fortran sources under src/), used solely as the parity checker for the CUDA
 * library and as the timed CPU baseline in bench.py.  Nothing in the product library links,
 * calls or falls back to this code.  Each function cites the Fortran routine it restates.
 *
 * Parity of this restatement is pinned against the reference's own printed outputs
 * (tests/golden/reference_golden.json, generated by tests/golden/make_fixtures.py):
 *   - the 2-step low_explicit `dtPhysical` and `res:` line,
 *   - the 2-step low_implicit sparse_residual.csv rows (8-slab emulation),
 *   - the static-equilibrium residual/update maxima of checks/VERIFICATION.json.
 *
 * Layout: single domain, cells c = j*nx + i (0-based, i fastest), velocity k fastest:
 *   h[c*nvel + k], b[c*nvel + k], W[c*4 + m].  x is periodic; y has diffuse moving walls.
 */
#ifndef UGKS_ORACLE_H
#define UGKS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nx, ny, nvel;
    double dx, dy;            /* cell lengths: Fortran ctr%length(1), ctr%length(2) */
    int ck;                   /* internal degrees of freedom (integer in the reference) */
    double pr, omega, mu_ref, gamma, cfl;
    double wall_ux[2];        /* WallUx(3:4): bottom (y=0), top (y=H) */
    double wall_tnative[2];   /* wall T_native (Tw); lambda_w = 1/Tw */
    double ncfl;              /* Implicit_nCFL (pseudo-time CFL) */
    int nslab;                /* number of 1-D slabs in y the reference's MPI blocking used (NP_Y) */
    int mass_rescale;         /* ClosedCouetteMassRescale */
    int macro_sweeps;         /* Implicit_MacroSweeps */
    double residual_tol, moment_tol, min_alpha;
    int high_order;           /* 1: HighOrderImplicit (S2 evolution, S2 physical collision, HO micro RHS) */
    /* the research S2CN2 wall variants (mod_ImportPara.f90:88-93, checks :455-471, :516-533); all zero is
     * the delivered configuration (FluxWall_type = 1, the multiscale wall) */
    int s2_kinetic_wall;      /* FluxWall_type = 0: the free-streaming diffuse wall s2w1_wall_node */
    int s2_time_centered;     /* S2W1_time_centered = 1: W1T, walls re-evaluated at a predicted midpoint */
    int s2_face_time;         /* S2W1D_face_time_consistent = 1: W1D, interior faces corrected there too */
    int s2_shared_predictor;  /* S2W2R_shared_predictor = 1: W2R, every face corrected at a shared predictor */
} uo_params;

typedef struct uo_ctx uo_ctx;

uo_ctx* uo_create(const uo_params* p, const double* u, const double* v, const double* w);
void    uo_destroy(uo_ctx* c);

/* state access: copy in/out of h, b (ncell*nvel) and W (ncell*4) */
void uo_set_state(uo_ctx* c, const double* h, const double* b, const double* W);
void uo_get_state(const uo_ctx* c, double* h, double* b, double* W);

/* InitFlow_Freestream + EnforceAcceptedMomentCompatibility (mod_InitializeFlow.f90:826-856,
 * mod_ImplicitMicro.f90 EnforceAcceptedMomentCompatibility, via InitializeSteadyImplicit). */
int uo_init_freestream(uo_ctx* c, double rho, double U, double V, double tnative);

/* TimeStep, Time_global_varying (mod_Solve.f90:373-421).  Returns dt_global. */
double uo_timestep(uo_ctx* c);

/* One full Explicit step: TimeStep, Interpolation, EvolutionNative, ComputeResidual,
 * ApplyExplicitUpdate (mod_Solve.f90:84-186).  res_out[4] = the `res` vector; returns 0 or a
 * reference abort code. */
int uo_explicit_step(uo_ctx* c, double* dt_out, double* res_out);

/* Pieces of the step, for piecewise parity checks. */
void uo_interpolation(uo_ctx* c);                 /* mod_Interpolation.f90:26-90 */
int  uo_evolution(uo_ctx* c, double dt);          /* mod_Evolution.f90:46-177 (Couette subset) */
int  uo_compute_residual(uo_ctx* c, double dt, int with_collision); /* mod_Residual.f90:17-132 */
int  uo_apply_explicit_update(uo_ctx* c, double dt, double* res_out); /* mod_TimeIntegrator.f90:16-134 */

/* Read-only views of the work arrays (valid until the next call). */
const double* uo_res_macro(const uo_ctx* c);     /* res_macro_flux_store  [ncell][4] */
const double* uo_res_h(const uo_ctx* c);         /* res_h_flux_store      [ncell][nvel] */
const double* uo_res_b(const uo_ctx* c);
const double* uo_wall_aero(const uo_ctx* c);     /* [2][nx][3] local-frame pnn, pnt, qn */
const double* uo_face_x_h(const uo_ctx* c);      /* x-face micro flux [ny][nx][nvel] (face i between i-1,i) */
const double* uo_face_y_h(const uo_ctx* c);      /* y-face micro flux [ny+1][nx][nvel] */
const double* uo_face_x_w(const uo_ctx* c);      /* [ny][nx][4] */
const double* uo_face_y_w(const uo_ctx* c);      /* [ny+1][nx][4] */
const double* uo_phys_eq_h(const uo_ctx* c);     /* physical_equilibrium_h [ncell][nvel] */
const double* uo_phys_col_h(const uo_ctx* c);    /* physical_collision_h */
const double* uo_phys_col_b(const uo_ctx* c);

/* Standalone kinetic-library entry points (mod_Tools.f90, mod_ImplicitCommon.f90). */
int uo_project_moments(int n, double* h, double* b, const double target[4], const double* u,
                       const double* v, const double* wl, const double* ref_h, const double* ref_b);
int uo_solve_dense4(const double m[16], const double rhs[4], double sol[4]);

/* ImplicitSteady pseudo-step (mod_SteadyImplicit.f90:379-462) with the reference's nslab
 * block-Jacobi seams.  out[] receives the diagnostics listed in ugks_oracle.c. */
int uo_implicit_step(uo_ctx* c, double* out, int nout);
int uo_implicit_init(uo_ctx* c);   /* persistent M0 of the cold start (InitializeClosedMass) */

/* High-order S2 path (ugks_oracle_s2.c): the S2 Evolution of HighOrderImplicit (targets, WENO-AO
 * reconstruction, Gauss-node UGKS fluxes, multiscale wall) publishing into the face arrays; the S2
 * residual/rates/physical collision; the S2 cold start (h, b := discrete closure Maxwellian of W). */
int uo_s2_evolution(uo_ctx* c, double dt);
int uo_s2_compute_residual(uo_ctx* c, double dt, int rates_only);
int uo_s2_init_state(uo_ctx* c);

/* S2CN2, the explicit high-order step (S2NativeEvolution + ComputeResidual + S2NativeApplyUpdate /
 * advance_step): uo_s2cn2_init sets the conservation ledger of the current state; each
 * uo_s2cn2_step advances one step or rejects it (state untouched).  out[UO_CN_OUT] is listed at
 * uo_s2cn2_step in ugks_oracle_s2.c. */
#define UO_CN_OUT 22
int uo_s2cn2_init(uo_ctx* c);
int uo_s2cn2_step(uo_ctx* c, double* out, int nout);

/* The reference's tangent routines of the high-order path, restated (ugks_oracle_reftan.c): return 1
 * when every output is finite.  n velocities u, v with weights wt; w the conserved state. */
int uo_ref_maxwellian_direction(const double w[4], const double dw[4], int ck, int n, const double* u, const double* v,
                                double* mh, double* mb, double* dmh, double* dmb);
int uo_ref_dq_direction(const double w[4], const double dw[4], const double m[4], const double dm[4], int ck, int n,
                        const double* u, const double* v, const double* wt, double* ch, double* cb, double* dch,
                        double* dcb);
int uo_ref_projector_direction(const double w[4], const double dw[4], const double* zh, const double* zb,
                               const double* dzh, const double* dzb, int ck, int n, const double* u, const double* v,
                               const double* wt, double* ph, double* pb, double* dph, double* dpb);
int uo_ref_weno_direction(const double q[5], const double dq[5], double xi, double* val, double* dval,
                          int* differentiable);

/* Worker threads used over faces and cells (0 = all host cores); returns the count in use.
 * Results do not depend on the thread count: faces and cells are independent and every sum over
 * cells is taken afterwards in cell order. */
int uo_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
