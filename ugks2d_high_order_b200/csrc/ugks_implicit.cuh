// ugks_implicit.cuh -- device state of the ImplicitSteady pseudo-step (second order).
#pragma once
#include "ugks_lo.cuh"
#include "ugks_s2.cuh"

namespace ugks {

// Scalars kept on the device across pseudo-steps (index into ImBuffers::state).
enum : int {
    IS_M0 = 0,          // persistent closed-mass target (InitializeClosedMass)
    IS_REF_H = 1,       // first-evaluation micro references (UpdateImplicitResidualDiagnostics)
    IS_REF_B = 2,
    IS_REF_INIT = 3,
    IS_MASS_SCALE = 4,  // M0 / mass of the proposed state
    IS_STREAK = 5,      // consecutive accepted states that passed the five-state gate
    IS_STOP = 6,        // 1: converged (streak reached 5) or a gate failed; kernels return at entry
    IS_STEPS = 7,       // accepted pseudo-steps so far
    IS_ALPHA = 8,       // micro alpha of the last step
    IS_MALPHA = 9,      // macro alpha of the last step
    IS_MOMENT = 10,     // implicit_moment_error of the last update
    IS_CONVERGED = 11,  // 1 once the streak reached 5
    IS_EVAL_VALID = 12, // 1: slopes, fluxes and steady rates still hold the evaluation of the current
    IS_EVAL_DT = 13,    //    state at dt = state[IS_EVAL_DT] (written by the accepted-state evaluation)
    IS_PRESCI = 16,     // [22] science_1..22 of that evaluation before the mass-rescale override
    IS_COUNT = 40
};
constexpr int kStatePublic = 16;   // leading state slots copied out by ugks_implicit_state

// Layout of the per-step report (the accepted state's sparse_residual.csv row):
// [0] gate pass, [1] moment, [2] M_W, [3] M_h, [4..11] R1..R8, [12..33] science_1..22,
// [34..49] flux_1..16, [50] reference_h, [51] reference_b, [52] c_minus_1, [53] alpha,
// [54] macro alpha, [55] dt, [56] streak, [57..78] science of the pre-update evaluation.
constexpr int kReport = 80;
constexpr int kImCell = 20;   // per-cell diagnostic terms
constexpr int kMaxSlabCells = 384;   // rows x nx of one slab held in shared memory by the sweep kernels

// Stages of one pseudo-step, in launch order, for the per-stage event timing of profile runs.
constexpr int kImStages = 12;
constexpr const char* kImStageNames[kImStages] = {
    "timestep", "pre_evaluation", "pr2_sweep", "equilibrium", "lusgs_forward", "wall_closure",
    "lusgs_backward", "micro_alpha", "apply", "rescale", "post_fluxes", "post_residual"};

// Streams and events of the pre-update evaluation's conditional graph body (graph capture only).
struct ImCapture {
    cudaStream_t s, s2;
    cudaEvent_t fork, join;
};

struct ImParams {
    int nslab;              // ranks of the reference's 1 x NP_Y blocking (rows per slab = ny / nslab)
    int mass_rescale;
    int macro_sweeps;
    int high_order;         // 1: HighOrderImplicit (S2 evolution, S2 physical collision, HO micro RHS)
    double ncfl, residual_tol, moment_tol, min_alpha;
    double wall_ux[2];
};

struct ImBuffers {
    double* stream_h;       // [nc][nvel] projected streaming rate (stream_h / stream_b)
    double* stream_b;
    double* rate_w;         // [nc][4]
    double* dwA;            // [nc][4] PR(2) corrections, two buffers (sweep input / output)
    double* dwB;
    double* pr_gamma;       // [nc][4] face spectral radius (ImplicitSpectralRadius)
    double* pr_foi;         // [nc][4 faces][4] Euler normal flux of the cell state
    double* pr_foj;         // [nc][4 faces][4] Euler normal flux of the neighbour (or Zhu ghost) state
    double* wt;             // [nc][4] w_tilde
    double* tau_t;          // [nc] tau_tilde
    double* rhs_h;          // [nc][nvel] stream + (G_predicted - h) / tau_tilde: the velocity-local part of
    double* rhs_b;          //            RelaxMicroPoint's right-hand side, shared by both LU-SGS stages
    double* dFh;            // [nc][nvel] forward-stage corrections
    double* dFb;
    double* dBh;            // [nc][nvel] backward-stage (final) corrections
    double* dBb;
    double* wall_hu;        // [2][nvel] unit-density wall Maxwellian h, b in each wall's frame
    double* wall_bu;
    double* wall_drho;      // [2][nx] frozen wall closure density correction of each wall cell
    double* cell;           // [nc][kImCell] per-cell terms for the global reductions
    double* state;          // [IS_COUNT]
    double* report;         // [kReport]
    S2Buffers s2;           // high-order volume targets and reconstruction cache (HighOrderImplicit)
    unsigned* mask;         // [2] admissible macro / micro alpha bitmasks (bit m: alpha = 2^-m)
    unsigned* counter;      // [1] last-CTA counter of the implicit kernels
    unsigned* stopw;        // [1] nonzero once the stop flag is set: the evaluation kernels of the step
                            // sequence see it through LoBuffers::halt and return at entry
    unsigned* prbar;        // [2] grid barrier between the PR(2) sweeps of one launch: arrivals, generation
};

}  // namespace ugks
