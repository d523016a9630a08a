// ugks_lo.cuh -- device-side state of one Couette domain and the second-order (Van-Leer UGKS)
// kernels' parameter blocks.
#pragma once
#include <cmath>

#include "../../include/ugks_b200.h"
#include "ugks_device.cuh"

namespace ugks {

constexpr int kMaxVel = 5 * 512;  // largest velocity set one CTA row covers (5 velocities x 512 threads)
constexpr int kRedSlots = 40;    // max values reduced together in one block_reduce
constexpr int kNDiag = 13;       // per-cell explicit residual-norm contributions

struct LoParams {
    int nx, ny, nvel, ck;
    double dx, dy, area, gm1, pr, omega, mu_ref, cfl, umax, vmax;
    double wall_ux[2];       // bottom, top wall speed (WallUx(3:4))
    double wall_lam[2];      // 1/Tw per wall
    double fixed_dt;         // > 0: Time_global_fixed
    double inv_dx, inv_dy;   // 1/dx, 1/dy for the slope stencils
    double inv_area;         // 1/area when area is a power of two (then x/area == x*inv_area exactly), else 0
    // the research S2CN2 wall variants (ugks_params): kinetic walls, W1T midpoint walls, W1D, W2R
    int s2_kinetic, s2_midpoint, s2_face_time, s2_shared;
};

// x / area, as a multiplication when that is exact (area a power of two: both operations round the
// same real number x * 2^-e once)
__device__ __forceinline__ double div_area(double x, const LoParams& P) {
    return P.inv_area != 0.0 ? x * P.inv_area : x / P.area;
}

struct LoBuffers {
    const double* u;         // [nvel] velocity table, k = i + j*Nu
    const double* v;
    const double* w;
    double* h;               // [nc][nvel] state, cell c = j*nx + i
    double* b;
    double* W;               // [nc][4] conservative variables
    double* sxh;             // [nc][nvel] Van-Leer slopes of h, b in x and y (Interpolation)
    double* syh;
    double* sxb;
    double* syb;
    double* fxh;             // [ny][nx][nvel] x-face micro flux (face i is between cells i-1 and i)
    double* fxb;
    double* fxw;             // [ny][nx][4] x-face macro flux
    double* fyh;             // [ny+1][nx][nvel] y-face micro flux (row 0 / ny are the walls)
    double* fyb;
    double* fyw;             // [ny+1][nx][4]
    double* res_w;           // [nc][4]   res_macro_flux_store
    double* res_h;           // [nc][nvel] res_h_flux_store (moment-projected stream * dt)
    double* res_b;
    double* peq_h;           // [nc][nvel] physical equilibrium (implicit paths)
    double* peq_b;
    double* pcol_h;          // [nc][nvel] physical collision
    double* pcol_b;
    double* dtl;             // [nc] dt_local of the next TimeStep
    double* dt;              // [2] dt_global of the next step; [1] dt of the last completed update
    double* cell_diag;       // [nc][kNDiag]
    double* diag;            // [kNDiag] reduced over cells by the last CTA
    double* wall_aero;       // [2][nx][3] local-frame pnn, pnt, qn per wall face
    unsigned* counter;       // [1] last-CTA counter (self-resetting)
    unsigned* status;        // [1] error bits
    const double* eval;      // [2] {valid, dt}: when valid and dt == dt[0], the slopes, fluxes and rates
                             // of the current state are already in place and the evaluation returns
                             // at entry (nullptr: always evaluate)
    const unsigned* halt;    // [1] nonzero after a rejected step of a multi-step launch sequence.  With
                             // halt set, a kernel returns at entry once this flag or any status bit
                             // is set, so a failure anywhere in a step ends the sequence there
                             // (nullptr: never halted)
};

__device__ __forceinline__ bool halted(const LoBuffers& B) {
    return B.halt != nullptr && (*B.halt != 0u || *B.status != 0u);
}

// true when the evaluation kernels have nothing to do: the cached evaluation is current, or the
// launch sequence has halted
__device__ __forceinline__ bool eval_cached(const LoBuffers& B) {
    return halted(B) || (B.eval != nullptr && B.eval[0] != 0.0 && B.eval[1] == B.dt[0]);
}

__device__ __forceinline__ int wrapx(int i, int nx) { return i < 0 ? i + nx : (i >= nx ? i - nx : i); }

// Velocity slot r of this thread: k, clamped index kk, and whether it is a real velocity.  Velocity
// loops are branch-free: a slot beyond nvel reads a valid velocity with weight 0 and skips stores.
struct Slot {
    int k, kk;
    bool ok;
};
__device__ __forceinline__ Slot slot(int r, int nv) {
    Slot s;
    s.k = threadIdx.x + r * blockDim.x;
    s.ok = s.k < nv;
    s.kk = s.ok ? s.k : nv - 1;
    return s;
}

// The kernels' parameter block of a domain described by the C ABI's ugks_params, with U_MAX / V_MAX
// of its velocity table (InitVelocityFromStructuredFile, mod_InitializeFlow.f90:508).  Host only;
// shared by the context path and the allocation-free entry point so that both derive the same block.
inline LoParams make_lo_params(const ugks_params& p, double umax, double vmax) {
    LoParams P{};
    P.nx = p.nx; P.ny = p.ny; P.nvel = p.nvel; P.ck = p.ck;
    P.dx = p.dx; P.dy = p.dy;
    P.area = std::fabs((-p.dx) * (-p.dy) - (p.dx) * (-p.dy)) * 0.5;
    {
        int e2 = 0;
        const double m2 = std::frexp(P.area, &e2);
        P.inv_area = (m2 == 0.5 && std::isfinite(P.area)) ? std::ldexp(1.0, 1 - e2) : 0.0;
    }
    P.gm1 = (double)(p.ck + 4) / (double)(p.ck + 2) - 1.0;
    P.pr = p.pr; P.omega = p.omega; P.mu_ref = p.mu_ref; P.cfl = p.cfl;
    P.umax = umax; P.vmax = vmax;
    for (int s = 0; s < 2; ++s) { P.wall_ux[s] = p.wall_ux[s]; P.wall_lam[s] = 1.0 / p.wall_tnative[s]; }
    P.fixed_dt = p.fixed_dt;
    P.inv_dx = 1.0 / p.dx;
    P.inv_dy = 1.0 / p.dy;
    P.s2_kinetic = p.s2_kinetic_wall != 0;
    P.s2_midpoint = p.s2_time_centered != 0;
    P.s2_face_time = p.s2_face_time != 0;
    P.s2_shared = p.s2_shared_predictor != 0;
    return P;
}

// The residual vector `res` of ApplyExplicitUpdate (mod_TimeIntegrator.f90:108-127) from the cell-reduced
// sums dg[kNDiag] (sum of squared rates [0..3], of |W| [4..7], of area^2 [8]).  Host only.
inline void finish_explicit_res(int nx, int ny, const double* dg, double* res) {
    const double SMV = 1.1754943508222875e-38;
    const double ncell = (double)nx * (double)ny;
    const double ords = std::fmax(std::fmax(dg[4], dg[7]), SMV);
    for (int m = 0; m < 4; ++m) {
        const double rel = std::sqrt(ncell * dg[m]) / (dg[4 + m] + SMV);
        const double ab = std::sqrt(dg[m] / std::fmax(dg[8], SMV));
        const bool near0 = dg[4 + m] <= std::sqrt(2.220446049250313e-16) * std::fmax(ords, 2.2250738585072014e-308);
        res[m] = near0 ? ab : rel;
    }
}

// Per-cell TimeStep (mod_Solve.f90:386-405): dt_local = CFL*area/(dy*max(U_MAX,|U|+c)+dx*max(V_MAX,|V|+c))
__device__ __forceinline__ double cell_dt(const LoParams& P, const double w[4], bool& ok) {
    Prim p;
    ok = get_primary(P.gm1, w, p);
    if (!ok) return 0.0;
    const double sos = sqrt(0.5 * (P.gm1 + 1.0) / p.L);
    const double a = fmax(P.umax, fabs(p.U) + sos), bq = fmax(P.vmax, fabs(p.V) + sos);
    return P.cfl * P.area / (P.dy * a + P.dx * bq);
}

}  // namespace ugks
