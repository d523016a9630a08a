// ugks_implicit.cu -- ImplicitSteady pseudo-step (second order) with the closed-Couette mass
// rescale and the accepted-state five-state gate, all on the device.
//
// Reference: ApplySteadyImplicitUpdate / ApplyOriginalSteadyImplicitUpdate
// (mod_SteadyImplicit.f90:379-462), SolveMacroPR2 (mod_ImplicitMacro.f90:57-123),
// BuildPredictedMacroState (:159-185), BuildPredictedEquilibrium (mod_ImplicitMicro.f90:43-88),
// SolveMicroLUSGS / RelaxMicroPoint / PrepareFrozenMicroWallState (:366-487, :647-791),
// ComputeDiffuseWallFaceDelta (mod_ImplicitBoundary.f90:282-326), FindAdmissibleMicroAlpha
// (mod_SteadyImplicit.f90:53-117), RecoverMacroFromKineticState (mod_ImplicitMicro.f90:628-645),
// RescaleClosedMass (mod_ClosedCouetteMass.f90:243-313), UpdateImplicitResidualDiagnostics
// (mod_ImplicitDiagnostics.f90:223-322) and the accepted-state evaluation of mod_R5Observe.f90.
//
// The reference runs NP_Y ranks stacked in y.  PR(2) and LU-SGS are Gauss-Seidel inside a rank and
// read the other ranks' corrections, and the x-periodic self-exchange, from halos refreshed only at
// the exchange points, so the device keeps the same seams ("slabs"):
//   * PR(2): one CTA per slab, an anti-diagonal wavefront of its cells; each sweep reads other slabs /
//     the x wrap from the previous sweep's complete buffer and its own cells Gauss-Seidel from the
//     current one (double buffer);
//   * LU-SGS: one thread per (slab, velocity) -- the per-velocity upwind sweep -- forward with zero
//     halos, backward with the forward result as halo, the diffuse-wall closure frozen per cell from
//     the forward correction between the two stages.
// Every kernel returns at entry once the stop flag is set (converged, or a gate failed), so a
// graph of several pseudo-steps can be replayed past convergence without changing the state.
#include "ugks_implicit.cuh"

namespace ugks {

__device__ __forceinline__ bool is_physical(const double w[4]) {   // IsPhysicalState (mod_ImplicitCommon.f90:10-20)
    if (!(isfinite(w[0]) && isfinite(w[1]) && isfinite(w[2]) && isfinite(w[3]))) return false;
    if (!(w[0] > 0.0)) return false;
    const double e = w[3] - 0.5 * (w[1] * w[1] + w[2] * w[2]) / w[0];
    return isfinite(e) && e > 0.0;
}

// EulerFluxNormal (mod_ImplicitCommon.f90:22-30)
// EulerFluxNormal (mod_ImplicitMacro.f90:265-280) split into the state's primitives (u, v, p), which
// hold the divisions and are shared by every face of a cell, and the normal flux.  Products are
// rounded before they are summed (no contraction), as in the reference's loop, so a flux built from
// cached primitives equals one built from scratch.
struct EulerPrim {
    double u, v, p;
};

__device__ __forceinline__ EulerPrim euler_prim(double gm1, const double w[4]) {
    EulerPrim e;
    e.u = w[1] / w[0];
    e.v = w[2] / w[0];
    const double ke = __dadd_rn(__dmul_rn(w[1], w[1]), __dmul_rn(w[2], w[2]));
    e.p = gm1 * (w[3] - 0.5 * ke / w[0]);
    return e;
}

__device__ __forceinline__ void euler_flux_prim(const double w[4], const EulerPrim& e, double nx, double ny,
                                                double f[4]) {
    const double un = __dadd_rn(__dmul_rn(e.u, nx), __dmul_rn(e.v, ny));
    f[0] = w[0] * un;
    f[1] = __dadd_rn(__dmul_rn(w[1], un), __dmul_rn(e.p, nx));
    f[2] = __dadd_rn(__dmul_rn(w[2], un), __dmul_rn(e.p, ny));
    f[3] = (w[3] + e.p) * un;
}

__device__ __forceinline__ void euler_flux(double gm1, const double w[4], double nx, double ny, double f[4]) {
    euler_flux_prim(w, euler_prim(gm1, w), nx, ny, f);
}

// ZhuMovingWallMap (mod_ImplicitBoundary.f90:187-194): ghost state and its exact tangent.
__device__ __forceinline__ void zhu_map(const double w[4], double uw, double vw, double g[4]) {
    g[0] = w[0];
    g[1] = __dsub_rn(__dmul_rn(2.0 * uw, w[0]), w[1]);
    g[2] = __dsub_rn(__dmul_rn(2.0 * vw, w[0]), w[2]);
    const double t = __dadd_rn(w[3], __dmul_rn(2.0 * __dadd_rn(__dmul_rn(uw, uw), __dmul_rn(vw, vw)), w[0]));
    g[3] = __dsub_rn(__dsub_rn(t, __dmul_rn(2.0 * uw, w[1])), __dmul_rn(2.0 * vw, w[2]));
}

// Face f (0 left, 1 right, 2 bottom, 3 top) of cell (i,j): outward normal of GetFaceGeometry
// (mod_ImplicitMacro.f90:236-263), length, neighbour, and whether the neighbour comes from a halo
// (other slab or x wrap) or is a wall.
struct FaceGeo {
    double nx, ny, len;
    int nb;
    bool ghost, wall;
};

__device__ __forceinline__ FaceGeo face_geo(const LoParams& P, int rows, int i, int j, int f) {
    FaceGeo g;
    g.wall = false;
    g.ghost = false;
    if (f == 0) {
        g.nx = -1.0; g.ny = 0.0; g.len = P.dy;
        g.ghost = i == 0; g.nb = j * P.nx + wrapx(i - 1, P.nx);
    } else if (f == 1) {
        g.nx = 1.0; g.ny = -0.0; g.len = P.dy;
        g.ghost = i == P.nx - 1; g.nb = j * P.nx + wrapx(i + 1, P.nx);
    } else if (f == 2) {
        g.nx = 0.0; g.ny = -1.0; g.len = P.dx;
        g.wall = j == 0; g.nb = g.wall ? -1 : (j - 1) * P.nx + i;
        g.ghost = !g.wall && (j - 1) / rows != j / rows;
    } else {
        g.nx = -0.0; g.ny = 1.0; g.len = P.dx;
        g.wall = j == P.ny - 1; g.nb = g.wall ? -1 : (j + 1) * P.nx + i;
        g.ghost = !g.wall && (j + 1) / rows != j / rows;
    }
    return g;
}

__device__ __forceinline__ int first_bit(unsigned m) { return m ? __ffs((int)m) - 1 : -1; }

__device__ __forceinline__ double pow2neg(int m) {
    double a = 1.0;
    for (int q = 0; q < m; ++q) a = 0.5 * a;
    return a;
}

// largest m with 2^-m >= min_alpha (the reference halves while alpha >= Implicit_MinAlpha)
__device__ __forceinline__ int alpha_levels(double min_alpha) {
    int m = 0;
    double a = 1.0;
    while (m < 30 && 0.5 * a >= min_alpha) { a = 0.5 * a; ++m; }
    return m;
}

__device__ __forceinline__ void stop_with(const ImBuffers& I, unsigned* status, unsigned bit) {
    set_status(status, bit);
    I.state[IS_STOP] = 1.0;
    *I.stopw = 1u;
}

// Wall frame of ComputeDiffuseWallFaceDelta: top = wall above row ny-1 (normal +y), else bottom.
__device__ __forceinline__ void wall_frame(const LoParams& P, int top, double uk, double vk, double& vn, double& hu,
                                           double& bu) {
    const double nxo = top ? -0.0 : 0.0, nyo = top ? 1.0 : -1.0;
    vn = uk * nxo + vk * nyo;
    const double vt = -uk * nyo + vk * nxo;
    // LocalFrame([1, Ux, 0, lambda_w], nxo, nyo) (mod_Tools.f90:150-162) with rho = 1
    const double pl1 = P.wall_ux[top] * nxo + 0.0 * nyo, pl2 = -P.wall_ux[top] * nyo + 0.0 * nxo;
    const double L = P.wall_lam[top];
    const double dvn = vn - pl1, dvt = vt - pl2;
    hu = 1.0 * (L / kPi) * exp(-L * (dvn * dvn + dvt * dvt));
    bu = hu * ((double)P.ck / (2.0 * L));
}

// -------------------------------------------------------------------------------------------
// ComputeResidual's steady-rate assembly (mod_Residual.f90:81-132) + UpdateImplicitResidualDiagnostics
// per cell.  POST = the accepted-state evaluation (PhysicalDiagnostic, mod_R5Observe.f90:40-141):
// its last CTA writes the report row and advances the five-state streak.
// Last-CTA part of the residual kernels: global sums (MPI_Allreduce SUM/MAX) of the per-cell
// terms, the science / flux columns, the five-state streak and the report row.
template <bool POST>
__device__ void im_residual_epilogue(const LoParams& P, const LoBuffers& B, const ImParams& Q, const ImBuffers& I,
                                     double* red, double* rout) {
    const int tid = threadIdx.x, nx = P.nx;
    const double dt = B.dt[0];
    __shared__ unsigned s_last;
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = (atomicAdd(I.counter, 1u) == (unsigned)(gridDim.x - 1)) ? 1u : 0u;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const int nc = P.nx * P.ny;
    // g[0..18]: sums of the per-cell terms; g[19..30]: boundary-face macro fluxes per unit time
    // (x wrap face, bottom wall, top wall; PhysicalDiagnostic flux, mod_R5Observe.f90:107-113);
    // g[31]: max moment error
    // g[32] (POST): max of -dt_local, the next pseudo-step's TimeStep
    double g[33];
#pragma unroll
    for (int m = 0; m < 32; ++m) g[m] = 0.0;
    g[32] = -INFINITY;
    for (int cc = tid; cc < nc; cc += blockDim.x) {
#pragma unroll
        for (int m = 0; m < 19; ++m) g[m] += __ldcg(I.cell + (size_t)cc * kImCell + m);
        g[31] = fmax(g[31], __ldcg(I.cell + (size_t)cc * kImCell + 19));
        if (POST) g[32] = fmax(g[32], -__ldcg(B.dtl + cc));
    }
    if (POST) {
        for (int jj = tid; jj < P.ny; jj += blockDim.x)
#pragma unroll
            for (int m = 0; m < 4; ++m) g[19 + m] += __ldcg(B.fxw + ((size_t)jj * nx + 0) * 4 + m) / dt;
        for (int ii = tid; ii < nx; ii += blockDim.x)
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                g[23 + m] += __ldcg(B.fyw + (size_t)ii * 4 + m) / dt;
                g[27 + m] += __ldcg(B.fyw + ((size_t)P.ny * nx + ii) * 4 + m) / dt;
            }
    }
    block_reduce<31, 2>(g, red, rout);
    if (tid != 0) return;
    const double SMV = kSMV;
    double sci[22];
    const double ncell = (double)nc;
    double ords = fmax(fmax(g[4], g[7]), SMV);
    for (int m = 0; m < 4; ++m) {
        const double rel = sqrt(ncell * g[m]) / (g[4 + m] + SMV);
        const double ab = sqrt(g[m] / fmax(g[8], SMV));
        sci[4 + m] = rel;
        sci[8 + m] = ab;
        sci[m] = (g[4 + m] <= sqrt(kEps) * fmax(ords, DBL_MIN)) ? ab : rel;
    }
    const double raw_h = sqrt(g[9]), raw_b = sqrt(g[10]);
    const double h_raw = sqrt(g[9] / fmax(g[11], SMV)), b_raw = sqrt(g[10] / fmax(g[12], SMV));
    if (I.state[IS_REF_INIT] == 0.0) {
        I.state[IS_REF_H] = h_raw;
        I.state[IS_REF_B] = b_raw;
        I.state[IS_REF_INIT] = 1.0;
    }
    const double rh = I.state[IS_REF_H], rb = I.state[IS_REF_B];
    const double nzr = fmax(100.0 * Q.residual_tol, 1000.0 * kEps);
    sci[12] = rh <= nzr ? h_raw : h_raw / rh;
    sci[13] = rb <= nzr ? b_raw : b_raw / rb;
    sci[14] = rh > DBL_MIN ? h_raw / rh : h_raw;
    sci[15] = rb > DBL_MIN ? b_raw / rb : b_raw;
    sci[16] = h_raw;
    sci[17] = b_raw;
    sci[18] = I.state[IS_MOMENT];
    sci[19] = fabs(g[13]);
    sci[20] = raw_h;
    sci[21] = raw_b;
    double* rep = I.report;
    if (!POST) {
        for (int m = 0; m < 22; ++m) rep[57 + m] = sci[m];
        *I.counter = 0u;
        return;
    }
    const double moment = g[31];
    for (int m = 0; m < 22; ++m) I.state[IS_PRESCI + m] = sci[m];
    I.state[IS_EVAL_DT] = dt;
    I.state[IS_EVAL_VALID] = 1.0;
    if (Q.mass_rescale) sci[18] = moment;   // implicit_moment_error = MassStatistics after the rescale
    // boundary-face totals per unit time: outflow through the left x face, inflow through the right
    // (the same periodic face), the bottom wall taken into the domain, the top wall out of it
    double flux[16];
    for (int m = 0; m < 4; ++m) {
        flux[m] = -g[19 + m];
        flux[4 + m] = g[19 + m];
        flux[8 + m] = -g[23 + m];
        flux[12 + m] = g[27 + m];
    }
    const double tol = Q.residual_tol;
    const bool pass = sci[0] <= tol && sci[1] <= tol && sci[2] <= tol && sci[3] <= tol && sci[12] <= tol &&
                      sci[13] <= tol && moment <= Q.moment_tol;
    const double streak = pass ? I.state[IS_STREAK] + 1.0 : 0.0;
    I.state[IS_STREAK] = streak;
    I.state[IS_STEPS] = I.state[IS_STEPS] + 1.0;
    const bool done = Q.mass_rescale ? streak >= 5.0 : pass;
    if (done) { I.state[IS_CONVERGED] = 1.0; I.state[IS_STOP] = 1.0; *I.stopw = 1u; }
    rep[0] = pass ? 1.0 : 0.0;
    rep[1] = moment;
    rep[2] = g[14];
    rep[3] = g[18];
    for (int m = 0; m < 4; ++m) rep[4 + m] = sci[8 + m];
    rep[8] = raw_h; rep[9] = raw_b; rep[10] = h_raw; rep[11] = b_raw;
    for (int m = 0; m < 22; ++m) rep[12 + m] = sci[m];
    for (int m = 0; m < 16; ++m) rep[34 + m] = flux[m];
    rep[50] = rh; rep[51] = rb;
    rep[52] = Q.mass_rescale ? I.state[IS_MASS_SCALE] - 1.0 : 0.0;
    rep[53] = I.state[IS_ALPHA]; rep[54] = I.state[IS_MALPHA]; rep[55] = dt; rep[56] = streak;
    // TimeStep of the next pseudo-step (mod_Solve.f90:373-421) from this accepted state, as k_lo_timestep
    // would take it at the next step's start
    B.dt[1] = B.dt[0];
    B.dt[0] = P.fixed_dt > 0.0 ? P.fixed_dt : -g[32];
    *I.counter = 0u;
}

template <int VPT, int NTMAX, bool POST>
__global__ void __launch_bounds__(NTMAX, 512 / NTMAX) k_im_residual(LoParams P, LoBuffers B, ImParams Q, ImBuffers I) {
    if (I.state[IS_STOP] != 0.0) return;
    if (!POST && eval_cached(B)) {   // the previous accepted-state evaluation is this evaluation
        if (blockIdx.x == 0 && threadIdx.x < 22) I.report[57 + threadIdx.x] = I.state[IS_PRESCI + threadIdx.x];
        return;
    }
    __shared__ double red[16 * 64];
    __shared__ double rout[kRedSlots];
    __shared__ double sc[32];   // [0..3] res_w [4..7] prim [8] tau [9] ok [12..15] stream lambda [16..19] eq lambda
    const int nv = P.nvel, tid = threadIdx.x, nx = P.nx;
    const int c = blockIdx.x, i = c % nx, j = c / nx;
    const double dt = B.dt[0], dti = 1.0 / dt;
    const size_t fl = (size_t)(j * nx + i), fr = (size_t)(j * nx + wrapx(i + 1, nx));
    const size_t gl = (size_t)(j * nx + i), gr = (size_t)((j + 1) * nx + i);
    if (tid == 0) {
        const double* Wo = B.W + c * 4;
#pragma unroll
        for (int m = 0; m < 4; ++m)
            sc[m] = (B.fxw[fl * 4 + m] - B.fxw[fr * 4 + m] + B.fyw[gl * 4 + m] - B.fyw[gr * 4 + m]) / P.area;
        Prim p;
        double tau = 1.0;
        bool ok = get_primary(P.gm1, Wo, p);
        ok = ok && get_tau(P.mu_ref, P.omega, p, tau);
        if (!ok) { p.r = 1.0; p.U = p.V = 0.0; p.L = 1.0; tau = 1.0; }
        sc[4] = p.r; sc[5] = p.U; sc[6] = p.V; sc[7] = p.L; sc[8] = tau; sc[9] = ok ? 1.0 : 0.0;
    }
    const double area_inv = 1.0 / P.area;
    double h[VPT], b[VPT], sh[VPT], sb[VPT], acc[14];
#pragma unroll
    for (int m = 0; m < 6; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const int k = s.kk;
        const double wk = s.ok ? B.w[k] : 0.0;
        h[r] = B.h[(size_t)c * nv + k];
        b[r] = B.b[(size_t)c * nv + k];
        sh[r] = (B.fxh[fl * nv + k] - B.fxh[fr * nv + k] + B.fyh[gl * nv + k] - B.fyh[gr * nv + k]) * area_inv * dti;
        sb[r] = (B.fxb[fl * nv + k] - B.fxb[fr * nv + k] + B.fyb[gl * nv + k] - B.fyb[gr * nv + k]) * area_inv * dti;
        moment_add(wk, B.u[k], B.v[k], sh[r], sb[r], acc);
        acc[4] = fmax(acc[4], s.ok ? fabs(h[r]) : 0.0);
        acc[5] = fmax(acc[5], s.ok ? fabs(b[r]) : 0.0);
    }
    block_reduce<4, 2>(acc, red, rout);
    // EnforceStreamingMomentCompatibility (mod_ImplicitMicro.f90:293-306): stream onto rate_w, weights |h|
    double smom[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) smom[m] = acc[m];
    const double shs = fmax(acc[4], 1.0), sbs = fmax(acc[5], 1.0);
#pragma unroll
    for (int m = 0; m < 10; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double wk = s.ok ? B.w[s.kk] : 0.0;
        gram_add(wk, fmax(fabs(h[r]), kEps * shs), fmax(fabs(b[r]), kEps * sbs), B.u[s.kk], B.v[s.kk], acc);
    }
    block_reduce_smem<10, 0>(acc, red, rout);
    if (tid == 0) {
        double rhs[4], gm[16], lam[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) rhs[m] = sc[m] * dti - smom[m];
        gram_expand(rout, gm);
        const bool ok = solve_dense4(gm, rhs, lam);
#pragma unroll
        for (int m = 0; m < 4; ++m) sc[12 + m] = ok ? lam[m] : 0.0;
        if (!ok) stop_with(I, B.status, ST_PROJECTION);
    }
    __syncthreads();
    const Prim p{sc[4], sc[5], sc[6], sc[7]};
    const double tau = sc[8];
    double lam[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) lam[m] = sc[12 + m];
#pragma unroll
    for (int m = 0; m < 6; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
        const double e = 0.5 * (uk * uk + vk * vk);
        sh[r] = sh[r] + fmax(fabs(h[r]), kEps * shs) * (lam[0] + uk * lam[1] + vk * lam[2] + e * lam[3]);
        sb[r] = sb[r] + 0.5 * fmax(fabs(b[r]), kEps * sbs) * lam[3];
        moment_add(wk, uk, vk, sh[r], sb[r], acc);
        const double dvn = uk - p.U, dvt = vk - p.V, v2 = dvn * dvn + dvt * dvt;
        const double t = 0.5 * wk * (v2 * h[r] + b[r]);
        acc[4] += t * dvn;
        acc[5] += t * dvt;
    }
    block_reduce_smem<6, 0>(acc, red, rout);
    if (tid == 0) {
        double rs = 1.0, err = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) { rs = fmax(rs, fabs(sc[m] * dti)); }
#pragma unroll
        for (int m = 0; m < 4; ++m) err = fmax(err, fabs(rout[m] - sc[m] * dti));
        if (!(err <= 1.0e-10 * rs)) stop_with(I, B.status, ST_PROJECTION);
        if (sc[9] == 0.0) stop_with(I, B.status, ST_GETPRIMARY);
    }
    const double q0 = rout[4], q1 = rout[5];
    // physical equilibrium (mod_Residual.f90:116-127): Maxwellian + Shakhov at W, projected onto W
    double E[VPT], F[VPT];
    {
        const double pref = p.r * (p.L / kPi), bfac = (double)P.ck / (2.0 * p.L);
        const double coeff = 0.8 * (1.0 - P.pr) * p.L * p.L / p.r, c2ck = 2.0 / (double)P.ck;
        acc[0] = acc[1] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            const double dvn = B.u[s.kk] - p.U, dvt = B.v[s.kk] - p.V, v2 = dvn * dvn + dvt * dvt;
            const double H = pref * exp(-p.L * v2), Bm = H * bfac;
            const double qd = dvn * q0 + dvt * q1, sH = 2.0 * p.L * v2 - 4.0;
            E[r] = H + coeff * qd * sH * H;
            F[r] = Bm + coeff * qd * (sH + c2ck) * Bm;
            acc[0] = fmax(acc[0], s.ok ? fabs(E[r]) : 0.0);
            acc[1] = fmax(acc[1], s.ok ? fabs(F[r]) : 0.0);
        }
        block_reduce<0, 2>(acc, red, rout);
    }
    const double se = fmax(acc[0], 1.0), sf = fmax(acc[1], 1.0);
#pragma unroll
    for (int m = 0; m < 14; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double wk = s.ok ? B.w[s.kk] : 0.0;
        moment_add(wk, B.u[s.kk], B.v[s.kk], E[r], F[r], acc);
        gram_add(wk, fmax(fabs(E[r]), kEps * se), fmax(fabs(F[r]), kEps * sf), B.u[s.kk], B.v[s.kk], acc + 4);
    }
    block_reduce_smem<14, 0>(acc, red, rout);
    if (tid == 0) {
        double rhs[4], gm[16], l[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) rhs[m] = B.W[c * 4 + m] - rout[m];
        gram_expand(rout + 4, gm);
        const bool ok = solve_dense4(gm, rhs, l);
#pragma unroll
        for (int m = 0; m < 4; ++m) sc[16 + m] = ok ? l[m] : 0.0;
        if (!ok) stop_with(I, B.status, ST_PROJECTION);
    }
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 4; ++m) lam[m] = sc[16 + m];
#pragma unroll
    for (int m = 0; m < 12; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0, e = 0.5 * (uk * uk + vk * vk);
        const double Ep = E[r] + fmax(fabs(E[r]), kEps * se) * (lam[0] + uk * lam[1] + vk * lam[2] + e * lam[3]);
        const double Fp = F[r] + 0.5 * fmax(fabs(F[r]), kEps * sf) * lam[3];
        const double ch = (Ep - h[r]) / tau, cb = (Fp - b[r]) / tau;
        moment_add(wk, uk, vk, Ep, Fp, acc);
        const double dh = sh[r] + ch, db = sb[r] + cb;
        acc[4] += wk * dh * dh;
        acc[5] += wk * db * db;
        acc[6] += wk * fmax(h[r] * h[r], Ep * Ep);
        acc[7] += wk * fmax(b[r] * b[r], Fp * Fp);
        moment_add(wk, uk, vk, h[r], b[r], acc + 8);
        if (s.ok) {   // the physical equilibrium and collision stay in registers: nothing later reads them
            const size_t q = (size_t)c * nv + s.k;
            I.stream_h[q] = sh[r];
            I.stream_b[q] = sb[r];
        }
    }
    block_reduce_smem<12, 0>(acc, red, rout);
    if (tid == 0) {
        const double* Wo = B.W + c * 4;
        double rs = 1.0, err = 0.0, merr = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) { rs = fmax(rs, fabs(Wo[m])); err = fmax(err, fabs(rout[m] - Wo[m])); }
        if (!(err <= 1.0e-10 * rs)) stop_with(I, B.status, ST_PROJECTION);
#pragma unroll
        for (int m = 0; m < 4; ++m) merr = fmax(merr, fabs(Wo[m] - rout[8 + m]) / fmax(fabs(Wo[m]), 1.0));
        double rate[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) { rate[m] = sc[m] * dti; I.rate_w[c * 4 + m] = rate[m]; }
        double* t = I.cell + (size_t)c * kImCell;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const double a = P.area * rate[m];
            t[m] = a * a;
            t[4 + m] = P.area * fabs(Wo[m] + dt * rate[m]);
            t[14 + m] = P.area * Wo[m];
        }
        t[8] = P.area * P.area;
        t[9] = P.area * rout[4];
        t[10] = P.area * rout[5];
        t[11] = P.area * rout[6];
        t[12] = P.area * rout[7];
        t[13] = rate[0] * P.area;
        t[18] = P.area * rout[8];
        t[19] = merr;
    }

    if (POST && tid == 0) {   // this cell's dt_local for the next pseudo-step's TimeStep
        bool okd;
        B.dtl[c] = cell_dt(P, B.W + c * 4, okd);
        if (!okd) set_status(B.status, ST_GETPRIMARY);
    }
    im_residual_epilogue<POST>(P, B, Q, I, red, rout);
}

// ComputeResidual + AssembleSteadyRateResiduals for HighOrderImplicit (mod_Residual.f90:81-108,
// IsS2CN2 branch) and S2NativePhysicalCollision (mod_S2NativeAdapter.f90:735-759): the steady rates
// without the streaming projection (the stream moments must equal rate_w to 2e-12), the physical
// collision C = (M + K_x q + K_y q - h) / tau with q = heat(h - M), tau = s2_tau(W), and the same
// per-cell diagnostic terms as the second-order evaluation.
template <int VPT, int NTMAX, bool POST>
__global__ void __launch_bounds__(NTMAX, 512 / NTMAX) k_im_residual_s2(LoParams P, LoBuffers B, ImParams Q,
                                                                       ImBuffers I) {
    if (I.state[IS_STOP] != 0.0) return;
    if (!POST && eval_cached(B)) {
        if (blockIdx.x == 0 && threadIdx.x < 22) I.report[57 + threadIdx.x] = I.state[IS_PRESCI + threadIdx.x];
        return;
    }
    __shared__ double red[16 * 64];
    __shared__ double rout[kRedSlots];
    __shared__ double sc[16];   // [0..3] res_w, [4] ux, [5] vy, [6] tau, [7] ok
    const int nv = P.nvel, tid = threadIdx.x, nx = P.nx;
    const int c = blockIdx.x, i = c % nx, j = c / nx;
    const double dt = B.dt[0], dti = 1.0 / dt;
    const size_t fl = (size_t)(j * nx + i), fr = (size_t)(j * nx + wrapx(i + 1, nx));
    const size_t gl = (size_t)(j * nx + i), gr = (size_t)((j + 1) * nx + i);
    const double* Wo = B.W + c * 4;
    if (tid == 0) {
#pragma unroll
        for (int m = 0; m < 4; ++m)
            sc[m] = (B.fxw[fl * 4 + m] - B.fxw[fr * 4 + m] + B.fyw[gl * 4 + m] - B.fyw[gr * 4 + m]) / P.area;
        double tau = 1.0;
        const bool ok = Wo[0] > 0.0 && s2_tau(P, Wo, tau);
        sc[4] = Wo[1] / Wo[0]; sc[5] = Wo[2] / Wo[0]; sc[6] = ok ? tau : 1.0; sc[7] = ok ? 1.0 : 0.0;
    }
    __syncthreads();
    const double ux = sc[4], vy = sc[5], tau = sc[6];
    const double area_inv = 1.0 / P.area;
    double h[VPT], b[VPT], sh[VPT], sb[VPT], acc[12];
#pragma unroll
    for (int m = 0; m < 6; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const int k = s.kk;
        const size_t q = (size_t)c * nv + k;
        const double wk = s.ok ? B.w[k] : 0.0, uk = B.u[k], vk = B.v[k];
        h[r] = B.h[q];
        b[r] = B.b[q];
        sh[r] = (B.fxh[fl * nv + k] - B.fxh[fr * nv + k] + B.fyh[gl * nv + k] - B.fyh[gr * nv + k]) * area_inv * dti;
        sb[r] = (B.fxb[fl * nv + k] - B.fxb[fr * nv + k] + B.fyb[gl * nv + k] - B.fyb[gr * nv + k]) * area_inv * dti;
        moment_add(wk, uk, vk, sh[r], sb[r], acc);
        const double cx = uk - ux, cy = vk - vy, c2 = cx * cx + cy * cy;
        const double dh = h[r] - I.s2.mh[q], db = b[r] - I.s2.mb[q];
        acc[4] += 0.5 * wk * cx * (c2 * dh + db);
        acc[5] += 0.5 * wk * cy * (c2 * dh + db);
    }
    block_reduce<6, 0>(acc, red, rout);
    if (tid == 0) {
        double rs = 1.0, err = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) { rs = fmax(rs, fabs(sc[m] * dti)); err = fmax(err, fabs(acc[m] - sc[m] * dti)); }
        if (!(err / rs <= 2.0e-12)) stop_with(I, B.status, ST_PROJECTION);
        if (sc[7] == 0.0) stop_with(I, B.status, ST_GETPRIMARY);
    }
    const double q0 = acc[4], q1 = acc[5];
#pragma unroll
    for (int m = 0; m < 12; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const size_t q = (size_t)c * nv + s.kk;
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
        const double Ep = I.s2.mh[q] + I.s2.kxh[q] * q0 + I.s2.kyh[q] * q1;
        const double Fp = I.s2.mb[q] + I.s2.kxb[q] * q0 + I.s2.kyb[q] * q1;
        const double ch = (Ep - h[r]) / tau, cb = (Fp - b[r]) / tau;
        moment_add(wk, uk, vk, ch, cb, acc);
        const double dh = sh[r] + ch, db = sb[r] + cb;
        acc[4] += wk * dh * dh;
        acc[5] += wk * db * db;
        acc[6] += wk * fmax(h[r] * h[r], Ep * Ep);
        acc[7] += wk * fmax(b[r] * b[r], Fp * Fp);
        moment_add(wk, uk, vk, h[r], b[r], acc + 8);
        if (s.ok) {
            I.stream_h[(size_t)c * nv + s.k] = sh[r];
            I.stream_b[(size_t)c * nv + s.k] = sb[r];
            B.pcol_h[(size_t)c * nv + s.k] = ch;
            B.pcol_b[(size_t)c * nv + s.k] = cb;
        }
    }
    block_reduce_smem<12, 0>(acc, red, rout);
    if (tid == 0) {
        double ws = 1.0, mx = 0.0, merr = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) { ws = fmax(ws, fabs(Wo[m])); mx = fmax(mx, fabs(rout[m])); }
        if (tau * mx / ws > 2.0e-12) stop_with(I, B.status, ST_PROJECTION);   // S2 collision moment gate
#pragma unroll
        for (int m = 0; m < 4; ++m) merr = fmax(merr, fabs(Wo[m] - rout[8 + m]) / fmax(fabs(Wo[m]), 1.0));
        double rate[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) { rate[m] = sc[m] * dti; I.rate_w[c * 4 + m] = rate[m]; }
        double* t = I.cell + (size_t)c * kImCell;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const double a = P.area * rate[m];
            t[m] = a * a;
            t[4 + m] = P.area * fabs(Wo[m] + dt * rate[m]);
            t[14 + m] = P.area * Wo[m];
        }
        t[8] = P.area * P.area;
        t[9] = P.area * rout[4];
        t[10] = P.area * rout[5];
        t[11] = P.area * rout[6];
        t[12] = P.area * rout[7];
        t[13] = rate[0] * P.area;
        t[18] = P.area * rout[8];
        t[19] = merr;
    }
    if (POST && tid == 0) {   // this cell's dt_local for the next pseudo-step's TimeStep
        bool okd;
        B.dtl[c] = cell_dt(P, B.W + c * 4, okd);
        if (!okd) set_status(B.status, ST_GETPRIMARY);
    }
    im_residual_epilogue<POST>(P, B, Q, I, red, rout);
}

// -------------------------------------------------------------------------------------------
// PR(2) set-up of one (cell, face): the spectral radius (ImplicitSpectralRadius,
// mod_ImplicitMacro.f90:15-55) and the Euler normal fluxes of the unperturbed cell and neighbour
// states, which stay fixed through the sweeps.  Written to global memory for the later sweeps.
// Returns false (after stopping the sequence) when gamma is not finite and positive.
__device__ __forceinline__ bool pr_prep_item(const LoParams& P, const LoBuffers& B, const ImParams& Q, const ImBuffers& I, int c,
                             int f, double& gam, double foi[4], double foj[4]) {
    const int i = c % P.nx, j = c / P.nx;
    const int rows = P.ny / Q.nslab;
    const FaceGeo g = face_geo(P, rows, i, j, f);
    double wi[4], wj[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) wi[m] = B.W[c * 4 + m];
    double dist;
    if (g.wall) {
        zhu_map(wi, (f == 2 ? Q.wall_ux[0] : Q.wall_ux[1]), 0.0, wj);
        dist = P.dy;   // ctr%length(dirc)
    } else {
#pragma unroll
        for (int m = 0; m < 4; ++m) wj[m] = B.W[g.nb * 4 + m];
        // ghost centres of the outer ranks are extrapolated (mod_InitializeFlow.f90:418-446): one cell
        dist = (f < 2) ? fabs(P.dx * g.nx) : fabs(P.dy * g.ny);
    }
    Prim pi_, pj;
    double ti = 1.0, tj = 1.0;
    bool ok = get_primary(P.gm1, wi, pi_) && get_primary(P.gm1, wj, pj);
    ok = ok && get_tau(P.mu_ref, P.omega, pi_, ti) && get_tau(P.mu_ref, P.omega, pj, tj);
    gam = NAN;
    if (ok) {
        const double rho_avg = 0.5 * (pi_.r + pj.r);
        const double u_avg = 0.5 * (pi_.U + pj.U), v_avg = 0.5 * (pi_.V + pj.V);
        const double p_i = 0.5 * pi_.r / pi_.L, p_j = 0.5 * pj.r / pj.L;
        const double p_avg = 0.5 * (p_i + p_j);
        const double mu_avg = 0.5 * (ti * p_i + tj * p_j);
        const double sos = sqrt((P.gm1 + 1.0) * p_avg / rho_avg);
        gam = fabs(u_avg * g.nx + v_avg * g.ny) + sos + 2.0 * mu_avg / (rho_avg * fmax(dist, 1000.0 * kEps));
    }
    const bool good = isfinite(gam) && gam > 0.0;
    if (!good) stop_with(I, B.status, ST_GETPRIMARY);
    I.pr_gamma[c * 4 + f] = gam;
    euler_flux(P.gm1, wi, g.nx, g.ny, foi);
    euler_flux(P.gm1, wj, g.nx, g.ny, foj);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        I.pr_foi[(c * 4 + f) * 4 + m] = foi[m];
        I.pr_foj[(c * 4 + f) * 4 + m] = foj[m];
    }
    return good;
}

// Cells of anti-diagonal d of a rows x nx slab (local row jl = 0..rows-1, column i), t-th cell.
__device__ __forceinline__ bool diag_cell(int d, int t, int rows, int nx, int& i, int& jl) {
    const int jl0 = d - (nx - 1) > 0 ? d - (nx - 1) : 0;
    jl = jl0 + t;
    i = d - jl;
    return jl < rows && i >= 0;
}

// One PR(2) sweep of one slab (SolveMacroPR2, mod_ImplicitMacro.f90:57-88; RelaxMacroPoint :90-123).
// Lexicographic Gauss-Seidel on the 5-point stencil equals an anti-diagonal wavefront: cell (i,j)
// reads the already-updated (i-1,j), (i,j-1) and the not-yet-updated (i+1,j), (i,j+1), and cells on
// one anti-diagonal never read each other.  Four lanes per cell, one per component: each sums its
// component of the four face terms len * (dF_i + dF_j) and len * gamma * delta_nb in face order and
// relaxes it.  The chain of dependent relaxations is kept short: what a relaxation reads is ready in
// shared memory when the wavefront reaches the cell.
//   * Every cell's normal Euler fluxes are kept as two vectors, F(T, (1,-0)) and F(T, (-0,1)) with
//     T = W + correction; the lanes that relax a cell refresh them for its new state (primitives and
//     fluxes, the divisions of EulerFluxNormal, once per relaxation).  A face with the opposite normal
//     (left, bottom) takes the negated vector: the products are rounded one by one (no contraction),
//     so F(T, -n) = -F(T, n) exactly, up to the sign of a zero.
//   * The wall faces' ghost-state flux and ghost correction depend on the cell's own correction only,
//     which changes only when the cell itself relaxes: they are built before each pass.
//   * The diagonal 1/dt_ps + 0.5 sum(L gamma)/area is fixed through the sweeps; the division by it is
//     a multiplication by its reciprocal with one remainder correction (div_by_recip).
// The halo cells (x wrap, slab seams) hold the previous sweep's corrections X; Y = this sweep's result.
// shared doubles of one slab: corrections, states and flux pairs of interior + halo cells, then W, rate,
// gamma, fixed fluxes, diagonal and its reciprocal of the interior cells, then the wall-face terms
__host__ __device__ constexpr int pr_smem_words(int rows, int nx) {
    return (rows * nx + 2 * rows + 2 * nx) * 16 + rows * nx * 46 + nx * 16;
}

// local index of the neighbour of interior cell (i, jl) across face f: interior cells first, then
// the halo (left wrap [rows], right wrap [rows], row below the slab [nx], row above [nx]); -1: wall
__device__ __forceinline__ int pr_neighbour(int i, int jl, int j, int f, int rows, int nx, int ny) {
    const int ncs = rows * nx, cl = jl * nx + i;
    if (f == 0) return i > 0 ? cl - 1 : ncs + jl;
    if (f == 1) return i < nx - 1 ? cl + 1 : ncs + rows + jl;
    if (f == 2) return j == 0 ? -1 : (jl > 0 ? cl - nx : ncs + 2 * rows + i);
    return j == ny - 1 ? -1 : (jl < rows - 1 ? cl + nx : ncs + 2 * rows + nx + i);
}

// a / d for a divisor used many times, from r = 1/d (correctly rounded, computed once): q0 = a r, the
// remainder a - d q0 is exact in one fused multiply-add, and q0 + remainder * r rounds to a/d
// (Markstein's division correction, IBM J. Res. Develop. 34(1):111-119, 1990).  Finite operands away
// from overflow and underflow, which the callers check.
__device__ __forceinline__ double div_by_recip(double a, double d, double r) {
    const double q0 = __dmul_rn(a, r);
    return __fma_rn(__fma_rn(-d, q0, a), r, q0);
}

// F(t, (1,-0)) and F(t, (-0,1)) of a state and its primitives (EulerFluxNormal with those normals)
__device__ __forceinline__ void euler_flux_pair(const double t[4], const EulerPrim& e, double fx[4], double fy[4]) {
    euler_flux_prim(t, e, 1.0, -0.0, fx);
    euler_flux_prim(t, e, -0.0, 1.0, fy);
}

// Wall-face terms of the wall rows of this slab: the ghost state Zhu(W) + Zhu(delta) of the cell's
// current correction, its Euler flux with the wall face's normal, and the ghost correction Zhu(delta).
// [side][i][4], side 0 the bottom wall (face 2, normal (0,-1)), 1 the top wall (face 3, normal (-0,1)).
__device__ __forceinline__ void pr_wall_terms(const LoParams& P, const ImParams& Q, int s, int rows, const double* sW,
                                              const double* sY, double* sWf, double* sWd) {
    for (int q = threadIdx.x; q < 2 * P.nx; q += blockDim.x) {
        const int side = q / P.nx, i = q - side * P.nx;
        const int jl = side == 0 ? 0 : rows - 1, j = s * rows + jl;
        if (side == 0 ? j != 0 : j != P.ny - 1) continue;
        const int cl = jl * P.nx + i;
        const double uw = side == 0 ? Q.wall_ux[0] : Q.wall_ux[1];
        double wi[4], di[4], wj[4], dnb[4], tj[4], fj[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) { wi[m] = sW[cl * 4 + m]; di[m] = sY[cl * 4 + m]; }
        zhu_map(wi, uw, 0.0, wj);
        zhu_map(di, uw, 0.0, dnb);
#pragma unroll
        for (int m = 0; m < 4; ++m) tj[m] = wj[m] + dnb[m];
        euler_flux(P.gm1, tj, side == 0 ? 0.0 : -0.0, side == 0 ? -1.0 : 1.0, fj);
#pragma unroll
        for (int m = 0; m < 4; ++m) { sWf[q * 4 + m] = fj[m]; sWd[q * 4 + m] = dnb[m]; }
    }
}

// Barrier of the wavefront warps alone (named barrier 1); the other warps of the CTA only fill
// and drain the slab's shared memory and meet the wavefront at barrier 0 afterwards.
__device__ __forceinline__ void pr_wave_sync(int warps) {
    if (warps == 1) __syncwarp();
    else asm volatile("bar.sync 1, %0;" ::"r"(warps * 32) : "memory");
}

// Launched with kPrThreads threads: all of them stage the slab (about 120 global loads a warp
// when one warp did it alone), the first 4 x min(dcells, 32) relax.
constexpr int kPrThreads = 256;

// Grid barrier between the sweeps of one launch (gridDim.x = nslab CTAs, all resident: a cooperative
// launch).  bar[0] counts the arrivals, bar[1] is the generation: every CTA reads the generation
// before it arrives, the last arrival resets the count and advances the generation, the others poll
// it.  The CTAs' global writes before the barrier are visible to every CTA after it (bar.sync, then a
// device-scope fence by the arriving thread; a fence after the wait).  Bounded: a CTA that polls
// kPrBarrierPolls times without the generation moving returns false.
constexpr long long kPrBarrierPolls = 1LL << 22;   // with 64 ns pauses: about 0.3-1 s
__device__ bool pr_grid_barrier(unsigned* bar) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile unsigned* gen = bar + 1;
        const unsigned g0 = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long n = 0;
            while (*gen == g0) {
                if (++n > kPrBarrierPolls) { ok = 0; break; }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// first: the launch also does the PR(2) set-up of its slab (pr_prep_item, straight into shared memory)
// and starts from the zero correction (X unused as input); when the launch does not also end with the
// last sweep, or does more than one sweep, CTA 0 resets the admissible-alpha masks.  last: the launch
// ends with the last sweep and also does BuildPredictedMacroState (mod_ImplicitMacro.f90:159-185) for
// its cells: the admissible alpha levels of W + alpha Y, ANDed into the macro mask.
// sweeps: the sweeps this launch does.  Sweep k reads the halo corrections of sweep k-1 from (k odd ? Y
// : X) and writes its own to the other buffer, so they end in Y when `sweeps` is odd, else in X, as
// `sweeps` one-sweep launches with the buffers swapped between them would leave them.  Between sweeps
// the CTAs meet at a grid barrier (sweeps > 1 needs a cooperative launch); each CTA keeps its
// interior cells' corrections, states and flux pairs in shared memory, which are bitwise those the
// next launch would rebuild from Y, and reloads only its halo.
__global__ void __launch_bounds__(kPrThreads, 1) k_im_pr2_sweep(LoParams P, LoBuffers B, ImParams Q, ImBuffers I,
                                                             double* X, double* Y, int first, int last, int sweeps) {
    if (I.state[IS_STOP] != 0.0) return;
    extern __shared__ double sm[];
    const int s = blockIdx.x, rows = P.ny / Q.nslab, nx = P.nx, ny = P.ny;
    const int ncs = rows * nx, nall = ncs + 2 * rows + 2 * nx, c0 = s * ncs;
    double* sY = sm;                  // [nall][4] corrections
    double* sT = sY + nall * 4;       // [nall][4] W + correction
    double* sF = sT + nall * 4;       // [nall][8] F(T, (1,-0)), F(T, (-0,1))
    double* sW = sF + nall * 8;       // [ncs][4]
    double* sR = sW + ncs * 4;        // [ncs][4] rate_w
    double* sG = sR + ncs * 4;        // [ncs][4] gamma per face
    double* sFi = sG + ncs * 4;       // [4 components][ncs * 4 faces] fixed Euler flux of the cell
    double* sFj = sFi + ncs * 16;     // [4 components][ncs * 4 faces] fixed Euler flux of the neighbour
    const int ncf = ncs * 4;          // component-major: the cells of a diagonal fall on distinct banks
    double* sD = sFj + ncs * 16;      // [ncs] diagonal
    double* sRd = sD + ncs;           // [ncs] 1 / diagonal
    double* sWf = sRd + ncs;          // [2][nx][4] wall-face flux (pr_wall_terms)
    double* sWd = sWf + nx * 8;       // [2][nx][4] wall-face ghost correction
    const int dcells = rows < nx ? rows : nx;                  // longest anti-diagonal
    const int wave = 4 * (dcells < 32 ? dcells : 32);          // relaxing lanes: 4 per cell
    const int wave_warps = (wave + 31) >> 5;
    const int m = threadIdx.x & 3, tc = threadIdx.x >> 2, D = wave >> 2;
    const double dtp = B.dt[0] * Q.ncfl / P.cfl;   // PseudoTimeStep (mod_ImplicitCommon.f90:115-119)
    int bad = 0;
    for (int q = threadIdx.x; q < ncs * 4; q += blockDim.x) {
        sW[q] = B.W[c0 * 4 + q];
        sR[q] = I.rate_w[c0 * 4 + q];
    }
    bool dead = false;   // the set-up failed in this slab (ST_GETPRIMARY set): the CTA only meets the barriers
    if (first) {
        if ((!last || sweeps > 1) && s == 0 && threadIdx.x == 0) { I.mask[0] = 0xffffffffu; I.mask[1] = 0xffffffffu; }
        int prep_bad = 0;
        for (int q = threadIdx.x; q < ncs * 4; q += blockDim.x) {
            double gam, foi[4], foj[4];
            if (!pr_prep_item(P, B, Q, I, c0 + (q >> 2), q & 3, gam, foi, foj)) prep_bad = 1;
            sG[q] = gam;
#pragma unroll
            for (int k = 0; k < 4; ++k) { sFi[k * ncf + q] = foi[k]; sFj[k * ncf + q] = foj[k]; }
        }
        dead = __syncthreads_or(prep_bad) != 0;   // the sequence has stopped (ST_GETPRIMARY)
        if (dead && sweeps == 1) return;
    } else {
        for (int q = threadIdx.x; q < ncs * 4; q += blockDim.x) sG[q] = I.pr_gamma[c0 * 4 + q];
        for (int q = threadIdx.x; q < ncs * 16; q += blockDim.x) {
            sFi[(q & 3) * ncf + (q >> 2)] = I.pr_foi[c0 * 16 + q];
            sFj[(q & 3) * ncf + (q >> 2)] = I.pr_foj[c0 * 16 + q];
        }
    }
    // interior and halo cells: correction, state, flux pair (halo rows beyond a wall stay unused); Xin
    // nullptr: the zero correction.  The halo corrections come from other CTAs of this launch after a
    // grid barrier, so they are read past L1.
    auto load_cells = [&](int l0, const double* Xin) {
        for (int l = l0 + (int)threadIdx.x; l < nall; l += blockDim.x) {
            int g;
            if (l < ncs) g = c0 + l;
            else if (l < ncs + rows) g = (s * rows + (l - ncs)) * nx + (nx - 1);
            else if (l < ncs + 2 * rows) g = (s * rows + (l - ncs - rows)) * nx;
            else if (l < ncs + 2 * rows + nx) g = s * rows > 0 ? (s * rows - 1) * nx + (l - ncs - 2 * rows) : -1;
            else g = (s + 1) * rows < ny ? ((s + 1) * rows) * nx + (l - ncs - 2 * rows - nx) : -1;
            double y[4] = {0.0, 0.0, 0.0, 0.0}, t[4] = {1.0, 0.0, 0.0, 1.0};
            if (g >= 0) {
#pragma unroll
                for (int k = 0; k < 4; ++k) { y[k] = Xin ? __ldcg(Xin + g * 4 + k) : 0.0; t[k] = B.W[g * 4 + k] + y[k]; }
            }
            double fx[4], fy[4];
            euler_flux_pair(t, euler_prim(P.gm1, t), fx, fy);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                sY[l * 4 + k] = y[k];
                sT[l * 4 + k] = t[k];
                sF[l * 8 + k] = fx[k];
                sF[l * 8 + 4 + k] = fy[k];
            }
        }
    };
    load_cells(0, first ? nullptr : X);
    // the diagonal 1/dt_ps + 0.5 * sum_faces(L * gamma) / area is fixed through the sweeps; the face
    // products are rounded before they are summed in face order, as the reference loop does
    __syncthreads();
    for (int cl = threadIdx.x; cl < ncs; cl += blockDim.x) {
        const double* gm = sG + cl * 4;
        double sg = 0.0;
        sg = sg + __dmul_rn(P.dy, gm[0]);
        sg = sg + __dmul_rn(P.dy, gm[1]);
        sg = sg + __dmul_rn(P.dx, gm[2]);
        sg = sg + __dmul_rn(P.dx, gm[3]);
        const double diag = 1.0 / dtp + div_area(0.5 * sg, P);
        if (!(isfinite(diag) && diag > 0.0)) bad = 1;
        sD[cl] = diag;
        sRd[cl] = 1.0 / diag;
    }
    pr_wall_terms(P, Q, s, rows, sW, sY, sWf, sWd);
    __syncthreads();
    const int ndiag = rows + nx - 1;
    for (int sw = 0; sw < sweeps; ++sw) {
        double* out = (sw & 1) ? X : Y;
        if (sw > 0) {   // the previous sweep's halo corrections, then this sweep's wall terms
            if (!pr_grid_barrier(I.prbar)) {
                if (threadIdx.x == 0) stop_with(I, B.status, ST_TIMEOUT);
                return;
            }
            if (__ldcg(I.state + IS_STOP) != 0.0) return;   // a slab of the previous sweep failed
            load_cells(ncs, (sw & 1) ? Y : X);
            __syncthreads();
            pr_wall_terms(P, Q, s, rows, sW, sY, sWf, sWd);
            __syncthreads();
        }
        for (int pass = 0; pass < 2 && !dead; ++pass) {
            if (pass == 1) {   // the wall-row cells relaxed in the first pass
                __syncthreads();
                pr_wall_terms(P, Q, s, rows, sW, sY, sWf, sWd);
                __syncthreads();
            }
            if ((int)threadIdx.x >= wave_warps * 32) continue;
            for (int dd = 0; dd < ndiag; ++dd) {
                const int d = pass == 0 ? dd : ndiag - 1 - dd;
                for (int t0 = 0; t0 < dcells; t0 += D) {
                    int i = 0, jl = 0;
                    const bool act = (int)threadIdx.x < wave && diag_cell(d, tc + t0, rows, nx, i, jl);
                    const int j = s * rows + jl, cl = jl * nx + i;
                    double tm = 0.0;
                    if (act) {   // lane = component m of cell (i, j)
                        double sdt = 0.0, sgn = 0.0;
    #pragma unroll
                        for (int f = 0; f < 4; ++f) {
                            const int dir = (f >> 1) * 4 + m;
                            const bool neg = (f & 1) == 0;   // left and bottom faces: normals (-1,0), (0,-1)
                            const double flen = f < 2 ? P.dy : P.dx;
                            const double fo = sF[cl * 8 + dir];
                            const double fi = neg ? -fo : fo;
                            const int nl = pr_neighbour(i, jl, j, f, rows, nx, ny);
                            double fj, dnb;
                            if (nl < 0) {
                                const int w = (f == 3 ? nx : 0) + i;
                                fj = sWf[w * 4 + m];
                                dnb = sWd[w * 4 + m];
                            } else {
                                const double fn = sF[nl * 8 + dir];
                                fj = neg ? -fn : fn;
                                dnb = sY[nl * 4 + m];
                            }
                            const double dti = fi - sFi[m * ncf + cl * 4 + f];
                            const double sm4 = dti + (fj - sFj[m * ncf + cl * 4 + f]);
                            if (!isfinite(sm4)) bad = 1;
                            sdt = __dadd_rn(sdt, __dmul_rn(flen, sm4));
                            sgn = __dadd_rn(sgn, __dmul_rn(__dmul_rn(flen, sG[cl * 4 + f]), dnb));
                        }
                        const double rhs = sR[cl * 4 + m] - div_area(0.5 * 1.0 * sdt, P) + div_area(0.5 * 1.0 * sgn, P);
                        if (!isfinite(rhs)) bad = 1;
                        const double y = div_by_recip(rhs, sD[cl], sRd[cl]);
                        tm = sW[cl * 4 + m] + y;
                        sY[cl * 4 + m] = y;
                        sT[cl * 4 + m] = tm;
                    }
                    // the relaxed state's flux pair, its components gathered from the cell's 4 lanes (every
                    // lane of the warp takes part in the shuffles)
                    double t[4];
    #pragma unroll
                    for (int k = 0; k < 4; ++k) t[k] = __shfl_sync(0xffffffffu, tm, (threadIdx.x & ~3) + k);
                    if (act) {
                        double fx[4], fy[4];
                        euler_flux_pair(t, euler_prim(P.gm1, t), fx, fy);
                        sF[cl * 8 + m] = m == 0 ? fx[0] : (m == 1 ? fx[1] : (m == 2 ? fx[2] : fx[3]));
                        sF[cl * 8 + 4 + m] = m == 0 ? fy[0] : (m == 1 ? fy[1] : (m == 2 ? fy[2] : fy[3]));
                    }
                }
                pr_wave_sync(wave_warps);
            }
        }
        __syncthreads();
        if (!dead)
            for (int q = threadIdx.x; q < ncs * 4; q += blockDim.x) out[c0 * 4 + q] = sY[q];
        if (sw < sweeps - 1 && __syncthreads_or(bad) && threadIdx.x == 0) stop_with(I, B.status, ST_NONFINITE_STATE);
    }
    if (dead) return;
    if (last) {
        const int lv = alpha_levels(Q.min_alpha);
        for (int cl = threadIdx.x; cl < ncs; cl += blockDim.x) {
            unsigned mask = 0u;
            double a = 1.0;
            for (int k = 0; k <= lv; ++k) {
                double t[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) t[q] = sW[cl * 4 + q] + a * sY[cl * 4 + q];
                if (is_physical(t)) mask |= 1u << k;
                a = 0.5 * a;
            }
            atomicAnd(I.mask, mask);
        }
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) stop_with(I, B.status, ST_NONFINITE_STATE);
}

// BuildPredictedEquilibrium (mod_ImplicitMicro.f90:43-88), second-order branch.
template <int VPT, int NTMAX>
__global__ void __launch_bounds__(NTMAX, 512 / NTMAX) k_im_equilibrium(LoParams P, LoBuffers B, ImParams Q,
                                                                       ImBuffers I, const double* D) {
    if (I.state[IS_STOP] != 0.0) return;
    __shared__ double red[16 * 64];
    __shared__ double rout[kRedSlots];
    __shared__ double sc[32];   // [0..3] prim_old [4..7] prim_tilde [8] tau_tilde [9] ok [12..15] lambda
                                // [16..19] old-state lambda, [20] tau_old (high order)
    const int nv = P.nvel, tid = threadIdx.x, c = blockIdx.x;
    if (tid == 0) {
        const int m = first_bit(I.mask[0]);
        const double a = m < 0 ? 0.0 : pow2neg(m);
        double wt[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) { wt[q] = B.W[c * 4 + q] + a * D[c * 4 + q]; I.wt[c * 4 + q] = wt[q]; }
        Prim po, pt;
        double tt = 1.0;
        bool ok = m >= 0 && get_primary(P.gm1, B.W + c * 4, po) && get_primary(P.gm1, wt, pt);
        ok = ok && get_tau(P.mu_ref, P.omega, pt, tt);
        double to = 1.0;
        if (Q.high_order) ok = ok && get_tau(P.mu_ref, P.omega, po, to);
        sc[20] = to;
        if (!ok) { po.r = pt.r = 1.0; po.U = po.V = pt.U = pt.V = 0.0; po.L = pt.L = 1.0; tt = 1.0; sc[20] = 1.0; }
        sc[0] = po.r; sc[1] = po.U; sc[2] = po.V; sc[3] = po.L;
        sc[4] = pt.r; sc[5] = pt.U; sc[6] = pt.V; sc[7] = pt.L; sc[8] = tt; sc[9] = ok ? 1.0 : 0.0;
        I.tau_t[c] = tt;
        if (c == 0) I.state[IS_MALPHA] = a;
        if (!ok) stop_with(I, B.status, m < 0 ? ST_ALPHA : ST_GETPRIMARY);
    }
    __syncthreads();
    const Prim po{sc[0], sc[1], sc[2], sc[3]}, pt{sc[4], sc[5], sc[6], sc[7]};
    double acc[14];
    acc[0] = acc[1] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {   // q_frozen = GetHeatFlux_Vec(h, b, prim_old)
        const Slot s = slot(r, nv);
        const double wk = s.ok ? B.w[s.kk] : 0.0;
        const double dvn = B.u[s.kk] - po.U, dvt = B.v[s.kk] - po.V, v2 = dvn * dvn + dvt * dvt;
        const size_t q = (size_t)c * nv + s.kk;
        const double t = 0.5 * wk * (v2 * B.h[q] + B.b[q]);
        acc[0] += t * dvn;
        acc[1] += t * dvt;
    }
    block_reduce<2, 0>(acc, red, rout);
    const double q0 = acc[0], q1 = acc[1];
    double E[VPT], F[VPT];
    {
        const double pref = pt.r * (pt.L / kPi), bfac = (double)P.ck / (2.0 * pt.L);
        const double coeff = 0.8 * (1.0 - P.pr) * pt.L * pt.L / pt.r, c2ck = 2.0 / (double)P.ck;
        acc[0] = acc[1] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            const double dvn = B.u[s.kk] - pt.U, dvt = B.v[s.kk] - pt.V, v2 = dvn * dvn + dvt * dvt;
            const double H = pref * exp(-pt.L * v2), Bm = H * bfac;
            const double qd = dvn * q0 + dvt * q1, sH = 2.0 * pt.L * v2 - 4.0;
            E[r] = H + coeff * qd * sH * H;
            F[r] = Bm + coeff * qd * (sH + c2ck) * Bm;
            acc[0] = fmax(acc[0], s.ok ? fabs(E[r]) : 0.0);
            acc[1] = fmax(acc[1], s.ok ? fabs(F[r]) : 0.0);
        }
        block_reduce<0, 2>(acc, red, rout);
    }
    const double se = fmax(acc[0], 1.0), sf = fmax(acc[1], 1.0);
#pragma unroll
    for (int m = 0; m < 14; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double wk = s.ok ? B.w[s.kk] : 0.0;
        moment_add(wk, B.u[s.kk], B.v[s.kk], E[r], F[r], acc);
        gram_add(wk, fmax(fabs(E[r]), kEps * se), fmax(fabs(F[r]), kEps * sf), B.u[s.kk], B.v[s.kk], acc + 4);
    }
    block_reduce_smem<14, 0>(acc, red, rout);
    if (tid == 0) {
        double rhs[4], gm[16], l[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) rhs[m] = I.wt[c * 4 + m] - rout[m];
        gram_expand(rout + 4, gm);
        const bool ok = solve_dense4(gm, rhs, l);
#pragma unroll
        for (int m = 0; m < 4; ++m) sc[12 + m] = ok ? l[m] : 0.0;
        if (!ok) stop_with(I, B.status, ST_PROJECTION);
    }
    // High order: the old-state Maxwell + Shakhov with q_frozen, projected onto W_old
    // (low_collision_old, mod_ImplicitMicro.f90:66-79)
    double Eo[VPT], Fo[VPT], seo = 1.0, sfo = 1.0;
    if (Q.high_order) {
        const double pref = po.r * (po.L / kPi), bfac = (double)P.ck / (2.0 * po.L);
        const double coeff = 0.8 * (1.0 - P.pr) * po.L * po.L / po.r, c2ck = 2.0 / (double)P.ck;
        double am[2] = {0.0, 0.0};
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            const double dvn = B.u[s.kk] - po.U, dvt = B.v[s.kk] - po.V, v2 = dvn * dvn + dvt * dvt;
            const double H = pref * exp(-po.L * v2), Bm = H * bfac;
            const double qd = dvn * q0 + dvt * q1, sH = 2.0 * po.L * v2 - 4.0;
            Eo[r] = H + coeff * qd * sH * H;
            Fo[r] = Bm + coeff * qd * (sH + c2ck) * Bm;
            am[0] = fmax(am[0], s.ok ? fabs(Eo[r]) : 0.0);
            am[1] = fmax(am[1], s.ok ? fabs(Fo[r]) : 0.0);
        }
        block_reduce<0, 2>(am, red, rout);
        seo = fmax(am[0], 1.0); sfo = fmax(am[1], 1.0);
        double ag[14];
#pragma unroll
        for (int m = 0; m < 14; ++m) ag[m] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            const double wk = s.ok ? B.w[s.kk] : 0.0;
            moment_add(wk, B.u[s.kk], B.v[s.kk], Eo[r], Fo[r], ag);
            gram_add(wk, fmax(fabs(Eo[r]), kEps * seo), fmax(fabs(Fo[r]), kEps * sfo), B.u[s.kk], B.v[s.kk], ag + 4);
        }
        block_reduce_smem<14, 0>(ag, red, rout);
        if (tid == 0) {
            double rhs[4], gm[16], l[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) rhs[m] = B.W[c * 4 + m] - rout[m];
            gram_expand(rout + 4, gm);
            const bool ok = solve_dense4(gm, rhs, l);
#pragma unroll
            for (int m = 0; m < 4; ++m) sc[16 + m] = ok ? l[m] : 0.0;
            if (!ok) stop_with(I, B.status, ST_PROJECTION);
        }
    }
    __syncthreads();
    double lam[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) lam[m] = sc[12 + m];
    double lamo[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) lamo[m] = sc[16 + m];
    const double tau_old = sc[20];
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0, e = 0.5 * (uk * uk + vk * vk);
        const double Ep = E[r] + fmax(fabs(E[r]), kEps * se) * (lam[0] + uk * lam[1] + vk * lam[2] + e * lam[3]);
        const double Fp = F[r] + 0.5 * fmax(fabs(F[r]), kEps * sf) * lam[3];
        moment_add(wk, uk, vk, Ep, Fp, acc);
        if (s.ok) {   // RelaxMicroPoint's velocity-local right-hand side (mod_ImplicitMicro.f90:458-470)
            const size_t q = (size_t)c * nv + s.k;
            double rh = I.stream_h[q] + (Ep - B.h[q]) / sc[8];
            double rb = I.stream_b[q] + (Fp - B.b[q]) / sc[8];
            if (Q.high_order) {
                const double Eop = Eo[r] + fmax(fabs(Eo[r]), kEps * seo) * (lamo[0] + uk * lamo[1] + vk * lamo[2] + e * lamo[3]);
                const double Fop = Fo[r] + 0.5 * fmax(fabs(Fo[r]), kEps * sfo) * lamo[3];
                const double lh = (Eop - B.h[q]) / tau_old, lb = (Fop - B.b[q]) / tau_old;
                rh = rh + B.pcol_h[q] - lh;
                rb = rb + B.pcol_b[q] - lb;
            }
            I.rhs_h[q] = rh;
            I.rhs_b[q] = rb;
        }
    }
    block_reduce_smem<4, 0>(acc, red, rout);
    if (tid == 0) {
        double rs = 1.0, err = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) { rs = fmax(rs, fabs(I.wt[c * 4 + m])); err = fmax(err, fabs(rout[m] - I.wt[c * 4 + m])); }
        if (!(err <= 1.0e-10 * rs)) stop_with(I, B.status, ST_PROJECTION);
    }
}

// -------------------------------------------------------------------------------------------
// One LU-SGS stage: RelaxMicroPoint (mod_ImplicitMicro.f90:444-487) as a hyperplane wavefront.
// Per velocity only upwind neighbours couple, and in the reference's sweep order (forward j up,
// i up; backward j down, i down) a cell reads updated values only from the previous cells of its
// row and column, so the cells of one anti-diagonal of a slab are independent.  A CTA owns one
// slab and 32 velocities: lane = velocity, warp = cell of the current diagonal.  The slab's
// corrections for those velocities stay in shared memory: zero at the start of the forward stage
// (all corrections were reset); the forward result at the start of the backward stage, overwritten
// cell by cell, so that a neighbour read there returns the backward value once that neighbour has
// been relaxed and the forward value before.  Halos (seams and the x wrap) read the forward result
// in global memory in the backward stage and 0 in the forward stage; wall faces use the closure
// frozen from the forward correction.
// A velocity has one inflow face per direction (u > 0: left, u < 0: right; v > 0: bottom, v < 0:
// top); the outflow faces add exact zeros to the right-hand side and their u_n L / area to the
// diagonal, so the sums below keep the reference's face order.  The next cell's right-hand side
// and diagonal are prefetched one diagonal ahead.
template <bool BACKWARD>
__global__ void __launch_bounds__(256) k_im_lusgs(LoParams P, LoBuffers B, ImParams Q, ImBuffers I) {
    if (I.state[IS_STOP] != 0.0) return;
    extern __shared__ double sm[];
    const int nv = P.nvel, nx = P.nx, ny = P.ny;
    const int s = blockIdx.y, rows = ny / Q.nslab, ncs = rows * nx, c0 = s * ncs;
    const int lane = threadIdx.x & 31, k = blockIdx.x * 32 + lane, tc = threadIdx.x >> 5, D = blockDim.x >> 5;
    const bool kok = k < nv;
    const int kk = kok ? k : nv - 1;
    double* sh = sm;              // [ncs][32]
    double* sb = sm + ncs * 32;
    for (int q = threadIdx.x; q < ncs * 32; q += blockDim.x) {
        const int kq = blockIdx.x * 32 + (q & 31);
        double vh = 0.0, vb = 0.0;
        if (BACKWARD && kq < nv) {
            const size_t g = (size_t)(c0 + (q >> 5)) * nv + kq;
            vh = I.dFh[g];
            vb = I.dFb[g];
        }
        sh[q] = vh;
        sb[q] = vb;
    }
    const double dtp = B.dt[0] * Q.ncfl / P.cfl;
    const double idtp = 1.0 / dtp;
    const double uk = B.u[kk], vk = B.v[kk];
    const double un[4] = {-uk, uk, -vk, vk};   // u*nx_out + v*ny_out of faces left, right, bottom, top
    const double len[4] = {P.dy, P.dy, P.dx, P.dx};
    double cd[4], cm[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        cd[f] = div_area(1.0 * fmax(un[f], 0.0) * len[f], P);   // outflow part of the diagonal
        cm[f] = 1.0 * fmin(un[f], 0.0) * len[f];                 // inflow coupling (divided by area below)
    }
    const int fx = un[0] < 0.0 ? 0 : (un[1] < 0.0 ? 1 : -1);   // inflow x face
    const int fy = un[2] < 0.0 ? 2 : (un[3] < 0.0 ? 3 : -1);   // inflow y face
    const double cmx = fx == 0 ? cm[0] : (fx == 1 ? cm[1] : 0.0);
    const double cmy = fy == 2 ? cm[2] : (fy == 3 ? cm[3] : 0.0);
    const double cdx = cd[0] + cd[1], cdy = cd[2] + cd[3];      // one of each pair is +0: exact
    double whu = 0.0, wbu = 0.0;
    if (BACKWARD && fy >= 2) { const int w = fy - 2; whu = I.wall_hu[w * nv + kk]; wbu = I.wall_bu[w * nv + kk]; }
    double* outh = BACKWARD ? I.dBh : I.dFh;
    double* outb = BACKWARD ? I.dBb : I.dFb;
    const int dcells = rows < nx ? rows : nx;
    const int nchunk = (dcells + D - 1) / D;
    const int nit = (rows + nx - 1) * nchunk;
    // work item `it`: diagonal it / nchunk, cell (it % nchunk) * D + tc of it (in sweep order)
    auto locate = [&](int it, int& i, int& jl) -> bool {
        const int d = it / nchunk;
        const bool a = diag_cell(d, (it - d * nchunk) * D + tc, rows, nx, i, jl);
        if (BACKWARD) { i = nx - 1 - i; jl = rows - 1 - jl; }
        return a && kok;
    };
    int ni = 0, njl = 0;
    bool nact = locate(0, ni, njl);
    double nrh = 0.0, nrb = 0.0, ndg = 1.0;
    if (nact) {
        const int c = c0 + njl * nx + ni;
        nrh = I.rhs_h[(size_t)c * nv + k]; nrb = I.rhs_b[(size_t)c * nv + k];
        ndg = ((idtp + 1.0 / I.tau_t[c]) + cdx) + cdy;
    }
    __syncthreads();
    bool ok = true;
    for (int it = 0; it < nit; ++it) {
        const bool act = nact;
        const int i = ni, jl = njl;
        double rh = nrh, rb = nrb;
        const double diag = ndg;
        if (it + 1 < nit) {
            nact = locate(it + 1, ni, njl);
            if (nact) {
                const int c = c0 + njl * nx + ni;
                nrh = I.rhs_h[(size_t)c * nv + k]; nrb = I.rhs_b[(size_t)c * nv + k];
                ndg = ((idtp + 1.0 / I.tau_t[c]) + cdx) + cdy;
            }
        }
        if (act) {
            const int j = s * rows + jl, cl = jl * nx + i;
            double nh = 0.0, nb = 0.0;   // x inflow neighbour
            if (fx == 0) {
                if (i > 0) { nh = sh[(cl - 1) * 32 + lane]; nb = sb[(cl - 1) * 32 + lane]; }
                else if (BACKWARD) { const size_t qn = (size_t)(j * nx + nx - 1) * nv + k; nh = I.dFh[qn]; nb = I.dFb[qn]; }
            } else if (fx == 1 && BACKWARD) {
                if (i < nx - 1) { nh = sh[(cl + 1) * 32 + lane]; nb = sb[(cl + 1) * 32 + lane]; }
                else { const size_t qn = (size_t)(j * nx) * nv + k; nh = I.dFh[qn]; nb = I.dFb[qn]; }
            }
            rh = rh - div_area(cmx * nh, P);
            rb = rb - div_area(cmx * nb, P);
            nh = 0.0; nb = 0.0;          // y inflow neighbour
            if (fy == 2) {
                if (j == 0) {
                    if (BACKWARD) { nh = I.wall_drho[i] * whu; nb = I.wall_drho[i] * wbu; }
                } else if (jl > 0) {
                    nh = sh[(cl - nx) * 32 + lane]; nb = sb[(cl - nx) * 32 + lane];
                } else if (BACKWARD) {
                    const size_t qn = (size_t)((j - 1) * nx + i) * nv + k;
                    nh = I.dFh[qn]; nb = I.dFb[qn];
                }
            } else if (fy == 3 && BACKWARD) {
                if (j == ny - 1) { nh = I.wall_drho[nx + i] * whu; nb = I.wall_drho[nx + i] * wbu; }
                else if (jl < rows - 1) { nh = sh[(cl + nx) * 32 + lane]; nb = sb[(cl + nx) * 32 + lane]; }
                else { const size_t qn = (size_t)((j + 1) * nx + i) * nv + k; nh = I.dFh[qn]; nb = I.dFb[qn]; }
            }
            rh = rh - div_area(cmy * nh, P);
            rb = rb - div_area(cmy * nb, P);
            ok = ok && diag > 0.0 && isfinite(diag) && isfinite(rh) && isfinite(rb);
            const double oh = rh / diag, ob = rb / diag;
            sh[cl * 32 + lane] = oh;
            sb[cl * 32 + lane] = ob;
            const size_t q = (size_t)(c0 + cl) * nv + k;
            outh[q] = oh;
            outb[q] = ob;
        }
        if ((it + 1) % nchunk == 0) __syncthreads();
    }
    if (!ok) stop_with(I, B.status, ST_NONFINITE_STATE);
}

// Frozen diffuse-wall closure of each wall cell for the backward stage (PrepareFrozenMicroWallState
// -> ComputeDiffuseWallFaceDelta, mod_ImplicitBoundary.f90:282-326), from its forward correction.
template <int VPT, int NTMAX>
__global__ void __launch_bounds__(NTMAX) k_im_wall_closure(LoParams P, LoBuffers B, ImParams Q, ImBuffers I) {
    if (I.state[IS_STOP] != 0.0) return;
    __shared__ double red[16 * 64];
    __shared__ double rout[kRedSlots];
    const int nv = P.nvel, nx = P.nx;
    const int top = blockIdx.x >= nx ? 1 : 0, i = blockIdx.x - top * nx;
    const int c = (top ? P.ny - 1 : 0) * nx + i;
    double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double wk = s.ok ? B.w[s.kk] : 0.0;
        double vn, hu, bu;
        wall_frame(P, top, B.u[s.kk], B.v[s.kk], vn, hu, bu);
        const double sel = vn < 0.0 ? 1.0 : 0.0;
        acc[0] += wk * vn * I.dFh[(size_t)c * nv + s.kk] * (1.0 - sel);
        acc[1] += wk * vn * hu * sel;
        acc[2] += fabs(wk * vn * hu * sel);
    }
    block_reduce_smem<3, 0>(acc, red, rout);
    if (threadIdx.x == 0) {
        const double refl = rout[1];
        if (fabs(refl) <= 1000.0 * kEps * fmax(rout[2], DBL_MIN)) stop_with(I, B.status, ST_NONFINITE_STATE);
        I.wall_drho[top * nx + i] = -rout[0] / refl;
    }
}

// FindAdmissibleMicroAlpha without the negative-fraction test (mod_SteadyImplicit.f90:53-117 with
// ClassifyMicroCandidate :200-270): per cell, finite candidates and physical candidate moments.
template <int VPT, int NTMAX>
__global__ void __launch_bounds__(NTMAX, 512 / NTMAX) k_im_micro_alpha(LoParams P, LoBuffers B, ImParams Q,
                                                                       ImBuffers I) {
    if (I.state[IS_STOP] != 0.0) return;
    __shared__ double red[16 * 64];
    __shared__ double rout[kRedSlots];
    const int nv = P.nvel, c = blockIdx.x;
    const int lv = alpha_levels(Q.min_alpha);
    // moments of h + a*dh for every level a (linear in a), and finiteness
    double acc[9];
#pragma unroll
    for (int m = 0; m < 9; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double wk = s.ok ? B.w[s.kk] : 0.0;
        const size_t q = (size_t)c * nv + s.kk;
        moment_add(wk, B.u[s.kk], B.v[s.kk], B.h[q], B.b[q], acc);
        moment_add(wk, B.u[s.kk], B.v[s.kk], I.dBh[q], I.dBb[q], acc + 4);
        const bool fin = isfinite(B.h[q]) && isfinite(B.b[q]) && isfinite(I.dBh[q]) && isfinite(I.dBb[q]);
        acc[8] = fmax(acc[8], fin ? 0.0 : 1.0);
    }
    block_reduce_smem<8, 1>(acc, red, rout);
    if (threadIdx.x == 0) {
        unsigned mask = 0u;
        double a = 1.0;
        for (int m = 0; m <= lv; ++m) {
            double t[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) t[q] = rout[q] + a * rout[4 + q];
            if (rout[8] == 0.0 && is_physical(t)) mask |= 1u << m;
            a = 0.5 * a;
        }
        atomicAnd(I.mask + 1, mask);
    }
}

// Update h, b with the admissible alpha, RecoverMacroFromKineticState, the moment gate, and the
// mass before the closed-mass rescale (MassStatistics, mod_ClosedCouetteMass.f90:173-204).
template <int VPT, int NTMAX>
__global__ void __launch_bounds__(NTMAX, 512 / NTMAX) k_im_apply(LoParams P, LoBuffers B, ImParams Q, ImBuffers I) {
    if (I.state[IS_STOP] != 0.0) return;
    __shared__ double red[16 * 64];
    __shared__ double rout[kRedSlots];
    __shared__ double s_alpha;
    const int nv = P.nvel, c = blockIdx.x, tid = threadIdx.x;
    if (tid == 0) {
        const int m = first_bit(I.mask[1]);
        s_alpha = m < 0 ? -1.0 : pow2neg(m);
    }
    __syncthreads();
    const double a = s_alpha;
    if (a < 0.0) {   // no admissible alpha down to Implicit_MinAlpha: the step is rejected
        if (tid == 0 && c == 0) stop_with(I, B.status, ST_ALPHA);
        return;
    }
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double wk = s.ok ? B.w[s.kk] : 0.0;
        const size_t q = (size_t)c * nv + s.kk;
        const double hn = B.h[q] + a * I.dBh[q], bn = B.b[q] + a * I.dBb[q];
        moment_add(wk, B.u[s.kk], B.v[s.kk], hn, bn, acc);
        if (s.ok) { B.h[q] = hn; B.b[q] = bn; }
    }
    block_reduce_smem<4, 0>(acc, red, rout);
    if (tid == 0) {
        double wn[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) { wn[m] = rout[m]; B.W[c * 4 + m] = wn[m]; }
        if (!is_physical(wn)) stop_with(I, B.status, ST_NONFINITE_STATE);
        I.cell[(size_t)c * kImCell + 0] = P.area * wn[0];
    }
    // last CTA: the alpha policy (CheckR5Policy) and mass_scale = M0 / mass (RescaleClosedMass)
    __shared__ unsigned s_last;
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = (atomicAdd(I.counter, 1u) == (unsigned)(gridDim.x - 1)) ? 1u : 0u;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double m0 = 0.0;
    for (int cc = tid; cc < P.nx * P.ny; cc += blockDim.x) m0 += __ldcg(I.cell + (size_t)cc * kImCell);
    block_reduce<1, 0>(&m0, red, rout);
    if (tid == 0) {
        I.state[IS_ALPHA] = a;
        I.state[IS_MOMENT] = 0.0;   // W was just set to the moments of (h, b)
        if (a != 1.0 || I.state[IS_MALPHA] != 1.0) stop_with(I, B.status, ST_ALPHA);
        const double scale = Q.mass_rescale ? I.state[IS_M0] / m0 : 1.0;
        if (!(isfinite(scale) && scale > 0.0)) stop_with(I, B.status, ST_NONFINITE_STATE);
        I.state[IS_MASS_SCALE] = scale;
        *I.counter = 0u;
    }
}

// RescaleClosedMass (mod_ClosedCouetteMass.f90:243-313): W, h, b *= M0 / mass.
__global__ void k_im_rescale(LoParams P, LoBuffers B, ImParams Q, ImBuffers I) {
    if (I.state[IS_STOP] != 0.0 || !Q.mass_rescale) return;
    const double s = I.state[IS_MASS_SCALE];
    const size_t n = (size_t)P.nx * P.ny * P.nvel;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        B.h[q] = s * B.h[q];
        B.b[q] = s * B.b[q];
        if (q < (size_t)P.nx * P.ny * 4) B.W[q] = s * B.W[q];
    }
}

// InitializeClosedMass (mod_ClosedCouetteMass.f90:212-241): persistent M0 of the cold start.
__global__ void k_im_init(LoParams P, LoBuffers B, ImParams Q, ImBuffers I) {
    __shared__ double red[16 * 64];
    __shared__ double rout[kRedSlots];
    double m = 0.0;
    for (int c = threadIdx.x; c < P.nx * P.ny; c += blockDim.x) m += P.area * B.W[c * 4];
    block_reduce<1, 0>(&m, red, rout);
    if (threadIdx.x == 0) {
        for (int q = 0; q < IS_COUNT; ++q) I.state[q] = 0.0;
        I.state[IS_M0] = m;
        I.state[IS_MASS_SCALE] = 1.0;
        I.state[IS_ALPHA] = 1.0;
        I.state[IS_MALPHA] = 1.0;
        *I.counter = 0u;
        *I.stopw = 0u;
    }
    for (int k = threadIdx.x; k < P.nvel; k += blockDim.x) {
        for (int w = 0; w < 2; ++w) {
            double vn, hu, bu;
            wall_frame(P, w, B.u[k], B.v[k], vn, hu, bu);
            I.wall_hu[w * P.nvel + k] = hu;
            I.wall_bu[w * P.nvel + k] = bu;
        }
    }
}

// -------------------------------------------------------------------------------------------
int lo_vpt(int nvel);
int lo_threads(int nvel);
cudaError_t launch_lo_slopes(const LoParams& P, const LoBuffers& B, cudaStream_t s);
cudaError_t launch_lo_faces(const LoParams& P, const LoBuffers& B, cudaStream_t s);
cudaError_t launch_lo_walls(const LoParams& P, const LoBuffers& B, cudaStream_t s);
cudaError_t launch_lo_timestep(const LoParams& P, const LoBuffers& B, cudaStream_t s);

cudaError_t launch_im_init(const LoParams& P, const LoBuffers& B, const ImParams& Q, const ImBuffers& I,
                           cudaStream_t s) {
    k_im_init<<<1, 256, 0, s>>>(P, B, Q, I);
    return cudaGetLastError();
}

template <int VPT, int NTMAX>
static void im_cell_kernels(int which, const LoParams& P, const LoBuffers& B, const ImParams& Q, const ImBuffers& I,
                            const double* D, cudaStream_t s) {
    const int nc = P.nx * P.ny, nt = lo_threads(P.nvel);
    switch (which) {
        case 0:
            if (Q.high_order) k_im_residual_s2<VPT, NTMAX, false><<<nc, nt, 0, s>>>(P, B, Q, I);
            else k_im_residual<VPT, NTMAX, false><<<nc, nt, 0, s>>>(P, B, Q, I);
            break;
        case 1:
            if (Q.high_order) k_im_residual_s2<VPT, NTMAX, true><<<nc, nt, 0, s>>>(P, B, Q, I);
            else k_im_residual<VPT, NTMAX, true><<<nc, nt, 0, s>>>(P, B, Q, I);
            break;
        case 2: k_im_equilibrium<VPT, NTMAX><<<nc, nt, 0, s>>>(P, B, Q, I, D); break;
        case 3: k_im_wall_closure<VPT, NTMAX><<<2 * P.nx, nt, 0, s>>>(P, B, Q, I); break;
        case 4: k_im_micro_alpha<VPT, NTMAX><<<nc, nt, 0, s>>>(P, B, Q, I); break;
        case 5: k_im_apply<VPT, NTMAX><<<nc, nt, 0, s>>>(P, B, Q, I); break;
    }
}

static cudaError_t im_cell(int which, const LoParams& P, const LoBuffers& B, const ImParams& Q, const ImBuffers& I,
                           const double* D, cudaStream_t s) {
    if (lo_vpt(P.nvel) == 4) im_cell_kernels<4, 256>(which, P, B, Q, I, D, s);
    else im_cell_kernels<5, 512>(which, P, B, Q, I, D, s);
    return cudaGetLastError();
}

// The flux evaluation of a pseudo-step (Interpolation + Evolution) on the main stream, the wall
// faces beside the interior faces on the side stream.
static cudaError_t im_fluxes(const LoParams& P, const LoBuffers& B, cudaStream_t s, cudaStream_t s2,
                             cudaEvent_t fork, cudaEvent_t join) {
    cudaError_t e = launch_lo_slopes(P, B, s);
    if (e == cudaSuccess) e = cudaEventRecord(fork, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s2, fork, 0);
    if (e == cudaSuccess) e = launch_lo_walls(P, B, s2);
    if (e == cudaSuccess) e = cudaEventRecord(join, s2);
    if (e == cudaSuccess) e = launch_lo_faces(P, B, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, join, 0);
    return e;
}

// Shared-memory opt-in of the sweep kernels for this slab size (slab rows x nx <= kMaxSlabCells).
cudaError_t prepare_implicit(const LoParams& P, const ImParams& Q) {
    const int rows = P.ny / Q.nslab, ncs = rows * P.nx;
    const int pr_bytes = pr_smem_words(rows, P.nx) * (int)sizeof(double);
    if (ncs > kMaxSlabCells || pr_bytes > 227 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_im_pr2_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize, pr_bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_im_lusgs<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, ncs * 64 * (int)sizeof(double));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_im_lusgs<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, ncs * 64 * (int)sizeof(double));
    return e;
}

// One ImplicitSteady pseudo-step (mod_Solve.f90:84-293 with TimeIntegration_method =
// 'ImplicitSteady' and ClosedCouetteMassRescale): 15 + macro_sweeps kernels with the second-order
// evaluations (3 kernels each), 6 more per evaluation with the S2 one of HighOrderImplicit, no host
// synchronisation.  The TimeStep of the next pseudo-step is taken in the accepted-state residual's last
// CTA, so it is no launch of its own; the caller launches k_lo_timestep once before the first pseudo-step
// of a sequence.
// Returns the number of kernels launched through *launches.
// marks (optional, profile runs only): kImStages + 1 events recorded on s at the start and after
// each stage of kImStageNames.
// Sets the condition of the pre-update evaluation's conditional graph node: 1 when the evaluation must
// run (the previous accepted-state evaluation does not apply: first pseudo-step, or dt changed), 0
// when it is reused, in which case its science columns are copied into the report here, as the
// skipped residual kernel would have done.  One warp.
__global__ void k_im_pre_gate(LoBuffers Bpre, ImBuffers I, cudaGraphConditionalHandle h) {
    const bool cached = eval_cached(Bpre);
    if (threadIdx.x == 0) cudaGraphSetConditional(h, cached ? 0u : 1u);
    if (cached && I.state[IS_STOP] == 0.0 && threadIdx.x < 22)
        I.report[57 + threadIdx.x] = I.state[IS_PRESCI + threadIdx.x];
}

// cond (graph capture only): the pre-update evaluation and its residual go into the body of a
// conditional node that k_im_pre_gate enables, so a reused evaluation launches none of its kernels;
// without it they are launched and return at entry.
cudaError_t enqueue_implicit_step(const LoParams& P, const LoBuffers& B, const ImParams& Q, const ImBuffers& I,
                                  cudaStream_t s, cudaStream_t s2, cudaEvent_t fork, cudaEvent_t join,
                                  long long* launches, cudaEvent_t* marks, const ImCapture* cond) {
    int stage = 0;
    // stage events; under stream capture they are captured as external event nodes, which the graph
    // records as it runs
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    if (marks) cudaStreamIsCapturing(s, &capturing);
    auto mark = [&](cudaError_t e) -> cudaError_t {
        if (e == cudaSuccess && marks)
            e = cudaEventRecordWithFlags(marks[stage++], s,
                                         capturing == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : 0);
        return e;
    };
    // The pre-update evaluation reuses the previous accepted-state evaluation when the state and dt
    // are unchanged since (dt is set by the velocity-table extent unless a cell outruns it).
    LoBuffers Bh = B;          // the evaluation kernels return at entry once the sequence has stopped
    Bh.halt = I.stopw;
    LoBuffers Bpre = Bh;
    Bpre.eval = I.state + IS_EVAL_VALID;
    cudaError_t e = mark(cudaSuccess);
    // TimeStep: taken by the previous pseudo-step's accepted-state residual (or, for the first pseudo-step
    // of a call, by the k_lo_timestep the call launches first)
    if (e == cudaSuccess) e = mark(cudaSuccess);
    if (e == cudaSuccess && cond) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        cudaGraphConditionalHandle h = 0;
        e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd);
        if (e == cudaSuccess && cs != cudaStreamCaptureStatusActive) e = cudaErrorStreamCaptureInvalidated;
        if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault);
        if (e == cudaSuccess) { k_im_pre_gate<<<1, 32, 0, s>>>(Bpre, I, h); e = cudaGetLastError(); }
        if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd);
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeIf;
        np.conditional.size = 1;
        cudaGraphNode_t node = nullptr;
        if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, deps, nd, &np);
        if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(cond->s, np.conditional.phGraph_out[0], nullptr,
                                                                nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t eb = Q.high_order ? s2_enqueue(1, P, Bpre, I.s2, cond->s, cond->s2, cond->fork, cond->join)
                                          : im_fluxes(P, Bpre, cond->s, cond->s2, cond->fork, cond->join);
            if (eb == cudaSuccess) eb = im_cell(0, P, Bpre, Q, I, nullptr, cond->s);
            cudaGraph_t body = nullptr;
            e = cudaStreamEndCapture(cond->s, &body);
            if (eb != cudaSuccess) e = eb;
        }
        if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
    } else {
        if (e == cudaSuccess)                                                     // Interpolation + Evolution
            e = Q.high_order ? s2_enqueue(1, P, Bpre, I.s2, s, s2, fork, join) : im_fluxes(P, Bpre, s, s2, fork, join);
        if (e == cudaSuccess) e = mark(im_cell(0, P, Bpre, Q, I, nullptr, s));   // ComputeResidual + diagnostics
    }
    double* X = I.dwA;
    double* Y = I.dwB;
    const int rows = P.ny / Q.nslab, ncs = rows * P.nx;
    const int dcells = rows < P.nx ? rows : P.nx;                              // longest anti-diagonal
    const int lu_warps = dcells < 8 ? dcells : 8;
    // SolveMacroPR2 with its set-up fused into the first sweep and BuildPredictedMacroState into the
    // last; a single sweep resets the alpha masks beforehand (its CTAs AND into them as they finish)
    if (e == cudaSuccess && Q.macro_sweeps == 1) e = cudaMemsetAsync(I.mask, 0xff, 2 * sizeof(unsigned), s);
    if (e == cudaSuccess) {   // all sweeps in one launch, its slabs meeting at a grid barrier between them
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)Q.nslab);
        cfg.blockDim = dim3(kPrThreads);
        cfg.dynamicSmemBytes = (size_t)pr_smem_words(rows, P.nx) * sizeof(double);
        cfg.stream = s;
        cudaLaunchAttribute coop[1];
        coop[0].id = cudaLaunchAttributeCooperative;
        coop[0].val.cooperative = 1;
        cfg.attrs = coop;
        cfg.numAttrs = Q.macro_sweeps > 1 ? 1 : 0;
        e = cudaLaunchKernelEx(&cfg, k_im_pr2_sweep, P, B, Q, I, X, Y, 1, 1, Q.macro_sweeps);
        if (Q.macro_sweeps % 2 == 1) X = Y;   // the last sweep's corrections (Y when the count is odd)
    }
    e = mark(e);
    if (e == cudaSuccess) e = mark(im_cell(2, P, B, Q, I, X, s));                // BuildPredictedEquilibrium
    const dim3 lu_grid((unsigned)((P.nvel + 31) / 32), (unsigned)Q.nslab);
    const size_t lu_smem = (size_t)ncs * 64 * sizeof(double);
    if (e == cudaSuccess) { k_im_lusgs<false><<<lu_grid, 32 * lu_warps, lu_smem, s>>>(P, B, Q, I); e = mark(cudaGetLastError()); }
    if (e == cudaSuccess) e = mark(im_cell(3, P, B, Q, I, nullptr, s));          // frozen wall closure
    if (e == cudaSuccess) { k_im_lusgs<true><<<lu_grid, 32 * lu_warps, lu_smem, s>>>(P, B, Q, I); e = mark(cudaGetLastError()); }
    if (e == cudaSuccess) e = mark(im_cell(4, P, B, Q, I, nullptr, s));          // FindAdmissibleMicroAlpha
    if (e == cudaSuccess) e = mark(im_cell(5, P, B, Q, I, nullptr, s));          // update + RecoverMacro
    if (e == cudaSuccess) { k_im_rescale<<<148 * 4, 256, 0, s>>>(P, B, Q, I); e = mark(cudaGetLastError()); }
    if (e == cudaSuccess)                                                         // accepted-state evaluation
        e = mark(Q.high_order ? s2_enqueue(1, P, Bh, I.s2, s, s2, fork, join) : im_fluxes(P, Bh, s, s2, fork, join));
    if (e == cudaSuccess) e = mark(im_cell(1, P, B, Q, I, nullptr, s));
    // im_fluxes: slopes, faces, walls.  With cond the pre-update evaluation (and its residual) are a
    // conditional body, not counted here: it runs only when no accepted-state evaluation applies
    // (counted once per sequence by ugks_implicit_init / ugks_implicit_restore); the gate replaces the
    // pre-update residual in the count
    const int evaluation = Q.high_order ? s2_enqueue_kernels(1) : 3;
    if (launches) *launches += 10 + (cond ? evaluation : 2 * evaluation);
    return e;
}

}  // namespace ugks
