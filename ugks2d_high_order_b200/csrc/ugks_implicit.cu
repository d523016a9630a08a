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
//   * PR(2): one thread per slab; each sweep reads other slabs / the x wrap from the previous
//     sweep's complete buffer and its own cells Gauss-Seidel from the current one (double buffer);
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
__device__ __forceinline__ void euler_flux(double gm1, const double w[4], double nx, double ny, double f[4]) {
    const double u = w[1] / w[0], v = w[2] / w[0], un = u * nx + v * ny;
    const double p = gm1 * (w[3] - 0.5 * (w[1] * w[1] + w[2] * w[2]) / w[0]);
    f[0] = w[0] * un;
    f[1] = w[1] * un + p * nx;
    f[2] = w[2] * un + p * ny;
    f[3] = (w[3] + p) * un;
}

// ZhuMovingWallMap (mod_ImplicitBoundary.f90:187-194): ghost state and its exact tangent.
__device__ __forceinline__ void zhu_map(const double w[4], double uw, double vw, double g[4]) {
    g[0] = w[0];
    g[1] = 2.0 * uw * w[0] - w[1];
    g[2] = 2.0 * vw * w[0] - w[2];
    g[3] = w[3] + 2.0 * (uw * uw + vw * vw) * w[0] - 2.0 * uw * w[1] - 2.0 * vw * w[2];
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
template <int VPT, int NTMAX, bool POST>
__global__ void __launch_bounds__(NTMAX, 512 / NTMAX) k_im_residual(LoParams P, LoBuffers B, ImParams Q, ImBuffers I) {
    if (I.state[IS_STOP] != 0.0) return;
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
        if (s.ok) {
            const size_t q = (size_t)c * nv + s.k;
            I.stream_h[q] = sh[r];
            I.stream_b[q] = sb[r];
            B.peq_h[q] = Ep;
            B.peq_b[q] = Fp;
            B.pcol_h[q] = ch;
            B.pcol_b[q] = cb;
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

    // ---- last CTA: global sums (MPI_Allreduce SUM/MAX) and the diagnostics derived from them
    __shared__ unsigned s_last;
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = (atomicAdd(I.counter, 1u) == (unsigned)(gridDim.x - 1)) ? 1u : 0u;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const int nc = P.nx * P.ny;
    double g[20];
#pragma unroll
    for (int m = 0; m < 19; ++m) g[m] = 0.0;
    g[19] = 0.0;
    for (int cc = tid; cc < nc; cc += blockDim.x) {
#pragma unroll
        for (int m = 0; m < 19; ++m) g[m] += __ldcg(I.cell + (size_t)cc * kImCell + m);
        g[19] = fmax(g[19], __ldcg(I.cell + (size_t)cc * kImCell + 19));
    }
    block_reduce<19, 1>(g, red, rout);
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
    const double moment = g[19];
    if (Q.mass_rescale) sci[18] = moment;   // implicit_moment_error = MassStatistics after the rescale
    // boundary-face totals per unit time (PhysicalDiagnostic flux, mod_R5Observe.f90:107-113)
    double flux[16];
    for (int m = 0; m < 16; ++m) flux[m] = 0.0;
    for (int jj = 0; jj < P.ny; ++jj)
        for (int m = 0; m < 4; ++m) {
            flux[m] = flux[m] - B.fxw[((size_t)jj * nx + 0) * 4 + m] / dt;
            flux[4 + m] = flux[4 + m] + B.fxw[((size_t)jj * nx + 0) * 4 + m] / dt;
        }
    for (int ii = 0; ii < nx; ++ii)
        for (int m = 0; m < 4; ++m) {
            flux[8 + m] = flux[8 + m] - B.fyw[(size_t)ii * 4 + m] / dt;
            flux[12 + m] = flux[12 + m] + B.fyw[((size_t)P.ny * nx + ii) * 4 + m] / dt;
        }
    const double tol = Q.residual_tol;
    const bool pass = sci[0] <= tol && sci[1] <= tol && sci[2] <= tol && sci[3] <= tol && sci[12] <= tol &&
                      sci[13] <= tol && moment <= Q.moment_tol;
    const double streak = pass ? I.state[IS_STREAK] + 1.0 : 0.0;
    I.state[IS_STREAK] = streak;
    I.state[IS_STEPS] = I.state[IS_STEPS] + 1.0;
    const bool done = Q.mass_rescale ? streak >= 5.0 : pass;
    if (done) { I.state[IS_CONVERGED] = 1.0; I.state[IS_STOP] = 1.0; }
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
    *I.counter = 0u;
}

// -------------------------------------------------------------------------------------------
// PR(2) set-up: per (cell, face) the spectral radius (ImplicitSpectralRadius, mod_ImplicitMacro.f90:
// 15-55) and the Euler normal fluxes of the unperturbed cell and neighbour states, which stay fixed
// through the sweeps; zero the first correction buffer and reset the admissible-alpha masks.
__global__ void k_im_pr2_prep(LoParams P, LoBuffers B, ImParams Q, ImBuffers I) {
    if (I.state[IS_STOP] != 0.0) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nc = P.nx * P.ny;
    if (t == 0) { I.mask[0] = 0xffffffffu; I.mask[1] = 0xffffffffu; }
    if (t >= nc * 4) return;
    const int c = t >> 2, f = t & 3, i = c % P.nx, j = c / P.nx;
    const int rows = P.ny / Q.nslab;
    const FaceGeo g = face_geo(P, rows, i, j, f);
    double wi[4], wj[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) wi[m] = B.W[c * 4 + m];
    double dist;
    if (g.wall) {
        zhu_map(wi, Q.wall_ux[f == 2 ? 0 : 1], 0.0, wj);
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
    double gam = NAN;
    if (ok) {
        const double rho_avg = 0.5 * (pi_.r + pj.r);
        const double u_avg = 0.5 * (pi_.U + pj.U), v_avg = 0.5 * (pi_.V + pj.V);
        const double p_i = 0.5 * pi_.r / pi_.L, p_j = 0.5 * pj.r / pj.L;
        const double p_avg = 0.5 * (p_i + p_j);
        const double mu_avg = 0.5 * (ti * p_i + tj * p_j);
        const double sos = sqrt((P.gm1 + 1.0) * p_avg / rho_avg);
        gam = fabs(u_avg * g.nx + v_avg * g.ny) + sos + 2.0 * mu_avg / (rho_avg * fmax(dist, 1000.0 * kEps));
    }
    if (!(isfinite(gam) && gam > 0.0)) stop_with(I, B.status, ST_GETPRIMARY);
    I.pr_gamma[c * 4 + f] = gam;
    double fo[4];
    euler_flux(P.gm1, wi, g.nx, g.ny, fo);
#pragma unroll
    for (int m = 0; m < 4; ++m) I.pr_foi[(c * 4 + f) * 4 + m] = fo[m];
    euler_flux(P.gm1, wj, g.nx, g.ny, fo);
#pragma unroll
    for (int m = 0; m < 4; ++m) I.pr_foj[(c * 4 + f) * 4 + m] = fo[m];
    if (f == 0) {
#pragma unroll
        for (int m = 0; m < 4; ++m) I.dwA[c * 4 + m] = 0.0;
    }
}

// RelaxMacroPoint (mod_ImplicitMacro.f90:90-123) for cell c; X = halo buffer (previous sweep),
// Y = this sweep's buffer (Gauss-Seidel inside the slab).
__device__ __forceinline__ bool relax_macro(const LoParams& P, const LoBuffers& B, const ImParams& Q,
                                            const ImBuffers& I, int rows, int i, int j, double dtp,
                                            const double* X, double* Y) {
    const int c = j * P.nx + i;
    double wi[4], di[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) { wi[m] = B.W[c * 4 + m]; di[m] = Y[c * 4 + m]; }
    double sdt[4] = {0.0, 0.0, 0.0, 0.0}, sgn[4] = {0.0, 0.0, 0.0, 0.0}, sg = 0.0;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        const FaceGeo g = face_geo(P, rows, i, j, f);
        double wj[4], dnb[4], t[4], fn[4];
        if (g.wall) {
            const double uw = Q.wall_ux[f == 2 ? 0 : 1];
            zhu_map(wi, uw, 0.0, wj);
            zhu_map(di, uw, 0.0, dnb);
        } else {
            const double* src = g.ghost ? X : Y;
#pragma unroll
            for (int m = 0; m < 4; ++m) { wj[m] = B.W[g.nb * 4 + m]; dnb[m] = src[g.nb * 4 + m]; }
        }
        const double gam = I.pr_gamma[c * 4 + f];
        const double* foi = I.pr_foi + (c * 4 + f) * 4;
        const double* foj = I.pr_foj + (c * 4 + f) * 4;
        double dti[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) t[m] = wi[m] + di[m];
        euler_flux(P.gm1, t, g.nx, g.ny, fn);
#pragma unroll
        for (int m = 0; m < 4; ++m) dti[m] = fn[m] - foi[m];
#pragma unroll
        for (int m = 0; m < 4; ++m) t[m] = wj[m] + dnb[m];
        euler_flux(P.gm1, t, g.nx, g.ny, fn);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const double s = dti[m] + (fn[m] - foj[m]);
            if (!isfinite(s)) return false;
            sdt[m] = sdt[m] + g.len * s;
            sgn[m] = sgn[m] + g.len * gam * dnb[m];
        }
        sg = sg + g.len * gam;
    }
    const double diag = 1.0 / dtp + 0.5 * sg / P.area;
    if (!(isfinite(diag) && diag > 0.0)) return false;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const double rhs = I.rate_w[c * 4 + m] - 0.5 * 1.0 * sdt[m] / P.area + 0.5 * 1.0 * sgn[m] / P.area;
        if (!isfinite(rhs)) return false;
        Y[c * 4 + m] = rhs / diag;
    }
    return true;
}

// One PR(2) sweep (forward then backward Gauss-Seidel) per slab.
__global__ void k_im_pr2_sweep(LoParams P, LoBuffers B, ImParams Q, ImBuffers I, const double* X, double* Y) {
    if (I.state[IS_STOP] != 0.0) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= Q.nslab) return;
    const int rows = P.ny / Q.nslab, nx = P.nx;
    const double dtp = B.dt[0] * Q.ncfl / P.cfl;   // PseudoTimeStep (mod_ImplicitCommon.f90:115-119)
    for (int j = s * rows; j < (s + 1) * rows; ++j)
        for (int i = 0; i < nx; ++i)
            for (int m = 0; m < 4; ++m) Y[(j * nx + i) * 4 + m] = X[(j * nx + i) * 4 + m];
    bool ok = true;
    for (int j = s * rows; j < (s + 1) * rows && ok; ++j)
        for (int i = 0; i < nx && ok; ++i) ok = relax_macro(P, B, Q, I, rows, i, j, dtp, X, Y);
    for (int j = (s + 1) * rows - 1; j >= s * rows && ok; --j)
        for (int i = nx - 1; i >= 0 && ok; --i) ok = relax_macro(P, B, Q, I, rows, i, j, dtp, X, Y);
    if (!ok) stop_with(I, B.status, ST_NONFINITE_STATE);
}

// BuildPredictedMacroState (mod_ImplicitMacro.f90:159-185): admissible alpha levels per cell.
__global__ void k_im_macro_alpha(LoParams P, LoBuffers B, ImParams Q, ImBuffers I, const double* D) {
    if (I.state[IS_STOP] != 0.0) return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.nx * P.ny) return;
    const int lv = alpha_levels(Q.min_alpha);
    unsigned mask = 0u;
    double a = 1.0;
    for (int m = 0; m <= lv; ++m) {
        double t[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) t[q] = B.W[c * 4 + q] + a * D[c * 4 + q];
        if (is_physical(t)) mask |= 1u << m;
        a = 0.5 * a;
    }
    atomicAnd(I.mask, mask);
}

// BuildPredictedEquilibrium (mod_ImplicitMicro.f90:43-88), second-order branch.
template <int VPT, int NTMAX>
__global__ void __launch_bounds__(NTMAX, 512 / NTMAX) k_im_equilibrium(LoParams P, LoBuffers B, ImParams Q,
                                                                       ImBuffers I, const double* D) {
    if (I.state[IS_STOP] != 0.0) return;
    __shared__ double red[16 * 64];
    __shared__ double rout[kRedSlots];
    __shared__ double sc[24];   // [0..3] prim_old [4..7] prim_tilde [8] tau_tilde [9] ok [12..15] lambda
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
        if (!ok) { po.r = pt.r = 1.0; po.U = po.V = pt.U = pt.V = 0.0; po.L = pt.L = 1.0; tt = 1.0; }
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
    __syncthreads();
    double lam[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) lam[m] = sc[12 + m];
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0, e = 0.5 * (uk * uk + vk * vk);
        const double Ep = E[r] + fmax(fabs(E[r]), kEps * se) * (lam[0] + uk * lam[1] + vk * lam[2] + e * lam[3]);
        const double Fp = F[r] + 0.5 * fmax(fabs(F[r]), kEps * sf) * lam[3];
        moment_add(wk, uk, vk, Ep, Fp, acc);
        if (s.ok) {
            I.eq_h[(size_t)c * nv + s.k] = Ep;
            I.eq_b[(size_t)c * nv + s.k] = Fp;
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
// One LU-SGS stage: RelaxMicroPoint (mod_ImplicitMicro.f90:444-487) over one slab for one velocity.
// Forward: cells j up, i up; corrections not yet relaxed, the halos and the wall closures are 0
// (everything was reset).  Backward: cells j down, i down; not-yet-relaxed neighbours, halos and the
// x wrap read the forward result, walls use the closure frozen from the forward correction.
template <bool BACKWARD>
__global__ void __launch_bounds__(256) k_im_lusgs(LoParams P, LoBuffers B, ImParams Q, ImBuffers I) {
    if (I.state[IS_STOP] != 0.0) return;
    const int nv = P.nvel, nx = P.nx, ny = P.ny;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = t / nv, k = t - s * nv;
    if (s >= Q.nslab) return;
    const int rows = ny / Q.nslab;
    const double dtp = B.dt[0] * Q.ncfl / P.cfl;
    const double uk = B.u[k], vk = B.v[k];
    const double un[4] = {-uk, uk, -vk, vk};   // u*nx_out + v*ny_out of faces left, right, bottom, top
    const double len[4] = {P.dy, P.dy, P.dx, P.dx};
    double whu[2], wbu[2];
    if (BACKWARD) {
#pragma unroll
        for (int w = 0; w < 2; ++w) { whu[w] = I.wall_hu[w * nv + k]; wbu[w] = I.wall_bu[w * nv + k]; }
    }
    double* outh = BACKWARD ? I.dBh : I.dFh;
    double* outb = BACKWARD ? I.dBb : I.dFb;
    bool ok = true;
    for (int jj = 0; jj < rows; ++jj) {
        const int j = BACKWARD ? (s + 1) * rows - 1 - jj : s * rows + jj;
        for (int ii = 0; ii < nx; ++ii) {
            const int i = BACKWARD ? nx - 1 - ii : ii;
            const int c = j * nx + i;
            const size_t q = (size_t)c * nv + k;
            const double tt = I.tau_t[c];
            double rh = I.stream_h[q] + (I.eq_h[q] - B.h[q]) / tt;
            double rb = I.stream_b[q] + (I.eq_b[q] - B.b[q]) / tt;
            double diag = 1.0 / dtp + 1.0 / tt;
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                double nh = 0.0, nb = 0.0;
                if (un[f] < 0.0) {   // only inflow faces couple (min(un,0) /= 0)
                    if (f == 0) {
                        const size_t qn = (size_t)(j * nx + wrapx(i - 1, nx)) * nv + k;
                        if (!BACKWARD) { if (i > 0) { nh = outh[qn]; nb = outb[qn]; } }
                        else { nh = I.dFh[qn]; nb = I.dFb[qn]; }
                    } else if (f == 1) {
                        const size_t qn = (size_t)(j * nx + wrapx(i + 1, nx)) * nv + k;
                        if (BACKWARD) {
                            if (i < nx - 1) { nh = outh[qn]; nb = outb[qn]; }
                            else { nh = I.dFh[qn]; nb = I.dFb[qn]; }
                        }
                    } else if (f == 2) {
                        if (j == 0) {
                            if (BACKWARD) { nh = I.wall_drho[i] * whu[0]; nb = I.wall_drho[i] * wbu[0]; }
                        } else {
                            const size_t qn = (size_t)((j - 1) * nx + i) * nv + k;
                            const bool same = (j - 1) / rows == j / rows;
                            if (!BACKWARD) { if (same) { nh = outh[qn]; nb = outb[qn]; } }
                            else { nh = I.dFh[qn]; nb = I.dFb[qn]; }
                        }
                    } else {
                        if (j == ny - 1) {
                            if (BACKWARD) { nh = I.wall_drho[nx + i] * whu[1]; nb = I.wall_drho[nx + i] * wbu[1]; }
                        } else {
                            const size_t qn = (size_t)((j + 1) * nx + i) * nv + k;
                            const bool same = (j + 1) / rows == j / rows;
                            if (BACKWARD) {
                                if (same) { nh = outh[qn]; nb = outb[qn]; }
                                else { nh = I.dFh[qn]; nb = I.dFb[qn]; }
                            }
                        }
                    }
                }
                diag = diag + 1.0 * fmax(un[f], 0.0) * len[f] / P.area;
                rh = rh - 1.0 * fmin(un[f], 0.0) * len[f] * nh / P.area;
                rb = rb - 1.0 * fmin(un[f], 0.0) * len[f] * nb / P.area;
            }
            ok = ok && diag > 0.0 && isfinite(diag) && isfinite(rh) && isfinite(rb);
            outh[q] = rh / diag;
            outb[q] = rb / diag;
        }
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
        case 0: k_im_residual<VPT, NTMAX, false><<<nc, nt, 0, s>>>(P, B, Q, I); break;
        case 1: k_im_residual<VPT, NTMAX, true><<<nc, nt, 0, s>>>(P, B, Q, I); break;
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

// One ImplicitSteady pseudo-step (mod_Solve.f90:84-293 with TimeIntegration_method =
// 'ImplicitSteady' and ClosedCouetteMassRescale): 19 kernels, no host synchronisation.
// Returns the number of kernels launched through *launches.
cudaError_t enqueue_implicit_step(const LoParams& P, const LoBuffers& B, const ImParams& Q, const ImBuffers& I,
                                  cudaStream_t s, cudaStream_t s2, cudaEvent_t fork, cudaEvent_t join,
                                  long long* launches) {
    const int nc = P.nx * P.ny;
    cudaError_t e = launch_lo_timestep(P, B, s);                              // TimeStep
    if (e == cudaSuccess) e = im_fluxes(P, B, s, s2, fork, join);            // Interpolation + Evolution
    if (e == cudaSuccess) e = im_cell(0, P, B, Q, I, nullptr, s);             // ComputeResidual + diagnostics
    if (e == cudaSuccess) { k_im_pr2_prep<<<(nc * 4 + 127) / 128, 128, 0, s>>>(P, B, Q, I); e = cudaGetLastError(); }
    const double* X = I.dwA;
    double* Y = I.dwB;
    for (int sw = 0; sw < Q.macro_sweeps && e == cudaSuccess; ++sw) {        // SolveMacroPR2
        k_im_pr2_sweep<<<(Q.nslab + 31) / 32, 32, 0, s>>>(P, B, Q, I, X, Y);
        e = cudaGetLastError();
        const double* t = Y; Y = const_cast<double*>(X); X = t;
    }
    if (e == cudaSuccess) { k_im_macro_alpha<<<(nc + 127) / 128, 128, 0, s>>>(P, B, Q, I, X); e = cudaGetLastError(); }
    if (e == cudaSuccess) e = im_cell(2, P, B, Q, I, X, s);                   // BuildPredictedEquilibrium
    const int nl = Q.nslab * P.nvel;
    if (e == cudaSuccess) { k_im_lusgs<false><<<(nl + 255) / 256, 256, 0, s>>>(P, B, Q, I); e = cudaGetLastError(); }
    if (e == cudaSuccess) e = im_cell(3, P, B, Q, I, nullptr, s);             // frozen wall closure
    if (e == cudaSuccess) { k_im_lusgs<true><<<(nl + 255) / 256, 256, 0, s>>>(P, B, Q, I); e = cudaGetLastError(); }
    if (e == cudaSuccess) e = im_cell(4, P, B, Q, I, nullptr, s);             // FindAdmissibleMicroAlpha
    if (e == cudaSuccess) e = im_cell(5, P, B, Q, I, nullptr, s);             // update + RecoverMacro
    if (e == cudaSuccess) { k_im_rescale<<<148 * 4, 256, 0, s>>>(P, B, Q, I); e = cudaGetLastError(); }
    if (e == cudaSuccess) e = im_fluxes(P, B, s, s2, fork, join);            // accepted-state evaluation
    if (e == cudaSuccess) e = im_cell(1, P, B, Q, I, nullptr, s);
    if (launches) *launches += 16 + Q.macro_sweeps;
    return e;
}

}  // namespace ugks
