// ugks_s2.cu -- the high-order "S2" evolution of HighOrderImplicit and S2CN2 on sm_100a (FP64).
//
//   k_s2_init         : S2 cold start, h, b := discrete closure Maxwellian of W (S2NativeInitializeState,
//                       mod_S2NativeAdapter.f90:192-445 with make_mke).  One warp per cell.
//   k_s2_macro        : macro WENO of W: the normal / tangential slopes of every interior face at its 3
//                       Gauss nodes (compute_flux :803-808,849-854) and the 9 mean-shifted volume node
//                       states of every cell (build_targets, mod_S2D1.f90:1246-1300).
//   k_s2_target_nodes : build_targets' closures: one warp per (cell, volume node) -> node scalars.
//   k_s2_target_sum   : the Gauss-weighted targets M, K_x, K_y per (cell, velocity) from those scalars.
//   k_s2_recon1/2     : tensor WENO-AO(5,3) reconstruction with one-sided wall quartics and the
//                       positivity limiter (mod_S2D1Reconstruction.f90, limit_cell_outputs
//                       mod_S2D1.f90:315-345): the shared first layer, then per cell the second-layer
//                       templates and the limiter; writes the face cache.
//   k_s2_face_nodes   : ugks_node (mod_S2D1.f90:421-521) at one Gauss node of one interior face per warp:
//                       closure, directions and time coefficients -> node scalars.
//   k_s2_face_flux    : the node's micro flux from those scalars, one CTA per face node.
//   k_s2_wall_nodes   : the multiscale diffuse wall node (s2w2_wall_node, mod_S2MultiscaleWall.f90:45-184)
//                       per warp.
//   k_s2_combine      : the Gauss-weighted node fluxes times the face length into the face arrays.
//
// The discrete closure (solve_q_first, mod_CorrectedWF2DClosure.f90:331-426) runs on one warp: its
// lanes stride over the velocities, every moment sum is a per-lane sum and a fixed butterfly whose
// totals every lane receives, and every lane runs the reference's accept / backtrack / stop logic on
// those identical totals.  Per-velocity closure quantities (the Maxwellian, the Shakhov directions,
// the slope directions) are recomputed from the closure's few scalars in each pass instead of being
// stored.
#include "ugks_implicit.cuh"
#include "ugks_s2.cuh"

namespace ugks {

__constant__ S2Maps c_s2;

// ------------------------------------------------------------------------------------------
// per-thread reconstruction arithmetic (mod_S2D1Reconstruction.f90), in the reference's order

// Every evaluation of the S2 path is at xi = -1/2, +1/2 or a Gauss node, so the value (or the
// xi-derivative) of candidate polynomial c at point p is a fixed linear combination of its stencil,
// sum_k E[p][c][k] q[k] with E = sum_d cmap[c][k][d] xi_p^d, tabulated on the host from the same
// maps.  The reference forms the polynomial coefficients first and then evaluates them
// (prepared_eval, :247-262); the same sums taken in this order agree to an ulp.
enum { S2_XM = 0, S2_XP = 1, S2_G0 = 2 };   // points -1/2, +1/2, then the Gauss nodes 0..2
struct S2PointW {
    double E[5][4][5];   // value weights [point][candidate][stencil sample]
    double D[5][4][5];   // derivative weights
};
__constant__ S2PointW c_s2p;

struct S2Weno {
    double fw[4];   // final weights of the 4 candidates
    double q[5];    // the stencil
};

// weno_coefficients (:168-204): the nonlinear weights of stencil q
__device__ __forceinline__ bool s2_weno(const double q[5], S2Weno& w) {
    double* fw = w.fw;
#pragma unroll
    for (int k = 0; k < 5; ++k) w.q[k] = q[k];
    const double q1 = q[0], q2 = q[1], q3 = q[2], q4 = q[3], q5 = q[4];
    double beta[4];
    double t = q1 - 2 * q2 + q3, u0 = q1 - 4 * q2 + 3 * q3;
    beta[0] = 13.0 / 12.0 * (t * t) + 0.25 * (u0 * u0);
    t = q2 - 2 * q3 + q4; u0 = q2 - q4;
    beta[1] = 13.0 / 12.0 * (t * t) + 0.25 * (u0 * u0);
    t = q3 - 2 * q4 + q5; u0 = 3 * q3 - 4 * q4 + q5;
    beta[2] = 13.0 / 12.0 * (t * t) + 0.25 * (u0 * u0);
    double s = 231153 * (q3 * q3);
    s = s + 104963 * (q2 * q2);
    s = s + 6908 * (q1 * q1);
    s = s - 38947 * q1 * q4;
    s = s + 104963 * (q4 * q4);
    s = s + q2 * (-(51001 * q1) + 179098 * q4 - 38947 * q5);
    s = s - 3 * q3 * (99692 * q2 - 22641 * q1 + 99692 * q4 - 22641 * q5);
    s = s + 8209 * q1 * q5;
    s = s - 51001 * q4 * q5;
    s = s + 6908 * (q5 * q5);
    // the reference's divisions by 5040, 3, sum(alpha) and gamma_4 are multiplications by the
    // reciprocals here (each weight moves by at most an ulp)
    beta[3] = s * (1.0 / 5040.0);
    double tau = fabs(beta[3] - beta[0]);
    tau = tau + fabs(beta[3] - beta[1]);
    tau = tau + fabs(beta[3] - beta[2]);
    tau = tau * (1.0 / 3.0);
    const double gam[4] = {0.01125, 0.1275, 0.01125, 0.85};
    // tau / (beta_c + 1e-8) for the 4 candidates from one reciprocal of the product of the 4
    // denominators (each quotient within a few ulps of the division); the product of values in
    // [1e-8, ~1e7] cannot leave the normal range, and a non-finite reciprocal falls back to division
    const double d0 = beta[0] + 1.0e-8, d1 = beta[1] + 1.0e-8, d2 = beta[2] + 1.0e-8, d3 = beta[3] + 1.0e-8;
    const double p01 = d0 * d1, p23 = d2 * d3, ip = 1.0 / (p01 * p23);
    double inv[4];
    if (isfinite(ip) && ip > 0.0) {
        const double a = p23 * ip, b = p01 * ip;
        inv[0] = d1 * a; inv[1] = d0 * a; inv[2] = d3 * b; inv[3] = d2 * b;
    } else {
        inv[0] = 1.0 / d0; inv[1] = 1.0 / d1; inv[2] = 1.0 / d2; inv[3] = 1.0 / d3;
    }
    double alpha[4], sa = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const double r = tau * inv[c];
        alpha[c] = gam[c] * (1.0 + r * r);
        sa = sa + alpha[c];
    }
    const double isa = 1.0 / sa;
    fw[3] = (alpha[3] * isa) * (1.0 / 0.85);
#pragma unroll
    for (int c = 0; c < 3; ++c) fw[c] = alpha[c] * isa - fw[3] * gam[c];
    return isfinite(fw[0]) && isfinite(fw[1]) && isfinite(fw[2]) && isfinite(fw[3]);
}

// sum_c fw[c] sum_k T[c][k] v[k] over each candidate's stencil samples (prepared_eval, :247-262)
__device__ __forceinline__ double s2_cand_sum(const double fw[4], const double v[5], const double (*T)[5]) {
    double r = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        double cand = 0.0;
#pragma unroll
        for (int k = (c < 3 ? c : 0); k <= (c < 3 ? c + 2 : 4); ++k) cand = cand + T[c][k] * v[k];
        r = r + fw[c] * cand;
    }
    return r;
}
__device__ __forceinline__ void s2_at(const S2Weno& w, int p, double& val, double& der) {
    val = s2_cand_sum(w.fw, w.q, c_s2p.E[p]);
    der = s2_cand_sum(w.fw, w.q, c_s2p.D[p]);
}
__device__ __forceinline__ double s2_at_v(const S2Weno& w, int p) { return s2_cand_sum(w.fw, w.q, c_s2p.E[p]); }

// companion_eval3 (:287-318): the weights of q applied to the companion samples comp as well
__device__ __forceinline__ bool s2_companion3(const double q[5], const double comp[5], double val[3], double der[3],
                                              double cval[3]) {
    S2Weno w;
    if (!s2_weno(q, w)) return false;
    bool ok = true;
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        s2_at(w, S2_G0 + s, val[s], der[s]);
        cval[s] = s2_cand_sum(w.fw, comp, c_s2p.E[S2_G0 + s]);
        ok = ok && isfinite(val[s]) && isfinite(der[s]) && isfinite(cval[s]);
    }
    return ok;
}

__device__ __forceinline__ bool s2_near_wall(int j, int ny) { return j + 1 <= 3 || j + 1 >= ny - 2; }
__device__ __forceinline__ int s2_wall_first(int j, int ny) { return (j + 1 <= 3) ? 0 : ny - 5; }

// wall_coeff + wall_eval (:113-136)
__device__ __forceinline__ void s2_wall_eval(const double q[5], int j, int ny, double xi, double& val, double& der) {
    const int side = (j + 1 <= 3) ? 0 : 1, dist = side == 0 ? j : ny - 1 - j;
    double c[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 5; ++k)
#pragma unroll
        for (int d = 0; d < 5; ++d) c[d] = c[d] + c_s2.wall[side][dist][k][d] * q[k];
    double v = c[4];
#pragma unroll
    for (int d = 3; d >= 0; --d) v = v * xi + c[d];
    double dv = 4.0 * c[4];
#pragma unroll
    for (int d = 3; d >= 1; --d) dv = dv * xi + (double)d * c[d];
    val = v;
    der = dv;
}

// a strided 2-D field: f[(j*nx + i)*stride], x periodic
struct S2Field {
    const double* f;
    int stride, nx, ny;
    __device__ __forceinline__ double at(int i, int j) const {
        i = i < 0 ? i + nx : (i >= nx ? i - nx : i);
        return f[(size_t)(j * nx + i) * stride];
    }
};

// s2d1_cell_faces9 / s2d1_cell_faces9_wall (:409-498)
__device__ bool s2_cell_faces9(const S2Field& F, int i, int j, double face[4][3], double dn[4][3], double dt[4][3],
                               double vol[3][3]) {
    double xv[5][2], xd[5][2], yv[5][2], yd[5][2], rows[5][3], q[5];
    S2Weno ww;
    const int ny = F.ny;
    if (!s2_near_wall(j, ny)) {
        for (int r = -2; r <= 2; ++r) {
#pragma unroll
            for (int s = -2; s <= 2; ++s) q[s + 2] = F.at(i + s, j + r);
            if (!s2_weno(q, ww)) return false;
            s2_at(ww, S2_XM, xv[r + 2][0], xd[r + 2][0]);
            s2_at(ww, S2_XP, xv[r + 2][1], xd[r + 2][1]);
#pragma unroll
            for (int a = 0; a < 3; ++a) rows[r + 2][a] = s2_at_v(ww, S2_G0 + a);
        }
        for (int r = -2; r <= 2; ++r) {
#pragma unroll
            for (int s = -2; s <= 2; ++s) q[s + 2] = F.at(i + r, j + s);
            if (!s2_weno(q, ww)) return false;
            s2_at(ww, S2_XM, yv[r + 2][0], yd[r + 2][0]);
            s2_at(ww, S2_XP, yv[r + 2][1], yd[r + 2][1]);
        }
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            double a5[5], b5[5];
#pragma unroll
            for (int r = 0; r < 5; ++r) { a5[r] = xv[r][s]; b5[r] = xd[r][s]; }
            if (!s2_companion3(a5, b5, face[s], dt[s], dn[s])) return false;
#pragma unroll
            for (int r = 0; r < 5; ++r) { a5[r] = yv[r][s]; b5[r] = yd[r][s]; }
            if (!s2_companion3(a5, b5, face[s + 2], dt[s + 2], dn[s + 2])) return false;
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            double a5[5];
#pragma unroll
            for (int r = 0; r < 5; ++r) a5[r] = rows[r][a];
            if (!s2_weno(a5, ww)) return false;
#pragma unroll
            for (int b = 0; b < 3; ++b) vol[a][b] = s2_at_v(ww, S2_G0 + b);
        }
    } else {
        const int first = s2_wall_first(j, ny);
        for (int r = 0; r < 5; ++r) {
#pragma unroll
            for (int s = -2; s <= 2; ++s) q[s + 2] = F.at(i + s, first + r);
            if (!s2_weno(q, ww)) return false;
            s2_at(ww, S2_XM, xv[r][0], xd[r][0]);
            s2_at(ww, S2_XP, xv[r][1], xd[r][1]);
#pragma unroll
            for (int a = 0; a < 3; ++a) rows[r][a] = s2_at_v(ww, S2_G0 + a);
        }
        for (int r = -2; r <= 2; ++r) {
#pragma unroll
            for (int s = 0; s < 5; ++s) q[s] = F.at(i + r, first + s);
            s2_wall_eval(q, j, ny, -0.5, yv[r + 2][0], yd[r + 2][0]);
            s2_wall_eval(q, j, ny, 0.5, yv[r + 2][1], yd[r + 2][1]);
        }
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            double a5[5], b5[5], dummy;
#pragma unroll
            for (int r = 0; r < 5; ++r) { a5[r] = xv[r][s]; b5[r] = xd[r][s]; }
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                s2_wall_eval(a5, j, ny, c_s2.gnode[a], face[s][a], dt[s][a]);
                s2_wall_eval(b5, j, ny, c_s2.gnode[a], dn[s][a], dummy);
            }
#pragma unroll
            for (int r = 0; r < 5; ++r) { a5[r] = yv[r][s]; b5[r] = yd[r][s]; }
            if (!s2_companion3(a5, b5, face[s + 2], dt[s + 2], dn[s + 2])) return false;
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            double a5[5], dummy;
#pragma unroll
            for (int r = 0; r < 5; ++r) a5[r] = rows[r][a];
#pragma unroll
            for (int b = 0; b < 3; ++b) s2_wall_eval(a5, j, ny, c_s2.gnode[b], vol[a][b], dummy);
        }
    }
    bool ok = true;
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int a = 0; a < 3; ++a) ok = ok && isfinite(face[s][a]) && isfinite(dn[s][a]) && isfinite(dt[s][a]);
    return ok;
}

// s2d1_side3 with wall_y for the macroscopic field (:320-354)
__device__ bool s2_side3(const S2Field& F, int axis, int cell, int tangent, double side, double val[3], double dn[3],
                         double dt[3]) {
    const int j = axis == 0 ? tangent : cell;
    if (s2_near_wall(j, F.ny)) {
        double f[4][3], n[4][3], t[4][3], vol[3][3];
        int slot;
        if (axis == 0) { if (!s2_cell_faces9(F, cell, j, f, n, t, vol)) return false; slot = side < 0.0 ? 0 : 1; }
        else { if (!s2_cell_faces9(F, tangent, j, f, n, t, vol)) return false; slot = side < 0.0 ? 2 : 3; }
#pragma unroll
        for (int a = 0; a < 3; ++a) { val[a] = f[slot][a]; dn[a] = n[slot][a]; dt[a] = t[slot][a]; }
        return true;
    }
    double nv5[5], nd5[5], q[5];
    S2Weno ww;
    for (int r = -2; r <= 2; ++r) {
#pragma unroll
        for (int s = -2; s <= 2; ++s) q[s + 2] = axis == 0 ? F.at(cell + s, tangent + r) : F.at(tangent + r, cell + s);
        if (!s2_weno(q, ww)) return false;
        s2_at(ww, side < 0.0 ? S2_XM : S2_XP, nv5[r + 2], nd5[r + 2]);
    }
    return s2_companion3(nv5, nd5, val, dt, dn);
}

// s2d1_cell9 (:378-403)
__device__ bool s2_cell9(const S2Field& F, int i, int j, double val[3][3]) {
    if (s2_near_wall(j, F.ny)) {
        double f[4][3], n[4][3], t[4][3];
        return s2_cell_faces9(F, i, j, f, n, t, val);
    }
    double rows[5][3], q[5];
    S2Weno ww;
    for (int r = -2; r <= 2; ++r) {
#pragma unroll
        for (int s = -2; s <= 2; ++s) q[s + 2] = F.at(i + s, j + r);
        if (!s2_weno(q, ww)) return false;
#pragma unroll
        for (int a = 0; a < 3; ++a) rows[r + 2][a] = s2_at_v(ww, S2_G0 + a);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double a5[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) a5[r] = rows[r][a];
        if (!s2_weno(a5, ww)) return false;
#pragma unroll
        for (int b = 0; b < 3; ++b) val[a][b] = s2_at_v(ww, S2_G0 + b);
    }
    return true;
}

// ------------------------------------------------------------------------------------------
// reconstruction + limiter in two passes.  Cache layout rec[((cell*72 + field*12 + side*3 + node)*nvel + k],
// fields: h, b, h_n, h_t, b_n, b_t; sides: x left, x right, y bottom, y top.
//
// k_s2_recon1, the first layer (prepare_first_layer_plane, mod_S2D1Reconstruction.f90:501-578):
// per (cell, velocity, field) the 1-D WENO along x of the cell's own row -- values and derivatives
// at xi = -1/2, +1/2 and values at the 3 Gauss nodes -- and, for rows away from the walls, along y
// of the cell's own column -- values and derivatives at -1/2, +1/2.  These are the first-layer
// results the tensor templates of the 5 neighbouring cells share.  l1[cell][field*11 + q][nvel]:
// q 0..3 = x value/derivative at -1/2, +1/2; 4..6 = x Gauss values; 7..10 = y value/derivative.
// CTA: 4 warps (field, direction) over 32 velocities of one cell.
__global__ void __launch_bounds__(128) k_s2_recon1(LoParams P, LoBuffers B, S2Buffers S) {
    if (eval_cached(B)) return;
    const int nv = P.nvel, nx = P.nx, ny = P.ny, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int f = warp >> 1, dir = warp & 1;
    const int k0 = blockIdx.x * 32 + lane;
    const bool kok = k0 < nv;
    const int k = kok ? k0 : nv - 1;
    const int cc = blockIdx.y, i = cc % nx, j = cc / nx;
    if (dir == 1 && s2_near_wall(j, ny)) return;   // walls use one-sided quartics instead
    const S2Field F{(f == 0 ? B.h : B.b) + k, nv, nx, ny};
    double q[5];
    S2Weno ww;
#pragma unroll
    for (int s = -2; s <= 2; ++s) q[s + 2] = dir == 0 ? F.at(i + s, j) : F.at(i, j + s);
    const bool ok = s2_weno(q, ww);
    double* o = S.l1 + ((size_t)cc * 22 + f * 11 + (dir == 0 ? 0 : 7)) * nv + k;
    double v0, d0, v1, d1;
    s2_at(ww, S2_XM, v0, d0);
    s2_at(ww, S2_XP, v1, d1);
    if (kok) {
        o[0] = v0; o[(size_t)nv] = d0; o[2 * (size_t)nv] = v1; o[3 * (size_t)nv] = d1;
        if (dir == 0)
#pragma unroll
            for (int a = 0; a < 3; ++a) o[(size_t)(4 + a) * nv] = s2_at_v(ww, S2_G0 + a);
        if (!ok) set_status(B.status, ST_NONFINITE_FLUX);
    }
}

// k_s2_recon2, the second layer (tensor_velocity_tile, :723-792; reconstruct_wall_tile, :918-971) and
// limit_cell_outputs (mod_S2D1.f90:315-345): CTA = 8 warps (field f = warp / 4, part p = warp % 4)
// over 32 velocities of one cell.  Part p reconstructs face side p (x left, x right, y bottom, y top)
// at its 3 Gauss nodes with value, normal and tangential derivative, and parts 0..2 also the volume
// Gauss row p; the positivity factor theta is the minimum over the 8 warps (both fields, all face and
// volume samples), then each warp writes its side's limited values.
__global__ void __launch_bounds__(256, 3) k_s2_recon2(LoParams P, LoBuffers B, S2Buffers S) {
    if (eval_cached(B)) return;
    __shared__ double s_th[8][32];
    const int nv = P.nvel, nx = P.nx, ny = P.ny, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int f = warp >> 2, p = warp & 3;
    const int k0 = blockIdx.x * 32 + lane;
    const bool kok = k0 < nv;
    const int k = kok ? k0 : nv - 1;
    const int cc = blockIdx.y, i = cc % nx, j = cc / nx;
    const bool nw = s2_near_wall(j, ny);
    const int first = nw ? s2_wall_first(j, ny) : j - 2;   // rows of the x first layer
    const double* L1 = S.l1 + (size_t)f * 11 * nv + k;
    auto X = [&](int r, int q) { return L1[((size_t)((first + r) * nx + i) * 22 + q) * nv]; };
    double face[3], dn[3], dt[3], vol[3];
    bool ok = true;
    if (p < 2) {   // x face p
        double a5[5], b5[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) { a5[r] = X(r, 2 * p); b5[r] = X(r, 2 * p + 1); }
        if (!nw) ok = s2_companion3(a5, b5, face, dt, dn);
        else {
            double dummy;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                s2_wall_eval(a5, j, ny, c_s2.gnode[a], face[a], dt[a]);
                s2_wall_eval(b5, j, ny, c_s2.gnode[a], dn[a], dummy);
            }
        }
    } else {       // y face p - 2
        const int s = p - 2;
        double a5[5], b5[5];
        if (!nw) {
#pragma unroll
            for (int r = 0; r < 5; ++r) {
                const double* y = L1 + ((size_t)(j * nx + wrapx(i + r - 2, nx)) * 22 + 7 + 2 * s) * nv;
                a5[r] = y[0];
                b5[r] = y[(size_t)nv];
            }
        } else {
            const S2Field F{(f == 0 ? B.h : B.b) + k, nv, nx, ny};
#pragma unroll
            for (int r = -2; r <= 2; ++r) {
                double q[5];
#pragma unroll
                for (int t = 0; t < 5; ++t) q[t] = F.at(i + r, first + t);
                s2_wall_eval(q, j, ny, s == 0 ? -0.5 : 0.5, a5[r + 2], b5[r + 2]);
            }
        }
        ok = s2_companion3(a5, b5, face, dt, dn);
    }
    if (p < 3) {   // volume Gauss row p
        double a5[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) a5[r] = X(r, 4 + p);
        if (!nw) {
            S2Weno ww;
            ok = ok && s2_weno(a5, ww);
#pragma unroll
            for (int b = 0; b < 3; ++b) vol[b] = s2_at_v(ww, S2_G0 + b);
        } else {
            double dummy;
#pragma unroll
            for (int b = 0; b < 3; ++b) s2_wall_eval(a5, j, ny, c_s2.gnode[b], vol[b], dummy);
        }
    }
    // positivity factor (limit_cell_outputs): min over both fields' face and volume samples
    const double hm = B.h[(size_t)cc * nv + k], bm = B.b[(size_t)cc * nv + k];
    const double mf = f == 0 ? hm : bm;
    const double margin = 64.0 * kEps;
    double cand = 1.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (face[a] < 0.0) cand = fmin(cand, (1.0 - margin) * mf / (mf - face[a]));
        if (p < 3 && vol[a] < 0.0) cand = fmin(cand, (1.0 - margin) * mf / (mf - vol[a]));
    }
    s_th[warp][lane] = cand;
    __syncthreads();
    double theta = s_th[0][lane];
#pragma unroll
    for (int w = 1; w < 8; ++w) theta = fmin(theta, s_th[w][lane]);
    theta = (hm <= 0.0 || bm <= 0.0) ? 0.0 : fmax(0.0, fmin(1.0, theta));
    // the derivatives are divided by the cell sizes (limit_cell_outputs): multiplied by the reciprocals
    // here, exact when dx and dy are powers of two (the delivered meshes), within an ulp otherwise
    const double ind = 1.0 / (p < 2 ? P.dx : P.dy), itd = 1.0 / (p < 2 ? P.dy : P.dx);
    double* r = S.rec + (size_t)cc * 72 * nv + k;
    const int fv = f == 0 ? 0 : 1, fn = f == 0 ? 2 : 4, ft = f == 0 ? 3 : 5;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double v = mf + theta * (face[a] - mf), n = theta * dn[a] * ind, t = theta * dt[a] * itd;
        if (kok) {
            r[(size_t)(fv * 12 + p * 3 + a) * nv] = v;
            r[(size_t)(fn * 12 + p * 3 + a) * nv] = n;
            r[(size_t)(ft * 12 + p * 3 + a) * nv] = t;
        }
        ok = ok && isfinite(v) && isfinite(n) && isfinite(t);
    }
    if (!ok && kok) set_status(B.status, ST_NONFINITE_FLUX);
}

// ------------------------------------------------------------------------------------------
// closure helpers

// solve_dense_4x4 (mod_CorrectedWF2DClosure.f90:631-661), m row-major
__device__ bool s2_solve4(const double* m, const double rhs[4], double x[4]) {
    double a[4][4], b[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
#pragma unroll
        for (int c = 0; c < 4; ++c) a[r][c] = m[r * 4 + c];
        b[r] = rhs[r];
    }
    x[0] = x[1] = x[2] = x[3] = 0.0;
#pragma unroll
    for (int p = 0; p < 3; ++p) {
        int row = p;
        double best = fabs(a[p][p]);
#pragma unroll
        for (int i = p + 1; i < 4; ++i) if (fabs(a[i][p]) > best) { best = fabs(a[i][p]); row = i; }
        double piv = a[p][p];
#pragma unroll
        for (int i = p + 1; i < 4; ++i) if (i == row) piv = a[i][p];
        if (fabs(piv) <= 100.0 * DBL_MIN || !isfinite(piv)) return false;
#pragma unroll
        for (int i = p + 1; i < 4; ++i)
            if (i == row) {
#pragma unroll
                for (int c = 0; c < 4; ++c) { const double t = a[p][c]; a[p][c] = a[i][c]; a[i][c] = t; }
                const double t = b[p]; b[p] = b[i]; b[i] = t;
            }
#pragma unroll
        for (int i = p + 1; i < 4; ++i) {
            const double f = a[i][p] / a[p][p];
#pragma unroll
            for (int c = p; c < 4; ++c) a[i][c] = a[i][c] - f * a[p][c];
            b[i] = b[i] - f * b[p];
        }
    }
    if (fabs(a[3][3]) <= 100.0 * DBL_MIN || !isfinite(a[3][3])) return false;
#pragma unroll
    for (int i = 3; i >= 0; --i) {
        double pv = b[i];
        if (i < 3) {
            double s = 0.0;
#pragma unroll
            for (int c = i + 1; c < 4; ++c) s = s + a[i][c] * x[c];
            pv = pv - s;
        }
        x[i] = pv / a[i][i];
    }
    return isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]) && isfinite(x[3]);
}

// the closure Maxwellian at theta for velocity (u, v) and its log-derivatives (q_state_first,
// mod_CorrectedWF2DClosure.f90:389-426).  The velocity-independent factors are formed once per
// theta (S2Th); the divisions by T and rho of the reference become multiplications by 1/T and 1/rho,
// which moves each value by at most an ulp.
struct S2Th {
    double r, u, v, tw;          // theta = (rho, u, v, T_native)
    double pref, itw, ir, ckh;   // rho / (pi T), 1 / T, 1 / rho, ck T / 2
};
__device__ __forceinline__ S2Th s2_th(const double th[4], int ck) {
    S2Th t;
    t.r = th[0]; t.u = th[1]; t.v = th[2]; t.tw = th[3];
    t.pref = t.r / (kPi * t.tw);
    t.itw = 1.0 / t.tw;
    t.ir = 1.0 / t.r;
    t.ckh = 0.5 * (double)ck * t.tw;
    return t;
}
struct S2Q {
    double qh, qb, ld[4], ldb[4];
};
__device__ __forceinline__ S2Q s2_q(const S2Th& t, double u, double v) {
    S2Q q;
    const double du = u - t.u, dv = v - t.v, c2 = du * du + dv * dv;
    q.qh = t.pref * exp(-c2 * t.itw);
    q.ld[0] = t.ir; q.ld[1] = 2.0 * du * t.itw; q.ld[2] = 2.0 * dv * t.itw; q.ld[3] = -t.itw + c2 * (t.itw * t.itw);
    q.qb = t.ckh * q.qh;
    q.ldb[0] = q.ld[0]; q.ldb[1] = q.ld[1]; q.ldb[2] = q.ld[2]; q.ldb[3] = q.ld[3] + t.itw;
    return q;
}

// dq for a moment direction m (closure_first_direction): td = solve(jac, m) by thread `who`,
// broadcast through S.v[base..base+3]
__device__ __forceinline__ void s2_dq(const S2Q& q, const double td[4], double& dh, double& db) {
    dh = 0.0; db = 0.0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        dh = dh + q.qh * q.ld[a] * td[a];
        db = db + q.qb * q.ldb[a] * td[a];
    }
}

// ------------------------------------------------------------------------------------------
// warp-level discrete closure.  One warp owns one closure-bearing node: lane l takes the
// velocities k = l, l + 32, ...; every velocity sum is a per-lane sequential sum followed by a
// fixed butterfly (warp_halving) and a broadcast, so all lanes hold bitwise-identical totals and
// run the same Newton / gate logic.  No shared memory and no block barriers.

struct WVel {
    int k;       // velocity index, clamped to a valid one
    bool ok;     // a real velocity of this lane
    double u, v, w;
};
__device__ __forceinline__ WVel wvel(const LoBuffers& B, int nv, int r) {
    WVel s;
    const int k = (threadIdx.x & 31) + 32 * r;
    s.ok = k < nv;
    s.k = s.ok ? k : nv - 1;
    s.u = __ldg(B.u + s.k);
    s.v = __ldg(B.v + s.k);
    s.w = s.ok ? __ldg(B.w + s.k) : 0.0;
    return s;
}

template <int N>
__device__ __forceinline__ void warp_sum_all(double* v) {
    constexpr int sh = 5 - ilog2(pow2_ceil(N));
    const double r = warp_halving<N, false>(v);
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = __shfl_sync(0xffffffffu, r, i << sh);
}
template <int N>
__device__ __forceinline__ void warp_max_all(double* v) {
    constexpr int sh = 5 - ilog2(pow2_ceil(N));
    const double r = warp_halving<N, true>(v);
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = __shfl_sync(0xffffffffu, r, i << sh);
}

__device__ __forceinline__ double s2_scaled(const double r[4], const double w[4]) {
    double s = 0.0;
#pragma unroll
    for (int m = 0; m < 4; ++m) s = fmax(s, fabs(r[m]) / fmax(1.0, fabs(w[m])));
    return s;
}

struct WClosure {
    double th[4];    // converged (rho, u, v, T_native)
    double* jac;     // [16] moment Jacobian at th, row-major (moment r, theta a), in the warp's slice of
                     // shared memory: lane 0 writes it, every lane reads it (it is warp-uniform)
};

enum { W_TRIAL = 0, W_DONE = 1, W_FAIL = 2 };

// the next trial after an accepted evaluation (new_iter) or a rejected one
__device__ __forceinline__ int w_newton_next(bool new_iter, const WClosure& C, const double res[4], double norm,
                                             int iter, double step[4], double& alpha, double trial[4]) {
    const double tol = 5.0e-13, floor_a = 9.5367431640625e-07;   // 2^-20
    if (new_iter) {
        if (norm <= tol) return W_DONE;
        if (iter > 12) return W_FAIL;
        const double mr[4] = {-res[0], -res[1], -res[2], -res[3]};
        if (!s2_solve4(C.jac, mr, step)) return W_FAIL;
        alpha = 1.0;
    }
    while (alpha >= floor_a) {
        double nt[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) nt[m] = C.th[m] + alpha * step[m];
        if (nt[0] > 0.0 && nt[3] > 0.0 && isfinite(nt[0]) && isfinite(nt[1]) && isfinite(nt[2]) && isfinite(nt[3])) {
#pragma unroll
            for (int m = 0; m < 4; ++m) trial[m] = nt[m];
            return W_TRIAL;
        }
        alpha = 0.5 * alpha;
    }
    return W_FAIL;
}

// solve_q_first (mod_CorrectedWF2DClosure.f90:331-426) for the target moments w by one warp
__device__ bool w_closure(const LoParams& P, const LoBuffers& B, const double w[4], WClosure& C) {
    const int nv = P.nvel, ck = P.ck, nr = (nv + 31) >> 5;
    double trial[4];
    {   // primitive_from_conserved_2d (mod_CorrectedWF2DEquilibrium.f90:25-41)
        if (!(isfinite(w[0]) && isfinite(w[1]) && isfinite(w[2]) && isfinite(w[3]) && w[0] > 0.0)) return false;
        const double u = w[1] / w[0], v = w[2] / w[0];
        const double kin = 0.5 * (u * u + v * v), ein = w[3] / w[0] - kin;
        const double temp = 4.0 * ein / (double)(ck + 2);
        if (!(isfinite(u) && isfinite(v) && isfinite(temp) && temp > 0.0)) return false;
        trial[0] = w[0]; trial[1] = u; trial[2] = v; trial[3] = temp;
    }
    double res[4] = {0.0, 0.0, 0.0, 0.0}, step[4] = {0.0, 0.0, 0.0, 0.0}, alpha = 1.0, norm = 0.0;
    int iter = 0;
    bool first = true;
    for (int guard = 0; guard < 1024; ++guard) {
        // 16 Jacobian moments, the 4 moments of (qh, qb), flags: nonfinite, nonpositive
        double acc[22];
#pragma unroll
        for (int m = 0; m < 22; ++m) acc[m] = 0.0;
        const S2Th tt = s2_th(trial, ck);
        for (int r = 0; r < nr; ++r) {
            const WVel s = wvel(B, nv, r);
            const S2Q q = s2_q(tt, s.u, s.v);
            const double e2 = s.u * s.u + s.v * s.v;
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const double hk = q.qh * q.ld[a], bk = q.qb * q.ldb[a];
                acc[0 * 4 + a] += s.w * hk;
                acc[1 * 4 + a] += s.w * s.u * hk;
                acc[2 * 4 + a] += s.w * s.v * hk;
                acc[3 * 4 + a] += 0.5 * s.w * (e2 * hk + bk);
            }
            acc[16] += s.w * q.qh;
            acc[17] += s.w * s.u * q.qh;
            acc[18] += s.w * s.v * q.qh;
            acc[19] += 0.5 * s.w * (e2 * q.qh + q.qb);
            if (s.ok) {
                acc[20] = fmax(acc[20], (isfinite(q.qh) && isfinite(q.qb)) ? 0.0 : 1.0);
                acc[21] = fmax(acc[21], (q.qh > 0.0 && q.qb > 0.0) ? 0.0 : 1.0);
            }
        }
        warp_sum_all<20>(acc);
        warp_max_all<2>(acc + 20);
        bool fin = acc[20] == 0.0;
#pragma unroll
        for (int m = 0; m < 20; ++m) fin = fin && isfinite(acc[m]);
        double nres[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) nres[m] = acc[16 + m] - w[m];
        int act;
        const double nn = fin ? s2_scaled(nres, w) : INFINITY;
        if (first ? fin : (fin && (nn < norm || nn <= 5.0e-13))) {   // accept the evaluation
#pragma unroll
            for (int m = 0; m < 4; ++m) { C.th[m] = trial[m]; res[m] = nres[m]; }
            if ((threadIdx.x & 31) == 0)
#pragma unroll
                for (int m = 0; m < 16; ++m) C.jac[m] = acc[m];
            __syncwarp();
            norm = nn;
            iter = first ? 1 : iter + 1;
            act = w_newton_next(true, C, res, norm, iter, step, alpha, trial);
            if (act == W_DONE && acc[21] != 0.0) act = W_FAIL;
        } else if (first) {
            return false;
        } else {
            alpha = 0.5 * alpha;
            act = w_newton_next(false, C, res, norm, iter, step, alpha, trial);
        }
        first = false;
        if (act == W_DONE) return true;
        if (act == W_FAIL) return false;
    }
    return false;
}

// make_mke_prepared (mod_S2D1.f90:111-151): the scalars that give, per velocity, the closure
// Maxwellian M and the projected Shakhov directions K_x, K_y (w_mke_at)
struct WMke {
    double ux, vy, lam, coeff;   // primitive of w (theta_gas) and the Shakhov coefficient
    double tdx[4], tdy[4];       // closure directions removed from the raw Shakhov terms
};

__device__ __forceinline__ void w_mke_raw(const WMke& M, const S2Q& q, int ck, double uk, double vk, double& kxh,
                                          double& kxb, double& kyh, double& kyb) {
    const double cx = uk - M.ux, cy = vk - M.vy, c2 = cx * cx + cy * cy;
    const double shh = 2.0 * M.lam * c2 - 4.0, shb = shh + 2.0 / (double)ck;
    kxh = M.coeff * cx * shh * q.qh; kxb = M.coeff * cx * shb * q.qb;
    kyh = M.coeff * cy * shh * q.qh; kyb = M.coeff * cy * shb * q.qb;
}

// M, K_x, K_y of one velocity from the node scalars
__device__ __forceinline__ void w_mke_at(const S2Th& th, const WMke& M, int ck, double uk, double vk, S2Q& q,
                                         double& mh, double& mb, double& kxh, double& kxb, double& kyh, double& kyb) {
    q = s2_q(th, uk, vk);
    mh = q.qh;
    mb = q.qb;
    w_mke_raw(M, q, ck, uk, vk, kxh, kxb, kyh, kyb);
    double dh, db;
    s2_dq(q, M.tdx, dh, db);
    kxh = kxh - dh; kxb = kxb - db;
    s2_dq(q, M.tdy, dh, db);
    kyh = kyh - dh; kyb = kyb - db;
}

// Returns the gate (moments of M equal w, K_x, K_y moment-free, all finite, to 2e-12).
__device__ bool w_make_mke(const LoParams& P, const LoBuffers& B, const double w[4], const WClosure& C, WMke& M) {
    const int nv = P.nvel, ck = P.ck, nr = (nv + 31) >> 5;
    double rho, th;
    const bool pok = s2_primitive(w, ck, rho, M.ux, M.vy, th);
    M.lam = 0.5 / th;
    M.coeff = 0.8 * (1.0 - P.pr) * M.lam * M.lam / rho;
    double acc[16];
#pragma unroll
    for (int m = 0; m < 8; ++m) acc[m] = 0.0;
    const S2Th tt = s2_th(C.th, ck);
    for (int r = 0; r < nr; ++r) {
        const WVel s = wvel(B, nv, r);
        const S2Q q = s2_q(tt, s.u, s.v);
        double kxh, kxb, kyh, kyb;
        w_mke_raw(M, q, ck, s.u, s.v, kxh, kxb, kyh, kyb);
        const double e2 = s.u * s.u + s.v * s.v;
        acc[0] += s.w * kxh; acc[1] += s.w * s.u * kxh; acc[2] += s.w * s.v * kxh; acc[3] += 0.5 * s.w * (e2 * kxh + kxb);
        acc[4] += s.w * kyh; acc[5] += s.w * s.u * kyh; acc[6] += s.w * s.v * kyh; acc[7] += 0.5 * s.w * (e2 * kyh + kyb);
    }
    warp_sum_all<8>(acc);
    {
        double td[4];
        const bool okx = s2_solve4(C.jac, acc, td);
#pragma unroll
        for (int m = 0; m < 4; ++m) M.tdx[m] = okx ? td[m] : NAN;
        const bool oky = s2_solve4(C.jac, acc + 4, td);
#pragma unroll
        for (int m = 0; m < 4; ++m) M.tdy[m] = oky ? td[m] : NAN;
    }
#pragma unroll
    for (int m = 0; m < 16; ++m) acc[m] = 0.0;
    for (int r = 0; r < nr; ++r) {
        const WVel s = wvel(B, nv, r);
        S2Q q;
        double mh, mb, kxh, kxb, kyh, kyb;
        w_mke_at(tt, M, ck, s.u, s.v, q, mh, mb, kxh, kxb, kyh, kyb);
        const double e2 = s.u * s.u + s.v * s.v, cx = s.u - M.ux, cy = s.v - M.vy, c2 = cx * cx + cy * cy;
        acc[0] += s.w * mh; acc[1] += s.w * s.u * mh; acc[2] += s.w * s.v * mh; acc[3] += 0.5 * s.w * (e2 * mh + mb);
        acc[4] += s.w * kxh; acc[5] += s.w * s.u * kxh; acc[6] += s.w * s.v * kxh; acc[7] += 0.5 * s.w * (e2 * kxh + kxb);
        acc[8] += s.w * kyh; acc[9] += s.w * s.u * kyh; acc[10] += s.w * s.v * kyh; acc[11] += 0.5 * s.w * (e2 * kyh + kyb);
        acc[12] += 0.5 * s.w * cx * (c2 * kxh + kxb);
        acc[13] += 0.5 * s.w * cy * (c2 * kxh + kxb);
        acc[14] += 0.5 * s.w * cx * (c2 * kyh + kyb);
        acc[15] += 0.5 * s.w * cy * (c2 * kyh + kyb);
    }
    warp_sum_all<16>(acc);
    double res = 0.0, sc = 1.0;
#pragma unroll
    for (int m = 0; m < 4; ++m) { res = fmax(res, fabs(acc[m] - w[m])); sc = fmax(sc, fabs(w[m])); }
    res = res / sc;
#pragma unroll
    for (int m = 4; m < 12; ++m) res = fmax(res, fabs(acc[m]));
    bool fin = isfinite(M.tdx[0]) && isfinite(M.tdy[0]);
#pragma unroll
    for (int m = 12; m < 16; ++m) fin = fin && isfinite(acc[m]);
    return pok && fin && res <= 2.0e-12;
}

// node scalars of a volume target: th[4], tdx[4], tdy[4], ux, vy, lam, coeff
constexpr int kS2TScal = 16;

__device__ __forceinline__ void w_store_scalars(double* o, const WClosure& C, const WMke& M) {
#pragma unroll
    for (int m = 0; m < 4; ++m) { o[m] = C.th[m]; o[4 + m] = M.tdx[m]; o[8 + m] = M.tdy[m]; }
    o[12] = M.ux; o[13] = M.vy; o[14] = M.lam; o[15] = M.coeff;
}
__device__ __forceinline__ void w_load_scalars(const double* o, double th[4], WMke& M) {
#pragma unroll
    for (int m = 0; m < 4; ++m) { th[m] = o[m]; M.tdx[m] = o[4 + m]; M.tdy[m] = o[8 + m]; }
    M.ux = o[12]; M.vy = o[13]; M.lam = o[14]; M.coeff = o[15];
}

// ------------------------------------------------------------------------------------------
// S2 cold start: one warp per cell, h, b := the discrete closure Maxwellian of W
__global__ void __launch_bounds__(256, 2) k_s2_init(LoParams P, LoBuffers B, S2Buffers SB) {
    const int nv = P.nvel, nc = P.nx * P.ny, lane = threadIdx.x & 31, nr = (nv + 31) >> 5;
    const int cc = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (cc >= nc) return;
    __shared__ double s_jac[8][16];
    double w[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) w[m] = B.W[cc * 4 + m];
    WClosure C;
    C.jac = s_jac[threadIdx.x >> 5];
    WMke M;
    const bool ok = w_closure(P, B, w, C) && w_make_mke(P, B, w, C, M);
    const S2Th tt = s2_th(C.th, P.ck);
    if (ok)
        for (int r = 0; r < nr; ++r) {
            const WVel s = wvel(B, nv, r);
            const S2Q q = s2_q(tt, s.u, s.v);
            if (s.ok) { B.h[(size_t)cc * nv + s.k] = q.qh; B.b[(size_t)cc * nv + s.k] = q.qb; }
        }
    if (!ok && lane == 0) set_status(B.status, ST_PROJECTION);
}

// ------------------------------------------------------------------------------------------
// Macro WENO of W in 8-lane groups: the 5 first-layer samples of a template are computed by lanes
// 0..4 of the group at once and gathered by shuffles, and lane 0 (or lanes 0..2) finish the template.
//
// s2d1_side3 with wall_y (:320-354) of one side: normal and tangential derivatives at the 3 Gauss
// nodes, valid in lane 0 of the group.  Near a wall the x faces take the one-sided quartic across the
// 5 true rows and the y faces the companion template of the columns' one-sided quartics
// (s2d1_cell_faces9_wall, :456-499), the same cases s2_side3 takes through s2_cell_faces9.
__device__ bool s2_side3_group(const S2Field& F, int axis, int cell, int tangent, double side, int gl, double dn[3],
                               double dt[3]) {
    const int ny = F.ny, j = axis == 0 ? tangent : cell, base = (threadIdx.x & 31) & ~7;
    const bool nw = s2_near_wall(j, ny);
    const int first = nw ? s2_wall_first(j, ny) : 0;
    double v = 0.0, d = 0.0;
    bool ok = true;
    if (gl < 5) {
        double q[5];
        if (nw && axis == 1) {   // column tangent + gl - 2, one-sided across the 5 true rows
#pragma unroll
            for (int t = 0; t < 5; ++t) q[t] = F.at(tangent + gl - 2, first + t);
            s2_wall_eval(q, j, ny, side, v, d);
        } else {
#pragma unroll
            for (int s = -2; s <= 2; ++s)
                q[s + 2] = nw ? F.at(cell + s, first + gl)
                              : (axis == 0 ? F.at(cell + s, tangent + gl - 2) : F.at(tangent + gl - 2, cell + s));
            S2Weno ww;
            ok = s2_weno(q, ww);
            s2_at(ww, side < 0.0 ? S2_XM : S2_XP, v, d);
        }
    }
    double v5[5], d5[5];
    int okc = ok ? 1 : 0;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        v5[r] = __shfl_sync(0xffffffffu, v, base + r);
        d5[r] = __shfl_sync(0xffffffffu, d, base + r);
        okc &= __shfl_sync(0xffffffffu, okc, base + r);
    }
    ok = okc != 0;
    if (gl == 0) {
        if (nw && axis == 0) {
            double dummy;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                s2_wall_eval(v5, j, ny, c_s2.gnode[a], dummy, dt[a]);
                s2_wall_eval(d5, j, ny, c_s2.gnode[a], dn[a], dummy);
            }
        } else {
            double val[3];
            ok = ok && s2_companion3(v5, d5, val, dt, dn);
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) ok = ok && isfinite(dn[a]) && isfinite(dt[a]);
    }
    return ok;
}

// s2d1_cell9 (:378-403; near a wall the volume part of s2d1_cell_faces9_wall) of one field: lanes
// 0..2 of the group return vol[gl][0..2]
__device__ bool s2_cell9_group(const S2Field& F, int i, int j, int gl, double vol[3]) {
    const int ny = F.ny, base = (threadIdx.x & 31) & ~7;
    const bool nw = s2_near_wall(j, ny);
    const int first = nw ? s2_wall_first(j, ny) : j - 2;
    double rw[3] = {0.0, 0.0, 0.0};
    bool ok = true;
    if (gl < 5) {   // the x first layer of row first + gl at the 3 Gauss nodes
        double q[5];
#pragma unroll
        for (int s = -2; s <= 2; ++s) q[s + 2] = F.at(i + s, first + gl);
        S2Weno ww;
        ok = s2_weno(q, ww);
#pragma unroll
        for (int a = 0; a < 3; ++a) rw[a] = s2_at_v(ww, S2_G0 + a);
    }
    double rows[5][3];
    int okc = ok ? 1 : 0;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
#pragma unroll
        for (int a = 0; a < 3; ++a) rows[r][a] = __shfl_sync(0xffffffffu, rw[a], base + r);
        okc &= __shfl_sync(0xffffffffu, okc, base + r);
    }
    ok = okc != 0;
    if (gl < 3) {
        double a5[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) a5[r] = rows[r][gl];
        if (!nw) {
            S2Weno ww;
            ok = ok && s2_weno(a5, ww);
#pragma unroll
            for (int b = 0; b < 3; ++b) vol[b] = s2_at_v(ww, S2_G0 + b);
        } else {
            double dummy;
#pragma unroll
            for (int b = 0; b < 3; ++b) s2_wall_eval(a5, j, ny, c_s2.gnode[b], vol[b], dummy);
        }
    }
    return ok;
}

// macro WENO of W: per interior face and component the normal slopes of both sides and the
// tangential slope at the 3 Gauss nodes (s2d1_face3, compute_flux :803-808,849-854), and per cell
// and component the 3x3 Gauss values and the mean-shifted volume node states (build_targets
// :1270-1279).  Faces: 2 warps per face, an 8-lane group per (component, side); cells: one warp per
// cell, an 8-lane group per component.
__global__ void __launch_bounds__(128) k_s2_macro(LoParams P, LoBuffers B, S2Buffers SB, int faces, int cells) {
    if (eval_cached(B)) return;
    const int nx = P.nx, ny = P.ny, nfx = nx * ny, nf = nfx + nx * (ny - 1), nc = nx * ny;
    int wid = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31, grp = lane >> 3, gl = lane & 7;
    const int nfw = faces ? nf * 2 : 0;
    if (wid < nfw) {
        const int fi = wid >> 1, m = (wid & 1) * 2 + (grp >> 1), right = grp & 1;
        const int axis = fi < nfx ? 0 : 1, f = axis == 0 ? fi : fi - nfx;
        const int i = f % nx, j = f / nx;
        const S2Field F{B.W + m, 4, nx, ny};
        double dn[3] = {0.0, 0.0, 0.0}, dt[3] = {0.0, 0.0, 0.0};
        bool ok;
        if (axis == 0) ok = s2_side3_group(F, 0, right ? (i + 1) % nx : i, j, right ? -0.5 : 0.5, gl, dn, dt);
        else ok = s2_side3_group(F, 1, right ? j + 1 : j, i, right ? -0.5 : 0.5, gl, dn, dt);
        // the right side's tangential derivatives to the left side's lane 0
        double tr[3];
#pragma unroll
        for (int g = 0; g < 3; ++g) tr[g] = __shfl_down_sync(0xffffffffu, dt[g], 8);
        if (gl == 0) {
            if (!ok) set_status(B.status, ST_NONFINITE_FLUX);
            const double dnrm = axis == 0 ? P.dx : P.dy, dtg = axis == 0 ? P.dy : P.dx;
#pragma unroll
            for (int g = 0; g < 3; ++g) {
                double* o = SB.mac + (size_t)(fi * 3 + g) * 12;
                o[(right ? 4 : 0) + m] = dn[g] / dnrm;
                if (!right) o[8 + m] = 0.5 * (dt[g] + tr[g]) / dtg;
            }
        }
        return;
    }
    wid -= nfw;
    if (!cells || wid >= nc) return;
    const int cc = wid, m = grp, i = cc % nx, j = cc / nx;
    const S2Field F{B.W + m, 4, nx, ny};
    double vol[3] = {0.0, 0.0, 0.0};
    const bool ok = s2_cell9_group(F, i, j, gl, vol);
    if (__any_sync(0xffffffffu, !ok) && lane == 0) set_status(B.status, ST_PROJECTION);
    // nodes[a][c] = vol of lane a, entry c; the mean over the 9 nodes in the reference's order
    const int base = lane & ~7;
    double nodes[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) nodes[a][c] = __shfl_sync(0xffffffffu, vol[c], base + a);
    const double gw[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
    double avg = 0.0;
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 3; ++a) avg = avg + gw[a] * gw[c] * nodes[a][c];
    const double wc = B.W[cc * 4 + m];
    if (gl < 3)
        for (int c = 0; c < 3; ++c) SB.wq[((size_t)cc * 9 + c * 3 + gl) * 4 + m] = nodes[gl][c] + wc - avg;
}

// The face-node closure kernel comes in two CTA shapes.  A single instance runs it in 128-thread
// CTAs, three per SM: up to 170 registers a thread (no spills) at 12 warps per SM, faster per step
// than two 256-thread CTAs per SM capped at 128 registers (which spill the closure's state).  Many
// instances on concurrent streams (S2Buffers::concurrent) gain more from the 16 resident warps of
// the 256-thread shape, which they keep.  The volume-node kernel is fastest in the 256-thread shape
// in both cases.
constexpr int kS2NodeThreads = 128;

// build_targets, closure part: one warp per (cell, volume node) -> the node scalars
__global__ void __launch_bounds__(256, 2) k_s2_target_nodes(LoParams P, LoBuffers B, S2Buffers SB) {
    if (eval_cached(B)) return;
    const int nc = P.nx * P.ny, lane = threadIdx.x & 31;
    const int wid = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (wid >= nc * 9) return;
    __shared__ double s_jac[8][16];
    double w[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) w[m] = SB.wq[(size_t)wid * 4 + m];
    WClosure C;
    C.jac = s_jac[threadIdx.x >> 5];
    WMke M;
    const bool ok = w_closure(P, B, w, C) && w_make_mke(P, B, w, C, M);
    if (lane == 0) {
        if (ok) w_store_scalars(SB.tscal + (size_t)wid * kS2TScal, C, M);
        else set_status(B.status, ST_PROJECTION);
    }
}

// build_targets, sum part: per (cell, velocity) the Gauss-weighted M, K_x, K_y of the 9 nodes
__global__ void __launch_bounds__(256) k_s2_target_sum(LoParams P, LoBuffers B, S2Buffers SB) {
    if (eval_cached(B)) return;
    const int nv = P.nvel, cc = blockIdx.y;
    const int k = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (k >= nv) return;
    const double uk = B.u[k], vk = B.v[k];
    const double gw[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
    double amh = 0.0, amb = 0.0, akxh = 0.0, akxb = 0.0, akyh = 0.0, akyb = 0.0;
    for (int p = 0; p < 9; ++p) {
        double th[4];
        WMke M;
        w_load_scalars(SB.tscal + ((size_t)cc * 9 + p) * kS2TScal, th, M);
        S2Q q;
        double mh, mb, kxh, kxb, kyh, kyb;
        w_mke_at(s2_th(th, P.ck), M, P.ck, uk, vk, q, mh, mb, kxh, kxb, kyh, kyb);
        const double wt2 = gw[p % 3] * gw[p / 3];
        amh = amh + wt2 * mh; amb = amb + wt2 * mb;
        akxh = akxh + wt2 * kxh; akxb = akxb + wt2 * kxb;
        akyh = akyh + wt2 * kyh; akyb = akyb + wt2 * kyb;
    }
    const size_t q = (size_t)cc * nv + k;
    SB.mh[q] = amh; SB.mb[q] = amb; SB.kxh[q] = akxh; SB.kxb[q] = akxb; SB.kyh[q] = akyh; SB.kyb[q] = akyb;
}

// ------------------------------------------------------------------------------------------
// interior face nodes (ugks_node, mod_S2D1.f90:421-521), scalar part: one warp per (face, Gauss
// node) -- the right x face of every cell, then the top y face of every cell below the last row --
// computes W0, the closure, make_mke, q0, the slope and time directions and Mt, and stores them as
// the node's scalars (SB.fscal) for k_s2_face_flux.
constexpr int kS2FScal = 48;   // [0] ok, [1..4] theta, [5..12] K directions, [13..16] ux vy lam coeff,
                               // [17..18] q0, [19..34] left/right/tangential/time directions, [35..39] Mt,
                               // [40..43] the time-direction moments wt
template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_s2_face_nodes(LoParams P, LoBuffers B, S2Buffers SB) {
    if (eval_cached(B)) return;
    const int nv = P.nvel, nx = P.nx, ny = P.ny, ck = P.ck, lane = threadIdx.x & 31, nr = (nv + 31) >> 5;
    const int nfx = nx * ny, nf = nfx + nx * (ny - 1);
    const int wid = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (wid >= nf * 3) return;
    const int fi = wid / 3, g = wid % 3;
    const int axis = fi < nfx ? 0 : 1, f = axis == 0 ? fi : fi - nfx;
    const int cl = f, i = cl % nx, j = cl / nx;
    const int cr = axis == 0 ? j * nx + (i + 1) % nx : (j + 1) * nx + i;
    const int sl = axis == 0 ? 1 : 3, sr = axis == 0 ? 0 : 2;
    const double dt = B.dt[0];
    const double* mac = SB.mac + (size_t)wid * 12;   // [nl | nr | t][component] of this node
    auto upwind = [&](const WVel& s, int field) {
        const double vn = axis == 0 ? s.u : s.v;
        const bool left = vn >= 0.0;
        return SB.rec[((size_t)(left ? cl : cr) * 72 + field * 12 + (left ? sl : sr) * 3 + g) * nv + s.k];
    };
    // W0: moments of the upwind face values
    double acc[16];
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[m] = 0.0;
    for (int r = 0; r < nr; ++r) {
        const WVel s = wvel(B, nv, r);
        moment_add(s.w, s.u, s.v, upwind(s, 0), upwind(s, 1), acc);
    }
    warp_sum_all<4>(acc);
    const double w0[4] = {acc[0], acc[1], acc[2], acc[3]};
    __shared__ double s_jac[NT / 32][16];
    WClosure C;
    C.jac = s_jac[threadIdx.x >> 5];
    WMke M;
    bool ok = w_closure(P, B, w0, C) && w_make_mke(P, B, w0, C, M);
    double q0x = 0.0, q0y = 0.0, tdl[4], tdr[4], tdt[4], tdm[4], wt[4], mt[5];
    if (ok) {   // q0 = heat(w0, f0 - analytic Maxwellian of w0)
        const double nrho = w0[0], nu = w0[1] / w0[0], nvv = w0[2] / w0[0];
        const double temp = 4.0 * (w0[3] / w0[0] - 0.5 * (nu * nu + nvv * nvv)) / (double)(ck + 2);
        const double lamn = 1.0 / temp;
        // directions of the macro normal slopes (left, right) and the tangential slope
        const bool okd = s2_solve4(C.jac, mac, tdl) & s2_solve4(C.jac, mac + 4, tdr) & s2_solve4(C.jac, mac + 8, tdt);
        if (!okd)
#pragma unroll
            for (int m = 0; m < 4; ++m) tdl[m] = tdr[m] = tdt[m] = NAN;
        // one pass over the velocities for q0 (qacc) and the direction moments (acc): two independent
        // chains per velocity, each summed in velocity order and reduced on its own
        double qacc[2] = {0.0, 0.0};
#pragma unroll
        for (int m = 0; m < 16; ++m) acc[m] = 0.0;
        const S2Th tt = s2_th(C.th, ck);
        for (int r = 0; r < nr; ++r) {
            const WVel s = wvel(B, nv, r);
            {
                const double du = s.u - nu, dv = s.v - nvv;
                const double eah = nrho * lamn / kPi * exp(-lamn * (du * du + dv * dv));
                const double eab = 0.5 * (double)ck * temp * eah;
                const double cx = s.u - M.ux, cy = s.v - M.vy, c2 = cx * cx + cy * cy;
                const double dh = upwind(s, 0) - eah, db = upwind(s, 1) - eab;
                qacc[0] += 0.5 * s.w * cx * (c2 * dh + db);
                qacc[1] += 0.5 * s.w * cy * (c2 * dh + db);
            }
            const S2Q q = s2_q(tt, s.u, s.v);
            double dlh, dlb, drh, drb, dth, dtb;
            s2_dq(q, tdl, dlh, dlb);
            s2_dq(q, tdr, drh, drb);
            s2_dq(q, tdt, dth, dtb);
            moment_add(s.w, s.u, s.v, dlh, dlb, acc);
            moment_add(s.w, s.u, s.v, drh, drb, acc + 4);
            moment_add(s.w, s.u, s.v, dth, dtb, acc + 8);
            const double vn = axis == 0 ? s.u : s.v, vt = axis == 0 ? s.v : s.u;
            const double fh = vn * (vn >= 0.0 ? dlh : drh) + vt * dth;
            const double fb = vn * (vn >= 0.0 ? dlb : drb) + vt * dtb;
            moment_add(s.w, s.u, s.v, fh, fb, acc + 12);
        }
        warp_sum_all<2>(qacc);
        q0x = qacc[0];
        q0y = qacc[1];
        warp_sum_all<16>(acc);
        for (int d = 0; d < 3; ++d) {   // gates of the three directions
            double mx = 0.0, sc = 1.0;
            for (int m = 0; m < 4; ++m) {
                mx = fmax(mx, fabs(acc[4 * d + m] - mac[4 * d + m]));
                sc = fmax(sc, fabs(mac[4 * d + m]));
            }
            ok = ok && mx / sc <= 2.0e-12;
        }
        // the time direction and the time coefficients Mt (mod_Evolution.f90:346-350)
#pragma unroll
        for (int m = 0; m < 4; ++m) wt[m] = -acc[12 + m];
        ok = ok && s2_solve4(C.jac, wt, tdm);
        double tau = 0.0;
        ok = ok && s2_tau(P, w0, tau);
        const double ex = exp(-dt / tau);
        mt[3] = tau * (1.0 - ex);
        mt[4] = -tau * dt * ex + tau * mt[3];
        mt[0] = dt - mt[3];
        mt[1] = -tau * mt[0] + mt[4];
        mt[2] = 0.5 * dt * dt - tau * mt[0];
    }
    // the node scalars of the flux pass (k_s2_face_flux)
    if (lane == 0) {
        double* o = SB.fscal + (size_t)wid * kS2FScal;
        o[0] = ok ? 1.0 : 0.0;
        if (ok) {
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                o[1 + m] = C.th[m]; o[5 + m] = M.tdx[m]; o[9 + m] = M.tdy[m];
                o[19 + m] = tdl[m]; o[23 + m] = tdr[m]; o[27 + m] = tdt[m]; o[31 + m] = tdm[m]; o[40 + m] = wt[m];
            }
            o[13] = M.ux; o[14] = M.vy; o[15] = M.lam; o[16] = M.coeff; o[17] = q0x; o[18] = q0y;
#pragma unroll
            for (int m = 0; m < 5; ++m) o[35 + m] = mt[m];
        } else {
            set_status(B.status, ST_NONFINITE_FLUX);
        }
    }
}

// ugks_node's flux at one face Gauss node (mod_S2D1.f90:486-507): one CTA per (face, node), VPT
// velocities per thread, from the node scalars; the node micro flux goes to SB.node, its moments to
// SB.nodew, and the time-direction moment gate (2e-12) is checked on the block-reduced moments.
// Three CTAs per SM (80 registers, small spills): the kernel waits on its face-cache loads, and 24
// resident warps hide that better than 16.
template <int VPT>
__global__ void __launch_bounds__(256, 3) k_s2_face_flux(LoParams P, LoBuffers B, S2Buffers SB) {
    if (eval_cached(B)) return;
    __shared__ double sc[kS2FScal];
    __shared__ double red[8 * 8];
    __shared__ double rout[kRedSlots];
    const int nv = P.nvel, nx = P.nx, ny = P.ny, ck = P.ck;
    const int nfx = nx * ny;
    const int wid = blockIdx.x, fi = wid / 3, g = wid % 3;
    const int axis = fi < nfx ? 0 : 1, f = axis == 0 ? fi : fi - nfx;
    const int cl = f, i = cl % nx, j = cl / nx;
    const int cr = axis == 0 ? j * nx + (i + 1) % nx : (j + 1) * nx + i;
    const int sl = axis == 0 ? 1 : 3, sr = axis == 0 ? 0 : 2;
    if (threadIdx.x < kS2FScal) sc[threadIdx.x] = SB.fscal[(size_t)wid * kS2FScal + threadIdx.x];
    __syncthreads();
    if (sc[0] == 0.0) return;   // the scalars kernel failed (status set there)
    double th[4], tdl[4], tdr[4], tdt[4], tdm[4], mt[5];
    WMke M;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        th[m] = sc[1 + m]; M.tdx[m] = sc[5 + m]; M.tdy[m] = sc[9 + m];
        tdl[m] = sc[19 + m]; tdr[m] = sc[23 + m]; tdt[m] = sc[27 + m]; tdm[m] = sc[31 + m];
    }
    M.ux = sc[13]; M.vy = sc[14]; M.lam = sc[15]; M.coeff = sc[16];
    const double q0x = sc[17], q0y = sc[18];
#pragma unroll
    for (int m = 0; m < 5; ++m) mt[m] = sc[35 + m];
    const S2Th tt = s2_th(th, ck);
    double* outh = SB.node + (size_t)wid * 2 * nv;
    double* outb = outh + nv;
    double acc[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) acc[m] = 0.0;
    int bad = 0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot sl_ = slot(r, nv);
        const int k = sl_.kk;
        const double uk = B.u[k], vk = B.v[k], wk = sl_.ok ? B.w[k] : 0.0;
        S2Q q;
        double mh, mb, kxh, kxb, kyh, kyb;
        w_mke_at(tt, M, ck, uk, vk, q, mh, mb, kxh, kxb, kyh, kyb);
        const double s0h = mh + kxh * q0x + kyh * q0y;
        const double s0b = mb + kxb * q0x + kyb * q0y;
        double dlh, dlb, drh, drb, dth, dtb, mth, mtb;
        s2_dq(q, tdl, dlh, dlb);
        s2_dq(q, tdr, drh, drb);
        s2_dq(q, tdt, dth, dtb);
        s2_dq(q, tdm, mth, mtb);
        moment_add(wk, uk, vk, mth, mtb, acc);
        const double vn = axis == 0 ? uk : vk, vt = axis == 0 ? vk : uk;
        const bool left = vn >= 0.0;
        const double* rc = SB.rec + ((size_t)(left ? cl : cr) * 72 + (left ? sl : sr) * 3 + g) * nv + k;
        const double f0h = rc[0], f0b = rc[(size_t)12 * nv], nh = rc[(size_t)24 * nv], th_ = rc[(size_t)36 * nv];
        const double nb = rc[(size_t)48 * nv], tb_ = rc[(size_t)60 * nv];
        const double sh = vn * (left ? dlh : drh) + vt * dth;
        const double sb = vn * (left ? dlb : drb) + vt * dtb;
        const double fhv = vn * (mt[0] * s0h + mt[1] * sh + mt[2] * mth + mt[3] * f0h - mt[4] * (vn * nh + vt * th_));
        const double fbv = vn * (mt[0] * s0b + mt[1] * sb + mt[2] * mtb + mt[3] * f0b - mt[4] * (vn * nb + vt * tb_));
        moment_add(wk, uk, vk, fhv, fbv, acc + 4);
        if (sl_.ok) {
            outh[sl_.k] = fhv;
            outb[sl_.k] = fbv;
            if (!(isfinite(fhv) && isfinite(fbv))) bad = 1;
        }
    }
    block_reduce_smem<8, 0>(acc, red, rout);
    bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) {
        double mx = 0.0, scl = 1.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) { mx = fmax(mx, fabs(rout[m] - sc[40 + m])); scl = fmax(scl, fabs(sc[40 + m])); }
#pragma unroll
        for (int m = 0; m < 4; ++m) SB.nodew[(size_t)wid * 4 + m] = rout[4 + m];
        if (bad || !(mx / scl <= 2.0e-12)) set_status(B.status, ST_NONFINITE_FLUX);
    }
}

// ------------------------------------------------------------------------------------------
// MicroSlope / CalcMoment / Moment_auvxi of mod_S2MultiscaleWall.f90:227-335
__device__ void s2w_micro_slope(int ck, const double pr[4], const double sw[4], double a[4]) {
    a[3] = 4.0 * (pr[3] * pr[3]) / ((double)(ck + 2) * pr[0]) *
           (2.0 * sw[3] - 2.0 * pr[1] * sw[1] - 2.0 * pr[2] * sw[2] +
            sw[0] * (pr[1] * pr[1] + pr[2] * pr[2] - 0.5 * (double)(ck + 2) / pr[3]));
    a[2] = 2.0 * pr[3] / pr[0] * (sw[2] - pr[2] * sw[0]) - pr[2] * a[3];
    a[1] = 2.0 * pr[3] / pr[0] * (sw[1] - pr[1] * sw[0]) - pr[1] * a[3];
    a[0] = sw[0] / pr[0] - pr[1] * a[1] - pr[2] * a[2] -
           0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + 0.5 * (double)(ck + 2) / pr[3]) * a[3];
}

__device__ void s2w_moments(int ck, const double pr[4], double Mu[7], double Mv[6], double Mxi[3]) {
    double MuL[7], MuR[7];
    MuL[0] = 0.5 * erfc(-sqrt(pr[3]) * pr[1]);
    MuL[1] = pr[1] * MuL[0] + 0.5 * exp(-pr[3] * (pr[1] * pr[1])) / sqrt(kPi * pr[3]);
    MuR[0] = 0.5 * erfc(sqrt(pr[3]) * pr[1]);
    MuR[1] = pr[1] * MuR[0] - 0.5 * exp(-pr[3] * (pr[1] * pr[1])) / sqrt(kPi * pr[3]);
    for (int i = 2; i <= 6; ++i) {
        MuL[i] = pr[1] * MuL[i - 1] + 0.5 * (double)(i - 1) * MuL[i - 2] / pr[3];
        MuR[i] = pr[1] * MuR[i - 1] + 0.5 * (double)(i - 1) * MuR[i - 2] / pr[3];
    }
    for (int i = 0; i <= 6; ++i) Mu[i] = MuL[i] + MuR[i];
    Mv[0] = 1.0;
    Mv[1] = pr[2];
    for (int i = 2; i <= 5; ++i) Mv[i] = pr[2] * Mv[i - 1] + 0.5 * (double)(i - 1) * Mv[i - 2] / pr[3];
    Mxi[0] = 1.0;
    Mxi[1] = 0.5 * (double)ck / pr[3];
    Mxi[2] = (double)ck * ((double)ck + 2.0) / (4.0 * (pr[3] * pr[3]));
}

__device__ void s2w_auvxi(const double a[4], const double Mu[7], const double Mv[6], const double Mxi[3], int al, int be,
                          double o[4]) {
    double t[6][4];
    const int A[6] = {al, al + 1, al, al + 2, al, al}, Bb[6] = {be, be, be + 1, be, be + 2, be}, D[6] = {0, 0, 0, 0, 0, 2};
    for (int q = 0; q < 6; ++q) {
        t[q][0] = Mu[A[q]] * Mv[Bb[q]] * Mxi[D[q] / 2];
        t[q][1] = Mu[A[q] + 1] * Mv[Bb[q]] * Mxi[D[q] / 2];
        t[q][2] = Mu[A[q]] * Mv[Bb[q] + 1] * Mxi[D[q] / 2];
        t[q][3] = 0.5 * (Mu[A[q] + 2] * Mv[Bb[q]] * Mxi[D[q] / 2] + Mu[A[q]] * Mv[Bb[q] + 2] * Mxi[D[q] / 2] +
                         Mu[A[q]] * Mv[Bb[q]] * Mxi[(D[q] + 2) / 2]);
    }
    for (int m = 0; m < 4; ++m)
        o[m] = a[0] * t[0][m] + a[1] * t[1][m] + a[2] * t[2][m] + 0.5 * a[3] * t[3][m] + 0.5 * a[3] * t[4][m] +
               0.5 * a[3] * t[5][m];
}

// s2w2_time_coefficients (:18-43)
__device__ void s2w_time_coeffs(double dt, double tau, double mt[5]) {
    const double x = dt / tau;
    if (x < 0.1) {
        double t = 1.0;
        for (int m = 0; m < 5; ++m) mt[m] = 0.0;
        for (int n = 1; n <= 24; ++n) {
            t = t * (-x) / (double)n;
            mt[3] = mt[3] - tau * t;
            if (n >= 2) { mt[0] = mt[0] + tau * t; mt[4] = mt[4] + tau * tau * (double)(n - 1) * t; }
            if (n >= 3) { mt[1] = mt[1] + tau * tau * (double)(n - 2) * t; mt[2] = mt[2] - tau * tau * t; }
        }
    } else {
        const double ex = exp(-x);
        mt[3] = tau * (1.0 - ex);
        mt[4] = -tau * dt * ex + tau * mt[3];
        mt[0] = dt - mt[3];
        mt[1] = -tau * mt[0] + mt[4];
        mt[2] = 0.5 * (dt * dt) - tau * mt[0];
    }
}


// wall face nodes (s2w2_wall_node, mod_S2MultiscaleWall.f90:45-184): one warp per (wall face,
// Gauss node); bottom faces of row 0, then top faces of row ny-1.  Node fluxes go to the node
// buffers after the interior faces.
__global__ void __launch_bounds__(256, 2) k_s2_wall_nodes(LoParams P, LoBuffers B, S2Buffers SB) {
    if (eval_cached(B)) return;
    const int nv = P.nvel, nx = P.nx, ny = P.ny, ck = P.ck, lane = threadIdx.x & 31, nr = (nv + 31) >> 5;
    const int nf = nx * ny + nx * (ny - 1);
    const int wid = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (wid >= 2 * nx * 3) return;
    const int wf = wid / 3, g = wid % 3;
    const int top = wf >= nx ? 1 : 0, i = wf - top * nx;
    const int cc = top ? (ny - 1) * nx + i : i, sidx = top ? 3 : 2;
    const size_t node = (size_t)(nf + wf) * 3 + g;
    const double side = top ? 1.0 : -1.0;
    const double ux = P.wall_ux[top], theta = 0.5 / P.wall_lam[top];
    const double dt = B.dt[0];
    const double* wcell = B.W + cc * 4;
    const double pp = (2.0 / (double)(ck + 2)) * (wcell[3] - 0.5 * (wcell[1] * wcell[1] + wcell[2] * wcell[2]) / wcell[0]);
    const double lambda = 0.5 / theta;
    const double prim_g[4] = {pp / theta, 0.0, -ux, lambda};
    const double wc[4] = {wcell[0], wcell[2], -wcell[1], wcell[3]};
    const double wg[4] = {prim_g[0], 0.0, -prim_g[0] * ux, prim_g[0] * ((double)(ck + 2) / (4.0 * lambda) + 0.5 * ux * ux)};
    // wall_equilibrium: the discrete closure of the wall state
    const double wwall[4] = {prim_g[0], prim_g[0] * ux, 0.0, prim_g[0] * ((double)(ck + 2) * theta / 2.0 + ux * ux / 2.0)};
    __shared__ double s_jac[8][16];
    WClosure C;
    C.jac = s_jac[threadIdx.x >> 5];
    bool ok = pp > 0.0 && isfinite(pp) && w_closure(P, B, wwall, C);
    auto rec = [&](const WVel& s, int field) {
        return SB.rec[((size_t)cc * 72 + field * 12 + sidx * 3 + g) * nv + s.k];
    };
    double acc[8];
    double an[4], at[4], atime[4], mt[5], mxi2 = 0.0, coeff = 0.0, hlx = 0.0, hly = 0.0;
    if (ok) {
#pragma unroll
        for (int m = 0; m < 6; ++m) acc[m] = 0.0;
        for (int r = 0; r < nr; ++r) {
            const WVel s = wvel(B, nv, r);
            const double hin = rec(s, 0), bin = rec(s, 1), ht = rec(s, 3), bt = rec(s, 5);
            const double vn = s.v, vt = -s.u, v2 = vn * vn + vt * vt;
            acc[0] += s.w * (-ht);
            acc[1] += s.w * (-(vn * ht));
            acc[2] += s.w * (-(vt * ht));
            acc[3] += s.w * (-(0.5 * (v2 * ht + bt)));
            const double vt2 = -s.u + ux, w2 = vn * vn + vt2 * vt2;
            acc[4] += 0.5 * s.w * vn * (w2 * hin + bin);
            acc[5] += 0.5 * s.w * vt2 * (w2 * hin + bin);
        }
        warp_sum_all<6>(acc);
        double sw[4], sw_t[4], Mu[7], Mv[6], Mxi[3], m1[4], m2[4];
        for (int m = 0; m < 4; ++m) { sw[m] = (wg[m] - wc[m]) / (side * 0.5 * P.dy); sw_t[m] = acc[m]; }
        s2w_micro_slope(ck, prim_g, sw, an);
        s2w_micro_slope(ck, prim_g, sw_t, at);
        s2w_moments(ck, prim_g, Mu, Mv, Mxi);
        s2w_auvxi(an, Mu, Mv, Mxi, 1, 0, m1);
        s2w_auvxi(at, Mu, Mv, Mxi, 0, 1, m2);
        for (int m = 0; m < 4; ++m) sw[m] = -prim_g[0] * (m1[m] + m2[m]);
        s2w_micro_slope(ck, prim_g, sw, atime);
        double tau_wall = 0.0;
        const double wgg[4] = {wg[0], -wg[2], wg[1], wg[3]};
        ok = s2_tau(P, wgg, tau_wall);
        s2w_time_coeffs(dt, tau_wall, mt);
        coeff = P.pr != 1.0 ? 0.8 * (1.0 - P.pr) * lambda * lambda / prim_g[0] : 0.0;
        mxi2 = Mxi[2];
        hlx = acc[4];
        hly = acc[5];
    }
    // the incident micro flux g_in and the reflected wall Maxwellian of one velocity
    const S2Th tt = s2_th(C.th, ck);
    auto gin = [&](const WVel& s, double& ginh, double& ginb, double& wallh, double& wallb) {
        const S2Q q = s2_q(tt, s.u, s.v);
        const double mh = q.qh, mb = q.qb;
        wallh = mh / prim_g[0];
        wallb = mb / prim_g[0];
        double corrh = 0.0, corrb = 0.0;
        if (P.pr != 1.0) {
            const double vn = s.v, vt = -s.u + ux, v2 = vn * vn + vt * vt;
            const double qdot = vn * hlx + vt * hly, shh = 2.0 * lambda * v2 - 4.0;
            corrh = coeff * qdot * shh * mh;
            corrb = coeff * qdot * (shh + 2.0 / (double)ck) * mb;
        }
        const double vn = s.v, vt = -s.u, v2 = vn * vn + vt * vt;
        const double Han = (an[0] + an[1] * vn + an[2] * vt) * mh + 0.5 * an[3] * (v2 * mh + mb);
        const double Hatan = (at[0] + at[1] * vn + at[2] * vt) * mh + 0.5 * at[3] * (v2 * mh + mb);
        const double Hatime = (atime[0] + atime[1] * vn + atime[2] * vt) * mh + 0.5 * atime[3] * (v2 * mh + mb);
        const double Ban = (an[0] + an[1] * vn + an[2] * vt) * mb + 0.5 * an[3] * (v2 * mb + mxi2 * mh);
        const double Batan = (at[0] + at[1] * vn + at[2] * vt) * mb + 0.5 * at[3] * (v2 * mb + mxi2 * mh);
        const double Batime = (atime[0] + atime[1] * vn + atime[2] * vt) * mb + 0.5 * atime[3] * (v2 * mb + mxi2 * mh);
        ginh = mt[0] * mh + mt[1] * (vn * Han + vt * Hatan) + mt[2] * Hatime + mt[3] * rec(s, 0) -
               mt[4] * (vn * rec(s, 2) + s.u * rec(s, 3));
        ginb = mt[0] * mb + mt[1] * (vn * Ban + vt * Batan) + mt[2] * Batime + mt[3] * rec(s, 1) -
               mt[4] * (vn * rec(s, 4) + s.u * rec(s, 5));
        ginh = ginh + mt[0] * corrh;
        ginb = ginb + mt[0] * corrb;
    };
    double inc = 0.0, rhow = 0.0;
    if (ok) {   // incidence and reflection -> wall density
        acc[0] = acc[1] = 0.0;
        for (int r = 0; r < nr; ++r) {
            const WVel s = wvel(B, nv, r);
            double ginh, ginb, wallh, wallb;
            gin(s, ginh, ginb, wallh, wallb);
            if (side * s.v > 0.0) acc[0] += s.w * s.v * ginh;
            else acc[1] += dt * s.w * s.v * wallh;
        }
        warp_sum_all<2>(acc);
        inc = acc[0];
        const double refl = acc[1];
        rhow = -inc / refl;
        ok = isfinite(refl) && fabs(refl) > DBL_MIN && isfinite(rhow) && rhow > 0.0;
    }
    if (ok) {
        double* outh = SB.node + node * 2 * nv;
        double* outb = outh + nv;
#pragma unroll
        for (int m = 0; m < 4; ++m) acc[m] = 0.0;
        for (int r = 0; r < nr; ++r) {
            const WVel s = wvel(B, nv, r);
            double ginh, ginb, wallh, wallb, fh, fb;
            gin(s, ginh, ginb, wallh, wallb);
            if (side * s.v > 0.0) { fh = s.v * ginh; fb = s.v * ginb; }
            else { fh = dt * s.v * rhow * wallh; fb = dt * s.v * rhow * wallb; }
            acc[0] += s.w * fh; acc[1] += s.w * (s.u * fh); acc[2] += s.w * (s.v * fh);
            acc[3] += s.w * (0.5 * ((s.u * s.u + s.v * s.v) * fh + fb));
            if (s.ok) {
                outh[s.k] = fh;
                outb[s.k] = fb;
                ok = ok && isfinite(fh) && isfinite(fb);
            }
        }
        warp_sum_all<4>(acc);
        ok = ok && isfinite(acc[0]) && fabs(acc[0]) <= 2.0e-12 * fmax(1.0, fabs(inc));
        if (lane < 4) SB.nodew[node * 4 + lane] = lane == 0 ? acc[0] : (lane == 1 ? acc[1] : (lane == 2 ? acc[2] : acc[3]));
    }
    ok = __all_sync(0xffffffffu, ok);
    if (!ok && lane == 0) set_status(B.status, ST_NONFINITE_FLUX);
}

// Gauss-weighted sum of the node fluxes of every face (interior, then the walls) times the face
// length, into the face arrays ComputeResidual reads; the walls' macro fluxes also unscaled into
// SB.wall_raw, and the walls' (pnn, pnt, qn) into B.wall_aero.  One thread per (face, velocity);
// threads k < 4 also do the macro flux.
__global__ void __launch_bounds__(256) k_s2_combine(LoParams P, LoBuffers B, S2Buffers SB) {
    if (eval_cached(B)) return;
    const int nv = P.nvel, nx = P.nx, ny = P.ny, nfx = nx * ny, nf = nfx + nx * (ny - 1);
    const int fi = blockIdx.y;
    const int k = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (k >= nv) return;
    const double gw[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
    size_t o;
    double len, *Fh, *Fb, *Fw;
    int wall = -1;
    if (fi < nfx) {
        const int i = fi % nx, j = fi / nx;
        o = (size_t)j * nx + (i + 1) % nx; len = P.dy; Fh = B.fxh; Fb = B.fxb; Fw = B.fxw;
    } else if (fi < nf) {
        const int f = fi - nfx, i = f % nx, j = f / nx;
        o = (size_t)(j + 1) * nx + i; len = P.dx; Fh = B.fyh; Fb = B.fyb; Fw = B.fyw;
    } else {
        wall = fi - nf;
        const int top = wall >= nx ? 1 : 0, i = wall - top * nx;
        o = top ? (size_t)ny * nx + i : (size_t)i; len = P.dx; Fh = B.fyh; Fb = B.fyb; Fw = B.fyw;
    }
    const double* nd = SB.node + (size_t)fi * 3 * 2 * nv;
    double afh = 0.0, afb = 0.0;
#pragma unroll
    for (int g = 0; g < 3; ++g) {
        afh = afh + gw[g] * nd[(size_t)(2 * g) * nv + k];
        afb = afb + gw[g] * nd[(size_t)(2 * g + 1) * nv + k];
    }
    Fh[o * nv + k] = afh * len;
    Fb[o * nv + k] = afb * len;
    if (k < 4) {
        double afw = 0.0;
#pragma unroll
        for (int g = 0; g < 3; ++g) afw = afw + gw[g] * SB.nodew[((size_t)fi * 3 + g) * 4 + k];
        Fw[o * 4 + k] = afw * len;
        if (wall >= 0 && SB.wall_raw != nullptr) SB.wall_raw[(size_t)wall * 4 + k] = afw;
    }
    if (wall >= 0 && k == 0) {   // PublishWallDiagnostics (mod_S2NativeAdapter.f90:1075-1097)
        const int top = wall >= nx ? 1 : 0;
        const double measure = B.dt[0] * len;
        double rate[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            double afw = 0.0;
#pragma unroll
            for (int g = 0; g < 3; ++g) afw = afw + gw[g] * SB.nodew[((size_t)fi * 3 + g) * 4 + m];
            rate[m] = afw * len / measure;
        }
        // native frame n = +y, t = -x; the heat removes the moving wall's mechanical work
        double* a = B.wall_aero + (size_t)wall * 3;
        a[0] = rate[2];
        a[1] = -rate[1];
        a[2] = rate[3] - P.wall_ux[top] * rate[1];
    }
}

// ------------------------------------------------------------------------------------------
// host side

// build_map / solve_small (mod_S2D1Reconstruction.f90:81-166), the same arithmetic on the host
static void s2_solve_small_host(int n, double a[5][5], double b[5], double x[5]) {
    for (int p = 0; p < n - 1; ++p) {
        int m = p;
        double best = std::fabs(a[p][p]);
        for (int i = p + 1; i < n; ++i) if (std::fabs(a[i][p]) > best) { best = std::fabs(a[i][p]); m = i; }
        if (m != p) {
            for (int j = 0; j < n; ++j) std::swap(a[p][j], a[m][j]);
            std::swap(b[p], b[m]);
        }
        for (int i = p + 1; i < n; ++i) {
            const double fac = a[i][p] / a[p][p];
            for (int j = p; j < n; ++j) a[i][j] = a[i][j] - fac * a[p][j];
            b[i] = b[i] - fac * b[p];
        }
    }
    x[n - 1] = b[n - 1] / a[n - 1][n - 1];
    for (int i = n - 2; i >= 0; --i) {
        double s = 0.0;
        for (int j = i + 1; j < n; ++j) s = s + a[i][j] * x[j];
        x[i] = (b[i] - s) / a[i][i];
    }
}

static void s2_build_map_host(int n, const int* off, bool ordered, double map[5][5]) {
    for (int k = 0; k < 5; ++k) for (int d = 0; d < 5; ++d) map[k][d] = 0.0;
    for (int c = 0; c < n; ++c) {
        double a[5][5], rhs[5], x[5];
        for (int r = 0; r < n; ++r)
            for (int d = 0; d < n; ++d)
                a[r][d] = (std::pow((double)off[r] + 0.5, d + 1) - std::pow((double)off[r] - 0.5, d + 1)) / (double)(d + 1);
        for (int r = 0; r < n; ++r) rhs[r] = 0.0;
        rhs[c] = 1.0;
        s2_solve_small_host(n, a, rhs, x);
        const int slot = ordered ? c : off[c] + 2;
        for (int d = 0; d < n; ++d) map[slot][d] = x[d];
    }
}

cudaError_t prepare_s2() {
    static S2Maps m;
    const int o1[3] = {-2, -1, 0}, o2[3] = {-1, 0, 1}, o3[3] = {0, 1, 2}, o5[5] = {-2, -1, 0, 1, 2};
    s2_build_map_host(3, o1, false, m.cmap[0]);
    s2_build_map_host(3, o2, false, m.cmap[1]);
    s2_build_map_host(3, o3, false, m.cmap[2]);
    s2_build_map_host(5, o5, false, m.cmap[3]);
    for (int j = 1; j <= 3; ++j) {
        int lo[5], hi[5];
        for (int s = 0; s < 5; ++s) { lo[s] = (s + 1) - j; hi[s] = (s - 4) + j - 1; }
        s2_build_map_host(5, lo, true, m.wall[0][j - 1]);
        s2_build_map_host(5, hi, true, m.wall[1][j - 1]);
    }
    const double g = 0.5 * std::sqrt(3.0 / 5.0);
    m.gnode[0] = -g; m.gnode[1] = 0.0; m.gnode[2] = g;
    // value and derivative weights of every candidate at the 5 evaluation points
    static S2PointW pw;
    const double xs[5] = {-0.5, 0.5, m.gnode[0], m.gnode[1], m.gnode[2]};
    for (int p = 0; p < 5; ++p)
        for (int c = 0; c < 4; ++c)
            for (int k = 0; k < 5; ++k) {
                double e = 0.0, d = 0.0, x = 1.0, xd = 0.0;   // x = xi^d, xd = d xi^(d-1)
                for (int q = 0; q < 5; ++q) {
                    e = e + m.cmap[c][k][q] * x;
                    d = d + m.cmap[c][k][q] * xd;
                    xd = (double)(q + 1) * x;
                    x = x * xs[p];
                }
                pw.E[p][c][k] = e;
                pw.D[p][c][k] = d;
            }
    cudaError_t e = cudaMemcpyToSymbol(c_s2, &m, sizeof m);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_s2p, &pw, sizeof pw);
    return e;
}


// which 0: the S2 cold start; 1: the S2 Evolution of one pseudo-step (targets, reconstruction,
// faces, walls); 2: the Evolution with the targets kept (S2CN2); 3: the targets of B.W only
cudaError_t s2_enqueue(int which, const LoParams& P, const LoBuffers& B, const S2Buffers& S, cudaStream_t s,
                       cudaStream_t s2, cudaEvent_t fork, cudaEvent_t join) {
    const int nx = P.nx, ny = P.ny, nv = P.nvel, nc = nx * ny, nf = nx * ny + nx * (ny - 1);
    auto warps = [](long long n) { return (unsigned)((n * 32 + 255) / 256); };
    auto node_ctas = [](long long n) { return (unsigned)((n * 32 + kS2NodeThreads - 1) / kS2NodeThreads); };
    if (which == 0) {
        k_s2_init<<<warps(nc), 256, 0, s>>>(P, B, S);
        return cudaGetLastError();
    }
    const int faces = which != 3, targets = which != 2;
    const long long nmacw = (faces ? (long long)nf * 2 : 0) + (targets ? (long long)nc : 0);   // warps
    k_s2_macro<<<(unsigned)((nmacw * 32 + 127) / 128), 128, 0, s>>>(P, B, S, faces, targets);
    cudaError_t e = cudaGetLastError();
    // which 1: the targets need only the macro pass and are first read after the face combine, so
    // they run on the side stream beside the reconstruction and the face nodes (the wall nodes
    // follow them there); which 3: on the main stream
    const bool side_targets = targets && faces;
    if (e == cudaSuccess && side_targets) {
        e = cudaEventRecord(fork, s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s2, fork, 0);
    }
    if (e == cudaSuccess && targets) {
        cudaStream_t ts = side_targets ? s2 : s;
        k_s2_target_nodes<<<warps((long long)nc * 9), 256, 0, ts>>>(P, B, S);
        e = cudaGetLastError();
        if (e == cudaSuccess) {
            k_s2_target_sum<<<dim3((unsigned)((nv + 255) / 256), (unsigned)nc), 256, 0, ts>>>(P, B, S);
            e = cudaGetLastError();
        }
    }
    if (e != cudaSuccess || which == 3) return e;
    const dim3 grid((unsigned)((nv + 31) / 32), (unsigned)nc);
    k_s2_recon1<<<grid, 128, 0, s>>>(P, B, S);
    e = cudaGetLastError();
    if (e == cudaSuccess) { k_s2_recon2<<<grid, 256, 0, s>>>(P, B, S); e = cudaGetLastError(); }
    if (e == cudaSuccess) e = cudaEventRecord(fork, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s2, fork, 0);
    if (e == cudaSuccess) { k_s2_wall_nodes<<<warps(2LL * nx * 3), 256, 0, s2>>>(P, B, S); e = cudaGetLastError(); }
    if (e == cudaSuccess) e = cudaEventRecord(join, s2);
    if (e == cudaSuccess) {
        if (S.concurrent) k_s2_face_nodes<256, 2><<<warps((long long)nf * 3), 256, 0, s>>>(P, B, S);
        else k_s2_face_nodes<kS2NodeThreads, 3><<<node_ctas((long long)nf * 3), kS2NodeThreads, 0, s>>>(P, B, S);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        if (nv <= 1024) k_s2_face_flux<4><<<(unsigned)(nf * 3), 256, 0, s>>>(P, B, S);
        else k_s2_face_flux<10><<<(unsigned)(nf * 3), 256, 0, s>>>(P, B, S);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, join, 0);
    if (e == cudaSuccess) {
        k_s2_combine<<<dim3((unsigned)((nv + 255) / 256), (unsigned)(nf + 2 * nx)), 256, 0, s>>>(P, B, S);
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace ugks
