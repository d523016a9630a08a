// ugks_s2_math.cuh -- device arithmetic of the high-order S2 path, shared by the forward kernels
// (ugks_s2.cu) and their adjoints (ugks_s2_adjoint.cu): the WENO-AO(5,3) reconstruction helpers, the
// warp-level discrete closure and make_mke, the multiscale-wall moments, the constant reconstruction
// tables and the node-scalar layouts.  Everything here has internal linkage: each translation unit
// compiles its own copy and uploads its own constant tables (s2_upload_tables).
#pragma once
#include <algorithm>
#include <cmath>

#include "ugks_implicit.cuh"
#include "ugks_s2.cuh"

namespace ugks {
namespace {

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

// intermediates of the weights that their transpose reads (the adjoint): the reciprocal denominators, the
// ratios tau / (beta_c + eps), 1 / sum(alpha), tau and the signs of beta_3 - beta_c
struct S2WenoX {
    double inv[4], r[4], isa, tau, sg[3];
};

// weno_coefficients (:168-204): the nonlinear weights of stencil q; X: also their intermediates into *x
template <bool X>
__device__ __forceinline__ bool s2_weno_x(const double q[5], S2Weno& w, S2WenoX* x) {
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
        if constexpr (X) { x->inv[c] = inv[c]; x->r[c] = r; }
    }
    const double isa = 1.0 / sa;
    fw[3] = (alpha[3] * isa) * (1.0 / 0.85);
#pragma unroll
    for (int c = 0; c < 3; ++c) fw[c] = alpha[c] * isa - fw[3] * gam[c];
    if constexpr (X) {
        x->isa = isa;
        x->tau = tau;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double dd = beta[3] - beta[c];
            x->sg[c] = dd > 0.0 ? 1.0 : (dd < 0.0 ? -1.0 : 0.0);
        }
    }
    return isfinite(fw[0]) && isfinite(fw[1]) && isfinite(fw[2]) && isfinite(fw[3]);
}
__device__ __forceinline__ bool s2_weno(const double q[5], S2Weno& w) { return s2_weno_x<false>(q, w, nullptr); }

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
// the closure Maxwellian's value alone: the one exponential of s2_q
__device__ __forceinline__ double s2_qh(const S2Th& t, double u, double v) {
    const double du = u - t.u, dv = v - t.v, c2 = du * du + dv * dv;
    return t.pref * exp(-c2 * t.itw);
}
// s2_q with that value given (the same theta and velocity), e.g. recorded by the closure's last
// Newton evaluation
__device__ __forceinline__ S2Q s2_q_at(const S2Th& t, double u, double v, double qh) {
    S2Q q;
    const double du = u - t.u, dv = v - t.v, c2 = du * du + dv * dv;
    q.qh = qh;
    q.ld[0] = t.ir; q.ld[1] = 2.0 * du * t.itw; q.ld[2] = 2.0 * dv * t.itw; q.ld[3] = -t.itw + c2 * (t.itw * t.itw);
    q.qb = t.ckh * q.qh;
    q.ldb[0] = q.ld[0]; q.ldb[1] = q.ld[1]; q.ldb[2] = q.ld[2]; q.ldb[3] = q.ld[3] + t.itw;
    return q;
}
__device__ __forceinline__ S2Q s2_q(const S2Th& t, double u, double v) { return s2_q_at(t, u, v, s2_qh(t, u, v)); }

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

// A warp's record of the closure Maxwellian's values at its converged theta, one per velocity
// (k = lane + 32 r at [r * 32 + lane]: every lane reads back only what it wrote).  The closure, the
// make_mke passes and the node kernels' later passes all evaluate the Maxwellian at that theta, so
// with a record they take its exponentials once.  nullptr: no record (each pass evaluates them).
struct WQRec {
    double* q;
    __device__ __forceinline__ S2Q at(const S2Th& t, const WVel& s, int r) const {
        return q ? s2_q_at(t, s.u, s.v, q[r * 32 + (threadIdx.x & 31)]) : s2_q(t, s.u, s.v);
    }
};


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
// With a record (qr.q != nullptr) every evaluation writes its Maxwellian values there, so on success
// it holds those of the converged theta C.th (the last evaluation is the accepted, converged one).
__device__ bool w_closure(const LoParams& P, const LoBuffers& B, const double w[4], WClosure& C, WQRec qr = {nullptr}) {
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
        // 16 Jacobian moments, the 4 moments of (qh, qb) (compensated: the Newton residual is their
        // difference from w), flags: nonfinite, nonpositive
        double acc[22], ms[4] = {0.0, 0.0, 0.0, 0.0}, mc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int m = 0; m < 22; ++m) acc[m] = 0.0;
        const S2Th tt = s2_th(trial, ck);
        for (int r = 0; r < nr; ++r) {
            const WVel s = wvel(B, nv, r);
            const S2Q q = s2_q(tt, s.u, s.v);
            if (qr.q) qr.q[r * 32 + (threadIdx.x & 31)] = q.qh;
            const double e2 = s.u * s.u + s.v * s.v;
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const double hk = q.qh * q.ld[a], bk = q.qb * q.ldb[a];
                acc[0 * 4 + a] += s.w * hk;
                acc[1 * 4 + a] += s.w * s.u * hk;
                acc[2 * 4 + a] += s.w * s.v * hk;
                acc[3 * 4 + a] += 0.5 * s.w * (e2 * hk + bk);
            }
            comp_add(ms[0], mc[0], s.w * q.qh);
            comp_add(ms[1], mc[1], s.w * s.u * q.qh);
            comp_add(ms[2], mc[2], s.w * s.v * q.qh);
            comp_add(ms[3], mc[3], 0.5 * s.w * (e2 * q.qh + q.qb));
            if (s.ok) {
                acc[20] = fmax(acc[20], (isfinite(q.qh) && isfinite(q.qb)) ? 0.0 : 1.0);
                acc[21] = fmax(acc[21], (q.qh > 0.0 && q.qb > 0.0) ? 0.0 : 1.0);
            }
        }
        warp_sum_all<16>(acc);
        warp_sum_all_comp<4>(ms, mc);
#pragma unroll
        for (int m = 0; m < 4; ++m) acc[16 + m] = ms[m];
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

// M, K_x, K_y of one velocity from the node scalars and the velocity's s2_q
__device__ __forceinline__ void w_mke_q(const WMke& M, int ck, double uk, double vk, const S2Q& q, double& mh,
                                        double& mb, double& kxh, double& kxb, double& kyh, double& kyb) {
    mh = q.qh;
    mb = q.qb;
    w_mke_raw(M, q, ck, uk, vk, kxh, kxb, kyh, kyb);
    double dh, db;
    s2_dq(q, M.tdx, dh, db);
    kxh = kxh - dh; kxb = kxb - db;
    s2_dq(q, M.tdy, dh, db);
    kyh = kyh - dh; kyb = kyb - db;
}
__device__ __forceinline__ void w_mke_at(const S2Th& th, const WMke& M, int ck, double uk, double vk, S2Q& q,
                                         double& mh, double& mb, double& kxh, double& kxb, double& kyh, double& kyb) {
    q = s2_q(th, uk, vk);
    w_mke_q(M, ck, uk, vk, q, mh, mb, kxh, kxb, kyh, kyb);
}

// Returns the gate (moments of M equal w, K_x, K_y moment-free, all finite, to 2e-12).
// qr: the closure's record of the Maxwellian at C.th, or none.
__device__ bool w_make_mke(const LoParams& P, const LoBuffers& B, const double w[4], const WClosure& C, WMke& M,
                           WQRec qr = {nullptr}) {
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
        const S2Q q = qr.at(tt, s, r);
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
        const S2Q q = qr.at(tt, s, r);
        double mh, mb, kxh, kxb, kyh, kyb;
        w_mke_q(M, ck, s.u, s.v, q, mh, mb, kxh, kxb, kyh, kyb);
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

__device__ __forceinline__ void w_store_scalars(double* o, const WClosure& C, const WMke& M) {
#pragma unroll
    for (int m = 0; m < 4; ++m) { o[m] = C.th[m]; o[4 + m] = M.tdx[m]; o[8 + m] = M.tdy[m]; }
    o[12] = M.ux; o[13] = M.vy; o[14] = M.lam; o[15] = M.coeff;
#pragma unroll
    for (int m = 0; m < 16; ++m) o[16 + m] = C.jac[m];
}
__device__ __forceinline__ void w_load_scalars(const double* o, double th[4], WMke& M) {
#pragma unroll
    for (int m = 0; m < 4; ++m) { th[m] = o[m]; M.tdx[m] = o[4 + m]; M.tdy[m] = o[8 + m]; }
    M.ux = o[12]; M.vy = o[13]; M.lam = o[14]; M.coeff = o[15];
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

// The reconstruction maps and point weights of this translation unit's constant tables: built on the
// host with the reference's own small solve, then copied to the device (each TU that includes this
// header has its own copy of c_s2 / c_s2p and uploads it once per device).
inline cudaError_t s2_upload_tables() {
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

}  // namespace
}  // namespace ugks
