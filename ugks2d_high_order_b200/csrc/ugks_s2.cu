// ugks_s2.cu -- the high-order "S2" evolution of HighOrderImplicit on sm_100a (FP64).
//
//   k_s2_init    : S2 cold start, h, b := discrete closure Maxwellian of W (S2NativeInitializeState,
//                  mod_S2NativeAdapter.f90:192-445 with make_mke).
//   k_s2_targets : build_targets (mod_S2D1.f90:1246-1300): per cell the Gauss-averaged closure
//                  targets M, K_x, K_y of 9 volume nodes.  One CTA per cell.
//   k_s2_recon   : tensor WENO-AO(5,3) reconstruction with one-sided wall quartics and the
//                  positivity limiter (mod_S2D1Reconstruction.f90, limit_cell_outputs
//                  mod_S2D1.f90:315-345).  One thread per (cell, velocity); writes the face cache.
//   k_s2_faces   : compute_flux's interior faces (mod_S2D1.f90:757-878): 3 Gauss nodes of
//                  ugks_node (:421-521) per face.  One CTA per face.
//   k_s2_walls   : the multiscale diffuse wall nodes (s2w2_wall_node, mod_S2MultiscaleWall.f90:45-184).
//
// The block-level discrete closure (solve_q_first, mod_CorrectedWF2DClosure.f90:331-426) runs its
// Newton iteration with one CTA: every trial state is one block reduction of the 16 Jacobian
// moments, the 4 moments and 2 flags; thread 0 keeps the reference's accept / backtrack / stop
// logic and broadcasts the next trial through shared memory.  The closure Maxwellian and its
// theta-derivatives are recomputed from theta where needed (the same rounded values), so a thread
// holds only its velocities' working arrays.
#include "ugks_implicit.cuh"
#include "ugks_s2.cuh"

namespace ugks {

__constant__ S2Maps c_s2;

// ------------------------------------------------------------------------------------------
// per-thread reconstruction arithmetic (mod_S2D1Reconstruction.f90), in the reference's order

__device__ __forceinline__ double s2_powi(double x, int n) {
    return n == 0 ? 1.0 : (n == 1 ? x : (n == 2 ? x * x : (n == 3 ? x * x * x : (x * x) * (x * x))));
}

// weno_coefficients (:168-204)
__device__ __forceinline__ bool s2_weno_coef(const double q[5], double fw[4], double coef[4][5]) {
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
    beta[3] = s / 5040.0;
    double tau = fabs(beta[3] - beta[0]);
    tau = tau + fabs(beta[3] - beta[1]);
    tau = tau + fabs(beta[3] - beta[2]);
    tau = tau / 3.0;
    const double gam[4] = {0.01125, 0.1275, 0.01125, 0.85};
    double alpha[4], sa = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const double r = tau / (beta[c] + 1.0e-8);
        alpha[c] = gam[c] * (1.0 + r * r);
        sa = sa + alpha[c];
    }
    fw[3] = (alpha[3] / sa) / gam[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) fw[c] = alpha[c] / sa - fw[3] * gam[c];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int d = 0; d < 5; ++d) coef[c][d] = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = c; k <= c + 2; ++k)
#pragma unroll
            for (int d = 0; d <= 2; ++d) coef[c][d] = coef[c][d] + c_s2.cmap[c][k][d] * q[k];
#pragma unroll
    for (int k = 0; k < 5; ++k)
#pragma unroll
        for (int d = 0; d <= 4; ++d) coef[3][d] = coef[3][d] + c_s2.cmap[3][k][d] * q[k];
    return isfinite(fw[0]) && isfinite(fw[1]) && isfinite(fw[2]) && isfinite(fw[3]);
}

// prepared_eval (:247-262)
__device__ __forceinline__ void s2_eval(const double fw[4], const double coef[4][5], double xi, double& val,
                                        double& der) {
    double pw[5], dp[5];
    pw[0] = 1.0; dp[0] = 0.0;
#pragma unroll
    for (int d = 1; d <= 4; ++d) { pw[d] = pw[d - 1] * xi; dp[d] = (double)d * s2_powi(xi, d - 1); }
    double v = 0.0, dv = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        double cand = 0.0, dcand = 0.0;
#pragma unroll
        for (int d = 0; d < 5; ++d) { cand = cand + coef[c][d] * pw[d]; dcand = dcand + coef[c][d] * dp[d]; }
        v = v + fw[c] * cand;
        dv = dv + fw[c] * dcand;
    }
    val = v;
    der = dv;
}

__device__ __forceinline__ double s2_eval_v(const double fw[4], const double coef[4][5], double xi) {
    double pw[5];
    pw[0] = 1.0;
#pragma unroll
    for (int d = 1; d <= 4; ++d) pw[d] = pw[d - 1] * xi;
    double v = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        double cand = 0.0;
#pragma unroll
        for (int d = 0; d < 5; ++d) cand = cand + coef[c][d] * pw[d];
        v = v + fw[c] * cand;
    }
    return v;
}

// companion_eval3 (:287-318)
__device__ __forceinline__ bool s2_companion3(const double q[5], const double comp[5], double val[3], double der[3],
                                              double cval[3]) {
    double fw[4], coef[4][5], ccoef[4][5];
    if (!s2_weno_coef(q, fw, coef)) return false;
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int d = 0; d < 5; ++d) ccoef[c][d] = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = c; k <= c + 2; ++k)
#pragma unroll
            for (int d = 0; d <= 2; ++d) ccoef[c][d] = ccoef[c][d] + c_s2.cmap[c][k][d] * comp[k];
#pragma unroll
    for (int k = 0; k < 5; ++k)
#pragma unroll
        for (int d = 0; d <= 4; ++d) ccoef[3][d] = ccoef[3][d] + c_s2.cmap[3][k][d] * comp[k];
    bool ok = true;
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        s2_eval(fw, coef, c_s2.gnode[s], val[s], der[s]);
        cval[s] = s2_eval_v(fw, ccoef, c_s2.gnode[s]);
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
    double xv[5][2], xd[5][2], yv[5][2], yd[5][2], rows[5][3], q[5], fw[4], coef[4][5];
    const int ny = F.ny;
    if (!s2_near_wall(j, ny)) {
        for (int r = -2; r <= 2; ++r) {
#pragma unroll
            for (int s = -2; s <= 2; ++s) q[s + 2] = F.at(i + s, j + r);
            if (!s2_weno_coef(q, fw, coef)) return false;
            s2_eval(fw, coef, -0.5, xv[r + 2][0], xd[r + 2][0]);
            s2_eval(fw, coef, 0.5, xv[r + 2][1], xd[r + 2][1]);
#pragma unroll
            for (int a = 0; a < 3; ++a) rows[r + 2][a] = s2_eval_v(fw, coef, c_s2.gnode[a]);
        }
        for (int r = -2; r <= 2; ++r) {
#pragma unroll
            for (int s = -2; s <= 2; ++s) q[s + 2] = F.at(i + r, j + s);
            if (!s2_weno_coef(q, fw, coef)) return false;
            s2_eval(fw, coef, -0.5, yv[r + 2][0], yd[r + 2][0]);
            s2_eval(fw, coef, 0.5, yv[r + 2][1], yd[r + 2][1]);
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
            if (!s2_weno_coef(a5, fw, coef)) return false;
#pragma unroll
            for (int b = 0; b < 3; ++b) vol[a][b] = s2_eval_v(fw, coef, c_s2.gnode[b]);
        }
    } else {
        const int first = s2_wall_first(j, ny);
        for (int r = 0; r < 5; ++r) {
#pragma unroll
            for (int s = -2; s <= 2; ++s) q[s + 2] = F.at(i + s, first + r);
            if (!s2_weno_coef(q, fw, coef)) return false;
            s2_eval(fw, coef, -0.5, xv[r][0], xd[r][0]);
            s2_eval(fw, coef, 0.5, xv[r][1], xd[r][1]);
#pragma unroll
            for (int a = 0; a < 3; ++a) rows[r][a] = s2_eval_v(fw, coef, c_s2.gnode[a]);
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
    double nv5[5], nd5[5], q[5], fw[4], coef[4][5];
    for (int r = -2; r <= 2; ++r) {
#pragma unroll
        for (int s = -2; s <= 2; ++s) q[s + 2] = axis == 0 ? F.at(cell + s, tangent + r) : F.at(tangent + r, cell + s);
        if (!s2_weno_coef(q, fw, coef)) return false;
        s2_eval(fw, coef, side, nv5[r + 2], nd5[r + 2]);
    }
    return s2_companion3(nv5, nd5, val, dt, dn);
}

// s2d1_cell9 (:378-403)
__device__ bool s2_cell9(const S2Field& F, int i, int j, double val[3][3]) {
    if (s2_near_wall(j, F.ny)) {
        double f[4][3], n[4][3], t[4][3];
        return s2_cell_faces9(F, i, j, f, n, t, val);
    }
    double rows[5][3], q[5], fw[4], coef[4][5];
    for (int r = -2; r <= 2; ++r) {
#pragma unroll
        for (int s = -2; s <= 2; ++s) q[s + 2] = F.at(i + s, j + r);
        if (!s2_weno_coef(q, fw, coef)) return false;
#pragma unroll
        for (int a = 0; a < 3; ++a) rows[r + 2][a] = s2_eval_v(fw, coef, c_s2.gnode[a]);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double a5[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) a5[r] = rows[r][a];
        if (!s2_weno_coef(a5, fw, coef)) return false;
#pragma unroll
        for (int b = 0; b < 3; ++b) val[a][b] = s2_eval_v(fw, coef, c_s2.gnode[b]);
    }
    return true;
}

// ------------------------------------------------------------------------------------------
// reconstruction + limiter: one thread per (cell, velocity); cache layout
// rec[((cell*72 + field*12 + side*3 + node)*nvel + k], fields: h, b, h_n, h_t, b_n, b_t
__global__ void __launch_bounds__(128) k_s2_recon(LoParams P, LoBuffers B, S2Buffers S) {
    if (eval_cached(B)) return;
    const int nv = P.nvel, nx = P.nx, ny = P.ny;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nv) return;
    const int cc = blockIdx.y, i = cc % nx, j = cc / nx;
    const S2Field Fh{B.h + k, nv, nx, ny}, Fb{B.b + k, nv, nx, ny};
    double hf[4][3], hn[4][3], ht[4][3], hv[3][3], bf[4][3], bn[4][3], bt[4][3], bv[3][3];
    bool ok = s2_cell_faces9(Fh, i, j, hf, hn, ht, hv) && s2_cell_faces9(Fb, i, j, bf, bn, bt, bv);
    const double hm = B.h[(size_t)cc * nv + k], bm = B.b[(size_t)cc * nv + k];
    const double margin = 64.0 * kEps;
    double theta = 1.0;
    if (hm <= 0.0 || bm <= 0.0) {
        theta = 0.0;
    } else {
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (hf[s][a] < 0.0) theta = fmin(theta, (1.0 - margin) * hm / (hm - hf[s][a]));
                if (bf[s][a] < 0.0) theta = fmin(theta, (1.0 - margin) * bm / (bm - bf[s][a]));
            }
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (hv[a][c] < 0.0) theta = fmin(theta, (1.0 - margin) * hm / (hm - hv[a][c]));
                if (bv[a][c] < 0.0) theta = fmin(theta, (1.0 - margin) * bm / (bm - bv[a][c]));
            }
        theta = fmax(0.0, fmin(1.0, theta));
    }
    double* r = S.rec + (size_t)cc * 72 * nv + k;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const double nd = s < 2 ? P.dx : P.dy, td = s < 2 ? P.dy : P.dx;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double v[6] = {hm + theta * (hf[s][a] - hm), bm + theta * (bf[s][a] - bm), theta * hn[s][a] / nd,
                                 theta * ht[s][a] / td, theta * bn[s][a] / nd, theta * bt[s][a] / td};
#pragma unroll
            for (int f = 0; f < 6; ++f) {
                r[(size_t)(f * 12 + s * 3 + a) * nv] = v[f];
                ok = ok && isfinite(v[f]);
            }
        }
    }
    if (!ok) set_status(B.status, ST_NONFINITE_FLUX);
}

// ------------------------------------------------------------------------------------------
// block-level discrete closure

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
// mod_CorrectedWF2DClosure.f90:389-426)
struct S2Q {
    double qh, qb, ld[4], ldb[4];
};
__device__ __forceinline__ S2Q s2_q(const double th[4], int ck, double u, double v) {
    S2Q q;
    const double r = th[0], tw = th[3];
    const double du = u - th[1], dv = v - th[2], c2 = du * du + dv * dv;
    q.qh = r / (kPi * tw) * exp(-c2 / tw);
    q.ld[0] = 1.0 / r; q.ld[1] = 2.0 * du / tw; q.ld[2] = 2.0 * dv / tw; q.ld[3] = -1.0 / tw + c2 / (tw * tw);
    q.qb = 0.5 * (double)ck * tw * q.qh;
    q.ldb[0] = q.ld[0]; q.ldb[1] = q.ld[1]; q.ldb[2] = q.ld[2]; q.ldb[3] = q.ld[3] + 1.0 / tw;
    return q;
}

// shared scalars of the block-level routines
struct S2Shared {
    double red[16 * 64];
    double rout[kRedSlots];
    double w[4];          // closure target
    double th[4];         // converged theta
    double trial[4];
    double jac[16];       // converged Jacobian (row-major: moment r, theta a)
    double tjac[16];
    double res[4], step[4], alpha, norm;
    double v[48];         // broadcast scalars of the callers
    int act, iter;
};

enum { S2_EVAL_INIT = 0, S2_EVAL_TRIAL = 1, S2_DONE = 2, S2_FAIL = 3 };

__device__ __forceinline__ double s2_scaled(const double r[4], const double w[4]) {
    double s = 0.0;
#pragma unroll
    for (int m = 0; m < 4; ++m) s = fmax(s, fabs(r[m]) / fmax(1.0, fabs(w[m])));
    return s;
}

// thread 0: choose the next trial after a rejected one or a new Newton iteration
__device__ void s2_newton_next(S2Shared& S, bool new_iter) {
    const double tol = 5.0e-13, floor_a = 9.5367431640625e-07;   // 2^-20
    if (new_iter) {
        if (S.norm <= tol) { S.act = S2_DONE; return; }
        if (S.iter > 12) { S.act = S2_FAIL; return; }
        const double mr[4] = {-S.res[0], -S.res[1], -S.res[2], -S.res[3]};
        double st[4];
        if (!s2_solve4(S.jac, mr, st)) { S.act = S2_FAIL; return; }
#pragma unroll
        for (int m = 0; m < 4; ++m) S.step[m] = st[m];
        S.alpha = 1.0;
    }
    while (S.alpha >= floor_a) {
        double nt[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) nt[m] = S.th[m] + S.alpha * S.step[m];
        if (nt[0] > 0.0 && nt[3] > 0.0 && isfinite(nt[0]) && isfinite(nt[1]) && isfinite(nt[2]) && isfinite(nt[3])) {
#pragma unroll
            for (int m = 0; m < 4; ++m) S.trial[m] = nt[m];
            S.act = S2_EVAL_TRIAL;
            return;
        }
        S.alpha = 0.5 * S.alpha;
    }
    S.act = S2_FAIL;
}

// solve_q_first with one CTA.  w must be in S.w (written by the caller before a barrier).
// Returns the converged theta / Jacobian in S.th / S.jac (uniform result).
template <int VPT>
__device__ bool s2_closure(const LoParams& P, const LoBuffers& B, S2Shared& S) {
    const int nv = P.nvel, ck = P.ck;
    if (threadIdx.x == 0) {
        const double* w = S.w;
        bool ok = isfinite(w[0]) && isfinite(w[1]) && isfinite(w[2]) && isfinite(w[3]) && w[0] > 0.0;
        if (ok) {   // primitive_from_conserved_2d (mod_CorrectedWF2DEquilibrium.f90:25-41)
            const double u = w[1] / w[0], v = w[2] / w[0];
            const double kin = 0.5 * (u * u + v * v), ein = w[3] / w[0] - kin;
            const double temp = 4.0 * ein / (double)(ck + 2);
            ok = isfinite(u) && isfinite(v) && isfinite(temp) && temp > 0.0;
            S.trial[0] = w[0]; S.trial[1] = u; S.trial[2] = v; S.trial[3] = temp;
        }
        S.act = ok ? S2_EVAL_INIT : S2_FAIL;
    }
    __syncthreads();
    for (int guard = 0; guard < 1024; ++guard) {
        const int act = S.act;
        if (act == S2_DONE || act == S2_FAIL) break;
        double th[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) th[m] = S.trial[m];
        // 16 Jacobian moments, 4 moments of (qh, qb), flags: nonfinite, nonpositive
        double acc[22];
#pragma unroll
        for (int m = 0; m < 22; ++m) acc[m] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
            const S2Q q = s2_q(th, ck, uk, vk);
            const double e2 = uk * uk + vk * vk;
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const double hk = q.qh * q.ld[a], bk = q.qb * q.ldb[a];
                acc[0 * 4 + a] += wk * hk;
                acc[1 * 4 + a] += wk * uk * hk;
                acc[2 * 4 + a] += wk * vk * hk;
                acc[3 * 4 + a] += 0.5 * wk * (e2 * hk + bk);
            }
            acc[16] += wk * q.qh;
            acc[17] += wk * uk * q.qh;
            acc[18] += wk * vk * q.qh;
            acc[19] += 0.5 * wk * (e2 * q.qh + q.qb);
            if (s.ok) {
                acc[20] = fmax(acc[20], (isfinite(q.qh) && isfinite(q.qb)) ? 0.0 : 1.0);
                acc[21] = fmax(acc[21], (q.qh > 0.0 && q.qb > 0.0) ? 0.0 : 1.0);
            }
        }
        block_reduce_smem<20, 2>(acc, S.red, S.rout);
        if (threadIdx.x == 0) {
            const double* o = S.rout;
            bool fin = o[20] == 0.0;
#pragma unroll
            for (int m = 0; m < 20; ++m) fin = fin && isfinite(o[m]);
            double nres[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) nres[m] = o[16 + m] - S.w[m];
            if (act == S2_EVAL_INIT) {
                if (!fin) S.act = S2_FAIL;
                else {
#pragma unroll
                    for (int m = 0; m < 4; ++m) { S.th[m] = th[m]; S.res[m] = nres[m]; }
#pragma unroll
                    for (int m = 0; m < 16; ++m) S.jac[m] = o[m];
                    S.norm = s2_scaled(nres, S.w);
                    S.iter = 1;
                    s2_newton_next(S, true);
                    if (S.act == S2_DONE && o[21] != 0.0) S.act = S2_FAIL;
                }
            } else {
                const double nn = fin ? s2_scaled(nres, S.w) : INFINITY;
                const bool accepted = fin && (nn < S.norm || nn <= 5.0e-13);
                if (accepted) {
#pragma unroll
                    for (int m = 0; m < 4; ++m) { S.th[m] = th[m]; S.res[m] = nres[m]; }
#pragma unroll
                    for (int m = 0; m < 16; ++m) S.jac[m] = o[m];
                    S.norm = nn;
                    S.iter = S.iter + 1;
                    s2_newton_next(S, true);
                    if (S.act == S2_DONE && o[21] != 0.0) S.act = S2_FAIL;
                } else {
                    S.alpha = 0.5 * S.alpha;
                    s2_newton_next(S, false);
                }
            }
        }
        __syncthreads();
    }
    return S.act == S2_DONE;
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

// make_mke_prepared (mod_S2D1.f90:111-151) after s2_closure on w = S.w: per velocity slot the
// closure Maxwellian M and the projected Shakhov directions K_x, K_y.  Returns the uniform gate.
template <int VPT>
__device__ bool s2_make_mke(const LoParams& P, const LoBuffers& B, S2Shared& S, double mh[VPT], double mb[VPT],
                            double kxh[VPT], double kxb[VPT], double kyh[VPT], double kyb[VPT]) {
    const int nv = P.nvel, ck = P.ck;
    double rho, ux, vy, th;
    const double w[4] = {S.w[0], S.w[1], S.w[2], S.w[3]};
    const bool pok = s2_primitive(w, ck, rho, ux, vy, th);
    const double lam = 0.5 / th;
    double thc[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) thc[m] = S.th[m];
    double acc[16];
#pragma unroll
    for (int m = 0; m < 8; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
        const S2Q q = s2_q(thc, ck, uk, vk);
        mh[r] = q.qh; mb[r] = q.qb;
        const double cx = uk - ux, cy = vk - vy, c2 = cx * cx + cy * cy;
        const double coeff = 0.8 * (1.0 - P.pr) * lam * lam / rho;
        const double shh = 2.0 * lam * c2 - 4.0, shb = shh + 2.0 / (double)ck;
        kxh[r] = coeff * cx * shh * mh[r]; kxb[r] = coeff * cx * shb * mb[r];
        kyh[r] = coeff * cy * shh * mh[r]; kyb[r] = coeff * cy * shb * mb[r];
        const double e2 = uk * uk + vk * vk;
        acc[0] += wk * kxh[r]; acc[1] += wk * uk * kxh[r]; acc[2] += wk * vk * kxh[r]; acc[3] += 0.5 * wk * (e2 * kxh[r] + kxb[r]);
        acc[4] += wk * kyh[r]; acc[5] += wk * uk * kyh[r]; acc[6] += wk * vk * kyh[r]; acc[7] += 0.5 * wk * (e2 * kyh[r] + kyb[r]);
    }
    block_reduce_smem<8, 0>(acc, S.red, S.rout);
    if (threadIdx.x == 0 || threadIdx.x == 32) {
        const int d = threadIdx.x == 0 ? 0 : 1;
        double m4[4], td[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) m4[m] = S.rout[4 * d + m];
        const bool ok = s2_solve4(S.jac, m4, td);
#pragma unroll
        for (int m = 0; m < 4; ++m) S.v[4 * d + m] = ok ? td[m] : NAN;
    }
    __syncthreads();
    double tdx[4], tdy[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) { tdx[m] = S.v[m]; tdy[m] = S.v[4 + m]; }
#pragma unroll
    for (int m = 0; m < 16; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
        const S2Q q = s2_q(thc, ck, uk, vk);
        double dh, db;
        s2_dq(q, tdx, dh, db);
        kxh[r] = kxh[r] - dh; kxb[r] = kxb[r] - db;
        s2_dq(q, tdy, dh, db);
        kyh[r] = kyh[r] - dh; kyb[r] = kyb[r] - db;
        const double e2 = uk * uk + vk * vk, cx = uk - ux, cy = vk - vy, c2 = cx * cx + cy * cy;
        acc[0] += wk * mh[r]; acc[1] += wk * uk * mh[r]; acc[2] += wk * vk * mh[r]; acc[3] += 0.5 * wk * (e2 * mh[r] + mb[r]);
        acc[4] += wk * kxh[r]; acc[5] += wk * uk * kxh[r]; acc[6] += wk * vk * kxh[r]; acc[7] += 0.5 * wk * (e2 * kxh[r] + kxb[r]);
        acc[8] += wk * kyh[r]; acc[9] += wk * uk * kyh[r]; acc[10] += wk * vk * kyh[r]; acc[11] += 0.5 * wk * (e2 * kyh[r] + kyb[r]);
        acc[12] += 0.5 * wk * cx * (c2 * kxh[r] + kxb[r]);
        acc[13] += 0.5 * wk * cy * (c2 * kxh[r] + kxb[r]);
        acc[14] += 0.5 * wk * cx * (c2 * kyh[r] + kyb[r]);
        acc[15] += 0.5 * wk * cy * (c2 * kyh[r] + kyb[r]);
    }
    block_reduce_smem<16, 0>(acc, S.red, S.rout);
    const double* o = S.rout;
    double res = 0.0, sc = 1.0;
#pragma unroll
    for (int m = 0; m < 4; ++m) { res = fmax(res, fabs(o[m] - w[m])); sc = fmax(sc, fabs(w[m])); }
    res = res / sc;
#pragma unroll
    for (int m = 4; m < 12; ++m) res = fmax(res, fabs(o[m]));
    bool fin = isfinite(tdx[0]) && isfinite(tdy[0]);
#pragma unroll
    for (int m = 12; m < 16; ++m) fin = fin && isfinite(o[m]);
    return pok && fin && res <= 2.0e-12;
}

// ------------------------------------------------------------------------------------------
// S2 cold start: one CTA per cell
template <int VPT, int NT>
__global__ void __launch_bounds__(NT) k_s2_init(LoParams P, LoBuffers B, S2Buffers SB) {
    __shared__ S2Shared S;
    const int nv = P.nvel, cc = blockIdx.x;
    if (threadIdx.x < 4) S.w[threadIdx.x] = B.W[cc * 4 + threadIdx.x];
    __syncthreads();
    bool ok = s2_closure<VPT>(P, B, S);
    if (ok) {
        double mh[VPT], mb[VPT], kxh[VPT], kxb[VPT], kyh[VPT], kyb[VPT];
        ok = s2_make_mke<VPT>(P, B, S, mh, mb, kxh, kxb, kyh, kyb);
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            if (s.ok) { B.h[(size_t)cc * nv + s.k] = mh[r]; B.b[(size_t)cc * nv + s.k] = mb[r]; }
        }
    }
    if (!ok && threadIdx.x == 0) set_status(B.status, ST_PROJECTION);
}

// build_targets: one CTA per cell, the 9 volume nodes in turn, accumulated in registers
template <int VPT, int NT>
__global__ void __launch_bounds__(NT) k_s2_targets(LoParams P, LoBuffers B, S2Buffers SB) {
    if (eval_cached(B)) return;
    __shared__ S2Shared S;
    __shared__ double s_wq[9][4];
    __shared__ int s_ok;
    const int nv = P.nvel, nx = P.nx, ny = P.ny, cc = blockIdx.x, i = cc % nx, j = cc / nx;
    if (threadIdx.x == 0) s_ok = 1;
    __syncthreads();
    if (threadIdx.x < 4) {   // s2d1_cell9 of the four macro fields
        const int m = threadIdx.x;
        const S2Field F{B.W + m, 4, nx, ny};
        double nodes[3][3];
        if (!s2_cell9(F, i, j, nodes)) s_ok = 0;
        S.v[m * 9 + 0] = nodes[0][0];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int c = 0; c < 3; ++c) S.v[m * 9 + a * 3 + c] = nodes[a][c];
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        const int m = threadIdx.x;
        const double gw[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
        double avg = 0.0;
        for (int c = 0; c < 3; ++c)
            for (int a = 0; a < 3; ++a) avg = avg + gw[a] * gw[c] * S.v[m * 9 + a * 3 + c];
        for (int c = 0; c < 3; ++c)
            for (int a = 0; a < 3; ++a) s_wq[c * 3 + a][m] = S.v[m * 9 + a * 3 + c] + B.W[cc * 4 + m] - avg;
    }
    __syncthreads();
    double amh[VPT], amb[VPT], akxh[VPT], akxb[VPT], akyh[VPT], akyb[VPT];
#pragma unroll
    for (int r = 0; r < VPT; ++r) amh[r] = amb[r] = akxh[r] = akxb[r] = akyh[r] = akyb[r] = 0.0;
    bool ok = s_ok != 0;
    const double gw[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
    for (int p = 0; p < 9 && ok; ++p) {
        if (threadIdx.x < 4) S.w[threadIdx.x] = s_wq[p][threadIdx.x];
        __syncthreads();
        ok = s2_closure<VPT>(P, B, S);
        if (!ok) break;
        double mh[VPT], mb[VPT], kxh[VPT], kxb[VPT], kyh[VPT], kyb[VPT];
        ok = s2_make_mke<VPT>(P, B, S, mh, mb, kxh, kxb, kyh, kyb);
        const double wt2 = gw[p % 3] * gw[p / 3];
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            amh[r] = amh[r] + wt2 * mh[r]; amb[r] = amb[r] + wt2 * mb[r];
            akxh[r] = akxh[r] + wt2 * kxh[r]; akxb[r] = akxb[r] + wt2 * kxb[r];
            akyh[r] = akyh[r] + wt2 * kyh[r]; akyb[r] = akyb[r] + wt2 * kyb[r];
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        if (!s.ok) continue;
        const size_t q = (size_t)cc * nv + s.k;
        SB.mh[q] = amh[r]; SB.mb[q] = amb[r]; SB.kxh[q] = akxh[r]; SB.kxb[q] = akxb[r]; SB.kyh[q] = akyh[r]; SB.kyb[q] = akyb[r];
    }
    if (!ok && threadIdx.x == 0) set_status(B.status, ST_PROJECTION);
}

// ------------------------------------------------------------------------------------------
// interior faces: one CTA per face (the right x face of every cell, then the top y face of every
// cell below the last row), the 3 Gauss nodes of ugks_node in turn
template <int VPT, int NT>
__global__ void __launch_bounds__(NT) k_s2_faces(LoParams P, LoBuffers B, S2Buffers SB) {
    if (eval_cached(B)) return;
    __shared__ S2Shared S;
    __shared__ double s_mac[3][4][3];   // [nl, nr, t][component][node]
    __shared__ int s_ok;
    const int nv = P.nvel, nx = P.nx, ny = P.ny;
    int f = blockIdx.x;
    const int axis = f < nx * ny ? 0 : 1;
    if (axis == 1) f -= nx * ny;
    const int cl = f, i = cl % nx, j = cl / nx;
    const int cr = axis == 0 ? j * nx + (i + 1) % nx : (j + 1) * nx + i;
    const double dt = B.dt[0];
    if (threadIdx.x == 0) s_ok = 1;
    __syncthreads();
    if (threadIdx.x < 4) {   // s2d1_face3 of W component m (the macro normal/tangential slopes)
        const int m = threadIdx.x;
        const S2Field F{B.W + m, 4, nx, ny};
        double vl[3], vr[3], nl[3], nr[3], tl[3], tr[3];
        bool ok;
        if (axis == 0) ok = s2_side3(F, 0, i, j, 0.5, vl, nl, tl) && s2_side3(F, 0, (i + 1) % nx, j, -0.5, vr, nr, tr);
        else ok = s2_side3(F, 1, j, i, 0.5, vl, nl, tl) && s2_side3(F, 1, j + 1, i, -0.5, vr, nr, tr);
        if (!ok) s_ok = 0;
        const double dn = axis == 0 ? P.dx : P.dy, dtg = axis == 0 ? P.dy : P.dx;
#pragma unroll
        for (int g = 0; g < 3; ++g) {
            s_mac[0][m][g] = nl[g] / dn;
            s_mac[1][m][g] = nr[g] / dn;
            s_mac[2][m][g] = 0.5 * (tl[g] + tr[g]) / dtg;
        }
    }
    __syncthreads();
    bool ok = s_ok != 0;
    const int sl = axis == 0 ? 1 : 3, sr = axis == 0 ? 0 : 2;
    const double gw[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
    double afh[VPT], afb[VPT], afw[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int r = 0; r < VPT; ++r) afh[r] = afb[r] = 0.0;
    for (int g = 0; g < 3 && ok; ++g) {
        // inputs of this node: upwind face values and micro derivatives
        double f0h[VPT], f0b[VPT], nh[VPT], nb[VPT], th_[VPT], tb_[VPT], acc[22];
#pragma unroll
        for (int m = 0; m < 4; ++m) acc[m] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
            const double vn = axis == 0 ? uk : vk;
            const bool left = vn >= 0.0;
            const double* rc = SB.rec + (size_t)(left ? cl : cr) * 72 * nv + s.kk;
            const int side = left ? sl : sr;
            f0h[r] = rc[(size_t)(0 * 12 + side * 3 + g) * nv];
            f0b[r] = rc[(size_t)(1 * 12 + side * 3 + g) * nv];
            nh[r] = rc[(size_t)(2 * 12 + side * 3 + g) * nv];
            th_[r] = rc[(size_t)(3 * 12 + side * 3 + g) * nv];
            nb[r] = rc[(size_t)(4 * 12 + side * 3 + g) * nv];
            tb_[r] = rc[(size_t)(5 * 12 + side * 3 + g) * nv];
            const double e2 = uk * uk + vk * vk;
            acc[0] += wk * f0h[r]; acc[1] += wk * uk * f0h[r]; acc[2] += wk * vk * f0h[r]; acc[3] += 0.5 * wk * (e2 * f0h[r] + f0b[r]);
        }
        block_reduce_smem<4, 0>(acc, S.red, S.rout);
        if (threadIdx.x < 4) S.w[threadIdx.x] = S.rout[threadIdx.x];
        __syncthreads();
        double w0[4] = {S.w[0], S.w[1], S.w[2], S.w[3]};
        ok = s2_closure<VPT>(P, B, S);
        if (!ok) break;
        double mh[VPT], mb[VPT], kxh[VPT], kxb[VPT], kyh[VPT], kyb[VPT];
        ok = s2_make_mke<VPT>(P, B, S, mh, mb, kxh, kxb, kyh, kyb);
        if (!ok) break;
        // q0 = heat(w0, f0 - analytic Maxwellian)
        double rho, ux, vy, thg;
        s2_primitive(w0, P.ck, rho, ux, vy, thg);
        double nrho = w0[0], nu = w0[1] / w0[0], nvv = w0[2] / w0[0];
        const double temp = 4.0 * (w0[3] / w0[0] - 0.5 * (nu * nu + nvv * nvv)) / (double)(P.ck + 2);
        const double lamn = 1.0 / temp;
        acc[0] = acc[1] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
            const double du = uk - nu, dv = vk - nvv;
            const double eah = nrho * lamn / kPi * exp(-lamn * (du * du + dv * dv));
            const double eab = 0.5 * (double)P.ck * temp * eah;
            const double cx = uk - ux, cy = vk - vy, c2 = cx * cx + cy * cy;
            const double dh = f0h[r] - eah, db = f0b[r] - eab;
            acc[0] += 0.5 * wk * cx * (c2 * dh + db);
            acc[1] += 0.5 * wk * cy * (c2 * dh + db);
        }
        block_reduce_smem<2, 0>(acc, S.red, S.rout);
        const double q0x = S.rout[0], q0y = S.rout[1];
        double s0h[VPT], s0b[VPT];
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            s0h[r] = mh[r] + kxh[r] * q0x + kyh[r] * q0y;
            s0b[r] = mb[r] + kxb[r] * q0x + kyb[r] * q0y;
        }
        // directions of the macro normal slopes (left, right) and the tangential slope
        if (threadIdx.x == 0 || threadIdx.x == 32 || threadIdx.x == 64) {
            const int d = threadIdx.x / 32;
            double m4[4], td[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) m4[m] = s_mac[d][m][g];
            const bool sok = s2_solve4(S.jac, m4, td);
#pragma unroll
            for (int m = 0; m < 4; ++m) S.v[8 + 4 * d + m] = sok ? td[m] : NAN;
        }
        __syncthreads();
        double thc[4], tdl[4], tdr[4], tdt[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) { thc[m] = S.th[m]; tdl[m] = S.v[8 + m]; tdr[m] = S.v[12 + m]; tdt[m] = S.v[16 + m]; }
        double dlh[VPT], dlb[VPT], drh[VPT], drb[VPT], dth[VPT], dtb[VPT];
#pragma unroll
        for (int m = 0; m < 16; ++m) acc[m] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
            const S2Q q = s2_q(thc, P.ck, uk, vk);
            s2_dq(q, tdl, dlh[r], dlb[r]);
            s2_dq(q, tdr, drh[r], drb[r]);
            s2_dq(q, tdt, dth[r], dtb[r]);
            const double e2 = uk * uk + vk * vk;
            acc[0] += wk * dlh[r]; acc[1] += wk * uk * dlh[r]; acc[2] += wk * vk * dlh[r]; acc[3] += 0.5 * wk * (e2 * dlh[r] + dlb[r]);
            acc[4] += wk * drh[r]; acc[5] += wk * uk * drh[r]; acc[6] += wk * vk * drh[r]; acc[7] += 0.5 * wk * (e2 * drh[r] + drb[r]);
            acc[8] += wk * dth[r]; acc[9] += wk * uk * dth[r]; acc[10] += wk * vk * dth[r]; acc[11] += 0.5 * wk * (e2 * dth[r] + dtb[r]);
            const double vn = axis == 0 ? uk : vk, vt = axis == 0 ? vk : uk;
            const double fh = vn * (vn >= 0.0 ? dlh[r] : drh[r]) + vt * dth[r];
            const double fb = vn * (vn >= 0.0 ? dlb[r] : drb[r]) + vt * dtb[r];
            acc[12] += wk * fh; acc[13] += wk * uk * fh; acc[14] += wk * vk * fh; acc[15] += 0.5 * wk * (e2 * fh + fb);
        }
        block_reduce_smem<16, 0>(acc, S.red, S.rout);
        if (threadIdx.x == 0) {   // gates of the three directions; the time direction and Mt
            bool gok = true;
            for (int d = 0; d < 3; ++d) {
                double mx = 0.0, sc = 1.0;
                for (int m = 0; m < 4; ++m) {
                    mx = fmax(mx, fabs(S.rout[4 * d + m] - s_mac[d][m][g]));
                    sc = fmax(sc, fabs(s_mac[d][m][g]));
                }
                gok = gok && mx / sc <= 2.0e-12;
            }
            double wt[4], td[4];
            for (int m = 0; m < 4; ++m) wt[m] = -S.rout[12 + m];
            gok = gok && s2_solve4(S.jac, wt, td);
            for (int m = 0; m < 4; ++m) { S.v[20 + m] = td[m]; S.v[24 + m] = wt[m]; }
            double tau = 0.0;
            gok = gok && s2_tau(P, w0, tau);
            const double ex = exp(-dt / tau);
            double mt[5];
            mt[3] = tau * (1.0 - ex);
            mt[4] = -tau * dt * ex + tau * mt[3];
            mt[0] = dt - mt[3];
            mt[1] = -tau * mt[0] + mt[4];
            mt[2] = 0.5 * dt * dt - tau * mt[0];
            for (int m = 0; m < 5; ++m) S.v[28 + m] = mt[m];
            S.v[33] = gok ? 1.0 : 0.0;
        }
        __syncthreads();
        if (S.v[33] == 0.0) { ok = false; break; }
        double tdm[4], mt[5];
#pragma unroll
        for (int m = 0; m < 4; ++m) tdm[m] = S.v[20 + m];
#pragma unroll
        for (int m = 0; m < 5; ++m) mt[m] = S.v[28 + m];
#pragma unroll
        for (int m = 0; m < 8; ++m) acc[m] = 0.0;
        double fhv[VPT], fbv[VPT];
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
            const S2Q q = s2_q(thc, P.ck, uk, vk);
            double mth, mtb;
            s2_dq(q, tdm, mth, mtb);
            const double e2 = uk * uk + vk * vk;
            acc[0] += wk * mth; acc[1] += wk * uk * mth; acc[2] += wk * vk * mth; acc[3] += 0.5 * wk * (e2 * mth + mtb);
            const double vn = axis == 0 ? uk : vk, vt = axis == 0 ? vk : uk;
            const double sh = vn * (vn >= 0.0 ? dlh[r] : drh[r]) + vt * dth[r];
            const double sb = vn * (vn >= 0.0 ? dlb[r] : drb[r]) + vt * dtb[r];
            fhv[r] = vn * (mt[0] * s0h[r] + mt[1] * sh + mt[2] * mth + mt[3] * f0h[r] - mt[4] * (vn * nh[r] + vt * th_[r]));
            fbv[r] = vn * (mt[0] * s0b[r] + mt[1] * sb + mt[2] * mtb + mt[3] * f0b[r] - mt[4] * (vn * nb[r] + vt * tb_[r]));
            acc[4] += wk * fhv[r]; acc[5] += wk * uk * fhv[r]; acc[6] += wk * vk * fhv[r]; acc[7] += 0.5 * wk * (e2 * fhv[r] + fbv[r]);
            afh[r] = afh[r] + gw[g] * fhv[r];
            afb[r] = afb[r] + gw[g] * fbv[r];
            if (s.ok) ok = ok && isfinite(fhv[r]) && isfinite(fbv[r]);
        }
        block_reduce_smem<8, 0>(acc, S.red, S.rout);
        {
            double mx = 0.0, sc = 1.0;
#pragma unroll
            for (int m = 0; m < 4; ++m) { mx = fmax(mx, fabs(S.rout[m] - S.v[24 + m])); sc = fmax(sc, fabs(S.v[24 + m])); }
            ok = ok && mx / sc <= 2.0e-12;
        }
#pragma unroll
        for (int m = 0; m < 4; ++m) afw[m] = afw[m] + gw[g] * S.rout[4 + m];
        ok = __syncthreads_and(ok) != 0;   // uniform before the loop test
    }
    if (!__syncthreads_and(ok)) {
        if (threadIdx.x == 0) set_status(B.status, ST_NONFINITE_FLUX);
        return;
    }
    // publish times the face length into the face arrays ComputeResidual reads
    const double len = axis == 0 ? P.dy : P.dx;
    size_t o;
    double *Fh, *Fb, *Fw;
    if (axis == 0) { o = (size_t)j * nx + (i + 1) % nx; Fh = B.fxh; Fb = B.fxb; Fw = B.fxw; }
    else { o = (size_t)(j + 1) * nx + i; Fh = B.fyh; Fb = B.fyb; Fw = B.fyw; }
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        if (s.ok) { Fh[o * nv + s.k] = afh[r] * len; Fb[o * nv + s.k] = afb[r] * len; }
    }
    if (threadIdx.x == 0)
        for (int m = 0; m < 4; ++m) Fw[o * 4 + m] = afw[m] * len;
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

// wall faces: one CTA per wall face (bottom faces of row 0, then top faces of row ny-1), the 3
// Gauss nodes of s2w2_wall_node in turn
template <int VPT, int NT>
__global__ void __launch_bounds__(NT) k_s2_walls(LoParams P, LoBuffers B, S2Buffers SB) {
    if (eval_cached(B)) return;
    __shared__ S2Shared S;
    const int nv = P.nvel, nx = P.nx, ny = P.ny, ck = P.ck;
    const int top = blockIdx.x >= nx ? 1 : 0, i = blockIdx.x - top * nx;
    const int cc = top ? (ny - 1) * nx + i : i, sidx = top ? 3 : 2;
    const double side = top ? 1.0 : -1.0;
    const double ux = P.wall_ux[top], theta = 0.5 / P.wall_lam[top];
    const double dt = B.dt[0];
    const double* wcell = B.W + cc * 4;
    const double pp = (2.0 / (double)(ck + 2)) * (wcell[3] - 0.5 * (wcell[1] * wcell[1] + wcell[2] * wcell[2]) / wcell[0]);
    const double lambda = 0.5 / theta;
    const double prim_g[4] = {pp / theta, 0.0, -ux, lambda};
    const double wc[4] = {wcell[0], wcell[2], -wcell[1], wcell[3]};
    const double wg[4] = {prim_g[0], 0.0, -prim_g[0] * ux, prim_g[0] * ((double)(ck + 2) / (4.0 * lambda) + 0.5 * ux * ux)};
    // wall_equilibrium: the discrete closure of the wall state (the same for the 3 nodes)
    if (threadIdx.x == 0) {
        S.w[0] = prim_g[0]; S.w[1] = prim_g[0] * ux; S.w[2] = 0.0;
        S.w[3] = prim_g[0] * ((double)(ck + 2) * theta / 2.0 + ux * ux / 2.0);
    }
    __syncthreads();
    bool ok = pp > 0.0 && isfinite(pp) && s2_closure<VPT>(P, B, S);
    const double gw[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
    double afh[VPT], afb[VPT], afw[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int r = 0; r < VPT; ++r) afh[r] = afb[r] = 0.0;
    double thc[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) thc[m] = S.th[m];
    for (int g = 0; g < 3 && ok; ++g) {
        double hin[VPT], bin[VPT], hn[VPT], bn[VPT], ht[VPT], bt[VPT], acc[8];
#pragma unroll
        for (int m = 0; m < 6; ++m) acc[m] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
            const double* rc = SB.rec + (size_t)cc * 72 * nv + s.kk;
            hin[r] = rc[(size_t)(0 * 12 + sidx * 3 + g) * nv];
            bin[r] = rc[(size_t)(1 * 12 + sidx * 3 + g) * nv];
            hn[r] = rc[(size_t)(2 * 12 + sidx * 3 + g) * nv];
            ht[r] = rc[(size_t)(3 * 12 + sidx * 3 + g) * nv];
            bn[r] = rc[(size_t)(4 * 12 + sidx * 3 + g) * nv];
            bt[r] = rc[(size_t)(5 * 12 + sidx * 3 + g) * nv];
            const double vn = vk, vt = -uk, v2 = vn * vn + vt * vt;
            acc[0] += wk * (-ht[r]);
            acc[1] += wk * (-(vn * ht[r]));
            acc[2] += wk * (-(vt * ht[r]));
            acc[3] += wk * (-(0.5 * (v2 * ht[r] + bt[r])));
            const double vt2 = -uk + ux, w2 = vn * vn + vt2 * vt2;
            acc[4] += 0.5 * wk * vn * (w2 * hin[r] + bin[r]);
            acc[5] += 0.5 * wk * vt2 * (w2 * hin[r] + bin[r]);
        }
        block_reduce_smem<6, 0>(acc, S.red, S.rout);
        if (threadIdx.x == 0) {
            double sw[4], sw_t[4], an[4], at[4], atime[4], Mu[7], Mv[6], Mxi[3], m1[4], m2[4], mt[5];
            for (int m = 0; m < 4; ++m) { sw[m] = (wg[m] - wc[m]) / (side * 0.5 * P.dy); sw_t[m] = S.rout[m]; }
            s2w_micro_slope(ck, prim_g, sw, an);
            s2w_micro_slope(ck, prim_g, sw_t, at);
            s2w_moments(ck, prim_g, Mu, Mv, Mxi);
            s2w_auvxi(an, Mu, Mv, Mxi, 1, 0, m1);
            s2w_auvxi(at, Mu, Mv, Mxi, 0, 1, m2);
            for (int m = 0; m < 4; ++m) sw[m] = -prim_g[0] * (m1[m] + m2[m]);
            s2w_micro_slope(ck, prim_g, sw, atime);
            double tau_wall = 0.0;
            const double wgg[4] = {wg[0], -wg[2], wg[1], wg[3]};
            const bool tok = s2_tau(P, wgg, tau_wall);
            s2w_time_coeffs(dt, tau_wall, mt);
            const double coeff = P.pr != 1.0 ? 0.8 * (1.0 - P.pr) * lambda * lambda / prim_g[0] : 0.0;
            for (int m = 0; m < 4; ++m) { S.v[m] = an[m]; S.v[4 + m] = at[m]; S.v[8 + m] = atime[m]; }
            for (int m = 0; m < 5; ++m) S.v[12 + m] = mt[m];
            S.v[17] = Mxi[2]; S.v[18] = coeff; S.v[19] = S.rout[4]; S.v[20] = S.rout[5]; S.v[21] = tok ? 1.0 : 0.0;
        }
        __syncthreads();
        if (S.v[21] == 0.0) { ok = false; break; }
        double an[4], at[4], atime[4], mt[5];
#pragma unroll
        for (int m = 0; m < 4; ++m) { an[m] = S.v[m]; at[m] = S.v[4 + m]; atime[m] = S.v[8 + m]; }
#pragma unroll
        for (int m = 0; m < 5; ++m) mt[m] = S.v[12 + m];
        const double mxi2 = S.v[17], coeff = S.v[18], hlx = S.v[19], hly = S.v[20];
        double ginh[VPT], ginb[VPT], wallh[VPT], wallb[VPT];
        acc[0] = acc[1] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
            const S2Q q = s2_q(thc, ck, uk, vk);
            const double mh = q.qh, mb = q.qb;
            wallh[r] = mh / prim_g[0]; wallb[r] = mb / prim_g[0];
            double corrh = 0.0, corrb = 0.0;
            if (P.pr != 1.0) {
                const double vn = vk, vt = -uk + ux, v2 = vn * vn + vt * vt;
                const double qdot = vn * hlx + vt * hly, shh = 2.0 * lambda * v2 - 4.0;
                corrh = coeff * qdot * shh * mh;
                corrb = coeff * qdot * (shh + 2.0 / (double)ck) * mb;
            }
            const double vn = vk, vt = -uk, v2 = vn * vn + vt * vt;
            const double Han = (an[0] + an[1] * vn + an[2] * vt) * mh + 0.5 * an[3] * (v2 * mh + mb);
            const double Hatan = (at[0] + at[1] * vn + at[2] * vt) * mh + 0.5 * at[3] * (v2 * mh + mb);
            const double Hatime = (atime[0] + atime[1] * vn + atime[2] * vt) * mh + 0.5 * atime[3] * (v2 * mh + mb);
            const double Ban = (an[0] + an[1] * vn + an[2] * vt) * mb + 0.5 * an[3] * (v2 * mb + mxi2 * mh);
            const double Batan = (at[0] + at[1] * vn + at[2] * vt) * mb + 0.5 * at[3] * (v2 * mb + mxi2 * mh);
            const double Batime = (atime[0] + atime[1] * vn + atime[2] * vt) * mb + 0.5 * atime[3] * (v2 * mb + mxi2 * mh);
            ginh[r] = mt[0] * mh + mt[1] * (vn * Han + vt * Hatan) + mt[2] * Hatime + mt[3] * hin[r] -
                      mt[4] * (vn * hn[r] + uk * ht[r]);
            ginb[r] = mt[0] * mb + mt[1] * (vn * Ban + vt * Batan) + mt[2] * Batime + mt[3] * bin[r] -
                      mt[4] * (vn * bn[r] + uk * bt[r]);
            ginh[r] = ginh[r] + mt[0] * corrh;
            ginb[r] = ginb[r] + mt[0] * corrb;
            if (side * vn > 0.0) acc[0] += wk * vn * ginh[r];
            else acc[1] += dt * wk * vn * wallh[r];
        }
        block_reduce_smem<2, 0>(acc, S.red, S.rout);
        const double inc = S.rout[0], refl = S.rout[1];
        const double rhow = -inc / refl;
        if (!isfinite(refl) || fabs(refl) <= DBL_MIN || !isfinite(rhow) || rhow <= 0.0) { ok = false; break; }
#pragma unroll
        for (int m = 0; m < 4; ++m) acc[m] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
            double fh, fb;
            if (side * vk > 0.0) { fh = vk * ginh[r]; fb = vk * ginb[r]; }
            else { fh = dt * vk * rhow * wallh[r]; fb = dt * vk * rhow * wallb[r]; }
            acc[0] += wk * fh; acc[1] += wk * (uk * fh); acc[2] += wk * (vk * fh);
            acc[3] += wk * (0.5 * ((uk * uk + vk * vk) * fh + fb));
            afh[r] = afh[r] + gw[g] * fh;
            afb[r] = afb[r] + gw[g] * fb;
            if (s.ok) ok = ok && isfinite(fh) && isfinite(fb);
        }
        block_reduce_smem<4, 0>(acc, S.red, S.rout);
        ok = ok && isfinite(S.rout[0]) && fabs(S.rout[0]) <= 2.0e-12 * fmax(1.0, fabs(inc));
#pragma unroll
        for (int m = 0; m < 4; ++m) afw[m] = afw[m] + gw[g] * S.rout[m];
        ok = __syncthreads_and(ok) != 0;   // uniform before the loop test
    }
    if (!__syncthreads_and(ok)) {
        if (threadIdx.x == 0) set_status(B.status, ST_NONFINITE_FLUX);
        return;
    }
    const size_t o = top ? (size_t)ny * nx + i : (size_t)i;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        if (s.ok) { B.fyh[o * nv + s.k] = afh[r] * P.dx; B.fyb[o * nv + s.k] = afb[r] * P.dx; }
    }
    if (threadIdx.x == 0) {
        for (int m = 0; m < 4; ++m) B.fyw[o * 4 + m] = afw[m] * P.dx;
        if (SB.wall_raw != nullptr)
            for (int m = 0; m < 4; ++m) SB.wall_raw[((size_t)top * nx + i) * 4 + m] = afw[m];
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
    return cudaMemcpyToSymbol(c_s2, &m, sizeof m);
}

template <int VPT, int NT>
static void s2_launch_all(int which, const LoParams& P, const LoBuffers& B, const S2Buffers& S, cudaStream_t s,
                          cudaStream_t s2, cudaEvent_t fork, cudaEvent_t join, cudaError_t& e) {
    const int nc = P.nx * P.ny;
    if (which == 0) {
        k_s2_init<VPT, NT><<<nc, NT, 0, s>>>(P, B, S);
        e = cudaGetLastError();
        return;
    }
    if (which != 2) {
        k_s2_targets<VPT, NT><<<nc, NT, 0, s>>>(P, B, S);
        e = cudaGetLastError();
        if (which == 3) return;
    }
    if (e == cudaSuccess) {
        const dim3 grid((unsigned)((P.nvel + 127) / 128), (unsigned)nc);
        k_s2_recon<<<grid, 128, 0, s>>>(P, B, S);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(fork, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s2, fork, 0);
    if (e == cudaSuccess) { k_s2_walls<VPT, NT><<<2 * P.nx, NT, 0, s2>>>(P, B, S); e = cudaGetLastError(); }
    if (e == cudaSuccess) e = cudaEventRecord(join, s2);
    if (e == cudaSuccess) { k_s2_faces<VPT, NT><<<P.nx * P.ny + P.nx * (P.ny - 1), NT, 0, s>>>(P, B, S); e = cudaGetLastError(); }
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, join, 0);
}

// which 0: the S2 cold start; 1: the S2 Evolution of one pseudo-step (targets, reconstruction, faces,
// walls); 2: the Evolution with the targets kept (S2CN2); 3: the targets of B.W only
cudaError_t s2_enqueue(int which, const LoParams& P, const LoBuffers& B, const S2Buffers& S, cudaStream_t s,
                       cudaStream_t s2, cudaEvent_t fork, cudaEvent_t join) {
    cudaError_t e = cudaSuccess;
    if (P.nvel <= 1024) s2_launch_all<2, 512>(which, P, B, S, s, s2, fork, join, e);
    else s2_launch_all<5, 512>(which, P, B, S, s, s2, fork, join, e);
    return e;
}

}  // namespace ugks
