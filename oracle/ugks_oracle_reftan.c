/*
 * ugks_oracle_reftan.c -- TEST INFRASTRUCTURE ONLY (included by ugks_oracle_s2.c).
 *
 * The reference's own forward-mode (tangent) routines of the high-order path, restated: the directional
 * derivatives its research code uses to check derivatives (mod_CorrectedWF2DEquilibrium.f90:67-101,
 * mod_CorrectedWF2DClosure.f90:211-243 and 560-625, mod_WENO5AOScalar.f90:98-201).  The tests compare
 * each with central differences of its own value outputs and with the tangent build of the oracle
 * (oracle/tangent.hpp), which differentiates the same arithmetic by (value, derivative) numbers: the
 * reference's hand-written tangents then pin the tangent build that the device adjoint is checked
 * against.  Nothing in the product library calls these.
 */

/* analytic_maxwellian_direction_2d (mod_CorrectedWF2DEquilibrium.f90:67-101): the analytic Maxwellian
 * of w (mh, mb) and its derivative along w_direction (dmh, dmb).  Returns 1 when all are finite. */
int uo_ref_maxwellian_direction(const double w[4], const double dw[4], int ck, int n, const double* u, const double* v,
                                double* mh, double* mb, double* dmh, double* dmb) {
    double rho, uu, vv, temp;
    for (int k = 0; k < n; ++k) { mh[k] = 0.0; mb[k] = 0.0; dmh[k] = 0.0; dmb[k] = 0.0; }
    if (!s2_prim_native(w, ck, &rho, &uu, &vv, &temp)) return 0;
    for (int m = 0; m < 4; ++m) if (!isfinite(dw[m])) return 0;
    const double drho = dw[0];
    const double du = (dw[1] - uu * drho) / rho;
    const double dv = (dw[2] - vv * drho) / rho;
    const double gamma_factor = 4.0 / (double)(ck + 2);
    const double dtemp = gamma_factor * (dw[3] / rho - (w[3] / (rho * rho)) * drho - uu * du - vv * dv);
    const double lambda = 1.0 / temp, pi = acos(-1.0);
    int ok = 1;
    for (int k = 0; k < n; ++k) {
        const double c2 = (u[k] - uu) * (u[k] - uu) + (v[k] - vv) * (v[k] - vv);
        mh[k] = rho * lambda / pi * exp(-lambda * c2);
        mb[k] = 0.5 * (double)ck * temp * mh[k];
        const double logd = drho / rho + 2.0 * ((u[k] - uu) * du + (v[k] - vv) * dv) / temp + (c2 / temp - 1.0) * dtemp / temp;
        dmh[k] = mh[k] * logd;
        dmb[k] = mb[k] * (dtemp / temp + logd);
        ok = ok && isfinite(mh[k]) && isfinite(mb[k]) && isfinite(dmh[k]) && isfinite(dmb[k]);
    }
    return ok;
}

/* second theta-derivatives of the closure pair at one velocity (q_state_and_derivatives,
 * mod_CorrectedWF2DClosure.f90, the hessian arrays): d2 q / d theta_a d theta_b = q (ld_a ld_b +
 * d ld_a / d theta_b), theta = (rho, u, v, T_native), ld the log-derivative row of q */
static void reftan_hessian(const double th[4], double u, double v, double qh, double qb, double hh[4][4], double hb[4][4]) {
    const double r = th[0], tw = th[3], du = u - th[1], dv = v - th[2], c2 = du * du + dv * dv;
    const double ld[4] = {1.0 / r, 2.0 * du / tw, 2.0 * dv / tw, -1.0 / tw + c2 / (tw * tw)};
    const double ldb[4] = {ld[0], ld[1], ld[2], ld[3] + 1.0 / tw};
    double dld[4][4];
    for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) dld[a][b] = 0.0;
    dld[0][0] = -1.0 / (r * r);
    dld[1][1] = -2.0 / tw;
    dld[1][3] = -2.0 * du / (tw * tw);
    dld[2][2] = -2.0 / tw;
    dld[2][3] = -2.0 * dv / (tw * tw);
    dld[3][1] = -2.0 * du / (tw * tw);
    dld[3][2] = -2.0 * dv / (tw * tw);
    dld[3][3] = 1.0 / (tw * tw) - 2.0 * c2 / (tw * tw * tw);
    for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) {
            const double dldb = (a == 3 && b == 3) ? dld[3][3] - 1.0 / (tw * tw) : dld[a][b];
            hh[a][b] = qh * (ld[a] * ld[b] + dld[a][b]);
            hb[a][b] = qb * (ldb[a] * ldb[b] + dldb);
        }
}

/* dq_value_and_direction (mod_CorrectedWF2DClosure.f90:560-625): the closure correction c = dq(w) theta_m
 * of the moment vector m, with theta_m = J^-1 m, and its derivative along (w_direction, m_direction):
 * dc = dq theta_md + d2q[theta_d, theta_m], theta_d = J^-1 dw, theta_md = J^-1 (dm - dJ[theta_d] theta_m). */
int uo_ref_dq_direction(const double w[4], const double dw[4], const double m[4], const double dm[4], int ck, int n,
                        const double* u, const double* v, const double* wt, double* ch, double* cb, double* dch,
                        double* dcb) {
    double* qh = (double*)calloc((size_t)n, sizeof(double));
    double* qb = (double*)calloc((size_t)n, sizeof(double));
    double* qht = (double*)calloc((size_t)n * 4, sizeof(double));
    double* qbt = (double*)calloc((size_t)n * 4, sizeof(double));
    double* scr = (double*)calloc((size_t)n * 10, sizeof(double));
    int ok = qh && qb && qht && qbt && scr;
    for (int k = 0; k < n; ++k) { ch[k] = cb[k] = dch[k] = dcb[k] = 0.0; }
    s2_closure C;
    if (ok) {
        C.qh = qh; C.qb = qb; C.qht = qht; C.qbt = qbt;
        ok = s2_closure_prepare(&C, w, ck, n, u, v, wt, scr);
    }
    double td[4], tm[4], tmd[4];
    ok = ok && s2_solve4(C.jac, dw, td) && s2_solve4(C.jac, m, tm);
    if (ok) {
        /* djac(:, a) = moments of sum_b hessian(:, a, b) theta_d(b) */
        double djac[4][4];
        for (int a = 0; a < 4; ++a) {
            double mom[4] = {0.0, 0.0, 0.0, 0.0};
            for (int k = 0; k < n; ++k) {
                double hh[4][4], hb[4][4];
                reftan_hessian(C.theta, u[k], v[k], qh[k], qb[k], hh, hb);
                double dh = 0.0, db = 0.0;
                for (int b = 0; b < 4; ++b) { dh = dh + hh[a][b] * td[b]; db = db + hb[a][b] * td[b]; }
                mom[0] = mom[0] + wt[k] * dh;
                mom[1] = mom[1] + wt[k] * u[k] * dh;
                mom[2] = mom[2] + wt[k] * v[k] * dh;
                mom[3] = mom[3] + 0.5 * wt[k] * ((u[k] * u[k] + v[k] * v[k]) * dh + db);
            }
            for (int r = 0; r < 4; ++r) djac[r][a] = mom[r];
        }
        double rhs[4];
        for (int r = 0; r < 4; ++r) {
            double s = 0.0;
            for (int a = 0; a < 4; ++a) s = s + djac[r][a] * tm[a];
            rhs[r] = dm[r] - s;
        }
        ok = s2_solve4(C.jac, rhs, tmd);
    }
    if (ok) {
        for (int k = 0; k < n; ++k) {
            double hh[4][4], hb[4][4];
            reftan_hessian(C.theta, u[k], v[k], qh[k], qb[k], hh, hb);
            double c_h = 0.0, c_b = 0.0, d_h = 0.0, d_b = 0.0;
            for (int a = 0; a < 4; ++a) {
                c_h = c_h + qht[(size_t)k * 4 + a] * tm[a];
                c_b = c_b + qbt[(size_t)k * 4 + a] * tm[a];
                d_h = d_h + qht[(size_t)k * 4 + a] * tmd[a];
                d_b = d_b + qbt[(size_t)k * 4 + a] * tmd[a];
                for (int b = 0; b < 4; ++b) { d_h = d_h + hh[a][b] * td[a] * tm[b]; d_b = d_b + hb[a][b] * td[a] * tm[b]; }
            }
            ch[k] = c_h; cb[k] = c_b; dch[k] = d_h; dcb[k] = d_b;
            ok = ok && isfinite(c_h) && isfinite(c_b) && isfinite(d_h) && isfinite(d_b);
        }
    }
    free(qh); free(qb); free(qht); free(qbt); free(scr);
    return ok;
}

/* projector_direction_2d (mod_CorrectedWF2DClosure.f90:211-243): p = z - dq(w) J^-1 moments(z) and its
 * derivative along (w_direction, z_direction). */
int uo_ref_projector_direction(const double w[4], const double dw[4], const double* zh, const double* zb,
                               const double* dzh, const double* dzb, int ck, int n, const double* u, const double* v,
                               const double* wt, double* ph, double* pb, double* dph, double* dpb) {
    double m[4], dm[4];
    if (!s2_moment(n, zh, zb, u, v, wt, m) || !s2_moment(n, dzh, dzb, u, v, wt, dm)) return 0;
    double* c = (double*)calloc((size_t)n * 4, sizeof(double));
    if (!c) return 0;
    const int ok = uo_ref_dq_direction(w, dw, m, dm, ck, n, u, v, wt, c, c + n, c + 2 * n, c + 3 * n);
    for (int k = 0; k < n; ++k) {
        ph[k] = zh[k] - c[k];
        pb[k] = zb[k] - c[n + k];
        dph[k] = dzh[k] - c[2 * n + k];
        dpb[k] = dzb[k] - c[3 * n + k];
    }
    free(c);
    return ok;
}

/* weno5ao_smoothness (mod_WENO5AOScalar.f90:203-219): the AO(5,3) smoothness indicators of a stencil */
static void reftan_beta(const double q[5], double beta[4]) {
    const double qm2 = q[0], qm1 = q[1], qi = q[2], qp1 = q[3], qp2 = q[4];
    const double t0 = qm2 - 2.0 * qm1 + qi, u0 = qm2 - 4.0 * qm1 + 3.0 * qi;
    const double t1 = qm1 - 2.0 * qi + qp1, u1 = qm1 - qp1;
    const double t2 = qi - 2.0 * qp1 + qp2, u2 = 3.0 * qi - 4.0 * qp1 + qp2;
    beta[0] = (13.0 / 12.0) * (t0 * t0) + 0.25 * (u0 * u0);
    beta[1] = (13.0 / 12.0) * (t1 * t1) + 0.25 * (u1 * u1);
    beta[2] = (13.0 / 12.0) * (t2 * t2) + 0.25 * (u2 * u2);
    beta[3] = (231153.0 * qi * qi + 104963.0 * qm1 * qm1 + 6908.0 * qm2 * qm2 - 38947.0 * qm2 * qp1 +
               104963.0 * qp1 * qp1 + qm1 * (-51001.0 * qm2 + 179098.0 * qp1 - 38947.0 * qp2) -
               3.0 * qi * (99692.0 * qm1 - 22641.0 * qm2 + 99692.0 * qp1 - 22641.0 * qp2) + 8209.0 * qm2 * qp2 -
               51001.0 * qp1 * qp2 + 6908.0 * qp2 * qp2) / 5040.0;
}

/* prepare_ / evaluate_weno5ao_cell_first_direction (mod_WENO5AOScalar.f90:98-201): the WENO-AO(5,3) value
 * at xi of the stencil q and its derivative along q_direction.  *differentiable = 0 where tau's |x| is at
 * its kink with a nonzero direction (the reference's branch test). */
int uo_ref_weno_direction(const double q[5], const double dq[5], double xi, double* val, double* dval,
                          int* differentiable) {
    s2_init_maps();
    const double eps = 1.0e-8, gam[4] = {0.01125, 0.1275, 0.01125, 0.85};
    double beta[4], bq[4], bs[4], qs[5], bd[4];
    for (int k = 0; k < 5; ++k) qs[k] = q[k] + dq[k];
    /* the direction of a quadratic form: beta(q + dq) - beta(q) - beta(dq) */
    reftan_beta(q, beta);
    reftan_beta(dq, bq);
    reftan_beta(qs, bs);
    for (int c = 0; c < 4; ++c) bd[c] = bs[c] - beta[c] - bq[c];
    double path = 0.0, pd = 0.0;
    for (int k = 0; k < 5; ++k) { path = fmax(path, fabs(q[k])); pd = fmax(pd, fabs(dq[k])); }
    path = fmax(path + pd, sqrt(DBL_MIN));
    const double btol = 1024.0 * DBL_EPSILON * path * path;
    double tau = 0.0, taud = 0.0;
    *differentiable = 1;
    for (int c = 0; c < 3; ++c) {
        const double d = beta[3] - beta[c], dd = bd[3] - bd[c];
        if (fabs(d) > DBL_MIN) { tau = tau + fabs(d); taud = taud + (d > 0.0 ? 1.0 : -1.0) * dd; }
        else if (fabs(dd) > btol) *differentiable = 0;
    }
    tau = tau / 3.0;
    taud = taud / 3.0;
    double alpha[4], alphad[4], sa = 0.0, sad = 0.0;
    for (int c = 0; c < 4; ++c) {
        const double den = beta[c] + eps, ratio = tau / den;
        const double ratiod = taud / den - tau * bd[c] / (den * den);
        alpha[c] = gam[c] * (1.0 + ratio * ratio);
        alphad[c] = 2.0 * gam[c] * ratio * ratiod;
        sa = sa + alpha[c];
        sad = sad + alphad[c];
    }
    double om[4], omd[4], fw[4], fwd[4];
    for (int c = 0; c < 4; ++c) { om[c] = alpha[c] / sa; omd[c] = alphad[c] / sa - alpha[c] * sad / (sa * sa); }
    fw[3] = om[3] / gam[3];
    fwd[3] = omd[3] / gam[3];
    for (int c = 0; c < 3; ++c) { fw[c] = om[c] - fw[3] * gam[c]; fwd[c] = omd[c] - fwd[3] * gam[c]; }
    fw[3] = 1.0 - (fw[0] + fw[1] + fw[2]);
    fwd[3] = -(fwd[0] + fwd[1] + fwd[2]);
    /* the candidate polynomials of q and of the direction at xi (cell_average_polynomial_coefficients) */
    double vv = 0.0, vd = 0.0;
    for (int c = 0; c < 4; ++c) {
        const int lo = c < 3 ? c : 0, hi = c < 3 ? c + 2 : 4;
        double pc = 0.0, pcd = 0.0;
        for (int d = 0; d < 5; ++d) {
            double cf = 0.0, cfd = 0.0;
            for (int k = lo; k <= hi; ++k) { cf = cf + s2_cmap[c][k][d] * q[k]; cfd = cfd + s2_cmap[c][k][d] * dq[k]; }
            const double xp = s2_powi(xi, d);
            pc = pc + cf * xp;
            pcd = pcd + cfd * xp;
        }
        vv = vv + fw[c] * pc;
        vd = vd + fwd[c] * pc + fw[c] * pcd;
    }
    *val = vv;
    *dval = vd;
    return isfinite(vv) && isfinite(vd);
}
