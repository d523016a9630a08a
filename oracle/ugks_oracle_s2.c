/*
 * ugks_oracle_s2.c -- TEST INFRASTRUCTURE ONLY.  Compiled as part of ugks_oracle.c (it is included
 * at the end of that file and shares its context and helpers).
 *
 * Plain-C restatement of the reference's high-order "S2" evolution for the HighOrderImplicit
 * Couette case (S2PhysicalGas=1, S2W1_wall_mode=1, FluxWall_type=1, S2CartesianMesh): tensor
 * WENO-AO(5,3) reconstruction with one-sided quartics at the walls, the discrete-conservative
 * Newton closure, 3-point Gauss quadrature UGKS face nodes, the multiscale diffuse wall node, the
 * volume targets and the S2 physical collision.  Summation and operation order follow the Fortran.
 */

#define S2_GATE 2.0e-12
static const double s2_gw[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};   /* mod_S2D1.f90:36 */
static const double s2_gamma_lin[4] = {0.01125, 0.1275, 0.01125, 0.85}; /* mod_S2D1Reconstruction.f90:13 */
#define S2_EPS_WENO 1.0e-8

/* reconstruction maps (mod_S2D1Reconstruction.f90:57-111): cmap[c][k][d] is the coefficient of xi^d
 * contributed by sample k of candidate c; wallmap[side][dist-1][k][d] the one-sided quartic. */
static double s2_cmap[4][5][5];
static double s2_wallmap[2][3][5][5];
static double s2_gnode[3];
static int s2_maps_ready = 0;
static pthread_mutex_t s2_maps_lock = PTHREAD_MUTEX_INITIALIZER;

/* solve_small (mod_S2D1Reconstruction.f90:143-166): partial-pivot elimination, back substitution */
static void s2_solve_small(int n, const double a[5][5], const double b[5], double x[5]) {
    double w[5][5], r[5];
    for (int i = 0; i < n; ++i) { for (int j = 0; j < n; ++j) w[i][j] = a[i][j]; r[i] = b[i]; }
    for (int p = 0; p < n - 1; ++p) {
        int m = p;
        double best = fabs(w[p][p]);
        for (int i = p + 1; i < n; ++i) if (fabs(w[i][p]) > best) { best = fabs(w[i][p]); m = i; }
        if (m != p) {
            for (int j = 0; j < n; ++j) { double t = w[p][j]; w[p][j] = w[m][j]; w[m][j] = t; }
            double t = r[p]; r[p] = r[m]; r[m] = t;
        }
        for (int i = p + 1; i < n; ++i) {
            double fac = w[i][p] / w[p][p];
            for (int j = p; j < n; ++j) w[i][j] = w[i][j] - fac * w[p][j];
            r[i] = r[i] - fac * r[p];
        }
    }
    x[n - 1] = r[n - 1] / w[n - 1][n - 1];
    for (int i = n - 2; i >= 0; --i) {
        double s = 0.0;
        for (int j = i + 1; j < n; ++j) s = s + w[i][j] * x[j];
        x[i] = (r[i] - s) / w[i][i];
    }
}

/* build_map (mod_S2D1Reconstruction.f90:81-108).  ordered: map index = sample position. */
static void s2_build_map(int n, const int* off, int ordered, double map[5][5] /* [k][d] */) {
    double a[5][5], rhs[5], x[5];
    for (int k = 0; k < 5; ++k) for (int d = 0; d < 5; ++d) map[k][d] = 0.0;
    for (int r = 0; r < n; ++r)
        for (int d = 0; d < n; ++d)
            a[r][d] = (pow((double)off[r] + 0.5, d + 1) - pow((double)off[r] - 0.5, d + 1)) / (double)(d + 1);
    for (int c = 0; c < n; ++c) {
        for (int r = 0; r < n; ++r) rhs[r] = 0.0;
        rhs[c] = 1.0;
        s2_solve_small(n, a, rhs, x);
        int slot = ordered ? c : off[c] + 2;
        for (int d = 0; d < n; ++d) map[slot][d] = x[d];
    }
}

static void s2_init_maps(void) {
    pthread_mutex_lock(&s2_maps_lock);
    if (!s2_maps_ready) {
        const int o1[3] = {-2, -1, 0}, o2[3] = {-1, 0, 1}, o3[3] = {0, 1, 2}, o5[5] = {-2, -1, 0, 1, 2};
        s2_build_map(3, o1, 0, s2_cmap[0]);
        s2_build_map(3, o2, 0, s2_cmap[1]);
        s2_build_map(3, o3, 0, s2_cmap[2]);
        s2_build_map(5, o5, 0, s2_cmap[3]);
        for (int j = 1; j <= 3; ++j) {
            int lo[5], hi[5];
            for (int s = 0; s < 5; ++s) { lo[s] = (s + 1) - j; hi[s] = (s - 4) + j - 1; }
            s2_build_map(5, lo, 1, s2_wallmap[0][j - 1]);
            s2_build_map(5, hi, 1, s2_wallmap[1][j - 1]);
        }
        const double g = 0.5 * sqrt(3.0 / 5.0);
        s2_gnode[0] = -g; s2_gnode[1] = 0.0; s2_gnode[2] = g;
        s2_maps_ready = 1;
    }
    pthread_mutex_unlock(&s2_maps_lock);
}

/* x**n with a small integer n as gfortran evaluates it (repeated squaring) */
static double s2_powi(double x, int n) {
    if (n == 0) return 1.0;
    if (n == 1) return x;
    if (n == 2) return x * x;
    if (n == 3) return x * x * x;
    return (x * x) * (x * x);
}

/* weno_coefficients (mod_S2D1Reconstruction.f90:168-204): fw[4], coef[c][d] */
static int s2_weno_coef(const double q[5], double fw[4], double coef[4][5]) {
    const double q1 = q[0], q2 = q[1], q3 = q[2], q4 = q[3], q5 = q[4];
    double beta[4], alpha[4], omega[4];
    double t;
    t = q1 - 2 * q2 + q3; double u0 = q1 - 4 * q2 + 3 * q3;
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
    double sa = 0.0;
    for (int c = 0; c < 4; ++c) {
        double r = tau / (beta[c] + S2_EPS_WENO);
        alpha[c] = s2_gamma_lin[c] * (1.0 + r * r);
        sa = sa + alpha[c];
    }
    for (int c = 0; c < 4; ++c) omega[c] = alpha[c] / sa;
    fw[3] = omega[3] / s2_gamma_lin[3];
    for (int c = 0; c < 3; ++c) fw[c] = omega[c] - fw[3] * s2_gamma_lin[c];
    for (int c = 0; c < 4; ++c) for (int d = 0; d < 5; ++d) coef[c][d] = 0.0;
    for (int c = 0; c < 3; ++c)
        for (int k = c; k <= c + 2; ++k)
            for (int d = 0; d <= 2; ++d) coef[c][d] = coef[c][d] + s2_cmap[c][k][d] * q[k];
    for (int k = 0; k < 5; ++k)
        for (int d = 0; d <= 4; ++d) coef[3][d] = coef[3][d] + s2_cmap[3][k][d] * q[k];
    int ok = 1;
    for (int c = 0; c < 4; ++c) { ok &= isfinite(fw[c]); for (int d = 0; d < 5; ++d) ok &= isfinite(coef[c][d]); }
    return ok;
}

/* coefficients of a companion field with the primary's weights (companion_eval3, :296-299) */
static void s2_companion_coef(const double q[5], double coef[4][5]) {
    for (int c = 0; c < 4; ++c) for (int d = 0; d < 5; ++d) coef[c][d] = 0.0;
    for (int c = 0; c < 3; ++c)
        for (int k = c; k <= c + 2; ++k)
            for (int d = 0; d <= 2; ++d) coef[c][d] = coef[c][d] + s2_cmap[c][k][d] * q[k];
    for (int k = 0; k < 5; ++k)
        for (int d = 0; d <= 4; ++d) coef[3][d] = coef[3][d] + s2_cmap[3][k][d] * q[k];
}

/* prepared_eval (mod_S2D1Reconstruction.f90:247-262) */
static void s2_eval(const double fw[4], const double coef[4][5], double xi, double* val, double* der) {
    double pw[5], dp[5];
    pw[0] = 1.0; dp[0] = 0.0;
    for (int d = 1; d <= 4; ++d) { pw[d] = pw[d - 1] * xi; dp[d] = (double)d * s2_powi(xi, d - 1); }
    double v = 0.0, dv = 0.0;
    for (int c = 0; c < 4; ++c) {
        double cand = 0.0, dcand = 0.0;
        for (int d = 0; d < 5; ++d) { cand = cand + coef[c][d] * pw[d]; dcand = dcand + coef[c][d] * dp[d]; }
        v = v + fw[c] * cand;
        dv = dv + fw[c] * dcand;
    }
    *val = v;
    if (der) *der = dv;
}

/* companion_eval3 (mod_S2D1Reconstruction.f90:287-318): value, derivative and the companion's
 * value at the three Gauss nodes */
static int s2_companion3(const double q[5], const double comp[5], double val[3], double der[3], double cval[3]) {
    double fw[4], coef[4][5], ccoef[4][5];
    if (!s2_weno_coef(q, fw, coef)) return 0;
    s2_companion_coef(comp, ccoef);
    for (int s = 0; s < 3; ++s) {
        s2_eval(fw, coef, s2_gnode[s], &val[s], &der[s]);
        double dummy;
        (void)dummy;
        double pw[5];
        pw[0] = 1.0;
        for (int d = 1; d <= 4; ++d) pw[d] = pw[d - 1] * s2_gnode[s];
        double cv = 0.0;
        for (int c = 0; c < 4; ++c) {
            double cc = 0.0;
            for (int d = 0; d < 5; ++d) cc = cc + ccoef[c][d] * pw[d];
            cv = cv + fw[c] * cc;
        }
        cval[s] = cv;
        if (!(isfinite(val[s]) && isfinite(der[s]) && isfinite(cval[s]))) return 0;
    }
    return 1;
}

/* near_wall / wall_first (mod_S2MPI1Layout.f90:280-284,386-389), 0-based rows */
static int s2_near_wall(int j, int ny) { return j + 1 <= 3 || j + 1 >= ny - 2; }
static int s2_wall_first(int j, int ny) { return (j + 1 <= 3) ? 0 : ny - 5; }

/* wall_coeff + wall_eval (mod_S2D1Reconstruction.f90:113-136) */
static void s2_wall_eval(const double q[5], int j, int ny, double xi, double* val, double* der) {
    const double (*map)[5] = (j + 1 <= 3) ? s2_wallmap[0][j] : s2_wallmap[1][ny - 1 - j];
    double c[5];
    for (int d = 0; d < 5; ++d) c[d] = 0.0;
    for (int k = 0; k < 5; ++k) for (int d = 0; d < 5; ++d) c[d] = c[d] + map[k][d] * q[k];
    double v = c[4];
    for (int d = 3; d >= 0; --d) v = v * xi + c[d];
    double dv = 4.0 * c[4];
    for (int d = 3; d >= 1; --d) dv = dv * xi + (double)d * c[d];
    *val = v;
    if (der) *der = dv;
}

/* field accessor: f[(j*nx + i)*stride + off] */
typedef struct { const double* f; int stride, nx, ny; } s2_field;
static inline double s2_at(const s2_field* F, int i, int j) {
    i = ((i % F->nx) + F->nx) % F->nx;
    j = ((j % F->ny) + F->ny) % F->ny;
    return F->f[(size_t)(j * F->nx + i) * F->stride];
}

/* s2d1_cell_faces9 / s2d1_cell_faces9_wall (mod_S2D1Reconstruction.f90:409-498): per cell the
 * four faces (x-, x+, y-, y+) at the 3 Gauss nodes (value, normal and tangential derivatives in
 * cell units) and the 3x3 volume nodes [a = x node][b = y node]. */
static int s2_cell_faces9(const s2_field* F, int i, int j, double face[4][3], double dn[4][3], double dt[4][3],
                          double vol[3][3]) {
    double xv[5][2], xd[5][2], yv[5][2], yd[5][2], rows[5][3], q[5], fw[4], coef[4][5];
    const int ny = F->ny;
    if (!s2_near_wall(j, ny)) {
        for (int r = -2; r <= 2; ++r) {
            for (int s = -2; s <= 2; ++s) q[s + 2] = s2_at(F, i + s, j + r);
            if (!s2_weno_coef(q, fw, coef)) return 0;
            s2_eval(fw, coef, -0.5, &xv[r + 2][0], &xd[r + 2][0]);
            s2_eval(fw, coef, 0.5, &xv[r + 2][1], &xd[r + 2][1]);
            for (int a = 0; a < 3; ++a) s2_eval(fw, coef, s2_gnode[a], &rows[r + 2][a], NULL);
        }
        for (int r = -2; r <= 2; ++r) {
            for (int s = -2; s <= 2; ++s) q[s + 2] = s2_at(F, i + r, j + s);
            if (!s2_weno_coef(q, fw, coef)) return 0;
            s2_eval(fw, coef, -0.5, &yv[r + 2][0], &yd[r + 2][0]);
            s2_eval(fw, coef, 0.5, &yv[r + 2][1], &yd[r + 2][1]);
        }
        for (int s = 0; s < 2; ++s) {
            double a5[5], b5[5];
            for (int r = 0; r < 5; ++r) { a5[r] = xv[r][s]; b5[r] = xd[r][s]; }
            if (!s2_companion3(a5, b5, face[s], dt[s], dn[s])) return 0;
            for (int r = 0; r < 5; ++r) { a5[r] = yv[r][s]; b5[r] = yd[r][s]; }
            if (!s2_companion3(a5, b5, face[s + 2], dt[s + 2], dn[s + 2])) return 0;
        }
        for (int a = 0; a < 3; ++a) {
            double a5[5];
            for (int r = 0; r < 5; ++r) a5[r] = rows[r][a];
            if (!s2_weno_coef(a5, fw, coef)) return 0;
            for (int b = 0; b < 3; ++b) s2_eval(fw, coef, s2_gnode[b], &vol[a][b], NULL);
        }
    } else {
        const int first = s2_wall_first(j, ny);
        for (int r = 0; r < 5; ++r) {
            for (int s = -2; s <= 2; ++s) q[s + 2] = s2_at(F, i + s, first + r);
            if (!s2_weno_coef(q, fw, coef)) return 0;
            s2_eval(fw, coef, -0.5, &xv[r][0], &xd[r][0]);
            s2_eval(fw, coef, 0.5, &xv[r][1], &xd[r][1]);
            for (int a = 0; a < 3; ++a) s2_eval(fw, coef, s2_gnode[a], &rows[r][a], NULL);
        }
        for (int r = -2; r <= 2; ++r) {
            for (int s = 0; s < 5; ++s) q[s] = s2_at(F, i + r, first + s);
            s2_wall_eval(q, j, ny, -0.5, &yv[r + 2][0], &yd[r + 2][0]);
            s2_wall_eval(q, j, ny, 0.5, &yv[r + 2][1], &yd[r + 2][1]);
        }
        for (int s = 0; s < 2; ++s) {
            double a5[5], b5[5];
            for (int r = 0; r < 5; ++r) { a5[r] = xv[r][s]; b5[r] = xd[r][s]; }
            for (int a = 0; a < 3; ++a) {
                s2_wall_eval(a5, j, ny, s2_gnode[a], &face[s][a], &dt[s][a]);
                s2_wall_eval(b5, j, ny, s2_gnode[a], &dn[s][a], NULL);
            }
            for (int r = 0; r < 5; ++r) { a5[r] = yv[r][s]; b5[r] = yd[r][s]; }
            if (!s2_companion3(a5, b5, face[s + 2], dt[s + 2], dn[s + 2])) return 0;
        }
        for (int a = 0; a < 3; ++a) {
            double a5[5];
            for (int r = 0; r < 5; ++r) a5[r] = rows[r][a];
            for (int b = 0; b < 3; ++b) s2_wall_eval(a5, j, ny, s2_gnode[b], &vol[a][b], NULL);
        }
    }
    for (int s = 0; s < 4; ++s)
        for (int a = 0; a < 3; ++a) if (!(isfinite(face[s][a]) && isfinite(dn[s][a]) && isfinite(dt[s][a]))) return 0;
    return 1;
}

/* limit_cell_outputs (mod_S2D1.f90:315-345) */
static int s2_limit(double hm, double bm, double dx, double dy, double hf[4][3], double bf[4][3], double hn[4][3],
                    double ht[4][3], double bn[4][3], double bt[4][3], double hv[3][3], double bv[3][3]) {
    const double margin = 64.0 * DBL_EPSILON;
    double theta = 1.0;
    if (hm <= 0.0 || bm <= 0.0) {
        theta = 0.0;
    } else {
        for (int s = 0; s < 4; ++s)
            for (int a = 0; a < 3; ++a) {
                if (hf[s][a] < 0.0) { double den = hm - hf[s][a]; theta = fmin(theta, (1.0 - margin) * hm / den); }
                if (bf[s][a] < 0.0) { double den = bm - bf[s][a]; theta = fmin(theta, (1.0 - margin) * bm / den); }
            }
        for (int c = 0; c < 3; ++c)
            for (int a = 0; a < 3; ++a) {
                if (hv[a][c] < 0.0) { double den = hm - hv[a][c]; theta = fmin(theta, (1.0 - margin) * hm / den); }
                if (bv[a][c] < 0.0) { double den = bm - bv[a][c]; theta = fmin(theta, (1.0 - margin) * bm / den); }
            }
        theta = fmax(0.0, fmin(1.0, theta));
    }
    for (int s = 0; s < 4; ++s)
        for (int a = 0; a < 3; ++a) {
            hf[s][a] = hm + theta * (hf[s][a] - hm);
            bf[s][a] = bm + theta * (bf[s][a] - bm);
            hn[s][a] = theta * hn[s][a]; ht[s][a] = theta * ht[s][a];
            bn[s][a] = theta * bn[s][a]; bt[s][a] = theta * bt[s][a];
        }
    for (int s = 0; s < 4; ++s)
        for (int a = 0; a < 3; ++a) {
            double nd = s < 2 ? dx : dy, td = s < 2 ? dy : dx;
            hn[s][a] = hn[s][a] / nd; ht[s][a] = ht[s][a] / td;
            bn[s][a] = bn[s][a] / nd; bt[s][a] = bt[s][a] / td;
        }
    int ok = isfinite(theta);
    for (int s = 0; s < 4; ++s)
        for (int a = 0; a < 3; ++a)
            ok &= isfinite(hf[s][a]) && isfinite(bf[s][a]) && isfinite(hn[s][a]) && isfinite(ht[s][a]) &&
                  isfinite(bn[s][a]) && isfinite(bt[s][a]);
    return ok;
}

/* s2d1_side3 with wall_y (mod_S2D1Reconstruction.f90:320-354) for the macroscopic field; x face
 * (axis 0): cell i, row j; y face (axis 1): cell row j, column i.  side +-0.5 selects the face. */
static int s2_side3(const s2_field* F, int axis, int cell, int tangent, double side, double val[3], double dn[3],
                    double dt[3]) {
    const int ny = F->ny;
    int j = axis == 0 ? tangent : cell;
    if (s2_near_wall(j, ny)) {
        double f[4][3], n[4][3], t[4][3], vol[3][3];
        int slot;
        if (axis == 0) { if (!s2_cell_faces9(F, cell, j, f, n, t, vol)) return 0; slot = side < 0.0 ? 0 : 1; }
        else { if (!s2_cell_faces9(F, tangent, j, f, n, t, vol)) return 0; slot = side < 0.0 ? 2 : 3; }
        for (int a = 0; a < 3; ++a) { val[a] = f[slot][a]; dn[a] = n[slot][a]; dt[a] = t[slot][a]; }
        return 1;
    }
    double nv5[5], nd5[5], q[5], fw[4], coef[4][5];
    for (int r = -2; r <= 2; ++r) {
        for (int s = -2; s <= 2; ++s) q[s + 2] = axis == 0 ? s2_at(F, cell + s, tangent + r) : s2_at(F, tangent + r, cell + s);
        if (!s2_weno_coef(q, fw, coef)) return 0;
        s2_eval(fw, coef, side, &nv5[r + 2], &nd5[r + 2]);
    }
    return s2_companion3(nv5, nd5, val, dt, dn);
}

/* ---------------------------------------------------------------- discrete closure */

/* moment_2d (mod_CorrectedWF2DClosure.f90:25-43) */
static int s2_moment(int n, const double* h, const double* b, const double* u, const double* v, const double* w,
                     double m[4]) {
    m[0] = m[1] = m[2] = m[3] = 0.0;
    for (int k = 0; k < n; ++k) {
        m[0] = m[0] + w[k] * h[k];
        m[1] = m[1] + w[k] * u[k] * h[k];
        m[2] = m[2] + w[k] * v[k] * h[k];
        m[3] = m[3] + 0.5 * w[k] * ((u[k] * u[k] + v[k] * v[k]) * h[k] + b[k]);
    }
    return isfinite(m[0]) && isfinite(m[1]) && isfinite(m[2]) && isfinite(m[3]);
}

/* solve_dense_4x4 (mod_CorrectedWF2DClosure.f90:631-661): column-major a[col][row] as in Fortran
 * matrix(row,col); here m[r][c]. */
static int s2_solve4(const double M[4][4], const double rhs[4], double x[4]) {
    double a[4][4], b[4];
    for (int r = 0; r < 4; ++r) { for (int c = 0; c < 4; ++c) a[r][c] = M[r][c]; b[r] = rhs[r]; }
    x[0] = x[1] = x[2] = x[3] = 0.0;
    for (int p = 0; p < 3; ++p) {
        int row = p;
        double best = fabs(a[p][p]);
        for (int i = p + 1; i < 4; ++i) if (fabs(a[i][p]) > best) { best = fabs(a[i][p]); row = i; }
        if (fabs(a[row][p]) <= 100.0 * DBL_MIN || !isfinite(a[row][p])) return 0;
        if (row != p) {
            for (int j = 0; j < 4; ++j) { double t = a[p][j]; a[p][j] = a[row][j]; a[row][j] = t; }
            double t = b[p]; b[p] = b[row]; b[row] = t;
        }
        for (int i = p + 1; i < 4; ++i) {
            double f = a[i][p] / a[p][p];
            for (int j = p; j < 4; ++j) a[i][j] = a[i][j] - f * a[p][j];
            b[i] = b[i] - f * b[p];
        }
    }
    if (fabs(a[3][3]) <= 100.0 * DBL_MIN || !isfinite(a[3][3])) return 0;
    for (int i = 3; i >= 0; --i) {
        double pv = b[i];
        if (i < 3) {
            double s = 0.0;
            for (int j = i + 1; j < 4; ++j) s = s + a[i][j] * x[j];
            pv = pv - s;
        }
        x[i] = pv / a[i][i];
    }
    return isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]) && isfinite(x[3]);
}

/* primitive_from_conserved_2d (mod_CorrectedWF2DEquilibrium.f90:25-41): temp = T_native */
static int s2_prim_native(const double w[4], int ck, double* rho, double* u, double* v, double* temp) {
    if (!(isfinite(w[0]) && isfinite(w[1]) && isfinite(w[2]) && isfinite(w[3]))) return 0;
    *rho = w[0];
    if (!(w[0] > 0.0)) return 0;
    *u = w[1] / w[0];
    *v = w[2] / w[0];
    double kin = 0.5 * ((*u) * (*u) + (*v) * (*v));
    double ein = w[3] / w[0] - kin;
    *temp = 4.0 * ein / (double)(ck + 2);
    return isfinite(*u) && isfinite(*v) && isfinite(*temp) && *temp > 0.0;
}

/* primitive (mod_S2D1.f90:66-79): theta_gas = p/rho */
static int s2_primitive(const double w[4], int ck, double* rho, double* ux, double* vy, double* theta, double* p) {
    *rho = w[0];
    if (!(isfinite(w[0]) && isfinite(w[1]) && isfinite(w[2]) && isfinite(w[3])) || w[0] <= 0.0) return 0;
    *ux = w[1] / w[0];
    *vy = w[2] / w[0];
    double eint = w[3] - 0.5 * w[0] * ((*ux) * (*ux) + (*vy) * (*vy));
    if (eint <= 0.0) return 0;
    *p = (2.0 / (double)(ck + 2)) * eint;
    *theta = *p / w[0];
    return isfinite(*theta) && isfinite(*p) && *theta > 0.0;
}

/* heat (mod_S2D1.f90:81-95) */
static int s2_heat(const double w[4], int ck, int n, const double* h, const double* b, const double* u,
                   const double* v, const double* wt, double q[2]) {
    double rho, ux, vy, th, p;
    q[0] = q[1] = 0.0;
    if (!s2_primitive(w, ck, &rho, &ux, &vy, &th, &p)) return 0;
    for (int k = 0; k < n; ++k) {
        double cx = u[k] - ux, cy = v[k] - vy, c2 = cx * cx + cy * cy;
        q[0] = q[0] + 0.5 * wt[k] * cx * (c2 * h[k] + b[k]);
        q[1] = q[1] + 0.5 * wt[k] * cy * (c2 * h[k] + b[k]);
    }
    return isfinite(q[0]) && isfinite(q[1]);
}

/* s2_tau (mod_S2PhysicalGas.f90:9-20) with GetTau */
static int s2_tau(const uo_params* p, const double w[4], double* tau) {
    double pr = 2.0 / (double)(p->ck + 2) * (w[3] - 0.5 * (w[1] * w[1] + w[2] * w[2]) / w[0]);
    double prim[4] = {w[0], w[1] / w[0], w[2] / w[0], 0.5 * w[0] / pr};
    return get_tau(p, prim, tau) == 0;
}

/* one prepared closure point: the Newton-fitted discrete Maxwellian and its theta-derivatives
 * (ClosureFirstOrderContext, mod_CorrectedWF2DClosure.f90:14-21) */
typedef struct {
    double w[4], theta[4], jac[4][4];
    double *qh, *qb, *qht, *qbt;   /* [n], [n], [n][4], [n][4] */
} s2_closure;

/* q_state_first (mod_CorrectedWF2DClosure.f90:389-426) */
static int s2_q_state(const double th[4], int ck, int n, const double* u, const double* v, const double* wt,
                      double* qh, double* qb, double* qht, double* qbt, double jac[4][4]) {
    if (th[0] <= 0.0 || th[3] <= 0.0) return 0;
    const double r = th[0], tw = th[3], pi = acos(-1.0);
    int ok = 1;
    for (int k = 0; k < n; ++k) {
        double du = u[k] - th[1], dv = v[k] - th[2], c2 = du * du + dv * dv;
        qh[k] = r / (pi * tw) * exp(-c2 / tw);
        double ld[4] = {1.0 / r, 2.0 * du / tw, 2.0 * dv / tw, -1.0 / tw + c2 / (tw * tw)};
        for (int a = 0; a < 4; ++a) qht[(size_t)k * 4 + a] = qh[k] * ld[a];
        if (ck > 0) {
            qb[k] = 0.5 * (double)ck * tw * qh[k];
            ld[3] = ld[3] + 1.0 / tw;
            for (int a = 0; a < 4; ++a) qbt[(size_t)k * 4 + a] = qb[k] * ld[a];
        } else {
            qb[k] = 0.0;
            for (int a = 0; a < 4; ++a) qbt[(size_t)k * 4 + a] = 0.0;
        }
        ok &= isfinite(qh[k]) && isfinite(qb[k]);
    }
    for (int a = 0; a < 4; ++a) {
        double m[4] = {0, 0, 0, 0};
        for (int k = 0; k < n; ++k) {
            double hk = qht[(size_t)k * 4 + a], bk = qbt[(size_t)k * 4 + a];
            m[0] = m[0] + wt[k] * hk;
            m[1] = m[1] + wt[k] * u[k] * hk;
            m[2] = m[2] + wt[k] * v[k] * hk;
            m[3] = m[3] + 0.5 * wt[k] * ((u[k] * u[k] + v[k] * v[k]) * hk + bk);
        }
        for (int r2 = 0; r2 < 4; ++r2) { jac[r2][a] = m[r2]; ok &= isfinite(m[r2]); }
    }
    return ok;
}

static double s2_scaled_res(const double r[4], const double w[4]) {
    double s = 0.0;
    for (int m = 0; m < 4; ++m) s = fmax(s, fabs(r[m]) / fmax(1.0, fabs(w[m])));
    return s;
}

/* solve_q_first (mod_CorrectedWF2DClosure.f90:331-387).  scratch: 2n + 8n doubles */
static int s2_closure_prepare(s2_closure* C, const double w[4], int ck, int n, const double* u, const double* v,
                              const double* wt, double* scratch) {
    const double tol = 5.0e-13, floor_a = ldexp(1.0, -20);
    double rho, uu, vv, temp, res[4], nres[4], step[4], nth[4], njac[4][4];
    double *nqh = scratch, *nqb = scratch + n, *nqht = scratch + 2 * n, *nqbt = scratch + 6 * n;
    memcpy(C->w, w, sizeof C->w);
    if (!s2_prim_native(w, ck, &rho, &uu, &vv, &temp)) return 0;
    double th[4] = {rho, uu, vv, temp};
    memcpy(C->theta, th, sizeof th);
    if (!s2_q_state(C->theta, ck, n, u, v, wt, C->qh, C->qb, C->qht, C->qbt, C->jac)) return 0;
    if (!s2_moment(n, C->qh, C->qb, u, v, wt, res)) return 0;
    for (int m = 0; m < 4; ++m) res[m] = res[m] - w[m];
    double norm = s2_scaled_res(res, w);
    for (int it = 1; it <= 12; ++it) {
        if (norm <= tol) break;
        double mr[4] = {-res[0], -res[1], -res[2], -res[3]};
        if (!s2_solve4(C->jac, mr, step)) return 0;
        double alpha = 1.0;
        int accepted = 0;
        while (alpha >= floor_a) {
            for (int m = 0; m < 4; ++m) nth[m] = C->theta[m] + alpha * step[m];
            if (nth[0] > 0.0 && nth[3] > 0.0 && isfinite(nth[0]) && isfinite(nth[1]) && isfinite(nth[2]) &&
                isfinite(nth[3])) {
                if (s2_q_state(nth, ck, n, u, v, wt, nqh, nqb, nqht, nqbt, njac) && s2_moment(n, nqh, nqb, u, v, wt, nres)) {
                    for (int m = 0; m < 4; ++m) nres[m] = nres[m] - w[m];
                    double nn = s2_scaled_res(nres, w);
                    if (nn < norm || nn <= tol) accepted = 1;
                    if (accepted) {
                        memcpy(C->theta, nth, sizeof nth);
                        memcpy(C->qh, nqh, sizeof(double) * n);
                        memcpy(C->qb, nqb, sizeof(double) * n);
                        memcpy(C->qht, nqht, sizeof(double) * 4 * n);
                        memcpy(C->qbt, nqbt, sizeof(double) * 4 * n);
                        memcpy(C->jac, njac, sizeof njac);
                        memcpy(res, nres, sizeof nres);
                        norm = nn;
                    }
                }
                if (accepted) break;
            }
            alpha = 0.5 * alpha;
        }
        if (!accepted) return 0;
    }
    int ok = norm <= tol;
    for (int k = 0; k < n && ok; ++k) ok = isfinite(C->qh[k]) && isfinite(C->qb[k]) && C->qh[k] > 0.0 && C->qb[k] > 0.0;
    return ok;
}

/* closure_first_direction (mod_CorrectedWF2DClosure.f90:92-109): dq = sum_a q_theta_a * solve(jac, m) */
static int s2_direction(const s2_closure* C, int n, const double m[4], double* dh, double* db) {
    double td[4];
    for (int k = 0; k < n; ++k) { dh[k] = 0.0; db[k] = 0.0; }
    if (!s2_solve4(C->jac, m, td)) return 0;
    for (int a = 0; a < 4; ++a)
        for (int k = 0; k < n; ++k) {
            dh[k] = dh[k] + C->qht[(size_t)k * 4 + a] * td[a];
            db[k] = db[k] + C->qbt[(size_t)k * 4 + a] * td[a];
        }
    int ok = 1;
    for (int k = 0; k < n && ok; ++k) ok = isfinite(dh[k]) && isfinite(db[k]);
    return ok;
}

/* closure_first_project (mod_CorrectedWF2DClosure.f90:111-131): p = z - direction(moments(z)) */
static int s2_project(const s2_closure* C, int n, const double* u, const double* v, const double* wt, const double* zh,
                      const double* zb, double* ph, double* pb, double* ch, double* cb) {
    double m[4];
    if (!s2_moment(n, zh, zb, u, v, wt, m)) return 0;
    if (!s2_direction(C, n, m, ch, cb)) return 0;
    for (int k = 0; k < n; ++k) { ph[k] = zh[k] - ch[k]; pb[k] = zb[k] - cb[k]; }
    return 1;
}

/* m_direction_prepared (mod_S2D1.f90:163-178) */
static int s2_m_direction(const s2_closure* C, int n, const double* u, const double* v, const double* wt,
                          const double dw[4], double* dh, double* db) {
    double mom[4];
    if (!s2_direction(C, n, dw, dh, db)) return 0;
    if (!s2_moment(n, dh, db, u, v, wt, mom)) return 0;
    double mx = 0.0, sc = 1.0;
    for (int m = 0; m < 4; ++m) { mx = fmax(mx, fabs(mom[m] - dw[m])); sc = fmax(sc, fabs(dw[m])); }
    return mx / sc <= S2_GATE;
}

/* analytic_maxwellian_2d (mod_CorrectedWF2DEquilibrium.f90:43-65) */
static int s2_analytic_maxwell(const double w[4], int ck, int n, const double* u, const double* v, double* mh,
                               double* mb) {
    double rho, uu, vv, temp;
    if (!s2_prim_native(w, ck, &rho, &uu, &vv, &temp)) return 0;
    double lam = 1.0 / temp, pi = acos(-1.0);
    for (int k = 0; k < n; ++k) {
        double du = u[k] - uu, dv = v[k] - vv;
        double c2 = du * du + dv * dv;
        mh[k] = rho * lam / pi * exp(-lam * c2);
        mb[k] = 0.5 * (double)ck * temp * mh[k];
    }
    return 1;
}

/* make_mke_prepared (mod_S2D1.f90:111-151): the Shakhov directions K_x, K_y projected by the
 * closure, kappa = heat of K, and the moment gate.  t: 6n scratch doubles */
static int s2_make_mke(const uo_params* p, const s2_closure* C, const double w[4], int n, const double* u,
                       const double* v, const double* wt, double* mh, double* mb, double* kxh, double* kxb,
                       double* kyh, double* kyb, double kappa[2][2], double* t) {
    double rho, ux, vy, th, pp, mom[4], q[2];
    if (!s2_primitive(w, p->ck, &rho, &ux, &vy, &th, &pp)) return 0;
    memcpy(mh, C->qh, sizeof(double) * n);
    memcpy(mb, C->qb, sizeof(double) * n);
    double lam = 0.5 / th;
    double *rh = t, *rb = t + n, *ch = t + 2 * n, *cb = t + 3 * n;
    for (int dir = 0; dir < 2; ++dir) {
        for (int k = 0; k < n; ++k) {
            double cx = u[k] - ux, cy = v[k] - vy, c2 = cx * cx + cy * cy;
            double coeff = 0.8 * (1.0 - p->pr) * lam * lam / rho;
            double shh = 2.0 * lam * c2 - 4.0, shb = shh + 2.0 / (double)p->ck;
            double cd = dir == 0 ? cx : cy;
            rh[k] = coeff * cd * shh * mh[k];
            rb[k] = coeff * cd * shb * mb[k];
        }
        if (!s2_project(C, n, u, v, wt, rh, rb, dir == 0 ? kxh : kyh, dir == 0 ? kxb : kyb, ch, cb)) return 0;
    }
    if (!s2_heat(w, p->ck, n, kxh, kxb, u, v, wt, q)) return 0;
    kappa[0][0] = q[0]; kappa[1][0] = q[1];
    if (!s2_heat(w, p->ck, n, kyh, kyb, u, v, wt, q)) return 0;
    kappa[0][1] = q[0]; kappa[1][1] = q[1];
    if (!s2_moment(n, mh, mb, u, v, wt, mom)) return 0;
    double mx = 0.0, sc = 1.0;
    for (int m = 0; m < 4; ++m) { mx = fmax(mx, fabs(mom[m] - w[m])); sc = fmax(sc, fabs(w[m])); }
    double res = mx / sc;
    if (!s2_moment(n, kxh, kxb, u, v, wt, mom)) return 0;
    for (int m = 0; m < 4; ++m) res = fmax(res, fabs(mom[m]));
    if (!s2_moment(n, kyh, kyb, u, v, wt, mom)) return 0;
    for (int m = 0; m < 4; ++m) res = fmax(res, fabs(mom[m]));
    return res <= S2_GATE && isfinite(kappa[0][0]) && isfinite(kappa[0][1]) && isfinite(kappa[1][0]) &&
           isfinite(kappa[1][1]);
}

/* per-thread S2 scratch: closure arrays and work vectors.  Work vector layout (units of nvel):
 * [0, 32) node / wall-node work, [32, 42) closure Newton scratch, [42, 64) the caller's arrays. */
typedef struct {
    s2_closure C;
    double* buf;
} s2_scratch;

#define S2_NBUF 64
#define S2_CALLER 42
static s2_scratch* s2_scr(uo_ctx* c, int tid) { return (s2_scratch*)c->s2_scr + tid; }

/* ugks_node (mod_S2D1.f90:421-521) at one face Gauss node.  axis 0: x face (vn = u, vt = v);
 * axis 1: y face (vn = v, vt = u).  in: 12 arrays hl hr bl br hnl hnr htl htr bnl bnr btl btr.
 * coef (NULL: not wanted): the optional f0_h, f0_b, k_h, k_b outputs (:501-505), the leading and the
 * time coefficients of the node flux, 4 x nvel. */
static int s2_ugks_node(uo_ctx* c, int tid, int axis, double dt, const double* const in[12], const double mnl4[4],
                        const double mnr4[4], const double mt4[4], double* fh, double* fb, double fw[4], double* coef) {
    const uo_params* p = &c->p;
    int n = p->nvel;
    const double *u = c->u, *v = c->v, *wt = c->w;
    s2_scratch* S = s2_scr(c, tid);
    double* B = S->buf;
    double *f0h = B, *f0b = B + n, *fnh = B + 2 * n, *fnb = B + 3 * n, *fth = B + 4 * n, *ftb = B + 5 * n;
    double *mh = B + 6 * n, *mb = B + 7 * n, *kxh = B + 8 * n, *kxb = B + 9 * n, *kyh = B + 10 * n, *kyb = B + 11 * n;
    double *eah = B + 12 * n, *eab = B + 13 * n, *s0h = B + 14 * n, *s0b = B + 15 * n;
    double *mnlh = B + 16 * n, *mnlb = B + 17 * n, *mnrh = B + 18 * n, *mnrb = B + 19 * n;
    double *mth = B + 20 * n, *mtb = B + 21 * n, *mtmh = B + 22 * n, *mtmb = B + 23 * n;
    double *tmp = B + 24 * n, *nscr = B + 32 * n;
    const double *hl = in[0], *hr = in[1], *bl = in[2], *br = in[3], *hnl = in[4], *hnr = in[5];
    const double *htl = in[6], *htr = in[7], *bnl = in[8], *bnr = in[9], *btl = in[10], *btr = in[11];
    double w0[4], q0[2], wtime[4], kap[2][2], mt[5];
    for (int k = 0; k < n; ++k) {
        double vn = axis == 0 ? u[k] : v[k];
        if (vn >= 0.0) { f0h[k] = hl[k]; f0b[k] = bl[k]; fnh[k] = hnl[k]; fnb[k] = bnl[k]; fth[k] = htl[k]; ftb[k] = btl[k]; }
        else { f0h[k] = hr[k]; f0b[k] = br[k]; fnh[k] = hnr[k]; fnb[k] = bnr[k]; fth[k] = htr[k]; ftb[k] = btr[k]; }
    }
    if (!s2_moment(n, f0h, f0b, u, v, wt, w0)) return 0;
    if (!s2_closure_prepare(&S->C, w0, p->ck, n, u, v, wt, nscr)) return 0;
    if (!s2_make_mke(p, &S->C, w0, n, u, v, wt, mh, mb, kxh, kxb, kyh, kyb, kap, tmp)) return 0;
    if (!s2_analytic_maxwell(w0, p->ck, n, u, v, eah, eab)) return 0;
    for (int k = 0; k < n; ++k) { tmp[k] = f0h[k] - eah[k]; tmp[n + k] = f0b[k] - eab[k]; }
    if (!s2_heat(w0, p->ck, n, tmp, tmp + n, u, v, wt, q0)) return 0;
    for (int k = 0; k < n; ++k) {
        s0h[k] = mh[k] + kxh[k] * q0[0] + kyh[k] * q0[1];
        s0b[k] = mb[k] + kxb[k] * q0[0] + kyb[k] * q0[1];
    }
    if (!s2_m_direction(&S->C, n, u, v, wt, mnl4, mnlh, mnlb)) return 0;
    if (!s2_m_direction(&S->C, n, u, v, wt, mnr4, mnrh, mnrb)) return 0;
    if (!s2_m_direction(&S->C, n, u, v, wt, mt4, mth, mtb)) return 0;
    for (int k = 0; k < n; ++k) {
        double vn = axis == 0 ? u[k] : v[k], vt = axis == 0 ? v[k] : u[k];
        double a = vn >= 0.0 ? mnlh[k] : mnrh[k], bq = vn >= 0.0 ? mnlb[k] : mnrb[k];
        tmp[k] = vn * a + vt * mth[k];
        tmp[n + k] = vn * bq + vt * mtb[k];
    }
    if (!s2_moment(n, tmp, tmp + n, u, v, wt, wtime)) return 0;
    for (int m = 0; m < 4; ++m) wtime[m] = -wtime[m];
    if (!s2_m_direction(&S->C, n, u, v, wt, wtime, mtmh, mtmb)) return 0;
    double tau;
    if (!s2_tau(p, w0, &tau)) return 0;
    double ex = exp(-dt / tau);
    mt[3] = tau * (1.0 - ex);
    mt[4] = -tau * dt * ex + tau * mt[3];
    mt[0] = dt - mt[3];
    mt[1] = -tau * mt[0] + mt[4];
    mt[2] = 0.5 * dt * dt - tau * mt[0];
    int ok = 1;
    for (int k = 0; k < n; ++k) {
        double vn = axis == 0 ? u[k] : v[k], vt = axis == 0 ? v[k] : u[k];
        double sh, sb;
        if (vn >= 0.0) { sh = vn * mnlh[k] + vt * mth[k]; sb = vn * mnlb[k] + vt * mtb[k]; }
        else { sh = vn * mnrh[k] + vt * mth[k]; sb = vn * mnrb[k] + vt * mtb[k]; }
        double nh = vn >= 0.0 ? hnl[k] : hnr[k], nb = vn >= 0.0 ? bnl[k] : bnr[k];
        fh[k] = vn * (mt[0] * s0h[k] + mt[1] * sh + mt[2] * mtmh[k] + mt[3] * f0h[k] - mt[4] * (vn * nh + vt * fth[k]));
        fb[k] = vn * (mt[0] * s0b[k] + mt[1] * sb + mt[2] * mtmb[k] + mt[3] * f0b[k] - mt[4] * (vn * nb + vt * ftb[k]));
        if (coef) {
            coef[k] = vn * f0h[k];
            coef[n + k] = vn * f0b[k];
            coef[2 * n + k] = vn * ((s0h[k] - f0h[k]) / tau - vn * nh - vt * fth[k]);
            coef[3 * n + k] = vn * ((s0b[k] - f0b[k]) / tau - vn * nb - vt * ftb[k]);
        }
        ok &= isfinite(fh[k]) && isfinite(fb[k]);
    }
    if (!s2_moment(n, fh, fb, u, v, wt, fw)) return 0;
    return ok;
}

/* ---------------------------------------------------------------- the multiscale wall node */

/* MicroSlope / CalcMoment / Moment_uvxi / Moment_auvxi of mod_S2MultiscaleWall.f90:227-335 */
static void s2w_micro_slope(int ck, const double pr[4], const double sw[4], double a[4]) {
    a[3] = 4.0 * (pr[3] * pr[3]) / ((double)(ck + 2) * pr[0]) *
           (2.0 * sw[3] - 2.0 * pr[1] * sw[1] - 2.0 * pr[2] * sw[2] +
            sw[0] * (pr[1] * pr[1] + pr[2] * pr[2] - 0.5 * (double)(ck + 2) / pr[3]));
    a[2] = 2.0 * pr[3] / pr[0] * (sw[2] - pr[2] * sw[0]) - pr[2] * a[3];
    a[1] = 2.0 * pr[3] / pr[0] * (sw[1] - pr[1] * sw[0]) - pr[1] * a[3];
    a[0] = sw[0] / pr[0] - pr[1] * a[1] - pr[2] * a[2] -
           0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + 0.5 * (double)(ck + 2) / pr[3]) * a[3];
}

static void s2w_calc_moment(int ck, const double pr[4], double Mu[7], double Mv[6], double Mxi[3]) {
    double MuL[7], MuR[7];
    const double pi = 4.0 * atan(1.0);
    MuL[0] = 0.5 * erfc(-sqrt(pr[3]) * pr[1]);
    MuL[1] = pr[1] * MuL[0] + 0.5 * exp(-pr[3] * (pr[1] * pr[1])) / sqrt(pi * pr[3]);
    MuR[0] = 0.5 * erfc(sqrt(pr[3]) * pr[1]);
    MuR[1] = pr[1] * MuR[0] - 0.5 * exp(-pr[3] * (pr[1] * pr[1])) / sqrt(pi * pr[3]);
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

static void s2w_uvxi(const double Mu[7], const double Mv[6], const double Mxi[3], int al, int be, int de, double o[4]) {
    o[0] = Mu[al] * Mv[be] * Mxi[de / 2];
    o[1] = Mu[al + 1] * Mv[be] * Mxi[de / 2];
    o[2] = Mu[al] * Mv[be + 1] * Mxi[de / 2];
    o[3] = 0.5 * (Mu[al + 2] * Mv[be] * Mxi[de / 2] + Mu[al] * Mv[be + 2] * Mxi[de / 2] + Mu[al] * Mv[be] * Mxi[(de + 2) / 2]);
}

static void s2w_auvxi(const double a[4], const double Mu[7], const double Mv[6], const double Mxi[3], int al, int be,
                      double o[4]) {
    double t0[4], t1[4], t2[4], t3[4], t4[4], t5[4];
    s2w_uvxi(Mu, Mv, Mxi, al, be, 0, t0);
    s2w_uvxi(Mu, Mv, Mxi, al + 1, be, 0, t1);
    s2w_uvxi(Mu, Mv, Mxi, al, be + 1, 0, t2);
    s2w_uvxi(Mu, Mv, Mxi, al + 2, be, 0, t3);
    s2w_uvxi(Mu, Mv, Mxi, al, be + 2, 0, t4);
    s2w_uvxi(Mu, Mv, Mxi, al, be, 2, t5);
    for (int m = 0; m < 4; ++m)
        o[m] = a[0] * t0[m] + a[1] * t1[m] + a[2] * t2[m] + 0.5 * a[3] * t3[m] + 0.5 * a[3] * t4[m] + 0.5 * a[3] * t5[m];
}

/* s2w2_time_coefficients (mod_S2MultiscaleWall.f90:18-43): series for dt/tau < 0.1 */
static void s2w_time_coeffs(double dt, double tau, double mt[5]) {
    double x = dt / tau;
    if (x < 0.1) {
        double t = 1.0;
        for (int m = 0; m < 5; ++m) mt[m] = 0.0;
        for (int n = 1; n <= 24; ++n) {
            t = t * (-x) / (double)n;
            mt[3] = mt[3] - tau * t;
            if (n >= 2) {
                mt[0] = mt[0] + tau * t;
                mt[4] = mt[4] + tau * tau * (double)(n - 1) * t;
            }
            if (n >= 3) {
                mt[1] = mt[1] + tau * tau * (double)(n - 2) * t;
                mt[2] = mt[2] - tau * tau * t;
            }
        }
    } else {
        double ex = exp(-x);
        mt[3] = tau * (1.0 - ex);
        mt[4] = -tau * dt * ex + tau * mt[3];
        mt[0] = dt - mt[3];
        mt[1] = -tau * mt[0] + mt[4];
        mt[2] = 0.5 * (dt * dt) - tau * mt[0];
    }
}

/* s2w2_wall_node, S2PhysicalGas=1 (mod_S2MultiscaleWall.f90:45-184).  side -1: bottom wall below
 * the first row; +1: top wall above the last row.  hin, bin, hn, bn, ht, bt: the wall-side face
 * values, normal (y) and tangential (x) derivatives at this Gauss node. */
static int s2_wall_node(uo_ctx* c, int tid, int side, double dt, double dn, const double wcell[4], const double* hin,
                        const double* bin, const double* hn, const double* bn, const double* ht, const double* bt,
                        double ux, double theta, double* fh, double* fb, double fw[4], double* coef) {
    const uo_params* p = &c->p;
    int n = p->nvel, ck = p->ck;
    const double *u = c->u, *v = c->v, *wt = c->w;
    s2_scratch* S = s2_scr(c, tid);
    double* B = S->buf;
    double *mh = B, *mb = B + n, *wall = B + 2 * n, *wallb = B + 3 * n, *ginh = B + 4 * n, *ginb = B + 5 * n;
    double *corrh = B + 6 * n, *corrb = B + 7 * n, *nscr = B + 32 * n;
    fw[0] = fw[1] = fw[2] = fw[3] = 0.0;
    if (!(isfinite(wcell[0]) && isfinite(wcell[1]) && isfinite(wcell[2]) && isfinite(wcell[3])) || wcell[0] <= 0.0) return 0;
    double pp = (2.0 / (double)(ck + 2)) * (wcell[3] - 0.5 * (wcell[1] * wcell[1] + wcell[2] * wcell[2]) / wcell[0]);
    if (pp <= 0.0 || !isfinite(pp)) return 0;
    double lambda = 0.5 / theta;
    double prim_g[4] = {pp / theta, 0.0, -ux, lambda};
    double wc[4] = {wcell[0], wcell[2], -wcell[1], wcell[3]};
    double wg[4] = {prim_g[0], 0.0, -prim_g[0] * ux, prim_g[0] * ((double)(ck + 2) / (4.0 * lambda) + 0.5 * ux * ux)};
    double sw[4], an[4], at[4], atime[4], sw_t[4] = {0, 0, 0, 0};
    for (int m = 0; m < 4; ++m) sw[m] = (wg[m] - wc[m]) / ((double)side * 0.5 * dn);
    s2w_micro_slope(ck, prim_g, sw, an);
    for (int k = 0; k < n; ++k) {
        double vn = v[k], vt = -u[k], v2 = vn * vn + vt * vt;
        double e[4] = {-ht[k], -(vn * ht[k]), -(vt * ht[k]), -(0.5 * (v2 * ht[k] + bt[k]))};
        for (int m = 0; m < 4; ++m) sw_t[m] = sw_t[m] + wt[k] * e[m];
    }
    /* wall_equilibrium (:212-220): the discrete closure of (rho, rho ux, 0, rho((ck+2)theta/2 + ux^2/2)) */
    double weq[4] = {prim_g[0], prim_g[0] * ux, 0.0,
                     prim_g[0] * ((double)(ck + 2) * theta / 2.0 + ux * ux / 2.0)};
    if (!s2_closure_prepare(&S->C, weq, ck, n, u, v, wt, nscr)) return 0;
    memcpy(mh, S->C.qh, sizeof(double) * n);
    memcpy(mb, S->C.qb, sizeof(double) * n);
    for (int k = 0; k < n; ++k) { wall[k] = mh[k] / prim_g[0]; wallb[k] = mb[k] / prim_g[0]; }
    s2w_micro_slope(ck, prim_g, sw_t, at);
    double Mu[7], Mv[6], Mxi[3], m1[4], m2[4];
    s2w_calc_moment(ck, prim_g, Mu, Mv, Mxi);
    s2w_auvxi(an, Mu, Mv, Mxi, 1, 0, m1);
    s2w_auvxi(at, Mu, Mv, Mxi, 0, 1, m2);
    for (int m = 0; m < 4; ++m) sw[m] = -prim_g[0] * (m1[m] + m2[m]);
    s2w_micro_slope(ck, prim_g, sw, atime);
    double tau_wall, mt[5];
    double wgg[4] = {wg[0], -wg[2], wg[1], wg[3]};
    if (!s2_tau(p, wgg, &tau_wall)) return 0;
    s2w_time_coeffs(dt, tau_wall, mt);
    for (int k = 0; k < n; ++k) { corrh[k] = 0.0; corrb[k] = 0.0; }
    if (p->pr != 1.0) {
        double hl[2] = {0.0, 0.0};
        for (int k = 0; k < n; ++k) {
            double vn = v[k], vt = -u[k] + ux, v2 = vn * vn + vt * vt;
            hl[0] = hl[0] + 0.5 * wt[k] * vn * (v2 * hin[k] + bin[k]);
            hl[1] = hl[1] + 0.5 * wt[k] * vt * (v2 * hin[k] + bin[k]);
        }
        double coeff = 0.8 * (1.0 - p->pr) * lambda * lambda / prim_g[0];
        for (int k = 0; k < n; ++k) {
            double vn = v[k], vt = -u[k] + ux, v2 = vn * vn + vt * vt;
            double qdot = vn * hl[0] + vt * hl[1], shh = 2.0 * lambda * v2 - 4.0;
            corrh[k] = coeff * qdot * shh * mh[k];
            corrb[k] = coeff * qdot * (shh + 2.0 / (double)ck) * mb[k];
        }
    }
    double inc = 0.0, refl = 0.0;
    for (int k = 0; k < n; ++k) {
        double vn = v[k], vt = -u[k], v2 = vn * vn + vt * vt;
        double Han = (an[0] + an[1] * vn + an[2] * vt) * mh[k] + 0.5 * an[3] * (v2 * mh[k] + mb[k]);
        double Hatan = (at[0] + at[1] * vn + at[2] * vt) * mh[k] + 0.5 * at[3] * (v2 * mh[k] + mb[k]);
        double Hatime = (atime[0] + atime[1] * vn + atime[2] * vt) * mh[k] + 0.5 * atime[3] * (v2 * mh[k] + mb[k]);
        double Ban = (an[0] + an[1] * vn + an[2] * vt) * mb[k] + 0.5 * an[3] * (v2 * mb[k] + Mxi[2] * mh[k]);
        double Batan = (at[0] + at[1] * vn + at[2] * vt) * mb[k] + 0.5 * at[3] * (v2 * mb[k] + Mxi[2] * mh[k]);
        double Batime = (atime[0] + atime[1] * vn + atime[2] * vt) * mb[k] + 0.5 * atime[3] * (v2 * mb[k] + Mxi[2] * mh[k]);
        ginh[k] = mt[0] * mh[k] + mt[1] * (vn * Han + vt * Hatan) + mt[2] * Hatime + mt[3] * hin[k] -
                  mt[4] * (vn * hn[k] + u[k] * ht[k]);
        ginb[k] = mt[0] * mb[k] + mt[1] * (vn * Ban + vt * Batan) + mt[2] * Batime + mt[3] * bin[k] -
                  mt[4] * (vn * bn[k] + u[k] * bt[k]);
        ginh[k] = ginh[k] + mt[0] * corrh[k];
        ginb[k] = ginb[k] + mt[0] * corrb[k];
        if ((double)side * vn > 0.0) inc = inc + wt[k] * vn * ginh[k];
        else refl = refl + dt * wt[k] * vn * wall[k];
    }
    if (!isfinite(refl) || fabs(refl) <= DBL_MIN) return 0;
    double rhow = -inc / refl;
    if (!isfinite(rhow) || rhow <= 0.0) return 0;
    int ok = 1;
    for (int k = 0; k < n; ++k) {
        if ((double)side * v[k] > 0.0) { fh[k] = v[k] * ginh[k]; fb[k] = v[k] * ginb[k]; }
        else { fh[k] = dt * v[k] * rhow * wall[k]; fb[k] = dt * v[k] * rhow * wallb[k]; }
        double e[4] = {fh[k], u[k] * fh[k], v[k] * fh[k], 0.5 * ((u[k] * u[k] + v[k] * v[k]) * fh[k] + fb[k])};
        for (int m = 0; m < 4; ++m) fw[m] = fw[m] + wt[k] * e[m];
        ok &= isfinite(fh[k]) && isfinite(fb[k]);
    }
    if (coef) {   /* the optional f0/k outputs (:155-177): the leading and time coefficients of the wall flux */
        double a0 = 0.0, a1 = 0.0, den = 0.0;
        for (int k = 0; k < n; ++k) {
            const double qh = (mh[k] + corrh[k] - hin[k]) / tau_wall - v[k] * hn[k] - u[k] * ht[k];
            if ((double)side * v[k] > 0.0) { a0 = a0 + wt[k] * v[k] * hin[k]; a1 = a1 + wt[k] * v[k] * qh; }
            else den = den + wt[k] * v[k] * wall[k];
        }
        const double r0 = -a0 / den, r1 = -a1 / den;
        if (!(isfinite(r0) && isfinite(r1)) || r0 <= 0.0) return 0;
        double s0 = 0.0, s1 = 0.0;
        for (int k = 0; k < n; ++k) {
            if ((double)side * v[k] > 0.0) {
                coef[k] = v[k] * hin[k];
                coef[n + k] = v[k] * bin[k];
                coef[2 * n + k] = v[k] * ((mh[k] + corrh[k] - hin[k]) / tau_wall - v[k] * hn[k] - u[k] * ht[k]);
                coef[3 * n + k] = v[k] * ((mb[k] + corrb[k] - bin[k]) / tau_wall - v[k] * bn[k] - u[k] * bt[k]);
            } else {
                coef[k] = v[k] * r0 * wall[k];
                coef[n + k] = v[k] * r0 * wallb[k];
                coef[2 * n + k] = v[k] * r1 * wall[k];
                coef[3 * n + k] = v[k] * r1 * wallb[k];
            }
            s0 = s0 + wt[k] * coef[k];
            s1 = s1 + wt[k] * coef[2 * n + k];
        }
        if (fabs(s0) > S2_GATE || fabs(s1) > S2_GATE) return 0;
    }
    return ok && isfinite(fw[0]) && fabs(fw[0]) <= S2_GATE * fmax(1.0, fabs(inc));
}

/* s2w1_wall_node (mod_S2D1.f90:961-995): the time-integrated free-streaming diffuse wall of
 * FluxWall_type 0 at one tangential Gauss node -- incident half from the face values, reflected half
 * the continuous wall Maxwellian scaled to zero mass flux. */
static int s2w1_wall_node(const uo_ctx* c, int side, double dt, const double* hin, const double* bin, double ux,
                          double theta, double* fh, double* fb, double fw[4]) {
    const int n = c->p.nvel;
    const double *u = c->u, *v = c->v, *wt = c->w;
    const double lambda = 0.5 / theta;
    double incidence = 0.0, reflection = 0.0;
    for (int k = 0; k < n; ++k) {
        const double mh = lambda / PI_D * exp(-lambda * ((u[k] - ux) * (u[k] - ux) + v[k] * v[k]));
        if ((double)side * v[k] > 0.0) incidence = incidence + wt[k] * v[k] * hin[k];
        else reflection = reflection + wt[k] * v[k] * mh;
    }
    if (!(isfinite(reflection) && fabs(reflection) > DBL_MIN)) return 0;
    const double rho_w = -incidence / reflection;
    if (!(isfinite(rho_w) && rho_w > 0.0)) return 0;
    for (int k = 0; k < n; ++k) {
        if ((double)side * v[k] > 0.0) { fh[k] = dt * v[k] * hin[k]; fb[k] = dt * v[k] * bin[k]; }
        else {
            const double mh = lambda / PI_D * exp(-lambda * ((u[k] - ux) * (u[k] - ux) + v[k] * v[k]));
            fh[k] = dt * v[k] * rho_w * mh;
            fb[k] = (double)c->p.ck * theta * fh[k];
        }
    }
    if (!s2_moment(n, fh, fb, u, v, wt, fw)) return 0;
    return fabs(fw[0]) <= S2_GATE * fmax(1.0, dt * fabs(incidence));
}

/* s2w2_instantaneous_node, S2PhysicalGas = 1 (mod_S2MultiscaleWall.f90:187-227): the un-integrated
 * diffuse wall flux of W2R's shared predictor -- incident half from the face values, reflected half the
 * discrete closure of the unit-density wall state (wall_equilibrium, :231-238) scaled to zero mass flux. */
static int s2w2_inst_node(uo_ctx* c, int tid, int side, const double* hin, const double* bin, double ux, double theta,
                          double* fh, double* fb, double fw[4]) {
    const int n = c->p.nvel, ck = c->p.ck;
    const double *u = c->u, *v = c->v, *wt = c->w;
    s2_scratch* S = s2_scr(c, tid);
    double* nscr = S->buf + 32 * (size_t)n;
    double inc = 0.0, den = 0.0;
    fw[0] = fw[1] = fw[2] = fw[3] = 0.0;
    const double weq[4] = {1.0, ux, 0.0, (double)(ck + 2) * theta / 2.0 + ux * ux / 2.0};
    if (!s2_closure_prepare(&S->C, weq, ck, n, u, v, wt, nscr)) return 0;
    const double *wall = S->C.qh, *wallb = S->C.qb;
    for (int k = 0; k < n; ++k) {
        if ((double)side * v[k] > 0.0) inc = inc + wt[k] * v[k] * hin[k];
        else den = den + wt[k] * v[k] * wall[k];
    }
    const double rho = -inc / den;
    if (!(isfinite(rho) && rho > 0.0)) return 0;
    int ok = 1;
    for (int k = 0; k < n; ++k) {
        if ((double)side * v[k] > 0.0) { fh[k] = v[k] * hin[k]; fb[k] = v[k] * bin[k]; }
        else { fh[k] = v[k] * rho * wall[k]; fb[k] = v[k] * rho * wallb[k]; }
        const double e[4] = {fh[k], u[k] * fh[k], v[k] * fh[k], 0.5 * ((u[k] * u[k] + v[k] * v[k]) * fh[k] + fb[k])};
        for (int m = 0; m < 4; ++m) fw[m] = fw[m] + wt[k] * e[m];
        ok &= isfinite(fh[k]) && isfinite(fb[k]);
    }
    return ok && fabs(fw[0]) <= S2_GATE * fmax(1.0, fabs(inc));
}

/* ---------------------------------------------------------------- evolution pieces */

/* reconstruction cache of one (cell, velocity): [field 0..5 = h face, b face, h normal, h
 * tangential, b normal, b tangential][side][node] */
#define S2_REC 72
static inline double* s2_rec(uo_ctx* c, int cc, int k) { return c->s2_rec + ((size_t)cc * c->p.nvel + k) * S2_REC; }

typedef struct { uo_ctx* c; int* err; int coef; } s2_arg;

/* velocity-by-velocity tensor reconstruction and positivity limiting of every cell (compute_flux,
 * mod_S2D1.f90:713-746 with S2_VELOCITY_TILE; limit_cell_outputs) */
static void s2_recon_body(void* vp, int cc, int tid) {
    s2_arg* a = (s2_arg*)vp;
    uo_ctx* c = a->c;
    const uo_params* p = &c->p;
    int nx = p->nx, ny = p->ny, nv = p->nvel, i = cc % nx, j = cc / nx;
    (void)tid;
    for (int k = 0; k < nv; ++k) {
        s2_field Fh = {c->h + k, nv, nx, ny}, Fb = {c->b + k, nv, nx, ny};
        double hf[4][3], hn[4][3], ht[4][3], hv[3][3], bf[4][3], bn[4][3], bt[4][3], bv[3][3];
        if (!s2_cell_faces9(&Fh, i, j, hf, hn, ht, hv) || !s2_cell_faces9(&Fb, i, j, bf, bn, bt, bv)) { a->err[cc] = 422; return; }
        if (!s2_limit(c->h[(size_t)cc * nv + k], c->b[(size_t)cc * nv + k], p->dx, p->dy, hf, bf, hn, ht, bn, bt, hv, bv)) {
            a->err[cc] = 422;
            return;
        }
        double* r = s2_rec(c, cc, k);
        for (int s = 0; s < 4; ++s)
            for (int g = 0; g < 3; ++g) {
                r[0 * 12 + s * 3 + g] = hf[s][g];
                r[1 * 12 + s * 3 + g] = bf[s][g];
                r[2 * 12 + s * 3 + g] = hn[s][g];
                r[3 * 12 + s * 3 + g] = ht[s][g];
                r[4 * 12 + s * 3 + g] = bn[s][g];
                r[5 * 12 + s * 3 + g] = bt[s][g];
            }
    }
}

/* the right x face and top y face of one cell (compute_flux :757-878), plus the wall faces of the
 * first and last rows (:880-955).  Fluxes include dt, not the face length. */
static void s2_face_body(void* vp, int cc, int tid) {
    s2_arg* a = (s2_arg*)vp;
    uo_ctx* c = a->c;
    const uo_params* p = &c->p;
    int nx = p->nx, ny = p->ny, nv = p->nvel, i = cc % nx, j = cc / nx;
    double dt = c->dt;
    s2_scratch* S = s2_scr(c, tid);
    double* base = S->buf + S2_CALLER * (size_t)nv;
    double* arr[12];
    for (int t = 0; t < 12; ++t) arr[t] = base + (size_t)t * nv;
    double *fh = base + 12 * (size_t)nv, *fb = base + 13 * (size_t)nv;
    double* acc = c->s2_facc + (size_t)cc * 3 * (2 * nv + 4);   /* [right x, top y, bottom wall][h nv, b nv, w 4] */
    /* the leading / time coefficients of the same three faces, when a variant corrects the faces */
    double* coef = a->coef ? c->s2_coef + (size_t)cc * 3 * 4 * nv : NULL;
    if (coef) for (size_t k = 0; k < (size_t)3 * 4 * nv; ++k) coef[k] = 0.0;
    for (int axis = 0; axis < 2; ++axis) {
        double* ah = acc + (size_t)axis * (2 * nv + 4);
        double *ab = ah + nv, *aw = ah + 2 * nv;
        for (int k = 0; k < 2 * nv + 4; ++k) ah[k] = 0.0;
        if (axis == 1 && j == ny - 1) continue;   /* the top wall face is the wall node's */
        int ic = axis == 0 ? (i + 1) % nx : i, jc = axis == 0 ? j : j + 1;
        int cr = jc * nx + ic;
        int sl = axis == 0 ? 1 : 3, sr = axis == 0 ? 0 : 2;   /* left cell's side, right cell's side */
        double d_n = axis == 0 ? p->dx : p->dy, d_t = axis == 0 ? p->dy : p->dx;
        double mnl[4][3], mnr[4][3], mtg[4][3];
        for (int m = 0; m < 4; ++m) {
            s2_field Fw = {c->W + m, 4, nx, ny};
            double vl[3], vr[3], nl[3], nr[3], tl[3], tr[3];
            if (axis == 0) {
                if (!s2_side3(&Fw, 0, i, j, 0.5, vl, nl, tl) || !s2_side3(&Fw, 0, (i + 1) % nx, j, -0.5, vr, nr, tr)) { a->err[cc] = 422; return; }
            } else {
                if (!s2_side3(&Fw, 1, j, i, 0.5, vl, nl, tl) || !s2_side3(&Fw, 1, (j + 1) % ny, i, -0.5, vr, nr, tr)) { a->err[cc] = 422; return; }
            }
            for (int g = 0; g < 3; ++g) {
                mnl[m][g] = nl[g] / d_n;
                mnr[m][g] = nr[g] / d_n;
                mtg[m][g] = 0.5 * (tl[g] + tr[g]) / d_t;
            }
        }
        for (int g = 0; g < 3; ++g) {
            for (int k = 0; k < nv; ++k) {
                const double* L = s2_rec(c, cc, k);
                const double* R = s2_rec(c, cr, k);
                arr[0][k] = L[0 * 12 + sl * 3 + g]; arr[1][k] = R[0 * 12 + sr * 3 + g];
                arr[2][k] = L[1 * 12 + sl * 3 + g]; arr[3][k] = R[1 * 12 + sr * 3 + g];
                arr[4][k] = L[2 * 12 + sl * 3 + g]; arr[5][k] = R[2 * 12 + sr * 3 + g];
                arr[6][k] = L[3 * 12 + sl * 3 + g]; arr[7][k] = R[3 * 12 + sr * 3 + g];
                arr[8][k] = L[4 * 12 + sl * 3 + g]; arr[9][k] = R[4 * 12 + sr * 3 + g];
                arr[10][k] = L[5 * 12 + sl * 3 + g]; arr[11][k] = R[5 * 12 + sr * 3 + g];
            }
            double m4l[4], m4r[4], m4t[4], fw[4];
            for (int m = 0; m < 4; ++m) { m4l[m] = mnl[m][g]; m4r[m] = mnr[m][g]; m4t[m] = mtg[m][g]; }
            const double* const in[12] = {arr[0], arr[1], arr[2], arr[3], arr[4], arr[5],
                                          arr[6], arr[7], arr[8], arr[9], arr[10], arr[11]};
            double* cn = coef ? base + 14 * (size_t)nv : NULL;
            if (!s2_ugks_node(c, tid, axis, dt, in, m4l, m4r, m4t, fh, fb, fw, cn)) { a->err[cc] = 422; return; }
            for (int k = 0; k < nv; ++k) { ah[k] = ah[k] + s2_gw[g] * fh[k]; ab[k] = ab[k] + s2_gw[g] * fb[k]; }
            for (int m = 0; m < 4; ++m) aw[m] = aw[m] + s2_gw[g] * fw[m];
            if (cn) {   /* leading_x/y and time_x/y (compute_flux :833-836, :879-882) */
                double* cs = coef + (size_t)axis * 4 * nv;
                for (int k = 0; k < 4 * nv; ++k) cs[k] = cs[k] + s2_gw[g] * cn[k];
            }
        }
    }
    /* wall faces: bottom of row 0 (into acc slot 2), top of row ny-1 (into the y slot) */
    for (int t = 0; t < 2; ++t) {
        if (!((t == 0 && j == 0) || (t == 1 && j == ny - 1))) continue;
        double* ah = acc + (size_t)(t == 0 ? 2 : 1) * (2 * nv + 4);
        double *ab = ah + nv, *aw = ah + 2 * nv;
        if (t == 0) for (int k = 0; k < 2 * nv + 4; ++k) ah[k] = 0.0;
        int side = t == 0 ? 2 : 3;
        for (int g = 0; g < 3; ++g) {
            for (int k = 0; k < nv; ++k) {
                const double* L = s2_rec(c, cc, k);
                arr[0][k] = L[0 * 12 + side * 3 + g];   /* hin */
                arr[1][k] = L[1 * 12 + side * 3 + g];   /* bin */
                arr[2][k] = L[2 * 12 + side * 3 + g];   /* hn  */
                arr[3][k] = L[4 * 12 + side * 3 + g];   /* bn  */
                arr[4][k] = L[3 * 12 + side * 3 + g];   /* ht  */
                arr[5][k] = L[5 * 12 + side * 3 + g];   /* bt  */
            }
            double fw[4];
            double* cn = coef ? base + 14 * (size_t)nv : NULL;
            int ok = p->s2_kinetic_wall
                         ? s2w1_wall_node(c, t == 0 ? -1 : 1, dt, arr[0], arr[1], p->wall_ux[t], 0.5 * p->wall_tnative[t],
                                          fh, fb, fw)
                         : s2_wall_node(c, tid, t == 0 ? -1 : 1, dt, p->dy, c->W + cc * 4, arr[0], arr[1], arr[2], arr[3],
                                        arr[4], arr[5], p->wall_ux[t], 0.5 * p->wall_tnative[t], fh, fb, fw, cn);
            if (!ok) { a->err[cc] = 422; return; }
            for (int k = 0; k < nv; ++k) { ah[k] = ah[k] + s2_gw[g] * fh[k]; ab[k] = ab[k] + s2_gw[g] * fb[k]; }
            for (int m = 0; m < 4; ++m) aw[m] = aw[m] + s2_gw[g] * fw[m];
            if (cn && !p->s2_kinetic_wall) {   /* lower0/lowerK, and the top wall into leading_y/time_y (:905-940) */
                double* cs = coef + (size_t)(t == 0 ? 2 : 1) * 4 * nv;
                for (int k = 0; k < 4 * nv; ++k) cs[k] = cs[k] + s2_gw[g] * cn[k];
            }
        }
    }
}

/* s2d1_cell9 (mod_S2D1Reconstruction.f90:378-403): 3x3 Gauss values of one field in one cell */
static int s2_cell9(const s2_field* F, int i, int j, double val[3][3]) {
    if (s2_near_wall(j, F->ny)) {
        double f[4][3], n[4][3], t[4][3];
        return s2_cell_faces9(F, i, j, f, n, t, val);
    }
    double rows[5][3], q[5], fw[4], coef[4][5];
    for (int r = -2; r <= 2; ++r) {
        for (int s = -2; s <= 2; ++s) q[s + 2] = s2_at(F, i + s, j + r);
        if (!s2_weno_coef(q, fw, coef)) return 0;
        for (int a = 0; a < 3; ++a) s2_eval(fw, coef, s2_gnode[a], &rows[r + 2][a], NULL);
    }
    for (int a = 0; a < 3; ++a) {
        double a5[5];
        for (int r = 0; r < 5; ++r) a5[r] = rows[r][a];
        if (!s2_weno_coef(a5, fw, coef)) return 0;
        for (int b = 0; b < 3; ++b) s2_eval(fw, coef, s2_gnode[b], &val[a][b], NULL);
    }
    return 1;
}

/* build_targets (mod_S2D1.f90:1246-1300): Gauss-averaged M, K_x, K_y of every cell of the macro
 * field Wsrc, and kappa = heat(Wsrc, K) */
typedef struct {
    uo_ctx* c;
    int* err;
    const double* Wsrc;
    double *mh, *mb, *kxh, *kxb, *kyh, *kyb, *kappa;
} s2tg_arg;

static void s2_target_body(void* vp, int cc, int tid) {
    s2tg_arg* a = (s2tg_arg*)vp;
    uo_ctx* c = a->c;
    const uo_params* p = &c->p;
    const double* Wsrc = a->Wsrc;
    int nx = p->nx, ny = p->ny, nv = p->nvel, i = cc % nx, j = cc / nx;
    s2_scratch* S = s2_scr(c, tid);
    double* B = S->buf + S2_CALLER * (size_t)nv;
    double *tmh = B, *tmb = B + nv, *tkxh = B + 2 * nv, *tkxb = B + 3 * nv, *tkyh = B + 4 * nv, *tkyb = B + 5 * nv;
    double *tt = B + 6 * nv, *nscr = S->buf + 32 * (size_t)nv;
    double nodes[4][3][3], avg[4] = {0, 0, 0, 0}, kap[2][2];
    double *mh = a->mh + (size_t)cc * nv, *mb = a->mb + (size_t)cc * nv;
    double *kxh = a->kxh + (size_t)cc * nv, *kxb = a->kxb + (size_t)cc * nv;
    double *kyh = a->kyh + (size_t)cc * nv, *kyb = a->kyb + (size_t)cc * nv;
    for (int k = 0; k < nv; ++k) mh[k] = mb[k] = kxh[k] = kxb[k] = kyh[k] = kyb[k] = 0.0;
    for (int m = 0; m < 4; ++m) {
        s2_field Fw = {Wsrc + m, 4, nx, ny};
        if (!s2_cell9(&Fw, i, j, nodes[m])) { a->err[cc] = 420; return; }
    }
    for (int cq = 0; cq < 3; ++cq)
        for (int aq = 0; aq < 3; ++aq)
            for (int m = 0; m < 4; ++m) avg[m] = avg[m] + s2_gw[aq] * s2_gw[cq] * nodes[m][aq][cq];
    for (int cq = 0; cq < 3; ++cq)
        for (int aq = 0; aq < 3; ++aq) {
            double wq[4], wt2 = s2_gw[aq] * s2_gw[cq];
            for (int m = 0; m < 4; ++m) wq[m] = nodes[m][aq][cq] + Wsrc[cc * 4 + m] - avg[m];
            if (!s2_closure_prepare(&S->C, wq, p->ck, nv, c->u, c->v, c->w, nscr) ||
                !s2_make_mke(p, &S->C, wq, nv, c->u, c->v, c->w, tmh, tmb, tkxh, tkxb, tkyh, tkyb, kap, tt)) {
                a->err[cc] = 420;
                return;
            }
            for (int k = 0; k < nv; ++k) {
                mh[k] = mh[k] + wt2 * tmh[k]; mb[k] = mb[k] + wt2 * tmb[k];
                kxh[k] = kxh[k] + wt2 * tkxh[k]; kxb[k] = kxb[k] + wt2 * tkxb[k];
                kyh[k] = kyh[k] + wt2 * tkyh[k]; kyb[k] = kyb[k] + wt2 * tkyb[k];
            }
        }
    double q[2];
    if (!s2_heat(Wsrc + cc * 4, p->ck, nv, kxh, kxb, c->u, c->v, c->w, q)) { a->err[cc] = 420; return; }
    a->kappa[cc * 4 + 0] = q[0]; a->kappa[cc * 4 + 1] = q[1];   /* kappa(1:2, 1) */
    if (!s2_heat(Wsrc + cc * 4, p->ck, nv, kyh, kyb, c->u, c->v, c->w, q)) { a->err[cc] = 420; return; }
    a->kappa[cc * 4 + 2] = q[0]; a->kappa[cc * 4 + 3] = q[1];   /* kappa(1:2, 2) */
}

static int s2_first_error(uo_ctx* c) {
    for (int cc = 0; cc < c->nc; ++cc) if (c->cell_err[cc]) return c->cell_err[cc];
    return 0;
}

static void s2_alloc(uo_ctx* c) {
    if (c->s2_rec) return;
    int nv = c->p.nvel;
    size_t S = (size_t)c->nc * nv;
    c->s2_rec = (double*)calloc(S * S2_REC, sizeof(double));
    c->s2_mh = (double*)calloc(S, sizeof(double)); c->s2_mb = (double*)calloc(S, sizeof(double));
    c->s2_kxh = (double*)calloc(S, sizeof(double)); c->s2_kxb = (double*)calloc(S, sizeof(double));
    c->s2_kyh = (double*)calloc(S, sizeof(double)); c->s2_kyb = (double*)calloc(S, sizeof(double));
    c->s2_kappa = (double*)calloc((size_t)c->nc * 4, sizeof(double));
    c->lco_h = (double*)calloc(S, sizeof(double)); c->lco_b = (double*)calloc(S, sizeof(double));
    c->s2_facc = (double*)calloc((size_t)c->nc * 3 * (2 * nv + 4), sizeof(double));
    if (c->p.s2_face_time || c->p.s2_shared_predictor) c->s2_coef = (double*)calloc(S * 3 * 4, sizeof(double));
    s2_scratch* sc = (s2_scratch*)calloc((size_t)c->nthr, sizeof(s2_scratch));
    for (int t = 0; t < c->nthr; ++t) {
        sc[t].buf = (double*)calloc((size_t)S2_NBUF * nv, sizeof(double));
        sc[t].C.qh = (double*)calloc(nv, sizeof(double));
        sc[t].C.qb = (double*)calloc(nv, sizeof(double));
        sc[t].C.qht = (double*)calloc((size_t)4 * nv, sizeof(double));
        sc[t].C.qbt = (double*)calloc((size_t)4 * nv, sizeof(double));
    }
    c->s2_scr = sc;
    s2_init_maps();
}

static void s2_free(uo_ctx* c) {
    if (!c->s2_rec) return;
    double* ptrs[] = {c->s2_rec, c->s2_mh, c->s2_mb, c->s2_kxh, c->s2_kxb, c->s2_kyh, c->s2_kyb, c->s2_kappa,
                      c->lco_h, c->lco_b, c->s2_facc, c->s2_coef, c->s2_facc0, c->v_inst};
    for (size_t q = 0; q < sizeof ptrs / sizeof ptrs[0]; ++q) free(ptrs[q]);
    s2_scratch* sc = (s2_scratch*)c->s2_scr;
    for (int t = 0; t < c->nthr; ++t) { free(sc[t].buf); free(sc[t].C.qh); free(sc[t].C.qb); free(sc[t].C.qht); free(sc[t].C.qbt); }
    free(sc);
}

/* S2NativeEvolution (mod_S2NativeAdapter.f90:469-490 and CartesianEvolution,
 * mod_S2CartesianMPI.f90:182-234): rebuild the volume targets of W when asked (HighOrderImplicit
 * invalidates them every call, :479; S2CN2 only when they are not ready, :480-484), reconstruct,
 * evaluate every face, and publish the face fluxes times the face length into the face arrays
 * ComputeResidual reads. */
static void s2_publish(uo_ctx* c);
static int s2_evaluate(uo_ctx* c, double dt, int coef);
static int s2_evolution_core(uo_ctx* c, double dt, int rebuild_targets) {
    int nthr = g_threads < c->nthr ? g_threads : c->nthr;
    s2_alloc(c);
    memset(c->cell_err, 0, sizeof(int) * c->nc);
    if (rebuild_targets) {
        s2tg_arg t = {c, c->cell_err, c->W, c->s2_mh, c->s2_mb, c->s2_kxh, c->s2_kxb, c->s2_kyh, c->s2_kyb, c->s2_kappa};
        par_for(c->nc, s2_target_body, &t, nthr);
        int e = s2_first_error(c);
        if (e) return e;
    }
    int e = s2_evaluate(c, dt, 0);
    if (e) return e;
    s2_publish(c);
    return 0;
}

/* compute_flux (mod_S2D1.f90:632-959) of the current state into the face accumulators: the
 * reconstruction, every interior face and the walls; with coef, also the leading and time coefficients
 * of every face (its optional leading_* / time_* / lower0* / lowerK* outputs) */
static int s2_evaluate(uo_ctx* c, double dt, int coef) {
    int nthr = g_threads < c->nthr ? g_threads : c->nthr;
    s2_alloc(c);
    c->dt = dt;
    memset(c->cell_err, 0, sizeof(int) * c->nc);
    s2_arg a = {c, c->cell_err, coef};
    int e;
    par_for(c->nc, s2_recon_body, &a, nthr);
    if ((e = s2_first_error(c))) return e;
    par_for(c->nc, s2_face_body, &a, nthr);
    return s2_first_error(c);
}

/* the face accumulators into the face arrays ComputeResidual reads, times the face lengths
 * (S2NativeEvolution's map, mod_S2NativeAdapter.f90:545-594) */
static void s2_publish(uo_ctx* c) {
    const uo_params* p = &c->p;
    int nx = p->nx, ny = p->ny, nv = p->nvel;
    const size_t st = 2 * (size_t)nv + 4;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            int cc = j * nx + i;
            const double* xr = c->s2_facc + (size_t)cc * 3 * st;
            const double* yt = xr + st;
            int fi = (i + 1) % nx;   /* face between cells i and i+1 */
            double* Fh = c->fxh + ((size_t)j * nx + fi) * nv;
            double* Fb = c->fxb + ((size_t)j * nx + fi) * nv;
            for (int k = 0; k < nv; ++k) { Fh[k] = xr[k] * p->dy; Fb[k] = xr[nv + k] * p->dy; }
            for (int m = 0; m < 4; ++m) c->fxw[((size_t)j * nx + fi) * 4 + m] = xr[2 * nv + m] * p->dy;
            size_t oy = ((size_t)(j + 1) * nx + i);
            for (int k = 0; k < nv; ++k) {
                c->fyLh[oy * nv + k] = c->fyRh[oy * nv + k] = yt[k] * p->dx;
                c->fyLb[oy * nv + k] = c->fyRb[oy * nv + k] = yt[nv + k] * p->dx;
            }
            for (int m = 0; m < 4; ++m) c->fyLw[oy * 4 + m] = c->fyRw[oy * 4 + m] = yt[2 * nv + m] * p->dx;
            if (j == 0) {
                const double* lw = xr + 2 * st;
                for (int k = 0; k < nv; ++k) {
                    c->fyLh[(size_t)i * nv + k] = c->fyRh[(size_t)i * nv + k] = lw[k] * p->dx;
                    c->fyLb[(size_t)i * nv + k] = c->fyRb[(size_t)i * nv + k] = lw[nv + k] * p->dx;
                }
                for (int m = 0; m < 4; ++m) c->fyLw[(size_t)i * 4 + m] = c->fyRw[(size_t)i * 4 + m] = lw[2 * nv + m] * p->dx;
            }
        }
}

int uo_s2_evolution(uo_ctx* c, double dt) { return s2_evolution_core(c, dt, 1); }

/* ComputeResidual + AssembleSteadyRateResiduals for the S2 path (mod_Residual.f90:17-132, IsS2CN2
 * branch) and S2NativePhysicalCollision (mod_S2NativeAdapter.f90:735-759): residuals from the
 * face arrays, rates without the streaming projection (a moment gate instead), and the physical
 * collision C_hi = (M + K_x q + K_y q - h) / tau with q = heat(h - M), tau = s2_tau(W). */
typedef struct { uo_ctx* c; double dt; int rates_only; } s2res_arg;

static void s2_residual_body(void* vp, int cc, int tid) {
    s2res_arg* a = (s2res_arg*)vp;
    uo_ctx* c = a->c;
    const uo_params* p = &c->p;
    int nx = p->nx, nv = p->nvel;
    double dt = a->dt, dti = 1.0 / dt, area_inv = 1.0 / c->area;
    int j = cc / nx, i = cc % nx, e = 0;
    double** T = scratch_t(c, tid);
    if (!a->rates_only) {
        const double *vl = c->fxw + ((size_t)j * nx + i) * 4, *vr = c->fxw + ((size_t)j * nx + (i + 1) % nx) * 4;
        const double *hl = c->fyLw + ((size_t)j * nx + i) * 4, *hr = c->fyRw + ((size_t)(j + 1) * nx + i) * 4;
        for (int m = 0; m < 4; ++m) c->res_w[cc * 4 + m] = (vl[m] - vr[m] + hl[m] - hr[m]) / c->area;
        const double *vlh = c->fxh + ((size_t)j * nx + i) * nv, *vrh = c->fxh + ((size_t)j * nx + (i + 1) % nx) * nv;
        const double *vlb = c->fxb + ((size_t)j * nx + i) * nv, *vrb = c->fxb + ((size_t)j * nx + (i + 1) % nx) * nv;
        const double *hlh = c->fyLh + ((size_t)j * nx + i) * nv, *hrh = c->fyRh + ((size_t)(j + 1) * nx + i) * nv;
        const double *hlb = c->fyLb + ((size_t)j * nx + i) * nv, *hrb = c->fyRb + ((size_t)(j + 1) * nx + i) * nv;
        for (int k = 0; k < nv; ++k) {
            c->res_h[(size_t)cc * nv + k] = (vlh[k] - vrh[k] + hlh[k] - hrh[k]) * area_inv;
            c->res_b[(size_t)cc * nv + k] = (vlb[k] - vrb[k] + hlb[k] - hrb[k]) * area_inv;
        }
    }
    for (int m = 0; m < 4; ++m) c->rate_w[cc * 4 + m] = c->res_w[cc * 4 + m] * dti;
    for (int k = 0; k < nv; ++k) {
        c->stream_h[(size_t)cc * nv + k] = c->res_h[(size_t)cc * nv + k] * dti;
        c->stream_b[(size_t)cc * nv + k] = c->res_b[(size_t)cc * nv + k] * dti;
    }
    const double *W = c->W + cc * 4, *h = c->h + (size_t)cc * nv, *b = c->b + (size_t)cc * nv;
    const double *mh = c->s2_mh + (size_t)cc * nv, *mb = c->s2_mb + (size_t)cc * nv;
    const double *kxh = c->s2_kxh + (size_t)cc * nv, *kxb = c->s2_kxb + (size_t)cc * nv;
    const double *kyh = c->s2_kyh + (size_t)cc * nv, *kyb = c->s2_kyb + (size_t)cc * nv;
    double q[2], tau, mom[4];
    for (int k = 0; k < nv; ++k) { T[0][k] = h[k] - mh[k]; T[1][k] = b[k] - mb[k]; }
    if (!s2_heat(W, p->ck, nv, T[0], T[1], c->u, c->v, c->w, q)) e = 443;
    if (!e && !s2_tau(p, W, &tau)) e = 443;
    if (!e) {
        double *eh = c->peq_h + (size_t)cc * nv, *eb = c->peq_b + (size_t)cc * nv;
        double *ch = c->pcol_h + (size_t)cc * nv, *cb = c->pcol_b + (size_t)cc * nv;
        for (int k = 0; k < nv; ++k) {
            eh[k] = mh[k] + kxh[k] * q[0] + kyh[k] * q[1];
            eb[k] = mb[k] + kxb[k] * q[0] + kyb[k] * q[1];
            ch[k] = (eh[k] - h[k]) / tau;
            cb[k] = (eb[k] - b[k]) / tau;
        }
        moment_conserved(nv, ch, cb, c->u, c->v, c->w, mom);
        double mx = 0.0, sc = 1.0;
        for (int m = 0; m < 4; ++m) { mx = fmax(mx, fabs(mom[m])); sc = fmax(sc, fabs(W[m])); }
        if (tau * mx / sc > S2_GATE) e = 444;
        /* AssembleSteadyRateResiduals' IsS2CN2 gate: the stream moments equal rate_w */
        moment_conserved(nv, c->stream_h + (size_t)cc * nv, c->stream_b + (size_t)cc * nv, c->u, c->v, c->w, mom);
        double rx = 0.0, rs = 1.0;
        for (int m = 0; m < 4; ++m) { rx = fmax(rx, fabs(mom[m] - c->rate_w[cc * 4 + m])); rs = fmax(rs, fabs(c->rate_w[cc * 4 + m])); }
        if (!e && !(rx / rs <= S2_GATE)) e = 444;
    }
    c->cell_err[cc] = e;
}

int uo_s2_compute_residual(uo_ctx* c, double dt, int rates_only) {
    s2res_arg a = {c, dt, rates_only};
    par_for(c->nc, s2_residual_body, &a, g_threads < c->nthr ? g_threads : c->nthr);
    return s2_first_error(c);
}

/* S2NativeInitializeState(native_state=.true., cold_start=.true.) (mod_S2NativeAdapter.f90:192-445):
 * h, b of every cell become the discrete closure Maxwellian of its W (make_mke). */
typedef struct { uo_ctx* c; } s2init_arg;
static void s2_init_body(void* vp, int cc, int tid) {
    uo_ctx* c = ((s2init_arg*)vp)->c;
    const uo_params* p = &c->p;
    int nv = p->nvel;
    s2_scratch* S = s2_scr(c, tid);
    double* B = S->buf + S2_CALLER * (size_t)nv;
    double kap[2][2];
    c->cell_err[cc] = 0;
    if (!s2_closure_prepare(&S->C, c->W + cc * 4, p->ck, nv, c->u, c->v, c->w, S->buf + 32 * (size_t)nv) ||
        !s2_make_mke(p, &S->C, c->W + cc * 4, nv, c->u, c->v, c->w, c->h + (size_t)cc * nv, c->b + (size_t)cc * nv,
                     B, B + nv, B + 2 * nv, B + 3 * nv, kap, B + 4 * nv))
        c->cell_err[cc] = 413;
}

int uo_s2_init_state(uo_ctx* c) {
    s2_alloc(c);
    s2init_arg a = {c};
    par_for(c->nc, s2_init_body, &a, g_threads < c->nthr ? g_threads : c->nthr);
    return s2_first_error(c);
}

/* ---------------------------------------------------------------- S2CN2 explicit step */

static void cn_alloc(uo_ctx* c) {
    if (c->cn_wn) return;
    size_t S = (size_t)c->nc * c->p.nvel;
    c->cn_mh = (double*)calloc(S, sizeof(double)); c->cn_mb = (double*)calloc(S, sizeof(double));
    c->cn_kxh = (double*)calloc(S, sizeof(double)); c->cn_kxb = (double*)calloc(S, sizeof(double));
    c->cn_kyh = (double*)calloc(S, sizeof(double)); c->cn_kyb = (double*)calloc(S, sizeof(double));
    c->cn_kappa = (double*)calloc((size_t)c->nc * 4, sizeof(double));
    c->cn_wn = (double*)calloc((size_t)c->nc * 4, sizeof(double));
    c->cn_hs = (double*)calloc(S, sizeof(double)); c->cn_bs = (double*)calloc(S, sizeof(double));
    c->cn_hn = (double*)calloc(S, sizeof(double)); c->cn_bn = (double*)calloc(S, sizeof(double));
    c->cn_cell = (double*)calloc((size_t)c->nc * UO_CN_CELL, sizeof(double));
}

static void cn_free(uo_ctx* c) {
    if (!c->cn_wn) return;
    double* ptrs[] = {c->cn_mh, c->cn_mb, c->cn_kxh, c->cn_kxb, c->cn_kyh, c->cn_kyb, c->cn_kappa,
                      c->cn_wn, c->cn_hs, c->cn_bs, c->cn_hn, c->cn_bn, c->cn_cell};
    for (size_t q = 0; q < sizeof ptrs / sizeof ptrs[0]; ++q) free(ptrs[q]);
}

/* the ledger of S2NativeInitializeState (mod_S2NativeAdapter.f90:323-349): total0 = sum of W over
 * the cells, an empty wall balance, targets not yet built */
int uo_s2cn2_init(uo_ctx* c) {
    s2_alloc(c);
    cn_alloc(c);
    for (int m = 0; m < 4; ++m) {
        double t = 0.0;
        for (int cc = 0; cc < c->nc; ++cc) t = t + c->W[cc * 4 + m];
        c->cn_total0[m] = t;
        c->cn_balance[m] = 0.0;
    }
    c->s2_ready = 0;
    return 0;
}

/* advance_step's per-cell Crank-Nicolson collision (mod_S2D1.f90:1355-1421, S2PhysicalGas=1):
 * beta = dt / (2 tau), the old-state Shakhov correction from q_old = heat(w, h - M), the 2x2 solve
 * for the new heat flux and h_new = (rh + beta eq) / (1 + beta); the cnres / mmerr gates. */
typedef struct { uo_ctx* c; double dt; } cn_arg;

static void s2_cn_body(void* vp, int cc, int tid) {
    cn_arg* a = (cn_arg*)vp;
    uo_ctx* c = a->c;
    const uo_params* p = &c->p;
    const int nv = p->nvel;
    const double dt = a->dt;
    const size_t o = (size_t)cc * nv;
    const double *w = c->W + cc * 4, *wn = c->cn_wn + cc * 4;
    const double *h = c->h + o, *b = c->b + o, *hs = c->cn_hs + o, *bs = c->cn_bs + o;
    const double *mh = c->s2_mh + o, *mb = c->s2_mb + o, *kxh = c->s2_kxh + o, *kxb = c->s2_kxb + o;
    const double *kyh = c->s2_kyh + o, *kyb = c->s2_kyb + o;
    const double *mhn = c->cn_mh + o, *mbn = c->cn_mb + o, *kxhn = c->cn_kxh + o, *kxbn = c->cn_kxb + o;
    const double *kyhn = c->cn_kyh + o, *kybn = c->cn_kyb + o, *kap = c->cn_kappa + cc * 4;
    double *hn = c->cn_hn + o, *bn = c->cn_bn + o, *d = c->cn_cell + (size_t)cc * UO_CN_CELL;
    double** T = scratch_t(c, tid);
    double *rh = T[0], *rb = T[1], *eqh = T[2], *eqb = T[3], *th = T[4], *tb = T[5];
    double tau_o, tau_n, rold[2], rhs[2], qtmp[2], rnew[2], rhat[2], mom[4];
    c->cell_err[cc] = 0;
    if (!s2_tau(p, w, &tau_o) || !s2_tau(p, wn, &tau_n)) { c->cell_err[cc] = 104; return; }
    const double beta_old = dt / (2.0 * tau_o), beta = dt / (2.0 * tau_n);
    d[0] = fmax(2.0 * beta_old, 2.0 * beta);
    for (int k = 0; k < nv; ++k) { th[k] = h[k] - mh[k]; tb[k] = b[k] - mb[k]; }
    if (!s2_heat(w, p->ck, nv, th, tb, c->u, c->v, c->w, rold)) { c->cell_err[cc] = 445; return; }
    for (int k = 0; k < nv; ++k) {
        rh[k] = hs[k] + beta_old * (mh[k] + kxh[k] * rold[0] + kyh[k] * rold[1] - h[k]);
        rb[k] = bs[k] + beta_old * (mb[k] + kxb[k] * rold[0] + kyb[k] * rold[1] - b[k]);
    }
    if (!s2_heat(wn, p->ck, nv, rh, rb, c->u, c->v, c->w, rhs) ||
        !s2_heat(wn, p->ck, nv, mhn, mbn, c->u, c->v, c->w, qtmp)) { c->cell_err[cc] = 445; return; }
    rhs[0] = rhs[0] - qtmp[0];
    rhs[1] = rhs[1] - qtmp[1];
    /* a22 = -beta kappa; a22(1,1), a22(2,2) += 1 + beta; kappa(r, col) = kap[2 col + r] */
    double a11 = -beta * kap[0], a21 = -beta * kap[1], a12 = -beta * kap[2], a22 = -beta * kap[3];
    a11 = a11 + 1.0 + beta;
    a22 = a22 + 1.0 + beta;
    const double det = a11 * a22 - a12 * a21;
    if (!isfinite(det) || det <= 0.0) { c->cell_err[cc] = 445; return; }
    rnew[0] = (rhs[0] * a22 - a12 * rhs[1]) / det;
    rnew[1] = (a11 * rhs[1] - rhs[0] * a21) / det;
    double scale = 1.0, cres = 0.0;
    for (int k = 0; k < nv; ++k) {
        eqh[k] = mhn[k] + kxhn[k] * rnew[0] + kyhn[k] * rnew[1];
        eqb[k] = mbn[k] + kxbn[k] * rnew[0] + kybn[k] * rnew[1];
        hn[k] = (rh[k] + beta * eqh[k]) / (1.0 + beta);
        bn[k] = (rb[k] + beta * eqb[k]) / (1.0 + beta);
    }
    /* scale = max(1, max|rh|, max|rb|, max|hn|, max|bn|), in the Fortran argument order */
    double mrh = 0.0, mrb = 0.0, mhn_ = 0.0, mbn_ = 0.0, erh = 0.0, erb = 0.0;
    for (int k = 0; k < nv; ++k) {
        mrh = fmax(mrh, fabs(rh[k])); mrb = fmax(mrb, fabs(rb[k]));
        mhn_ = fmax(mhn_, fabs(hn[k])); mbn_ = fmax(mbn_, fabs(bn[k]));
        erh = fmax(erh, fabs((1.0 + beta) * hn[k] - rh[k] - beta * eqh[k]));
        erb = fmax(erb, fabs((1.0 + beta) * bn[k] - rb[k] - beta * eqb[k]));
    }
    scale = fmax(fmax(fmax(fmax(1.0, mrh), mrb), mhn_), mbn_);
    cres = fmax(erh, erb) / scale;
    for (int k = 0; k < nv; ++k) { th[k] = hn[k] - mhn[k]; tb[k] = bn[k] - mbn[k]; }
    if (!s2_heat(wn, p->ck, nv, th, tb, c->u, c->v, c->w, rhat)) { c->cell_err[cc] = 445; return; }
    cres = fmax(cres, fmax(fabs(rhat[0] - rnew[0]), fabs(rhat[1] - rnew[1])) /
                          fmax(fmax(1.0, fmax(fabs(rhat[0]), fabs(rhat[1]))), fmax(fabs(rnew[0]), fabs(rnew[1]))));
    if (!s2_moment(nv, hn, bn, c->u, c->v, c->w, mom)) { c->cell_err[cc] = 445; return; }
    double mx = 0.0, sc = 1.0;
    for (int m = 0; m < 4; ++m) { mx = fmax(mx, fabs(mom[m] - wn[m])); sc = fmax(sc, fabs(wn[m])); }
    d[1] = cres;
    d[2] = mx / sc;
    double lo_h = INFINITY, hi_h = -INFINITY, lo_b = INFINITY, hi_b = -INFINITY;
    for (int k = 0; k < nv; ++k) {
        lo_h = fmin(lo_h, hn[k]); hi_h = fmax(hi_h, hn[k]);
        lo_b = fmin(lo_b, bn[k]); hi_b = fmax(hi_b, bn[k]);
    }
    d[3] = lo_h; d[4] = hi_h; d[5] = lo_b; d[6] = hi_b;
}

/* ---------------------------------------------------------------- research wall variants */

static const double s2_tau0 = 0.1;   /* the frozen relaxation time of W2R's predictor, mod_S2D1.f90:32 */

/* the option checks of mod_ImportPara.f90:455-471 and :516-533 for the S2CN2 Couette case; 200 is the
 * reference's AbortInvalidImplicitOption code */
static int s2_variant_check(const uo_params* p) {
    if (p->s2_time_centered && !p->s2_kinetic_wall) return 200;        /* W2 type1 requires centered=0 */
    if (p->s2_face_time && !p->s2_time_centered) return 200;          /* W1D requires the W1T midpoint wall */
    if (p->s2_shared_predictor &&
        (p->s2_kinetic_wall || p->ck != 1 || p->pr != 1.0 || p->s2_time_centered || p->s2_face_time))
        return 200;                                                    /* W2R: flat type1 BGK only */
    return 0;
}

static void s2v_alloc(uo_ctx* c) {
    const size_t nc = (size_t)c->nc, nv = (size_t)c->p.nvel;
    if (!c->s2_facc0) c->s2_facc0 = (double*)calloc(nc * 3 * (2 * nv + 4), sizeof(double));
    if (!c->v_inst) c->v_inst = (double*)calloc(nc * 3 * 2 * nv, sizeof(double));
}

/* one face's reconstructed value of field f (0 h, 1 b) at Gauss node g on side s of cell cc */
static inline double s2_face_value(uo_ctx* c, int cc, int k, int f, int s, int g) {
    return s2_rec(c, cc, k)[f * 12 + s * 3 + g];
}

/* the unchanged instantaneous upwind transport flux of the current reconstruction at the right x face
 * and (below the top row) the top y face of every cell (s2w1d_instantaneous_flux, mod_S2D1.f90:1052-1095;
 * s2w2r_instantaneous, :1098-1150), into v_inst slots 0 and 1 */
static void s2_inst_faces(uo_ctx* c) {
    const int nx = c->p.nx, ny = c->p.ny, nv = c->p.nvel;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const int cc = j * nx + i, ir = j * nx + (i + 1) % nx, up = cc + nx;
            double* xi = c->v_inst + (size_t)cc * 3 * 2 * nv;
            double* yi = xi + 2 * (size_t)nv;
            for (int k = 0; k < 2 * nv; ++k) { xi[k] = 0.0; yi[k] = 0.0; }
            for (int g = 0; g < 3; ++g)
                for (int k = 0; k < nv; ++k) {
                    const int xl = c->u[k] >= 0.0;
                    const double rh = xl ? s2_face_value(c, cc, k, 0, 1, g) : s2_face_value(c, ir, k, 0, 0, g);
                    const double rb = xl ? s2_face_value(c, cc, k, 1, 1, g) : s2_face_value(c, ir, k, 1, 0, g);
                    xi[k] = xi[k] + s2_gw[g] * c->u[k] * rh;
                    xi[nv + k] = xi[nv + k] + s2_gw[g] * c->u[k] * rb;
                    if (j < ny - 1) {
                        const int yl = c->v[k] >= 0.0;
                        const double sh = yl ? s2_face_value(c, cc, k, 0, 3, g) : s2_face_value(c, up, k, 0, 2, g);
                        const double sb = yl ? s2_face_value(c, cc, k, 1, 3, g) : s2_face_value(c, up, k, 1, 2, g);
                        yi[k] = yi[k] + s2_gw[g] * c->v[k] * sh;
                        yi[nv + k] = yi[nv + k] + s2_gw[g] * c->v[k] * sb;
                    }
                }
        }
}

/* the reconstruction of the state (h, b) into s2_rec, the accepted state staying in place */
static int s2_recon_of(uo_ctx* c, double* h, double* b) {
    int nthr = g_threads < c->nthr ? g_threads : c->nthr;
    double *h0 = c->h, *b0 = c->b;
    c->h = h;
    c->b = b;
    memset(c->cell_err, 0, sizeof(int) * c->nc);
    s2_arg a = {c, c->cell_err, 0};
    par_for(c->nc, s2_recon_body, &a, nthr);
    c->h = h0;
    c->b = b0;
    return s2_first_error(c);
}

/* the corrected micro flux of one face: f + dt (instantaneous - leading) - dt^2/2 time, in the two
 * groupings the reference writes (W1D: 0.5*dt**2, W2R: 0.5*dt*dt) */
static inline double s2_correct(double f, double inst, double lead, double time, double dt) {
    return f + dt * (inst - lead) - 0.5 * (dt * dt) * time;
}

/* S2W1PredictMidpointWall (mod_S2NativeAdapter.f90:605-685), with the W1D face correction (:660-680):
 * an isolated half step of the accepted state (compute_flux at dt/2 with the kinetic walls, the
 * transport, advance_step's CN collision at dt/2) predicts the state at t + dt/2; the walls are then
 * re-evaluated there at the full dt (s2w1_compute_wall_flux, mod_S2D1.f90:1000-1048) and replace the
 * official walls.  W1D also moves every interior face's leading-order flux to the midpoint:
 * f + dt (f_inst(mid) - f_lead) - dt^2/2 f_time, and re-takes its macro flux.  A failure anywhere is the
 * reference's abort 449. */
static int s2w1t_predict(uo_ctx* c, double dt) {
    const uo_params* p = &c->p;
    const int nx = p->nx, ny = p->ny, nv = p->nvel, nc = c->nc;
    const int nthr = g_threads < c->nthr ? g_threads : c->nthr;
    const size_t st = 2 * (size_t)nv + 4;
    const double half = 0.5 * dt;
    s2v_alloc(c);
    cn_alloc(c);
    memcpy(c->s2_facc0, c->s2_facc, sizeof(double) * (size_t)nc * 3 * st);
    if (s2_evaluate(c, half, 0)) return 449;
    /* the transport of the accepted state with the half-step fluxes (:630-647) */
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const int cc = j * nx + i, im = j * nx + (i + nx - 1) % nx;
            const double* xr = c->s2_facc + (size_t)cc * 3 * st;
            const double* xl = c->s2_facc + (size_t)im * 3 * st;
            const double* yt = xr + st;
            const double* yb = j == 0 ? xr + 2 * st : c->s2_facc + (size_t)(cc - nx) * 3 * st + st;
            for (int m = 0; m < 4; ++m) {
                double w = c->W[cc * 4 + m] - (xr[2 * nv + m] - xl[2 * nv + m]) / p->dx;
                c->cn_wn[cc * 4 + m] = w - (yt[2 * nv + m] - yb[2 * nv + m]) / p->dy;
            }
            for (int k = 0; k < nv; ++k) {
                const size_t q = (size_t)cc * nv + k;
                double sh = c->h[q] - (xr[k] - xl[k]) / p->dx, sb = c->b[q] - (xr[nv + k] - xl[nv + k]) / p->dx;
                c->cn_hs[q] = sh - (yt[k] - yb[k]) / p->dy;
                c->cn_bs[q] = sb - (yt[nv + k] - yb[nv + k]) / p->dy;
            }
        }
    /* advance_step on the stream state at dt/2 (mod_S2D1.f90:1302-1435): targets, CN collision, gates */
    memset(c->cell_err, 0, sizeof(int) * nc);
    s2tg_arg t = {c, c->cell_err, c->cn_wn, c->cn_mh, c->cn_mb, c->cn_kxh, c->cn_kxb, c->cn_kyh, c->cn_kyb, c->cn_kappa};
    par_for(nc, s2_target_body, &t, nthr);
    if (s2_first_error(c)) return 449;
    cn_arg ca = {c, half};
    par_for(nc, s2_cn_body, &ca, nthr);
    if (s2_first_error(c)) return 449;
    double cnres = 0.0, mmerr = 0.0;
    int fin = 1;
    for (int cc = 0; cc < nc; ++cc) {
        cnres = fmax(cnres, c->cn_cell[(size_t)cc * UO_CN_CELL + 1]);
        mmerr = fmax(mmerr, c->cn_cell[(size_t)cc * UO_CN_CELL + 2]);
    }
    for (size_t q = 0; q < (size_t)nc * 4; ++q) fin &= isfinite(c->cn_wn[q]);
    for (size_t q = 0; q < (size_t)nc * nv; ++q) fin &= isfinite(c->cn_hn[q]) && isfinite(c->cn_bn[q]);
    if (!fin || cnres > S2_GATE || mmerr > S2_GATE) return 449;
    /* the predicted state's reconstruction; its kinetic walls at the full dt replace the official ones */
    if (s2_recon_of(c, c->cn_hn, c->cn_bn)) return 449;
    memcpy(c->s2_facc, c->s2_facc0, sizeof(double) * (size_t)nc * 3 * st);
    s2_scratch* S = s2_scr(c, 0);
    double *hin = S->buf + 42 * (size_t)nv, *bin = hin + nv, *fh = bin + nv, *fb = fh + nv;
    for (int i = 0; i < nx; ++i)
        for (int t2 = 0; t2 < 2; ++t2) {
            const int cc = t2 == 0 ? i : (ny - 1) * nx + i, side = t2 == 0 ? 2 : 3;
            double* acc = c->s2_facc + (size_t)cc * 3 * st + (size_t)(t2 == 0 ? 2 : 1) * st;
            for (size_t k = 0; k < st; ++k) acc[k] = 0.0;
            for (int g = 0; g < 3; ++g) {
                for (int k = 0; k < nv; ++k) { hin[k] = s2_face_value(c, cc, k, 0, side, g); bin[k] = s2_face_value(c, cc, k, 1, side, g); }
                double fw[4];
                if (!s2w1_wall_node(c, t2 == 0 ? -1 : 1, dt, hin, bin, p->wall_ux[t2], 0.5 * p->wall_tnative[t2], fh, fb, fw))
                    return 449;
                for (int k = 0; k < nv; ++k) { acc[k] = acc[k] + s2_gw[g] * fh[k]; acc[nv + k] = acc[nv + k] + s2_gw[g] * fb[k]; }
                for (int m = 0; m < 4; ++m) acc[2 * nv + m] = acc[2 * nv + m] + s2_gw[g] * fw[m];
            }
        }
    if (!p->s2_face_time) return 0;
    s2_inst_faces(c);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const int cc = j * nx + i;
            for (int f = 0; f < (j < ny - 1 ? 2 : 1); ++f) {
                double* a = c->s2_facc + (size_t)cc * 3 * st + (size_t)f * st;
                const double* in = c->v_inst + ((size_t)cc * 3 + f) * 2 * nv;
                const double* cf = c->s2_coef + ((size_t)cc * 3 + f) * 4 * nv;
                for (int k = 0; k < nv; ++k) {
                    a[k] = s2_correct(a[k], in[k], cf[k], cf[2 * nv + k], dt);
                    a[nv + k] = s2_correct(a[nv + k], in[nv + k], cf[nv + k], cf[3 * nv + k], dt);
                }
                if (!s2_moment(nv, a, a + nv, c->u, c->v, c->w, a + 2 * nv)) return 449;
            }
        }
    return 0;
}

/* s2w2r_correct (mod_S2D1.f90:1152-1244): W2R's shared predictor.  From compute_flux's leading
 * coefficients a half step of transport and BGK relaxation with the frozen tau0 predicts the state at
 * t + dt/2 (its moment gate 2e-12); the instantaneous upwind faces and the instantaneous multiscale walls
 * there replace every face's leading-order flux: f + dt (f_inst - f_lead) - dt^2/2 f_time, the walls
 * included, whose mass flux must then vanish (gate 2e-12); every macro flux is re-taken.  A failure is
 * the reference's abort 456. */
static int s2w2r_correct(uo_ctx* c, double dt) {
    const uo_params* p = &c->p;
    const int nx = p->nx, ny = p->ny, nv = p->nvel, nc = c->nc, ck = p->ck;
    const size_t st = 2 * (size_t)nv + 4;
    s2v_alloc(c);
    cn_alloc(c);
    double** T = scratch_t(c, 0);
    double *dlh = T[0], *dlb = T[1];
    double diag1 = 0.0;
    int lok = 1;
    /* the predictor (:1175-1193): ws, hs, bs into cn_wn, cn_hn, cn_bn */
    for (int j = 0; j < ny && lok; ++j)
        for (int i = 0; i < nx; ++i) {
            const int cc = j * nx + i, im = j * nx + (i + nx - 1) % nx;
            const double* x0 = c->s2_coef + (size_t)cc * 3 * 4 * nv;
            const double* x0m = c->s2_coef + (size_t)im * 3 * 4 * nv;
            const double* y0 = x0 + 4 * (size_t)nv;
            const double* y0l = j == 0 ? x0 + 8 * (size_t)nv : c->s2_coef + ((size_t)(cc - nx) * 3 + 1) * 4 * nv;
            for (int k = 0; k < nv; ++k) {
                dlh[k] = -(x0[k] - x0m[k]) / p->dx;
                dlb[k] = -(x0[nv + k] - x0m[nv + k]) / p->dx;
                dlh[k] = dlh[k] - (y0[k] - y0l[k]) / p->dy;
                dlb[k] = dlb[k] - (y0[nv + k] - y0l[nv + k]) / p->dy;
            }
            double mom[4];
            if (!s2_moment(nv, dlh, dlb, c->u, c->v, c->w, mom)) return 456;
            double* ws = c->cn_wn + cc * 4;
            for (int m = 0; m < 4; ++m) ws[m] = c->W[cc * 4 + m] + 0.5 * dt * mom[m];
            for (int k = 0; k < nv; ++k) {
                const size_t q = (size_t)cc * nv + k;
                c->cn_hn[q] = c->h[q] + 0.5 * dt * (dlh[k] + (c->s2_mh[q] - c->h[q]) / s2_tau0);
                c->cn_bn[q] = c->b[q] + 0.5 * dt * (dlb[k] + (c->s2_mb[q] - c->b[q]) / s2_tau0);
            }
            double rho, ux, vy, th, pp;
            if (!s2_primitive(ws, ck, &rho, &ux, &vy, &th, &pp)) { lok = 0; break; }
            if (!s2_moment(nv, c->cn_hn + (size_t)cc * nv, c->cn_bn + (size_t)cc * nv, c->u, c->v, c->w, mom)) return 456;
            double mx = 0.0, sc = 0.0;
            for (int m = 0; m < 4; ++m) { mx = fmax(mx, fabs(mom[m] - ws[m])); sc = fmax(sc, fabs(ws[m])); }
            diag1 = fmax(diag1, mx / fmax(1.0, sc));
        }
    int fin = 1;
    for (size_t q = 0; q < (size_t)nc * nv; ++q) fin &= isfinite(c->cn_hn[q]) && isfinite(c->cn_bn[q]);
    if (!lok || diag1 > S2_GATE || !fin) return 456;
    /* the instantaneous faces and walls at the predictor (s2w2r_instantaneous) */
    if (s2_recon_of(c, c->cn_hn, c->cn_bn)) return 456;
    s2_inst_faces(c);
    s2_scratch* S = s2_scr(c, 0);
    double *hin = S->buf + 42 * (size_t)nv, *bin = hin + nv, *fh = bin + nv, *fb = fh + nv;
    for (int i = 0; i < nx; ++i)
        for (int t2 = 0; t2 < 2; ++t2) {
            const int cc = t2 == 0 ? i : (ny - 1) * nx + i, side = t2 == 0 ? 2 : 3;
            double* in = c->v_inst + ((size_t)cc * 3 + (t2 == 0 ? 2 : 1)) * 2 * nv;
            for (int k = 0; k < 2 * nv; ++k) in[k] = 0.0;
            for (int g = 0; g < 3; ++g) {
                for (int k = 0; k < nv; ++k) { hin[k] = s2_face_value(c, cc, k, 0, side, g); bin[k] = s2_face_value(c, cc, k, 1, side, g); }
                double fw[4];
                if (!s2w2_inst_node(c, 0, t2 == 0 ? -1 : 1, hin, bin, p->wall_ux[t2], 0.5 * p->wall_tnative[t2], fh, fb, fw))
                    return 456;
                for (int k = 0; k < nv; ++k) { in[k] = in[k] + s2_gw[g] * fh[k]; in[nv + k] = in[nv + k] + s2_gw[g] * fb[k]; }
            }
        }
    /* the corrected faces (:1214-1233): every x face, every y face with the top wall, the bottom wall */
    double diag6 = 0.0;
    fin = 1;
    for (int cc = 0; cc < nc; ++cc) {
        const int j = cc / nx;
        for (int f = 0; f < 3; ++f) {
            if (f == 2 && j != 0) continue;
            double* a = c->s2_facc + (size_t)cc * 3 * st + (size_t)f * st;
            const double* in = c->v_inst + ((size_t)cc * 3 + f) * 2 * nv;
            const double* cf = c->s2_coef + ((size_t)cc * 3 + f) * 4 * nv;
            for (int k = 0; k < nv; ++k) {
                a[k] = s2_correct(a[k], in[k], cf[k], cf[2 * nv + k], dt);
                a[nv + k] = s2_correct(a[nv + k], in[nv + k], cf[nv + k], cf[3 * nv + k], dt);
                if (f < 2) fin &= isfinite(a[k]) && isfinite(a[nv + k]);
            }
            if (f == 2 || (f == 1 && j == ny - 1)) {
                double mom[4];
                if (!s2_moment(nv, a, a + nv, c->u, c->v, c->w, mom)) return 456;
                diag6 = fmax(diag6, fabs(mom[0]));
            }
        }
    }
    if (diag6 > S2_GATE || !fin) return 456;
    for (int cc = 0; cc < nc; ++cc)
        for (int f = 0; f < 3; ++f) {
            if (f == 2 && cc >= nx) continue;
            double* a = c->s2_facc + (size_t)cc * 3 * st + (size_t)f * st;
            if (!s2_moment(nv, a, a + nv, c->u, c->v, c->w, a + 2 * nv)) return 456;
        }
    return 0;
}

/* One S2CN2 step of the explicit high-order method (TimeStep; S2NativeEvolution with the targets
 * kept between steps, mod_S2NativeAdapter.f90:469-490; ComputeResidual; S2NativeApplyUpdate,
 * :867-940, with advance_step on the stream state, mod_S2D1.f90:1302-1435): the proposal
 * wn = W + res, hs = h + res_h; targets of wn; the CN collision; the cnres / mmerr gates (2e-12);
 * the global conservation drift with the wall ledger.  A rejected step leaves W, h, b, the targets
 * and the ledger untouched and returns the reference abort code (203, AbortSteadyImplicit, for a rejection).
 * out[UO_CN_OUT]: [0] dt, [1] cnres, [2] mmerr, [3] max 2 beta, [4] transport CFL, [5..8] min/max
 * of h and b, [9] drift, [10..13] bottom wall flux / dy, [14..17] top wall flux / dy,
 * [18..21] wall balance after the step. */
int uo_s2cn2_step(uo_ctx* c, double* out, int nout) {
    const uo_params* p = &c->p;
    const int nx = p->nx, ny = p->ny, nv = p->nvel, nc = c->nc;
    int nthr = g_threads < c->nthr ? g_threads : c->nthr;
    s2_alloc(c);
    cn_alloc(c);
    double o[UO_CN_OUT];
    for (int q = 0; q < UO_CN_OUT; ++q) o[q] = 0.0;
    const double dt = uo_timestep(c);
    if (!isfinite(dt)) return 101;
    o[0] = dt;
    int e;
    if (!c->s2_ready) {   /* native_build_targets of the accepted state (:480-484) */
        memset(c->cell_err, 0, sizeof(int) * nc);
        s2tg_arg t = {c, c->cell_err, c->W, c->s2_mh, c->s2_mb, c->s2_kxh, c->s2_kxb, c->s2_kyh, c->s2_kyb, c->s2_kappa};
        par_for(nc, s2_target_body, &t, nthr);
        if ((e = s2_first_error(c))) return e;
        c->s2_ready = 1;
    }
    if ((e = s2_variant_check(p))) return e;
    if ((e = s2_evaluate(c, dt, p->s2_face_time || p->s2_shared_predictor))) return e;
    if (p->s2_shared_predictor && (e = s2w2r_correct(c, dt))) return e;
    if (p->s2_time_centered && (e = s2w1t_predict(c, dt))) return e;
    c->dt = dt;
    s2_publish(c);
    if ((e = uo_s2_compute_residual(c, dt, 0))) return e;
    /* the stream state (S2NativeApplyUpdate :884-890) */
    for (int cc = 0; cc < nc; ++cc) {
        for (int m = 0; m < 4; ++m) c->cn_wn[cc * 4 + m] = c->W[cc * 4 + m] + c->res_w[cc * 4 + m];
        for (int k = 0; k < nv; ++k) {
            c->cn_hs[(size_t)cc * nv + k] = c->h[(size_t)cc * nv + k] + c->res_h[(size_t)cc * nv + k];
            c->cn_bs[(size_t)cc * nv + k] = c->b[(size_t)cc * nv + k] + c->res_b[(size_t)cc * nv + k];
        }
    }
    memset(c->cell_err, 0, sizeof(int) * nc);
    s2tg_arg t = {c, c->cell_err, c->cn_wn, c->cn_mh, c->cn_mb, c->cn_kxh, c->cn_kxb, c->cn_kyh, c->cn_kyb, c->cn_kappa};
    par_for(nc, s2_target_body, &t, nthr);
    if ((e = s2_first_error(c))) return e;
    cn_arg ca = {c, dt};
    par_for(nc, s2_cn_body, &ca, nthr);
    if ((e = s2_first_error(c))) return e;
    double cnres = 0.0, mmerr = 0.0, b2 = 0.0, lo_h = INFINITY, hi_h = 0.0, lo_b = INFINITY, hi_b = 0.0;
    double umx = 0.0, vmx = 0.0;
    for (int cc = 0; cc < nc; ++cc) {
        const double* d = c->cn_cell + (size_t)cc * UO_CN_CELL;
        b2 = fmax(b2, d[0]); cnres = fmax(cnres, d[1]); mmerr = fmax(mmerr, d[2]);
        lo_h = fmin(lo_h, d[3]); hi_h = fmax(hi_h, d[4]); lo_b = fmin(lo_b, d[5]); hi_b = fmax(hi_b, d[6]);
    }
    for (int k = 0; k < nv; ++k) { umx = fmax(umx, fabs(c->u[k])); vmx = fmax(vmx, fabs(c->v[k])); }
    o[1] = cnres; o[2] = mmerr; o[3] = b2; o[4] = dt * (umx / p->dx + vmx / p->dy);
    o[5] = lo_h; o[6] = hi_h; o[7] = lo_b; o[8] = hi_b;
    int reject = !(cnres <= S2_GATE) || !(mmerr <= S2_GATE);
    for (size_t q = 0; q < (size_t)nc * 4 && !reject; ++q) if (!isfinite(c->cn_wn[q])) reject = 1;
    for (size_t q = 0; q < (size_t)nc * nv && !reject; ++q)
        if (!isfinite(c->cn_hn[q]) || !isfinite(c->cn_bn[q])) reject = 1;
    /* global conservation: total of the proposal plus the wall ledger against total0 (:907-926) */
    double total[4], bottom[4] = {0, 0, 0, 0}, top[4] = {0, 0, 0, 0}, drift = 0.0;
    const size_t st = 2 * (size_t)nv + 4;
    for (int m = 0; m < 4; ++m) {
        double s = 0.0;
        for (int cc = 0; cc < nc; ++cc) s = s + c->cn_wn[cc * 4 + m];
        total[m] = s;
    }
    for (int i = 0; i < nx; ++i) {
        const double* lw = c->s2_facc + (size_t)i * 3 * st + 2 * st + 2 * nv;
        const double* tw = c->s2_facc + ((size_t)(ny - 1) * nx + i) * 3 * st + st + 2 * nv;
        for (int m = 0; m < 4; ++m) { bottom[m] = bottom[m] + lw[m] / p->dy; top[m] = top[m] + tw[m] / p->dy; }
    }
    for (int m = 0; m < 4; ++m) {
        const double bal = c->cn_balance[m] + top[m] - bottom[m];
        drift = fmax(drift, fabs(total[m] + bal - c->cn_total0[m]) / fmax(1.0, fabs(c->cn_total0[m])));
        o[10 + m] = bottom[m]; o[14 + m] = top[m]; o[18 + m] = bal;
    }
    o[9] = drift;
    if (!(drift <= S2_GATE)) reject = 1;
    if (out) for (int q = 0; q < nout && q < UO_CN_OUT; ++q) out[q] = o[q];
    if (reject) return 203;
    /* accept: publish the proposal, keep its targets, advance the ledger */
    memcpy(c->W, c->cn_wn, sizeof(double) * 4 * (size_t)nc);
    memcpy(c->h, c->cn_hn, sizeof(double) * (size_t)nc * nv);
    memcpy(c->b, c->cn_bn, sizeof(double) * (size_t)nc * nv);
    double* sw;
    sw = c->s2_mh; c->s2_mh = c->cn_mh; c->cn_mh = sw;
    sw = c->s2_mb; c->s2_mb = c->cn_mb; c->cn_mb = sw;
    sw = c->s2_kxh; c->s2_kxh = c->cn_kxh; c->cn_kxh = sw;
    sw = c->s2_kxb; c->s2_kxb = c->cn_kxb; c->cn_kxb = sw;
    sw = c->s2_kyh; c->s2_kyh = c->cn_kyh; c->cn_kyh = sw;
    sw = c->s2_kyb; c->s2_kyb = c->cn_kyb; c->cn_kyb = sw;
    sw = c->s2_kappa; c->s2_kappa = c->cn_kappa; c->cn_kappa = sw;
    for (int m = 0; m < 4; ++m) c->cn_balance[m] = o[18 + m];
    return 0;
}

#include "ugks_oracle_reftan.c"
